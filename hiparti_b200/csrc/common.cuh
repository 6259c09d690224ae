// common.cuh -- error reporting, device memory and stream plumbing shared by
// every translation unit of libhiparti_b200.so.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/hiparti_b200.h"

namespace pti {

// Records the error in the calling thread's last-error slot (the behaviour of
// src/helper_funcs/error.c:27-74 in the reference) and prints it to stderr
// unless HIPARTI_B200_QUIET is set.  Returns errcode for `return complain(...)`.
int complain(const char *module, int errcode, const char *file, unsigned line, const char *reason);

}  // namespace pti

#define PTI_FAIL(code, module, reason) \
    return ::pti::complain((module), (code), __FILE__, __LINE__, (reason))

#define PTI_CHECK(cond, code, module, reason)       \
    do {                                            \
        if (__builtin_expect(!(cond), 0)) PTI_FAIL((code), (module), (reason)); \
    } while (0)

// CUDA runtime errors map to PTIERR_CUDA_ERROR + cudaError_t, as in
// include/includes/error.h:79-85 of the reference.
#define PTI_CUDA(call, module)                                                   \
    do {                                                                         \
        cudaError_t _e = (call);                                                 \
        if (__builtin_expect(_e != cudaSuccess, 0)) {                            \
            cudaGetLastError();                                                  \
            PTI_FAIL(PTIERR_CUDA_ERROR + (int)_e, (module), cudaGetErrorString(_e)); \
        }                                                                        \
    } while (0)

// Propagates a non-zero return code of a nested call.
#define PTI_TRY(expr)                     \
    do {                                  \
        int _r = (expr);                  \
        if (_r != 0) return _r;           \
    } while (0)

namespace pti {

// Stream used by the synchronous reference entry points: one non-blocking
// stream per device, created on first use.
cudaStream_t sync_stream();
// A second stream per device, for host-to-device copies that overlap work on
// sync_stream().
cudaStream_t copy_stream();
// Two non-blocking side streams per device (0 is copy_stream()), for kernels
// that run beside the caller's stream; created on first use.
cudaStream_t side_stream(int which);

// Stream-ordered device allocation from the runtime's default memory pool
// (cudaMallocAsync).  The pool keeps freed memory for reuse, so repeated calls
// do not return to the driver.
struct DevBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
    cudaStream_t stream = nullptr;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    DevBuf(DevBuf &&o) noexcept { swap(o); }
    DevBuf &operator=(DevBuf &&o) noexcept { reset(); swap(o); return *this; }
    ~DevBuf() { reset(); }
    void swap(DevBuf &o) {
        std::swap(ptr, o.ptr); std::swap(bytes, o.bytes); std::swap(stream, o.stream);
    }
    cudaError_t alloc(size_t n, cudaStream_t s) {
        reset();
        stream = s;
        bytes = n;
        if (n == 0) return cudaSuccess;
        return cudaMallocAsync(&ptr, n, s);
    }
    void reset() {
        if (ptr) cudaFreeAsync(ptr, stream);
        ptr = nullptr;
        bytes = 0;
    }
    template <class T> T *as() const { return static_cast<T *>(ptr); }
};

// Sets the runtime's default pool to keep freed memory (release threshold =
// unlimited) so that stream-ordered allocations are served from the pool.
void configure_pool_once();

// Allocation sizes are rounded up to 64 bytes plus one 64-byte guard so that
// vectorised and bulk copies of a final partial tile stay inside the buffer.
inline size_t padded(size_t bytes) { return ((bytes + 63) / 64) * 64 + 64; }

inline unsigned ceil_div(uint64_t a, uint64_t b) { return (unsigned)((a + b - 1) / b); }

int sm_count();

}  // namespace pti
