// probe.cu -- the L2 read bandwidth of this GPU, measured by a kernel of this
// library: the ceiling against which the MTTKRP's factor-row gathers (2 rows
// of R values per nonzero for a 3-D tensor, served from L1 and L2) are read.
// A buffer well inside L2 is streamed with 16-byte loads; the first pass
// brings it into L2 and is not timed.
#include "common.cuh"

namespace pti {
namespace {

__global__ void l2_read_kernel(const uint4 *buf, uint64_t n16, unsigned reps, uint32_t *sink)
{
    uint32_t acc = 0;
    for (unsigned r = 0; r < reps; ++r)
        for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n16; i += (uint64_t)gridDim.x * blockDim.x) {
            uint4 v;
            // L2 only (.cg: the loads do not allocate in L1)
            asm volatile("ld.global.cg.v4.u32 {%0,%1,%2,%3}, [%4];"
                         : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                         : "l"(buf + i));
            acc ^= v.x ^ v.y ^ v.z ^ v.w;
        }
    if (acc == 0x9e3779b9u) sink[0] = acc;  // keeps the loads; practically never written
}

}  // namespace
}  // namespace pti

extern "C" int ptiB200ProbeL2ReadBandwidth(unsigned long long bytes, unsigned reps, double *gbps)
{
    using namespace pti;
    const char *mod = "B200 L2 read probe";
    PTI_CHECK(gbps && bytes >= (1u << 20) && bytes <= (1ull << 30) && reps >= 1 && reps <= 1000, PTIERR_VALUE_ERROR,
              mod, "bytes must be in [1 MiB, 1 GiB] and reps in [1, 1000]");
    cudaStream_t s = sync_stream();
    DevBuf buf, sink;
    const uint64_t n16 = bytes / 16;
    PTI_CUDA(buf.alloc(padded(n16 * 16), s), mod);
    PTI_CUDA(sink.alloc(64, s), mod);
    PTI_CUDA(cudaMemsetAsync(buf.ptr, 1, n16 * 16, s), mod);
    const unsigned grid = (unsigned)sm_count() * 8;
    l2_read_kernel<<<grid, 256, 0, s>>>(buf.as<uint4>(), n16, 1, sink.as<uint32_t>());  // into L2
    cudaEvent_t e0, e1;
    PTI_CUDA(cudaEventCreate(&e0), mod);
    PTI_CUDA(cudaEventCreate(&e1), mod);
    cudaEventRecord(e0, s);
    l2_read_kernel<<<grid, 256, 0, s>>>(buf.as<uint4>(), n16, reps, sink.as<uint32_t>());
    cudaEventRecord(e1, s);
    const cudaError_t e = cudaStreamSynchronize(s);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    PTI_CUDA(e, mod);
    PTI_CUDA(cudaGetLastError(), mod);
    *gbps = (double)n16 * 16 * reps / (ms * 1e-3) / 1e9;
    return 0;
}
