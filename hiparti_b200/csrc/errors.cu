// errors.cu -- last-error slot, device selection, shared stream and pool.
#include "common.cuh"

#include <mutex>

namespace {
struct LastError {
    int code = 0;
    const char *module = nullptr;
    const char *file = nullptr;
    unsigned line = 0;
    char reason[512] = {0};
};
thread_local LastError g_last;
}  // namespace

namespace pti {

int complain(const char *module, int errcode, const char *file, unsigned line, const char *reason)
{
    g_last.code = errcode;
    g_last.module = module;
    g_last.file = file;
    g_last.line = line;
    std::snprintf(g_last.reason, sizeof g_last.reason, "%s", reason ? reason : "");
    if (!std::getenv("HIPARTI_B200_QUIET")) {
        std::fprintf(stderr, "[%s] error 0x%x at %s:%u, %s\n", module ? module : "", errcode,
                     file ? file : "", line, reason ? reason : "");
    }
    return errcode;
}

cudaStream_t sync_stream()
{
    static std::mutex mu;
    static std::vector<cudaStream_t> streams;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(mu);
    if ((int)streams.size() <= dev) streams.resize(dev + 1, nullptr);
    if (!streams[dev]) cudaStreamCreateWithFlags(&streams[dev], cudaStreamNonBlocking);
    return streams[dev];
}

cudaStream_t copy_stream() { return side_stream(0); }

cudaStream_t side_stream(int which)
{
    static std::mutex mu;
    static std::vector<cudaStream_t> streams;  // [device][2]
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(mu);
    if ((int)streams.size() <= 2 * dev + 1) streams.resize(2 * dev + 2, nullptr);
    cudaStream_t &st = streams[2 * dev + (which & 1)];
    if (!st) cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    return st;
}

void configure_pool_once()
{
    static std::mutex mu;
    static std::vector<char> done;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(mu);
    if ((int)done.size() <= dev) done.resize(dev + 1, 0);
    if (done[dev]) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t threshold = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold);
    }
    done[dev] = 1;
}

int sm_count()
{
    static std::vector<int> counts;
    static std::mutex mu;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(mu);
    if ((int)counts.size() <= dev) counts.resize(dev + 1, 0);
    if (!counts[dev]) cudaDeviceGetAttribute(&counts[dev], cudaDevAttrMultiProcessorCount, dev);
    return counts[dev];
}

}  // namespace pti

extern "C" {

int ptiGetLastError(const char **module, const char **file, unsigned *line, const char **reason)
{
    if (module) *module = g_last.module;
    if (file) *file = g_last.file;
    if (line) *line = g_last.line;
    if (reason) *reason = g_last.reason;
    return g_last.code;
}

void ptiClearLastError(void)
{
    g_last = LastError();
}

int ptiCudaSetDevice(int device)
{
    PTI_CUDA(cudaSetDevice(device), "CUDA SetDevice");
    return 0;
}

int ptiCudaGetLastError(void)
{
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : PTIERR_CUDA_ERROR + (int)e;
}

}  // extern "C"
