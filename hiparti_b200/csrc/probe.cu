// probe.cu -- the L2 read bandwidth of this GPU, measured by a kernel of this
// library: the ceiling against which the MTTKRP's factor-row gathers (2 rows
// of R values per nonzero for a 3-D tensor, served from L1 and L2) are read.
// A buffer inside L2 is streamed with 16-byte loads; the first pass brings
// it into L2 and is not timed.  Each thread needs several loads per pass for
// all eight to be in flight: on B200 buffers of 64-96 MiB read at the same
// rate (18.8 TB/s), 16 MiB (under four loads per thread) at half of it.
#include "common.cuh"

namespace pti {
namespace {

constexpr int kProbeLoads = 8;  // independent 16-byte loads in flight per thread

// Every thread issues kProbeLoads independent 16-byte L2-only loads (__ldcg:
// ld.global.cg, no L1 allocation) before it uses any of them, so the figure
// is the L2's read rate rather than the latency of one load per thread.
__global__ void l2_read_kernel(const uint4 *buf, uint64_t n16, unsigned reps, uint32_t *sink)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    uint32_t acc = 0;
    for (unsigned r = 0; r < reps; ++r)
        for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n16; i += kProbeLoads * stride) {
            uint4 v[kProbeLoads];
#pragma unroll
            for (int k = 0; k < kProbeLoads; ++k)
                v[k] = i + k * stride < n16 ? __ldcg(buf + i + k * stride) : make_uint4(0, 0, 0, 0);
#pragma unroll
            for (int k = 0; k < kProbeLoads; ++k) acc ^= v[k].x ^ v[k].y ^ v[k].z ^ v[k].w;
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
