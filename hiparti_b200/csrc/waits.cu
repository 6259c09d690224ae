// waits.cu -- a self-check of the bounded mbarrier wait that every bulk-copy
// kernel here uses (tma.cuh).  One CTA arms an mbarrier for 16 bytes that no
// copy ever delivers and waits with the normal bound, which must give up and
// report it; a second barrier, whose arrival completes its phase, must be
// seen complete.  No copy is issued, so nothing is left in flight when the
// CTA exits.
#include "common.cuh"
#include "tma.cuh"

namespace pti {
namespace {

__global__ void mbar_probe_kernel(uint32_t polls, int *out)
{
    __shared__ uint64_t withheld, delivered;
    if (threadIdx.x == 0) {
        mbar_init(&withheld, 1);
        mbar_init(&delivered, 1);
        mbar_fence_init();
        mbar_arrive_expect_tx(&withheld, 16);  // 16 bytes expected, none ever sent
        mbar_arrive_expect_tx(&delivered, 0);  // arrival alone completes this phase
    }
    __syncthreads();
    const bool gave_up = !mbar_wait_bounded(&withheld, 0, polls);
    const bool done = mbar_wait_bounded(&delivered, 0, polls);
    if (threadIdx.x == 0) {
        out[0] = gave_up ? 1 : 0;
        out[1] = done ? 1 : 0;
    }
}

}  // namespace
}  // namespace pti

extern "C" int ptiB200MbarrierWaitProbe(unsigned polls, int *gave_up, int *completed)
{
    using namespace pti;
    const char *mod = "B200 mbarrier wait probe";
    PTI_CHECK(gave_up && completed && polls >= 1 && polls <= (1u << 22), PTIERR_VALUE_ERROR, mod,
              "polls must be in [1, 2^22]");
    cudaStream_t s = sync_stream();
    DevBuf out;
    PTI_CUDA(out.alloc(64, s), mod);
    PTI_CUDA(cudaMemsetAsync(out.ptr, 0xff, 8, s), mod);
    mbar_probe_kernel<<<1, 32, 0, s>>>(polls, out.as<int>());
    PTI_CUDA(cudaGetLastError(), mod);
    int h[2] = {-1, -1};
    PTI_CUDA(cudaMemcpyAsync(h, out.ptr, sizeof h, cudaMemcpyDeviceToHost, s), mod);
    PTI_CUDA(cudaStreamSynchronize(s), mod);
    *gave_up = h[0];
    *completed = h[1];
    return 0;
}
