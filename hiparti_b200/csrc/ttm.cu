// ttm.cu -- sparse tensor times a dense matrix (TTM) and times a vector (TTV)
// along one mode, on the GPU.
//
// The reference (src/sptensor/mmul.c:36-86, vmul.c:26-70, with the fibers of
// src/ssptensor/setinds.c:33-71) sorts the nonzeros with the mode last
// (msort.c:33-57), cuts them into fibers -- runs with equal coordinates in
// every other mode -- and for every fiber f and column k adds up
//     Y[f, k] += x_j * U[i_mode(j), k]
// over the fiber's nonzeros in order, in FP32 with a rounded product and a
// rounded sum.  The result is a semi-sparse tensor: the fibers' coordinates
// plus a dense nfibers x stride block (stride = R rounded up to 8, padding
// zero).
//
// Here the sort is a stable LSD radix sort (the mode first, then the other
// modes from the last to the first) and the fibers come from a scan over
// "coordinates changed" flags; the fiber structure is kept per mode.  The TTM
// kernel gives each fiber a group of G lanes (G = 8, 16 or 32 by R), each lane
// CPL columns; the group loads G nonzeros of its fiber at a time and then
// walks them in order, so every Y element is the same sequence of FP32
// multiply-then-add steps as the reference's loop, and the result is
// bit-identical for tensors with distinct coordinates.
#include <cerrno>

#include "primitives.cuh"
#include "tensor.cuh"

namespace pti {
namespace {

unsigned grid_t(uint64_t n)
{
    return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, (uint64_t)sm_count() * 8));
}

#define GRID_LOOP(i, n) \
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += (uint64_t)gridDim.x * blockDim.x)

__global__ void iota_t(uint32_t *v, uint64_t n) { GRID_LOOP(i, n) v[i] = (uint32_t)i; }

__global__ void gather_key_t(const uint32_t *ind, const uint32_t *perm, uint64_t n, uint64_t *key)
{
    GRID_LOOP(i, n) key[i] = ind[perm[i]];
}

__global__ void gather_u32_t(const uint32_t *ind, const uint32_t *perm, uint64_t n, uint32_t *out)
{
    GRID_LOOP(i, n) out[i] = ind[perm[i]];
}

struct FiberArgs {
    uint32_t nmodes, mode;
    const uint32_t *inds[kMaxModes];
    const float *vals;
    const uint32_t *perm;
    uint64_t *fptr;
    uint32_t *finds[kMaxModes];
    uint32_t *sind;
    float *sval;
};
struct FiberHeadIn {
    FiberArgs a;
    __device__ uint64_t operator()(uint64_t i) const
    {
        if (i == 0) return 1;
        const uint32_t p = a.perm[i], q = a.perm[i - 1];
        for (uint32_t m = 0; m < a.nmodes; ++m)
            if (m != a.mode && a.inds[m][p] != a.inds[m][q]) return 1;
        return 0;
    }
};
struct FiberOut {
    FiberArgs a;
    __device__ void operator()(uint64_t i, uint64_t prefix, uint64_t head) const
    {
        const uint32_t p = a.perm[i];
        a.sind[i] = a.inds[a.mode][p];
        a.sval[i] = a.vals[p];
        if (!head) return;
        a.fptr[prefix] = i;  // fiber `prefix` starts at sorted position i
        for (uint32_t m = 0; m < a.nmodes; ++m)
            if (m != a.mode) a.finds[m][prefix] = a.inds[m][p];
    }
};

__global__ void set_last_t(uint64_t *fptr, uint64_t nfib, uint64_t nnz) { fptr[nfib] = nnz; }

// One group of G lanes per fiber; lane l of the group owns columns
// l, l + G, ..., l + (CPL-1) G.  Pad columns [R, ldy) are written as zero.
template <int CPL>
__global__ void __launch_bounds__(256) ttm_kernel(const uint64_t *__restrict__ fptr, uint64_t nfib,
                                                  const uint32_t *__restrict__ sind,
                                                  const float *__restrict__ sval, const float *__restrict__ U,
                                                  uint32_t ldu, uint32_t R, float *__restrict__ Y, uint32_t ldy,
                                                  int G)
{
    const int lane = threadIdx.x & 31;
    const int gl = lane % G;                       // lane in the group
    const unsigned gmask = (G == 32 ? 0xffffffffu : ((1u << G) - 1u)) << (lane - gl);
    const uint64_t groups = (uint64_t)gridDim.x * (blockDim.x / G);
    const uint64_t g0 = (uint64_t)blockIdx.x * (blockDim.x / G) + threadIdx.x / G;
    for (uint64_t f = g0; f < nfib; f += groups) {
        float acc[CPL];
#pragma unroll
        for (int c = 0; c < CPL; ++c) acc[c] = 0.f;
        const uint64_t b = fptr[f], e = fptr[f + 1];
        for (uint64_t j0 = b; j0 < e; j0 += G) {
            // the group's next G nonzeros, one per lane
            const uint64_t mine = j0 + gl;
            const uint32_t r_mine = mine < e ? sind[mine] : 0u;
            const float x_mine = mine < e ? sval[mine] : 0.f;
            const int cnt = (e - j0) < (uint64_t)G ? (int)(e - j0) : G;
            int t = 0;
            for (; t + 4 <= cnt; t += 4) {
                uint32_t r[4];
                float x[4], u[4][CPL];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    r[q] = __shfl_sync(gmask, r_mine, (lane - gl) + t + q);
                    x[q] = __shfl_sync(gmask, x_mine, (lane - gl) + t + q);
                }
#pragma unroll
                for (int q = 0; q < 4; ++q)
#pragma unroll
                    for (int c = 0; c < CPL; ++c) {
                        const uint32_t k = gl + c * G;
                        u[q][c] = k < R ? __ldg(U + (size_t)r[q] * ldu + k) : 0.f;
                    }
#pragma unroll
                for (int q = 0; q < 4; ++q)
#pragma unroll
                    for (int c = 0; c < CPL; ++c) acc[c] = __fadd_rn(acc[c], __fmul_rn(x[q], u[q][c]));
            }
            for (; t < cnt; ++t) {
                const uint32_t r = __shfl_sync(gmask, r_mine, (lane - gl) + t);
                const float x = __shfl_sync(gmask, x_mine, (lane - gl) + t);
#pragma unroll
                for (int c = 0; c < CPL; ++c) {
                    const uint32_t k = gl + c * G;
                    const float u = k < R ? __ldg(U + (size_t)r * ldu + k) : 0.f;
                    acc[c] = __fadd_rn(acc[c], __fmul_rn(x, u));
                }
            }
        }
        float *y = Y + (size_t)f * ldy;
#pragma unroll
        for (int c = 0; c < CPL; ++c) {
            const uint32_t k = gl + c * G;
            if (k < R) y[k] = acc[c];
        }
        for (uint32_t k = R + gl; k < ldy; k += G) y[k] = 0.f;
    }
}

// TTV: one lane per fiber.  Y[f * ldy] = sum of x_j * v[i_mode(j)] in order;
// the other ldy - 1 entries of the row are zero.
__global__ void ttv_kernel(const uint64_t *__restrict__ fptr, uint64_t nfib, const uint32_t *__restrict__ sind,
                           const float *__restrict__ sval, const float *__restrict__ v, float *__restrict__ Y,
                           uint32_t ldy)
{
    GRID_LOOP(f, nfib)
    {
        float acc = 0.f;
        for (uint64_t j = fptr[f]; j < fptr[f + 1]; ++j) acc = __fadd_rn(acc, __fmul_rn(sval[j], __ldg(v + sind[j])));
        float *y = Y + (size_t)f * ldy;
        y[0] = acc;
        for (uint32_t k = 1; k < ldy; ++k) y[k] = 0.f;
    }
}

int bits_t(uint64_t maxval)
{
    int b = 0;
    while (b < 64 && (maxval >> b)) ++b;
    return b;
}

}  // namespace

// Builds t's fibers along `mode`.  sort == false keeps the nonzeros in their
// input order (the reference does not sort a tensor whose sortorder already
// names this order).
int fiber_plan(ptiB200Tensor *t, uint32_t mode, bool sort, cudaStream_t s)
{
    const char *mod = "B200 TTM";
    PTI_CHECK(t && !t->hicoo, PTIERR_VALUE_ERROR, mod, "needs a device COO tensor");
    PTI_CHECK(mode < t->nmodes, PTIERR_SHAPE_MISMATCH, mod, "mode out of range");
    FiberPlan &P = t->fiber_plan[mode];
    const uint64_t n = t->nnz;
    const uint32_t N = t->nmodes;
    PTI_CHECK(n < 0xFFFFFFFFull, PTIERR_VALUE_ERROR, mod, "too many nonzeros");
    DevBuf key, tmp;
    RadixScratch sc;
    PTI_CUDA(P.perm.alloc(padded(n * 4), s), mod);
    PTI_CUDA(P.sind.alloc(padded(n * 4), s), mod);
    PTI_CUDA(P.sval.alloc(padded(n * 4), s), mod);
    if (n) iota_t<<<grid_t(n), 256, 0, s>>>(P.perm.as<uint32_t>(), n);
    if (n > 1 && sort) {
        PTI_CUDA(key.alloc(padded(n * 8), s), mod);
        PTI_TRY(sc.alloc(n, s));
        // least significant first: the mode itself, then the other modes from
        // the last to the first
        for (int k = (int)N; k >= 0; --k) {
            const uint32_t m = k == (int)N ? mode : (uint32_t)k;
            if (k != (int)N && m == mode) continue;
            gather_key_t<<<grid_t(n), 256, 0, s>>>(t->inds[m].as<uint32_t>(), P.perm.as<uint32_t>(), n,
                                                  key.as<uint64_t>());
            PTI_TRY(radix_sort_pairs(key, P.perm, n, ((bits_t(t->ndims[m] ? t->ndims[m] - 1 : 0) + 7) / 8) * 8, sc, s));
        }
    }
    FiberArgs a;
    a.nmodes = N;
    a.mode = mode;
    for (uint32_t m = 0; m < N; ++m) a.inds[m] = t->inds[m].as<uint32_t>();
    a.vals = t->vals.as<float>();
    a.perm = P.perm.as<uint32_t>();
    a.sind = P.sind.as<uint32_t>();
    a.sval = P.sval.as<float>();
    // fibers: at most n; allocate for n, then the count is known
    PTI_CUDA(P.fptr.alloc(padded((n + 1) * 8), s), mod);
    for (uint32_t m = 0; m < N; ++m) {
        if (m == mode) continue;
        PTI_CUDA(P.finds[m].alloc(padded(n * 4), s), mod);
        a.finds[m] = P.finds[m].as<uint32_t>();
    }
    a.fptr = P.fptr.as<uint64_t>();
    uint64_t nfib = 0;
    if (n) {
        PTI_CUDA(tmp.alloc(padded(scan_tmp_elems<uint64_t>(n) * 8), s), mod);
        PTI_TRY((exclusive_scan<uint64_t>(FiberHeadIn{a}, FiberOut{a}, n, tmp.as<uint64_t>(), &nfib, s)));
    }
    set_last_t<<<1, 1, 0, s>>>(P.fptr.as<uint64_t>(), nfib, n);
    PTI_CUDA(cudaGetLastError(), mod);
    P.nfib = nfib;
    P.ready = true;
    return 0;
}

// Y (device, nfib x ldy) = fibers of t along `mode` times U (device, rows of
// ldu floats, R columns used).  R == 0 with ldu == 1 is TTV (U a vector).
int ttm_device(ptiB200Tensor *t, uint32_t mode, const float *U, uint32_t R, uint32_t ldu, float *Y, uint32_t ldy,
               bool ttv, cudaStream_t s)
{
    const char *mod = "B200 TTM";
    FiberPlan &P = t->fiber_plan[mode];
    PTI_CHECK(P.ready, PTIERR_VALUE_ERROR, mod, "fibers not built");
    if (!P.nfib) return 0;
    const unsigned sms = (unsigned)sm_count();
    if (ttv) {
        ttv_kernel<<<grid_t(P.nfib), 256, 0, s>>>(P.fptr.as<uint64_t>(), P.nfib, P.sind.as<uint32_t>(),
                                                  P.sval.as<float>(), U, Y, ldy);
        PTI_CUDA(cudaGetLastError(), mod);
        return 0;
    }
    PTI_CHECK(R >= 1 && R <= 256 && ldu >= R && ldy >= R, PTIERR_VALUE_ERROR, mod, "rank must be in [1, 256]");
    const int G = R > 16 ? 32 : (R > 8 ? 16 : 8);
    const int cpl = (int)((R + G - 1) / G);
    const uint64_t groups_needed = P.nfib;
    const unsigned per_cta = 256 / G;
    const unsigned grid =
        (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((groups_needed + per_cta - 1) / per_cta, (uint64_t)sms * 16));
    const uint64_t *fp = P.fptr.as<uint64_t>();
    const uint32_t *si = P.sind.as<uint32_t>();
    const float *sv = P.sval.as<float>();
    if (cpl <= 1) ttm_kernel<1><<<grid, 256, 0, s>>>(fp, P.nfib, si, sv, U, ldu, R, Y, ldy, G);
    else if (cpl <= 2) ttm_kernel<2><<<grid, 256, 0, s>>>(fp, P.nfib, si, sv, U, ldu, R, Y, ldy, G);
    else if (cpl <= 4) ttm_kernel<4><<<grid, 256, 0, s>>>(fp, P.nfib, si, sv, U, ldu, R, Y, ldy, G);
    else ttm_kernel<8><<<grid, 256, 0, s>>>(fp, P.nfib, si, sv, U, ldu, R, Y, ldy, G);
    PTI_CUDA(cudaGetLastError(), mod);
    return 0;
}

namespace {

int new_index_vector(ptiIndexVector *v, uint64_t len)
{
    v->len = len;
    v->cap = len ? len : 1;
    v->data = static_cast<ptiIndex *>(std::malloc(v->cap * sizeof(ptiIndex)));
    PTI_CHECK(v->data, PTIERR_OS_ERROR + ENOMEM, "SspTns New", "out of memory");
    return 0;
}

// The reference's sortorder test (msort.c:33-57): the tensor is sorted only
// if its sortorder does not already read "the other modes ascending, then
// `mode`"; afterwards it does.
bool needs_sort_and_mark(ptiSparseTensor *X, uint32_t mode)
{
    bool need = false;
    const uint32_t N = X->nmodes;
    for (uint32_t m = 0; m < mode; ++m)
        if (X->sortorder[m] != m) {
            X->sortorder[m] = m;
            need = true;
        }
    for (uint32_t m = mode + 1; m < N; ++m)
        if (X->sortorder[m - 1] != m) {
            X->sortorder[m - 1] = m;
            need = true;
        }
    if (X->sortorder[N - 1] != mode) {
        X->sortorder[N - 1] = mode;
        need = true;
    }
    return need;
}

// Host entry: the reference's SpTTM / SpTTV with X and U (or V) on the host.
int host_ttm(ptiSemiSparseTensor *Y, ptiSparseTensor *X, const ptiValue *Uvals, uint32_t Urows, uint32_t R,
             uint32_t ldu, ptiIndex mode, bool ttv, const char *mod)
{
    PTI_CHECK(Y && X, PTIERR_VALUE_ERROR, mod, "null argument");
    PTI_CHECK(mode < X->nmodes, PTIERR_SHAPE_MISMATCH, mod, "shape mismatch");
    PTI_CHECK(X->ndims[mode] == Urows, PTIERR_SHAPE_MISMATCH, mod, "shape mismatch");
    PTI_CHECK(X->nmodes >= 2, PTIERR_SHAPE_MISMATCH, mod, "nmodes < 2");
    cudaStream_t s = sync_stream();
    ptiB200Tensor t;
    PTI_TRY(upload_coo(&t, X, s));
    const bool sort = needs_sort_and_mark(X, mode);
    PTI_TRY(fiber_plan(&t, mode, sort, s));
    const FiberPlan &P = t.fiber_plan[mode];
    const uint64_t nfib = P.nfib, nnz = X->nnz;
    const uint32_t N = X->nmodes;
    const uint32_t width = ttv ? 1 : R;               // Y's size in `mode`
    const uint32_t stride = ((width - 1) / 8 + 1) * 8;
    DevBuf dU, dY;
    PTI_CUDA(dU.alloc(padded((size_t)Urows * ldu * 4), s), mod);
    if (Urows) PTI_CUDA(cudaMemcpyAsync(dU.ptr, Uvals, (size_t)Urows * ldu * 4, cudaMemcpyHostToDevice, s), mod);
    PTI_CUDA(dY.alloc(padded(nfib * stride * 4), s), mod);
    PTI_TRY(ttm_device(&t, mode, dU.as<float>(), R, ldu, dY.as<float>(), stride, ttv, s));

    // The reference leaves X sorted in the fiber order when it sorted it.
    DevBuf sorted[kMaxModes];
    if (sort && nnz) {
        for (uint32_t m = 0; m < N; ++m) {
            if (m == mode) continue;
            PTI_CUDA(sorted[m].alloc(padded(nnz * 4), s), mod);
            gather_u32_t<<<grid_t(nnz), 256, 0, s>>>(t.inds[m].as<uint32_t>(), P.perm.as<uint32_t>(), nnz,
                                                    sorted[m].as<uint32_t>());
            PTI_CUDA(cudaMemcpyAsync(X->inds[m].data, sorted[m].ptr, nnz * 4, cudaMemcpyDeviceToHost, s), mod);
        }
        PTI_CUDA(cudaMemcpyAsync(X->inds[mode].data, P.sind.ptr, nnz * 4, cudaMemcpyDeviceToHost, s), mod);
        PTI_CUDA(cudaMemcpyAsync(X->values.data, P.sval.ptr, nnz * 4, cudaMemcpyDeviceToHost, s), mod);
    }

    // Y: ptiNewSemiSparseTensor (src/ssptensor/ssptensor.c:32-54) and the
    // fibers of setinds.c:33-71.
    Y->nmodes = N;
    Y->ndims = static_cast<ptiIndex *>(std::malloc(N * sizeof(ptiIndex)));
    PTI_CHECK(Y->ndims, PTIERR_OS_ERROR + ENOMEM, mod, "out of memory");
    for (uint32_t m = 0; m < N; ++m) Y->ndims[m] = m == mode ? width : X->ndims[m];
    Y->mode = mode;
    Y->nnz = nfib;
    Y->stride = stride;
    Y->inds = static_cast<ptiIndexVector *>(std::malloc(N * sizeof(ptiIndexVector)));
    PTI_CHECK(Y->inds, PTIERR_OS_ERROR + ENOMEM, mod, "out of memory");
    for (uint32_t m = 0; m < N; ++m) {
        PTI_TRY(new_index_vector(&Y->inds[m], m == mode ? 0 : nfib));
        if (m != mode && nfib)
            PTI_CUDA(cudaMemcpyAsync(Y->inds[m].data, P.finds[m].ptr, nfib * 4, cudaMemcpyDeviceToHost, s), mod);
    }
    PTI_TRY(ptiNewMatrix(&Y->values, (ptiIndex)nfib, stride));
    if (nfib)
        PTI_CUDA(cudaMemcpyAsync(Y->values.values, dY.ptr, nfib * stride * 4, cudaMemcpyDeviceToHost, s), mod);
    PTI_CUDA(cudaStreamSynchronize(s), mod);
    return 0;
}

}  // namespace
}  // namespace pti

extern "C" {

int ptiNewSemiSparseTensor(ptiSemiSparseTensor *tsr, ptiIndex nmodes, ptiIndex mode, const ptiIndex ndims[])
{
    using namespace pti;
    const char *mod = "SspTns New";
    PTI_CHECK(tsr && ndims, PTIERR_VALUE_ERROR, mod, "null argument");
    PTI_CHECK(nmodes >= 2, PTIERR_SHAPE_MISMATCH, mod, "nmodes < 2");
    PTI_CHECK(mode < nmodes, PTIERR_SHAPE_MISMATCH, mod, "mode out of range");
    tsr->nmodes = nmodes;
    tsr->ndims = static_cast<ptiIndex *>(std::malloc(nmodes * sizeof(ptiIndex)));
    PTI_CHECK(tsr->ndims, PTIERR_OS_ERROR + ENOMEM, mod, "out of memory");
    std::memcpy(tsr->ndims, ndims, nmodes * sizeof(ptiIndex));
    tsr->mode = mode;
    tsr->nnz = 0;
    tsr->inds = static_cast<ptiIndexVector *>(std::malloc(nmodes * sizeof(ptiIndexVector)));
    PTI_CHECK(tsr->inds, PTIERR_OS_ERROR + ENOMEM, mod, "out of memory");
    for (ptiIndex m = 0; m < nmodes; ++m) PTI_TRY(new_index_vector(&tsr->inds[m], 0));
    tsr->stride = ((ndims[mode] - 1) / 8 + 1) * 8;
    return ptiNewMatrix(&tsr->values, 0, tsr->stride);
}

void ptiFreeSemiSparseTensor(ptiSemiSparseTensor *tsr)
{
    if (!tsr) return;
    if (tsr->inds)
        for (ptiIndex m = 0; m < tsr->nmodes; ++m) std::free(tsr->inds[m].data);
    std::free(tsr->inds);
    std::free(tsr->ndims);
    ptiFreeMatrix(&tsr->values);
    tsr->inds = nullptr;
    tsr->ndims = nullptr;
    tsr->nmodes = 0;
    tsr->nnz = 0;
}

int ptiSparseTensorMulMatrix(ptiSemiSparseTensor *Y, ptiSparseTensor *const X, ptiMatrix *const U, ptiIndex mode)
{
    PTI_CHECK(U, PTIERR_VALUE_ERROR, "CPU  SpTns * Mtx", "null matrix");
    return pti::host_ttm(Y, X, U->values, U->nrows, U->ncols, U->stride, mode, false, "CPU  SpTns * Mtx");
}
int ptiOmpSparseTensorMulMatrix(ptiSemiSparseTensor *Y, ptiSparseTensor *const X, ptiMatrix *const U, ptiIndex mode)
{
    PTI_CHECK(U, PTIERR_VALUE_ERROR, "OMP  SpTns * Mtx", "null matrix");
    return pti::host_ttm(Y, X, U->values, U->nrows, U->ncols, U->stride, mode, false, "OMP  SpTns * Mtx");
}
int ptiCudaSparseTensorMulMatrix(ptiSemiSparseTensor *Y, ptiSparseTensor *X, const ptiMatrix *U, ptiIndex const mode)
{
    PTI_CHECK(U, PTIERR_VALUE_ERROR, "CUDA SpTns * Mtx", "null matrix");
    return pti::host_ttm(Y, X, U->values, U->nrows, U->ncols, U->stride, mode, false, "CUDA SpTns * Mtx");
}
int ptiCudaSparseTensorMulMatrixOneKernel(ptiSemiSparseTensor *Y, ptiSparseTensor *X, const ptiMatrix *U,
                                          ptiIndex const mode, ptiIndex const impl_num, ptiNnzIndex const smen_size)
{
    (void)impl_num;
    (void)smen_size;
    PTI_CHECK(U, PTIERR_VALUE_ERROR, "CUDA SpTns * Mtx", "null matrix");
    return pti::host_ttm(Y, X, U->values, U->nrows, U->ncols, U->stride, mode, false, "CUDA SpTns * Mtx");
}
int ptiSparseTensorMulVector(ptiSemiSparseTensor *Y, ptiSparseTensor *const X, ptiValueVector *const V,
                             ptiIndex mode)
{
    PTI_CHECK(V, PTIERR_VALUE_ERROR, "CPU  SpTns * Vec", "null vector");
    return pti::host_ttm(Y, X, V->data, (uint32_t)V->len, 0, 1, mode, true, "CPU  SpTns * Vec");
}

int ptiB200TTMFibers(ptiB200Tensor *t, ptiIndex mode, ptiNnzIndex *nfibers, ptiIndex * const *dev_fiber_inds,
                     void *stream)
{
    using namespace pti;
    const char *mod = "B200 TTM";
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    PTI_CHECK(t && mode < t->nmodes, PTIERR_VALUE_ERROR, mod, "bad tensor or mode");
    if (!t->fiber_plan[mode].ready) PTI_TRY(fiber_plan(t, mode, true, s));
    const FiberPlan &P = t->fiber_plan[mode];
    if (nfibers) *nfibers = P.nfib;
    if (dev_fiber_inds)
        for (uint32_t m = 0; m < t->nmodes; ++m)
            if (m != mode && dev_fiber_inds[m] && P.nfib)
                PTI_CUDA(cudaMemcpyAsync(dev_fiber_inds[m], P.finds[m].ptr, P.nfib * 4, cudaMemcpyDeviceToDevice, s),
                         mod);
    return 0;
}

int ptiB200TTM(ptiB200Tensor *t, ptiIndex mode, const float *dev_U, ptiIndex rank, ptiIndex ldu, float *dev_Y,
               ptiIndex ldy, void *stream)
{
    using namespace pti;
    const char *mod = "B200 TTM";
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    PTI_CHECK(t && mode < t->nmodes && dev_U && dev_Y, PTIERR_VALUE_ERROR, mod, "null argument or bad mode");
    if (!t->fiber_plan[mode].ready) PTI_TRY(fiber_plan(t, mode, true, s));
    return ttm_device(t, mode, dev_U, rank, ldu, dev_Y, ldy, rank == 0, s);
}

}  // extern "C"
