// mttkrp.cu -- sparse MTTKRP on sm_100a for COO and HiCOO tensors.
//
// Math (src/sptensor/mttkrp.c:39-163, src/sptensor/hicoo/mttkrp.c:61-310):
//   out[i_mode, r] = sum_z v_z * prod_{k=1..N-1} A_{order[k]}[i_{order[k]}, r]
// Products are taken left to right in mats_order order, as in the reference.
//
// Thread mapping: a group of G lanes owns one nonzero; each lane owns 4
// consecutive rank columns (one 16-byte factor load per operand and one
// 16-byte vector atomic per output quad).  G = R/4 rounded up to a power of
// two, at most 32 (more columns loop).
#include "kutil.cuh"
#include "tensor.cuh"

#include <mutex>

namespace pti {

constexpr int kThreads = 256;
constexpr int kHiTile = 1024;  // nonzeros per HiCOO tile (one CTA)

struct CooArgs {
    uint64_t nnz;
    uint32_t nin;  // N-1 operand modes
    uint32_t R, stride;
    const uint32_t *out_ind;
    const uint32_t *in_ind[kMaxModes - 1];
    const void *in_mat[kMaxModes - 1];
    const float *vals;
    float *out;
};

template <int G, class FT>
__global__ void __launch_bounds__(kThreads) coo_atomic_kernel(CooArgs a)
{
    const uint32_t lane = threadIdx.x % G;
    const uint64_t ngroups = ((uint64_t)gridDim.x * kThreads) / G;
    for (uint64_t z = ((uint64_t)blockIdx.x * kThreads + threadIdx.x) / G; z < a.nnz; z += ngroups) {
        const float v = __ldg(a.vals + z);
        const uint32_t orow = __ldg(a.out_ind + z);
        uint32_t rows[kMaxModes - 1];
#pragma unroll
        for (int i = 0; i < kMaxModes - 1; ++i)
            if (i < (int)a.nin) rows[i] = __ldg(a.in_ind[i] + z);
        for (uint32_t col = lane * 4; col < a.R; col += 4 * G) {
            float4 p = scale4(load4(static_cast<const FT *>(a.in_mat[0]) + (size_t)rows[0] * a.stride, col), v);
#pragma unroll
            for (int i = 1; i < kMaxModes - 1; ++i)
                if (i < (int)a.nin)
                    p = mul4(p, load4(static_cast<const FT *>(a.in_mat[i]) + (size_t)rows[i] * a.stride, col));
            red_add4(a.out + (size_t)orow * a.stride + col, mask4(p, col, a.R));
        }
    }
}

struct HicooArgs {
    uint64_t nnz, nb;
    uint32_t nin;
    uint32_t R, stride;
    uint32_t sb;
    const uint64_t *bptr;
    const uint32_t *tile_block;
    const uint32_t *out_bind;
    const uint8_t *out_eind;
    uint32_t out_dim;
    const uint32_t *in_bind[kMaxModes - 1];
    const uint8_t *in_eind[kMaxModes - 1];
    uint32_t in_dim[kMaxModes - 1];
    const void *in_mat[kMaxModes - 1];
    const float *vals;
    float *out;
    uint32_t *err;
};

// First block of every nonzero tile: tile t starts at nonzero t*kHiTile, which
// lies in exactly one non-empty block b (bptr[b] <= t*kHiTile < bptr[b+1]).
__global__ void tile_block_kernel(const uint64_t *bptr, uint64_t nb, uint32_t ntiles,
                                  uint32_t *tile_block)
{
    uint64_t b = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    uint64_t zs = bptr[b], ze = bptr[b + 1];
    for (uint64_t t = (zs + kHiTile - 1) / kHiTile; t * kHiTile < ze && t < ntiles; ++t)
        tile_block[t] = (uint32_t)b;
    if (b == nb - 1) tile_block[ntiles] = (uint32_t)b;
}

// One CTA per tile of kHiTile nonzeros.  The tile's block coordinates are
// staged in shared memory pre-shifted by sb, each nonzero is tagged with its
// tile-local block, and groups of G lanes then decode the 8-bit element
// offsets, gather the operand rows and add into the output rows.
template <int G, class FT>
__global__ void __launch_bounds__(kThreads) hicoo_tile_kernel(HicooArgs a)
{
    extern __shared__ uint32_t smem[];
    uint32_t *s_out = smem;                            // [kHiTile + 1]
    uint32_t *s_in = smem + (kHiTile + 1);             // [nin][kHiTile + 1]
    uint16_t *s_blk = reinterpret_cast<uint16_t *>(s_in + a.nin * (kHiTile + 1));  // [kHiTile]

    const uint64_t z0 = (uint64_t)blockIdx.x * kHiTile;
    const uint64_t z1 = min(z0 + kHiTile, a.nnz);
    const uint32_t b0 = a.tile_block[blockIdx.x];
    if (b0 >= a.nb) {  // only a malformed bptr leaves a tile without a block
        if (threadIdx.x == 0) atomicOr(a.err, 1u);
        return;
    }
    uint32_t nblk = a.tile_block[blockIdx.x + 1] - b0 + 1;
    if (nblk > kHiTile + 1) nblk = kHiTile + 1;
    if (b0 + (uint64_t)nblk > a.nb) nblk = (uint32_t)(a.nb - b0);

    for (uint32_t z = threadIdx.x; z < kHiTile; z += kThreads) s_blk[z] = 0;
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < nblk; i += kThreads) {
        const uint64_t b = b0 + i;
        s_out[i] = __ldg(a.out_bind + b) << a.sb;
#pragma unroll
        for (int k = 0; k < kMaxModes - 1; ++k)
            if (k < (int)a.nin) s_in[k * (kHiTile + 1) + i] = __ldg(a.in_bind[k] + b) << a.sb;
        const uint64_t zs = max(__ldg(a.bptr + b), z0), ze = min(__ldg(a.bptr + b + 1), z1);
        for (uint64_t z = zs; z < ze; ++z) s_blk[z - z0] = (uint16_t)i;
    }
    __syncthreads();

    const uint32_t lane = threadIdx.x % G;
    constexpr int kGroups = kThreads / G;
    for (uint64_t z = z0 + threadIdx.x / G; z < z1; z += kGroups) {
        const uint32_t i = s_blk[z - z0];
        const uint32_t orow = s_out[i] + __ldg(a.out_eind + z);
        uint32_t rows[kMaxModes - 1];
        bool ok = orow < a.out_dim;
#pragma unroll
        for (int k = 0; k < kMaxModes - 1; ++k)
            if (k < (int)a.nin) {
                rows[k] = s_in[k * (kHiTile + 1) + i] + __ldg(a.in_eind[k] + z);
                ok = ok && rows[k] < a.in_dim[k];
            }
        if (!ok) {
            if (lane == 0) atomicOr(a.err, 1u);
            continue;
        }
        const float v = __ldg(a.vals + z);
        for (uint32_t col = lane * 4; col < a.R; col += 4 * G) {
            float4 p = scale4(load4(static_cast<const FT *>(a.in_mat[0]) + (size_t)rows[0] * a.stride, col), v);
#pragma unroll
            for (int k = 1; k < kMaxModes - 1; ++k)
                if (k < (int)a.nin)
                    p = mul4(p, load4(static_cast<const FT *>(a.in_mat[k]) + (size_t)rows[k] * a.stride, col));
            red_add4(a.out + (size_t)orow * a.stride + col, mask4(p, col, a.R));
        }
    }
}

// Checks every COO index against its mode size; sets err on violation.
__global__ void check_coo_kernel(const uint32_t *ind, uint64_t nnz, uint32_t dim, uint32_t *err)
{
    for (uint64_t z = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; z < nnz;
         z += (uint64_t)gridDim.x * blockDim.x)
        if (ind[z] >= dim) atomicOr(err, 1u);
}

// bptr must start at 0, end at nnz and increase strictly (no empty blocks:
// the kernels size their per-tile block tables by that).
__global__ void check_bptr_kernel(const uint64_t *bptr, uint64_t nb, uint64_t nnz, uint32_t *err)
{
    for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; b <= nb;
         b += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t v = bptr[b];
        if ((b == 0 && v != 0) || (b == nb && v != nnz) || (b < nb && bptr[b + 1] <= v) || v > nnz)
            atomicOr(err, 1u);
    }
}

namespace {

int group_lanes(uint32_t R)
{
    uint32_t q = (R + 3) / 4;
    int g = 1;
    while ((uint32_t)g < q && g < 32) g *= 2;
    return g;
}

unsigned grid_for(uint64_t items, int per_cta)
{
    uint64_t want = (items + per_cta - 1) / per_cta;
    uint64_t cap = (uint64_t)sm_count() * 16;
    if (want > cap) want = cap;
    return (unsigned)(want ? want : 1);
}

template <class FT>
void launch_coo(const CooArgs &a, int G, cudaStream_t s)
{
    unsigned grid = grid_for(a.nnz, kThreads / G);
    switch (G) {
        case 1: coo_atomic_kernel<1, FT><<<grid, kThreads, 0, s>>>(a); break;
        case 2: coo_atomic_kernel<2, FT><<<grid, kThreads, 0, s>>>(a); break;
        case 4: coo_atomic_kernel<4, FT><<<grid, kThreads, 0, s>>>(a); break;
        case 8: coo_atomic_kernel<8, FT><<<grid, kThreads, 0, s>>>(a); break;
        case 16: coo_atomic_kernel<16, FT><<<grid, kThreads, 0, s>>>(a); break;
        default: coo_atomic_kernel<32, FT><<<grid, kThreads, 0, s>>>(a); break;
    }
}

template <class FT>
void launch_hicoo(const HicooArgs &a, int G, unsigned ntiles, cudaStream_t s)
{
    size_t smem = (size_t)(kHiTile + 1) * 4 * (1 + a.nin) + kHiTile * 2;
    switch (G) {
        case 1: hicoo_tile_kernel<1, FT><<<ntiles, kThreads, smem, s>>>(a); break;
        case 2: hicoo_tile_kernel<2, FT><<<ntiles, kThreads, smem, s>>>(a); break;
        case 4: hicoo_tile_kernel<4, FT><<<ntiles, kThreads, smem, s>>>(a); break;
        case 8: hicoo_tile_kernel<8, FT><<<ntiles, kThreads, smem, s>>>(a); break;
        case 16: hicoo_tile_kernel<16, FT><<<ntiles, kThreads, smem, s>>>(a); break;
        default: hicoo_tile_kernel<32, FT><<<ntiles, kThreads, smem, s>>>(a); break;
    }
}

}  // namespace

int ensure_err_word(ptiB200Tensor *t, cudaStream_t s);
uint32_t *err_word(ptiB200Tensor *t);
int mttkrp_scheduled(ptiB200Tensor *t, const void *const *mats, int ft, uint32_t R, uint32_t stride,
                     const uint32_t *mats_order, uint32_t mode, float *out, cudaStream_t s,
                     const float *vals_override);
bool schedule_supported(const ptiB200Tensor *t, uint32_t R, uint32_t stride);

// The output-privatised kernels (sched.cu) cover orders 2-4, R <= 128 and
// (HiCOO) factors of fewer than 2^32 elements; HIPARTI_B200_SCHEDULE=0 selects
// the direct-atomic kernels instead.
static bool use_schedule(const ptiB200Tensor *t, uint32_t R, uint32_t stride)
{
    static int env = -1;
    if (env < 0) {
        const char *e = std::getenv("HIPARTI_B200_SCHEDULE");
        env = (e && e[0] == '0') ? 0 : 1;
    }
    return env == 1 && schedule_supported(t, R, stride);
}

int mttkrp_device(ptiB200Tensor *t, const void *const *mats, int ft, uint32_t R, uint32_t stride,
                  const uint32_t *mats_order, uint32_t mode, float *out, cudaStream_t s, const float *vals_override,
                  const Arrivals *arr)
{
    const char *mod = "B200 MTTKRP";
    const uint32_t N = t->nmodes;
    PTI_CHECK(N >= 2 && N <= (uint32_t)kMaxModes, PTIERR_VALUE_ERROR, mod, "unsupported number of modes");
    PTI_CHECK(mode < N, PTIERR_VALUE_ERROR, mod, "mode out of range");
    PTI_CHECK(ft == PTI_B200_F32 || ft == PTI_B200_BF16, PTIERR_VALUE_ERROR, mod, "bad factor type");
    PTI_CHECK(R >= 1 && stride >= R && stride % 4 == 0, PTIERR_SHAPE_MISMATCH, mod,
              "stride must be >= rank and a multiple of 4");
    PTI_CHECK(((uintptr_t)out & 15) == 0, PTIERR_VALUE_ERROR, mod, "output must be 16-byte aligned");
    // mats_order must be a permutation whose first entry is `mode`.
    uint32_t seen = 0;
    for (uint32_t i = 0; i < N; ++i) {
        PTI_CHECK(mats_order[i] < N && !(seen >> mats_order[i] & 1u), PTIERR_VALUE_ERROR, mod,
                  "mats_order must be a permutation of the modes");
        seen |= 1u << mats_order[i];
    }
    PTI_CHECK(mats_order[0] == mode, PTIERR_VALUE_ERROR, mod, "mats_order[0] must equal mode");
    PTI_CHECK(!vals_override || !t->hicoo, PTIERR_VALUE_ERROR, mod, "substituted values need a COO tensor");
    const size_t esz = ft == PTI_B200_F32 ? 4 : 2;
    for (uint32_t i = 1; i < N; ++i) {
        PTI_CHECK(mats[mats_order[i]], PTIERR_VALUE_ERROR, mod, "null factor");
        PTI_CHECK(((uintptr_t)mats[mats_order[i]] & (4 * esz - 1)) == 0, PTIERR_VALUE_ERROR, mod,
                  "factors must be aligned to 4 elements");
    }
    PTI_CUDA(cudaMemsetAsync(out, 0, (size_t)t->ndims[mode] * stride * sizeof(float), s), mod);
    if (t->nnz == 0) return 0;
    const int G = group_lanes(R);
    if (use_schedule(t, R, stride)) {
        PTI_TRY(prepare_mode(t, mode, s, arr));
        if (arr && arr->all) PTI_CUDA(cudaStreamWaitEvent(s, arr->all, 0), mod);
        return mttkrp_scheduled(t, mats, ft, R, stride, mats_order, mode, out, s, vals_override);
    }
    if (arr && arr->all) PTI_CUDA(cudaStreamWaitEvent(s, arr->all, 0), mod);

    if (!t->hicoo) {
        CooArgs a{};
        a.nnz = t->nnz;
        a.nin = N - 1;
        a.R = R;
        a.stride = stride;
        a.out_ind = t->inds[mode].as<uint32_t>();
        for (uint32_t i = 1; i < N; ++i) {
            a.in_ind[i - 1] = t->inds[mats_order[i]].as<uint32_t>();
            a.in_mat[i - 1] = mats[mats_order[i]];
        }
        a.vals = vals_override ? vals_override : t->vals.as<float>();
        a.out = out;
        if (ft == PTI_B200_F32) launch_coo<float>(a, G, s);
        else launch_coo<__nv_bfloat16>(a, G, s);
        PTI_CUDA(cudaGetLastError(), mod);
        return 0;
    }

    PTI_TRY(ensure_err_word(t, s));
    HicooArgs a{};
    a.nnz = t->nnz;
    a.nb = t->nb;
    a.nin = N - 1;
    a.R = R;
    a.stride = stride;
    a.sb = t->sb;
    a.bptr = t->bptr.as<uint64_t>();
    a.tile_block = t->tile_block.as<uint32_t>();
    a.out_bind = t->binds[mode].as<uint32_t>();
    a.out_eind = t->einds[mode].as<uint8_t>();
    a.out_dim = t->ndims[mode];
    for (uint32_t i = 1; i < N; ++i) {
        uint32_t k = mats_order[i];
        a.in_bind[i - 1] = t->binds[k].as<uint32_t>();
        a.in_eind[i - 1] = t->einds[k].as<uint8_t>();
        a.in_dim[i - 1] = t->ndims[k];
        a.in_mat[i - 1] = mats[k];
    }
    a.vals = t->vals.as<float>();
    a.out = out;
    a.err = err_word(t);
    if (ft == PTI_B200_F32) launch_hicoo<float>(a, G, t->ntiles, s);
    else launch_hicoo<__nv_bfloat16>(a, G, t->ntiles, s);
    PTI_CUDA(cudaGetLastError(), mod);
    return 0;
}

// ----------------------------------------------------------------------------
// Device error word of a tensor: set by kernels that meet an out-of-range
// coordinate or give up a bounded wait.  One word per tensor handle, so calls
// on different tensors (different streams or host threads) do not see each
// other's errors.
// ----------------------------------------------------------------------------
int ensure_err_word(ptiB200Tensor *t, cudaStream_t s)
{
    if (!t->err.ptr) {
        PTI_CUDA(t->err.alloc(padded(sizeof(uint32_t)), s), "B200 err");
        PTI_CUDA(cudaMemsetAsync(t->err.ptr, 0, sizeof(uint32_t), s), "B200 err");
    }
    return 0;
}

uint32_t *err_word(ptiB200Tensor *t) { return t->err.as<uint32_t>(); }

// Reads and clears the tensor's device error word (synchronises `s`).
int take_device_error(ptiB200Tensor *t, cudaStream_t s, const char *mod)
{
    uint32_t *w = err_word(t);
    if (!w) return 0;
    uint32_t h = 0;
    PTI_CUDA(cudaMemcpyAsync(&h, w, sizeof h, cudaMemcpyDeviceToHost, s), mod);
    PTI_CUDA(cudaMemsetAsync(w, 0, sizeof h, s), mod);
    PTI_CUDA(cudaStreamSynchronize(s), mod);
    PTI_CHECK(!(h & 2u), PTIERR_CUDA_ERROR, mod, "a bulk copy did not complete within its wait limit");
    PTI_CHECK(h == 0, PTIERR_VALUE_ERROR, mod, "tensor coordinate out of range");
    return 0;
}

// ----------------------------------------------------------------------------
// Upload
// ----------------------------------------------------------------------------
int upload_coo(ptiB200Tensor *t, const ptiSparseTensor *X, cudaStream_t s)
{
    const char *mod = "B200 Upload";
    PTI_CHECK(X && X->nmodes >= 2 && X->nmodes <= (uint32_t)kMaxModes, PTIERR_VALUE_ERROR, mod,
              "unsupported number of modes");
    configure_pool_once();
    cudaGetDevice(&t->device);
    t->hicoo = false;
    t->nmodes = X->nmodes;
    t->ndims.assign(X->ndims, X->ndims + X->nmodes);
    t->nnz = X->nnz;
    for (uint32_t m = 0; m < X->nmodes; ++m) {
        PTI_CUDA(t->inds[m].alloc(padded(t->nnz * 4), s), mod);
        if (t->nnz)
            PTI_CUDA(cudaMemcpyAsync(t->inds[m].ptr, X->inds[m].data, t->nnz * 4, cudaMemcpyHostToDevice, s), mod);
    }
    PTI_CUDA(t->vals.alloc(padded(t->nnz * 4), s), mod);
    if (t->nnz)
        PTI_CUDA(cudaMemcpyAsync(t->vals.ptr, X->values.data, t->nnz * 4, cudaMemcpyHostToDevice, s), mod);
    return check_coo_ranges(t, s);
}

int check_coo_ranges(ptiB200Tensor *t, cudaStream_t s)
{
    const char *mod = "B200 Upload";
    PTI_TRY(ensure_err_word(t, s));
    if (t->nnz) {
        for (uint32_t m = 0; m < t->nmodes; ++m)
            check_coo_kernel<<<grid_for(t->nnz, 256), 256, 0, s>>>(t->inds[m].as<uint32_t>(), t->nnz,
                                                                   t->ndims[m], err_word(t));
        PTI_CUDA(cudaGetLastError(), mod);
        PTI_TRY(take_device_error(t, s, mod));
    }
    return 0;
}

// Checks every index of a device COO tensor against the mode sizes.
int validate_coo(ptiB200Tensor *t, cudaStream_t s)
{
    const char *mod = "B200 Upload";
    PTI_TRY(ensure_err_word(t, s));
    if (t->nnz) {
        for (uint32_t m = 0; m < t->nmodes; ++m)
            check_coo_kernel<<<grid_for(t->nnz, 256), 256, 0, s>>>(t->inds[m].as<uint32_t>(), t->nnz,
                                                                   t->ndims[m], err_word(t));
        PTI_CUDA(cudaGetLastError(), mod);
        PTI_TRY(take_device_error(t, s, mod));
    }
    return 0;
}

int finish_hicoo_layout(ptiB200Tensor *t, cudaStream_t s)
{
    const char *mod = "B200 Upload";
    t->ntiles = (uint32_t)((t->nnz + kHiTile - 1) / kHiTile);
    PTI_CUDA(t->tile_block.alloc(padded(((size_t)t->ntiles + 1) * 4), s), mod);
    if (t->nb) {
        tile_block_kernel<<<ceil_div(t->nb, 256), 256, 0, s>>>(t->bptr.as<uint64_t>(), t->nb, t->ntiles,
                                                               t->tile_block.as<uint32_t>());
        PTI_CUDA(cudaGetLastError(), mod);
    }
    return 0;
}

int upload_hicoo(ptiB200Tensor *t, const ptiSparseTensorHiCOO *H, cudaStream_t s, int first_mode, cudaStream_t s2,
                 Arrivals *arr)
{
    const char *mod = "B200 Upload";
    PTI_CHECK(H && H->nmodes >= 2 && H->nmodes <= (uint32_t)kMaxModes, PTIERR_VALUE_ERROR, mod,
              "unsupported number of modes");
    PTI_CHECK(H->sb_bits <= 8, PTIERR_VALUE_ERROR, mod, "sb_bits must be <= 8");
    configure_pool_once();
    cudaGetDevice(&t->device);
    t->hicoo = true;
    t->nmodes = H->nmodes;
    t->ndims.assign(H->ndims, H->ndims + H->nmodes);
    t->nnz = H->nnz;
    t->sb = H->sb_bits;
    t->sk = H->sk_bits;
    t->sc = H->sc_bits;
    t->nb = H->bptr.len ? H->bptr.len - 1 : 0;
    PTI_CHECK(t->nnz == 0 || t->nb > 0, PTIERR_VALUE_ERROR, mod, "HiCOO tensor has nonzeros but no blocks");
    PTI_CHECK(H->values.len >= t->nnz, PTIERR_SHAPE_MISMATCH, mod, "values shorter than nnz");
    PTI_CHECK(t->nb < 0xFFFFFFFFull, PTIERR_VALUE_ERROR, mod, "too many blocks");
    for (uint32_t m = 0; m < H->nmodes; ++m)
        PTI_CHECK(H->binds[m].len >= t->nb && H->einds[m].len >= t->nnz, PTIERR_SHAPE_MISMATCH, mod,
                  "binds/einds shorter than nb/nnz");
    PTI_CUDA(t->bptr.alloc(padded((t->nb + 1) * 8), s), mod);
    for (uint32_t m = 0; m < H->nmodes; ++m) {
        PTI_CUDA(t->binds[m].alloc(padded(t->nb * 4), s), mod);
        PTI_CUDA(t->einds[m].alloc(padded(t->nnz), s), mod);
    }
    PTI_CUDA(t->vals.alloc(padded(t->nnz * 4), s), mod);
    auto copy_mode = [&](uint32_t m, cudaStream_t cs) -> int {
        if (t->nb)
            PTI_CUDA(cudaMemcpyAsync(t->binds[m].ptr, H->binds[m].data, t->nb * 4, cudaMemcpyHostToDevice, cs), mod);
        if (t->nnz)
            PTI_CUDA(cudaMemcpyAsync(t->einds[m].ptr, H->einds[m].data, t->nnz, cudaMemcpyHostToDevice, cs), mod);
        return 0;
    };
    PTI_CUDA(cudaMemcpyAsync(t->bptr.ptr, H->bptr.data, (t->nb + 1) * 8, cudaMemcpyHostToDevice, s), mod);
    if (s2) {
        // The arrays the schedule starts from go first, alone on the host
        // link; the rest starts on s2 when they have landed (and the buffers'
        // stream-ordered allocations are done), so it overlaps the schedule
        // build instead of slowing down its inputs.
        if (first_mode >= 0) PTI_TRY(copy_mode((uint32_t)first_mode, s));
        cudaEvent_t ev;
        PTI_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), mod);
        cudaEventRecord(ev, s);
        cudaStreamWaitEvent(s2, ev, 0);
        cudaEventDestroy(ev);
        if (t->nnz)
            PTI_CUDA(cudaMemcpyAsync(t->vals.ptr, H->values.data, t->nnz * 4, cudaMemcpyHostToDevice, s2), mod);
        if (arr && arr->vals) PTI_CUDA(cudaEventRecord(arr->vals, s2), mod);
        for (uint32_t m = 0; m < H->nmodes; ++m)
            if ((int)m != first_mode) {
                PTI_TRY(copy_mode(m, s2));
                if (arr && arr->mode[m]) PTI_CUDA(cudaEventRecord(arr->mode[m], s2), mod);
            }
        if (arr && arr->all) PTI_CUDA(cudaEventRecord(arr->all, s2), mod);
    } else {
        for (uint32_t m = 0; m < H->nmodes; ++m) PTI_TRY(copy_mode(m, s));
        if (t->nnz)
            PTI_CUDA(cudaMemcpyAsync(t->vals.ptr, H->values.data, t->nnz * 4, cudaMemcpyHostToDevice, s), mod);
    }
    PTI_TRY(ensure_err_word(t, s));
    if (t->nb) {
        check_bptr_kernel<<<grid_for(t->nb + 1, 256), 256, 0, s>>>(t->bptr.as<uint64_t>(), t->nb, t->nnz,
                                                                   err_word(t));
        PTI_CUDA(cudaGetLastError(), mod);
        PTI_TRY(take_device_error(t, s, mod));
    }
    return finish_hicoo_layout(t, s);
}

// ----------------------------------------------------------------------------
// Host-struct MTTKRP (the reference entry points)
// ----------------------------------------------------------------------------
namespace {

int check_mats(uint32_t N, const uint32_t *ndims, ptiMatrix **mats, const char *mod)
{
    PTI_CHECK(mats, PTIERR_VALUE_ERROR, mod, "null mats");
    for (uint32_t i = 0; i <= N; ++i) PTI_CHECK(mats[i], PTIERR_VALUE_ERROR, mod, "null matrix");
    // src/sptensor/mttkrp.c:58-65
    for (uint32_t i = 0; i < N; ++i) {
        if (mats[i]->ncols != mats[N]->ncols)
            PTI_FAIL(PTIERR_SHAPE_MISMATCH, mod, "mats[i]->cols != mats[nmodes]->ncols");
        if (mats[i]->nrows != ndims[i])
            PTI_FAIL(PTIERR_SHAPE_MISMATCH, mod, "mats[i]->nrows != ndims[i]");
        if (mats[i]->stride != mats[0]->stride)
            PTI_FAIL(PTIERR_SHAPE_MISMATCH, mod, "factor strides differ");
    }
    return 0;
}

// With s2 and arr (the tensor's remaining arrays being copied on s2), the
// factors are copied on s2 behind them and arr->all is recorded again after
// them: the schedule build on s does not wait for the factors, the kernel does.
int run_host(ptiB200Tensor *t, ptiMatrix **mats, const ptiIndex *mats_order, ptiIndex mode,
             cudaStream_t s, const char *mod, Arrivals *arr = nullptr, cudaStream_t s2 = nullptr)
{
    const uint32_t N = t->nmodes;
    const uint32_t R = mats[mode]->ncols, stride = mats[0]->stride;
    PTI_CHECK(mats[N]->cap >= t->ndims[mode], PTIERR_SHAPE_MISMATCH, mod, "mats[nmodes] has too few rows");
    DevBuf dm[kMaxModes], dout;
    const void *ptrs[kMaxModes] = {nullptr};
    const cudaStream_t fs = s2 && arr && arr->all ? s2 : s;
    for (uint32_t k = 0; k < N; ++k) {
        if (k == mode) continue;
        size_t bytes = (size_t)t->ndims[k] * stride * 4;
        PTI_CUDA(dm[k].alloc(padded(bytes), fs), mod);
        PTI_CUDA(cudaMemcpyAsync(dm[k].ptr, mats[k]->values, bytes, cudaMemcpyHostToDevice, fs), mod);
        ptrs[k] = dm[k].ptr;
    }
    if (fs != s) PTI_CUDA(cudaEventRecord(arr->all, s2), mod);
    size_t obytes = (size_t)t->ndims[mode] * stride * 4;
    PTI_CUDA(dout.alloc(padded(obytes), s), mod);
    PTI_TRY(mttkrp_device(t, ptrs, PTI_B200_F32, R, stride, mats_order, mode, dout.as<float>(), s, nullptr, arr));
    PTI_CUDA(cudaMemcpyAsync(mats[N]->values, dout.ptr, obytes, cudaMemcpyDeviceToHost, s), mod);
    PTI_TRY(take_device_error(t, s, mod));
    return 0;
}

}  // namespace

int mttkrp_host_coo(const ptiSparseTensor *X, ptiMatrix **mats, const ptiIndex *mats_order, ptiIndex mode)
{
    const char *mod = "B200 SpTns MTTKRP";
    PTI_CHECK(X && mode < X->nmodes, PTIERR_VALUE_ERROR, mod, "bad tensor or mode");
    PTI_TRY(check_mats(X->nmodes, X->ndims, mats, mod));
    cudaStream_t s = sync_stream();
    ptiB200Tensor t;
    PTI_TRY(upload_coo(&t, X, s));
    return run_host(&t, mats, mats_order, mode, s, mod);
}

int mttkrp_host_hicoo(const ptiSparseTensorHiCOO *H, ptiMatrix **mats, const ptiIndex *mats_order, ptiIndex mode)
{
    const char *mod = "B200 HiSpTns MTTKRP";
    PTI_CHECK(H && mode < H->nmodes, PTIERR_VALUE_ERROR, mod, "bad tensor or mode");
    PTI_TRY(check_mats(H->nmodes, H->ndims, mats, mod));
    // The arrays mode `mode`'s schedule starts from (block pointers, the
    // mode's coordinates and offsets) are copied first on s; the rest follows
    // on a second stream while the schedule is being built.
    cudaStream_t s = sync_stream(), s2 = copy_stream();
    Arrivals arr;
    int r = 0;
    auto make = [&](cudaEvent_t *ev) {
        if (r == 0 && cudaEventCreateWithFlags(ev, cudaEventDisableTiming) != cudaSuccess) r = PTIERR_CUDA_ERROR;
    };
    make(&arr.all);
    make(&arr.vals);
    for (uint32_t m = 0; m < H->nmodes && m < (uint32_t)kMaxModes; ++m)
        if (m != mode) make(&arr.mode[m]);
    PTI_CHECK(r == 0, r, mod, "event creation failed");
    {
        ptiB200Tensor t;
        r = upload_hicoo(&t, H, s, (int)mode, s2, &arr);
        if (r == 0) r = run_host(&t, mats, mats_order, mode, s, mod, &arr, s2);
        cudaStreamWaitEvent(s, arr.all, 0);  // the tensor is released on s only after the second stream's copies
    }
    cudaEventDestroy(arr.all);
    cudaEventDestroy(arr.vals);
    for (uint32_t m = 0; m < (uint32_t)kMaxModes; ++m)
        if (arr.mode[m]) cudaEventDestroy(arr.mode[m]);
    return r;
}

}  // namespace pti

extern "C" {

int ptiMTTKRP(ptiSparseTensor const *const X, ptiMatrix *mats[], ptiIndex const mats_order[], ptiIndex const mode)
{
    return pti::mttkrp_host_coo(X, mats, mats_order, mode);
}
int ptiOmpMTTKRP(ptiSparseTensor const *const X, ptiMatrix *mats[], ptiIndex const mats_order[],
                 ptiIndex const mode, const int tk)
{
    (void)tk;
    return pti::mttkrp_host_coo(X, mats, mats_order, mode);
}
int ptiOmpMTTKRP_Reduce(ptiSparseTensor const *const X, ptiMatrix *mats[], ptiMatrix *copy_mats[],
                        ptiIndex const mats_order[], ptiIndex const mode, const int tk)
{
    (void)copy_mats;
    (void)tk;
    return pti::mttkrp_host_coo(X, mats, mats_order, mode);
}
struct ptiMutexPool {
    uint32_t nlocks, padsize;  // recorded only: the GPU path takes no locks
};
ptiMutexPool *SptMutexAllocCustom(ptiIndex const num_locks, ptiIndex const pad_size)
{
    auto *p = static_cast<ptiMutexPool *>(std::malloc(sizeof(ptiMutexPool)));
    if (p) {
        p->nlocks = num_locks;
        p->padsize = pad_size;
    }
    return p;
}
ptiMutexPool *ptiMutexAlloc(void) { return SptMutexAllocCustom(1024, 16); }
void ptiMutexFree(ptiMutexPool *pool) { std::free(pool); }

int ptiOmpMTTKRP_Lock(ptiSparseTensor const *const X, ptiMatrix *mats[], ptiIndex const mats_order[],
                      ptiIndex const mode, const int tk, ptiMutexPool *lock_pool)
{
    (void)tk;
    (void)lock_pool;
    return pti::mttkrp_host_coo(X, mats, mats_order, mode);
}

int ptiCudaMTTKRP(ptiSparseTensor const *const X, ptiMatrix *mats[], ptiIndex *const mats_order,
                  ptiIndex const mode, ptiIndex const impl_num)
{
    (void)impl_num;
    return pti::mttkrp_host_coo(X, mats, mats_order, mode);
}
int ptiCudaMTTKRPOneKernel(ptiSparseTensor const *const X, ptiMatrix **const mats, ptiIndex *const mats_order,
                           ptiIndex const mode, ptiIndex const impl_num)
{
    (void)impl_num;
    return pti::mttkrp_host_coo(X, mats, mats_order, mode);
}
int ptiCudaMTTKRPDevice(const ptiIndex mode, const ptiIndex nmodes, const ptiNnzIndex nnz, const ptiIndex rank,
                        const ptiIndex stride, const ptiIndex *Xndims, ptiIndex **const Xinds, const ptiValue *Xvals,
                        const ptiIndex *dev_mats_order, ptiValue **dev_mats, ptiValue *dev_scratch)
{
    using namespace pti;
    (void)Xndims;
    (void)dev_scratch;
    const char *mod = "CUDA SpTns MTTKRP (device)";
    PTI_CHECK(nmodes >= 2 && nmodes <= (uint32_t)kMaxModes && mode < nmodes, PTIERR_VALUE_ERROR, mod,
              "unsupported number of modes or mode out of range");
    PTI_CHECK(rank >= 1 && stride >= rank && stride % 4 == 0, PTIERR_SHAPE_MISMATCH, mod,
              "stride must be >= rank and a multiple of 4");
    if (nnz == 0) return 0;
    PTI_CHECK(Xinds && Xvals && dev_mats_order && dev_mats, PTIERR_VALUE_ERROR, mod, "null device array");
    // the pointer arrays and the mode order live in device memory, as the
    // reference's kernel reads them there (mttkrp_cuda_kernels.cu:374-427)
    cudaStream_t s = sync_stream();
    std::vector<ptiIndex *> inds(nmodes);
    std::vector<ptiValue *> mats(nmodes + 1);
    std::vector<ptiIndex> order(nmodes);
    PTI_CUDA(cudaMemcpyAsync(inds.data(), Xinds, nmodes * sizeof(ptiIndex *), cudaMemcpyDeviceToHost, s), mod);
    PTI_CUDA(cudaMemcpyAsync(mats.data(), dev_mats, (nmodes + 1) * sizeof(ptiValue *), cudaMemcpyDeviceToHost, s),
             mod);
    PTI_CUDA(cudaMemcpyAsync(order.data(), dev_mats_order, nmodes * sizeof(ptiIndex), cudaMemcpyDeviceToHost, s),
             mod);
    PTI_CUDA(cudaStreamSynchronize(s), mod);
    uint32_t seen = 0;
    for (uint32_t i = 0; i < nmodes; ++i) {
        PTI_CHECK(order[i] < nmodes && !(seen >> order[i] & 1u), PTIERR_VALUE_ERROR, mod,
                  "mats_order must be a permutation of the modes");
        seen |= 1u << order[i];
    }
    PTI_CHECK(order[0] == mode, PTIERR_VALUE_ERROR, mod, "mats_order[0] must equal mode");
    PTI_CHECK(mats[nmodes] && ((uintptr_t)mats[nmodes] & 15) == 0, PTIERR_VALUE_ERROR, mod,
              "output must be non-null and 16-byte aligned");
    CooArgs a{};
    a.nnz = nnz;
    a.nin = nmodes - 1;
    a.R = rank;
    a.stride = stride;
    a.out_ind = inds[mode];
    for (uint32_t i = 1; i < nmodes; ++i) {
        const uint32_t k = order[i];
        PTI_CHECK(inds[k] && mats[k] && ((uintptr_t)mats[k] & 15) == 0, PTIERR_VALUE_ERROR, mod,
                  "factors must be non-null and 16-byte aligned");
        a.in_ind[i - 1] = inds[k];
        a.in_mat[i - 1] = mats[k];
    }
    PTI_CHECK(a.out_ind, PTIERR_VALUE_ERROR, mod, "null index array");
    a.vals = Xvals;
    a.out = mats[nmodes];
    launch_coo<float>(a, group_lanes(rank), s);
    PTI_CUDA(cudaGetLastError(), mod);
    PTI_CUDA(cudaStreamSynchronize(s), mod);
    return 0;
}

int ptiMTTKRPHiCOO(ptiSparseTensorHiCOO const *const hitsr, ptiMatrix *mats[], ptiIndex const mats_order[],
                   ptiIndex const mode)
{
    return pti::mttkrp_host_hicoo(hitsr, mats, mats_order, mode);
}
int ptiOmpMTTKRPHiCOO(ptiSparseTensorHiCOO const *const hitsr, ptiMatrix *mats[], ptiIndex const mats_order[],
                      ptiIndex const mode, const int tk, const int tb)
{
    (void)tk;
    (void)tb;
    return pti::mttkrp_host_hicoo(hitsr, mats, mats_order, mode);
}
// ptiRankMatrix (8-bit ncols and stride) viewed as ptiMatrix for the shared
// MTTKRP path; the values are shared, so the result lands in mats[N] itself.
static int mttkrp_rank_hicoo(ptiSparseTensorHiCOO const *const hitsr, ptiRankMatrix *mats[],
                             ptiIndex const mats_order[], ptiIndex const mode)
{
    const char *mod = "B200 HiSpTns MTTKRP";
    PTI_CHECK(hitsr && mats, PTIERR_VALUE_ERROR, mod, "null argument");
    const uint32_t N = hitsr->nmodes;
    PTI_CHECK(N >= 2 && N <= (uint32_t)pti::kMaxModes, PTIERR_VALUE_ERROR, mod, "unsupported number of modes");
    ptiMatrix views[pti::kMaxModes + 1];
    ptiMatrix *ptrs[pti::kMaxModes + 1];
    for (uint32_t m = 0; m <= N; ++m) {
        PTI_CHECK(mats[m], PTIERR_VALUE_ERROR, mod, "null matrix");
        views[m].nrows = mats[m]->nrows;
        views[m].ncols = mats[m]->ncols;
        views[m].cap = mats[m]->cap;
        views[m].stride = mats[m]->stride;
        views[m].values = mats[m]->values;
        ptrs[m] = &views[m];
    }
    return pti::mttkrp_host_hicoo(hitsr, ptrs, mats_order, mode);
}

int ptiMTTKRPHiCOO_MatrixTiling(ptiSparseTensorHiCOO const *const hitsr, ptiRankMatrix *mats[],
                                ptiIndex const mats_order[], ptiIndex const mode)
{
    return mttkrp_rank_hicoo(hitsr, mats, mats_order, mode);
}
int ptiOmpMTTKRPHiCOO_MatrixTiling(ptiSparseTensorHiCOO const *const hitsr, ptiRankMatrix *mats[],
                                   ptiIndex const mats_order[], ptiIndex const mode, const int tk, const int tb)
{
    (void)tk;
    (void)tb;
    return mttkrp_rank_hicoo(hitsr, mats, mats_order, mode);
}
int ptiOmpMTTKRPHiCOO_MatrixTiling_Scheduled(ptiSparseTensorHiCOO const *const hitsr, ptiRankMatrix *mats[],
                                             ptiIndex const mats_order[], ptiIndex const mode, const int tk,
                                             const int tb, int balanced)
{
    (void)tk;
    (void)tb;
    (void)balanced;
    return mttkrp_rank_hicoo(hitsr, mats, mats_order, mode);
}
int ptiOmpMTTKRPHiCOO_MatrixTiling_Scheduled_Reduce(ptiSparseTensorHiCOO const *const hitsr, ptiRankMatrix *mats[],
                                                    ptiRankMatrix *copy_mats[], ptiIndex const mats_order[],
                                                    ptiIndex const mode, const int tk, const int tb, int balanced)
{
    (void)copy_mats;
    (void)tk;
    (void)tb;
    (void)balanced;
    return mttkrp_rank_hicoo(hitsr, mats, mats_order, mode);
}
int ptiOmpMTTKRPHiCOO_MatrixTiling_Scheduled_Reduce_Two(ptiSparseTensorHiCOO const *const hitsr,
                                                        ptiRankMatrix *mats[], ptiRankMatrix *copy_mats[],
                                                        ptiIndex const mats_order[], ptiIndex const mode,
                                                        const int tk, const int tb)
{
    (void)copy_mats;
    (void)tk;
    (void)tb;
    return mttkrp_rank_hicoo(hitsr, mats, mats_order, mode);
}

int ptiCudaMTTKRPHiCOO(ptiSparseTensorHiCOO const *const hitsr, ptiMatrix **const mats, ptiIndex *const mats_order,
                       ptiIndex const mode, ptiNnzIndex const max_nnzb, int const impl_num)
{
    (void)max_nnzb;
    (void)impl_num;
    return pti::mttkrp_host_hicoo(hitsr, mats, mats_order, mode);
}

int ptiB200UploadSparseTensor(ptiB200Tensor **out, ptiSparseTensor const *X)
{
    PTI_CHECK(out, PTIERR_VALUE_ERROR, "B200 Upload", "null handle pointer");
    auto *t = new ptiB200Tensor();
    cudaStream_t s = pti::sync_stream();
    int r = pti::upload_coo(t, X, s);
    if (r == 0) r = cudaStreamSynchronize(s) == cudaSuccess ? 0 : PTIERR_CUDA_ERROR;
    if (r) { delete t; return r; }
    *out = t;
    return 0;
}

int ptiB200UploadSparseTensorHiCOO(ptiB200Tensor **out, ptiSparseTensorHiCOO const *H)
{
    PTI_CHECK(out, PTIERR_VALUE_ERROR, "B200 Upload", "null handle pointer");
    auto *t = new ptiB200Tensor();
    cudaStream_t s = pti::sync_stream();
    int r = pti::upload_hicoo(t, H, s);
    if (r == 0) r = cudaStreamSynchronize(s) == cudaSuccess ? 0 : PTIERR_CUDA_ERROR;
    if (r) { delete t; return r; }
    *out = t;
    return 0;
}

int ptiB200FreeTensor(ptiB200Tensor *t)
{
    if (!t) return 0;
    int dev = 0;
    cudaGetDevice(&dev);
    cudaSetDevice(t->device);
    cudaStream_t s = pti::sync_stream();
    cudaStreamSynchronize(s);
    delete t;
    cudaStreamSynchronize(s);
    cudaSetDevice(dev);
    return 0;
}

int ptiB200DownloadHiCOO(ptiB200Tensor const *t, ptiNnzIndex *bptr, void *const *binds, void *const *einds,
                         ptiValue *vals)
{
    const char *mod = "B200 Download";
    PTI_CHECK(t && t->hicoo && bptr && binds && einds && vals, PTIERR_VALUE_ERROR, mod, "need a HiCOO handle");
    cudaStream_t s = pti::sync_stream();
    PTI_CUDA(cudaMemcpyAsync(bptr, t->bptr.ptr, (t->nb + 1) * 8, cudaMemcpyDeviceToHost, s), mod);
    for (uint32_t m = 0; m < t->nmodes; ++m) {
        if (t->nb) PTI_CUDA(cudaMemcpyAsync(binds[m], t->binds[m].ptr, t->nb * 4, cudaMemcpyDeviceToHost, s), mod);
        if (t->nnz) PTI_CUDA(cudaMemcpyAsync(einds[m], t->einds[m].ptr, t->nnz, cudaMemcpyDeviceToHost, s), mod);
    }
    if (t->nnz) PTI_CUDA(cudaMemcpyAsync(vals, t->vals.ptr, t->nnz * 4, cudaMemcpyDeviceToHost, s), mod);
    PTI_CUDA(cudaStreamSynchronize(s), mod);
    return 0;
}

int ptiB200TensorInfo(ptiB200Tensor const *t, ptiNnzIndex info[7], ptiIndex *ndims_out)
{
    PTI_CHECK(t && info, PTIERR_VALUE_ERROR, "B200 Info", "null argument");
    info[0] = t->nmodes;
    info[1] = t->nnz;
    info[2] = t->nb;
    info[3] = t->sb;
    info[4] = t->sk;
    info[5] = t->sc;
    info[6] = t->hicoo ? 1 : 0;
    if (ndims_out)
        for (uint32_t m = 0; m < t->nmodes; ++m) ndims_out[m] = t->ndims[m];
    return 0;
}

int ptiB200MTTKRP(ptiB200Tensor *t, const void *const *dev_mats, int factor_type, ptiIndex rank,
                  ptiIndex stride, const ptiIndex *mats_order, ptiIndex mode, float *dev_out, void *stream)
{
    PTI_CHECK(t && dev_mats && mats_order && dev_out, PTIERR_VALUE_ERROR, "B200 MTTKRP", "null argument");
    return pti::mttkrp_device(t, dev_mats, factor_type, rank, stride, mats_order, mode, dev_out,
                              static_cast<cudaStream_t>(stream));
}

int ptiB200Prepare(ptiB200Tensor *t, ptiIndex mode, void *stream)
{
    PTI_CHECK(t, PTIERR_VALUE_ERROR, "B200 Prepare", "null handle");
    return pti::prepare_mode(t, mode, static_cast<cudaStream_t>(stream));
}

int ptiB200CheckTensor(ptiB200Tensor *t, void *stream)
{
    PTI_CHECK(t, PTIERR_VALUE_ERROR, "B200 Check", "null handle");
    return pti::take_device_error(t, static_cast<cudaStream_t>(stream), "B200 Check");
}

}  // extern "C"

// ---------------------------------------------------------------------------
// HiCOO MTTKRP that allocates nothing.
//
// Some callers cannot allocate device memory while they run this operation:
// code inside a host framework that owns every byte of device memory through
// its own pool, services with a fixed memory budget that must not grow or fail
// mid-request, and real-time loops where a cudaMalloc would block.  This entry
// point therefore keeps its only scratch -- the tile-to-block table the kernel
// needs and the error word -- in fixed arrays in device global memory that are
// part of the library image.  Every GPU that loads the library holds them
// (about 1 MiB) until the process exits.
// ---------------------------------------------------------------------------
namespace pti {
namespace {

constexpr uint32_t kNoAllocMaxTiles = 1u << 18;  // tiles of kHiTile nonzeros: up to 268,435,456 nonzeros

static __device__ __align__(256) uint32_t g_noalloc_tile_block[kNoAllocMaxTiles + 1];
static __device__ __align__(256) uint32_t g_noalloc_err[64];

constexpr int kNoAllocMaxDevices = 64;
struct NoAllocScratch {
    uint32_t *tile_block;
    uint32_t *err;
};
NoAllocScratch g_noalloc_scratch[kNoAllocMaxDevices];
std::mutex g_noalloc_mu;

// Device addresses of the scratch arrays for the current device, looked up
// once per device (host code must not use the symbols' host-side names as
// device pointers).  They stay valid for the life of the device's primary
// context; a cudaDeviceReset would leave them stale, which the header states.
int noalloc_scratch(NoAllocScratch &out, const char *mod)
{
    int dev = 0;
    PTI_CUDA(cudaGetDevice(&dev), mod);
    PTI_CHECK(dev >= 0 && dev < kNoAllocMaxDevices, PTIERR_VALUE_ERROR, mod, "device ordinal too large");
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    NoAllocScratch &sc = g_noalloc_scratch[dev];
    if (!sc.tile_block) {
        void *tb = nullptr, *er = nullptr;
        PTI_CUDA(cudaGetSymbolAddress(&tb, g_noalloc_tile_block), mod);
        PTI_CUDA(cudaGetSymbolAddress(&er, g_noalloc_err), mod);
        sc.err = static_cast<uint32_t *>(er);
        sc.tile_block = static_cast<uint32_t *>(tb);
    }
    out = sc;
    return 0;
}

}  // namespace
}  // namespace pti

extern "C" int ptiB200MTTKRPHiCOONoAlloc(ptiIndex nmodes, const ptiIndex *ndims, ptiNnzIndex nnz, ptiNnzIndex nb,
                                         ptiElementIndex sb_bits, const ptiNnzIndex *dev_bptr,
                                         const ptiBlockIndex *const *dev_binds,
                                         const ptiElementIndex *const *dev_einds, const ptiValue *dev_vals,
                                         const float *const *dev_mats, ptiIndex rank, ptiIndex stride,
                                         const ptiIndex *mats_order, ptiIndex mode, float *dev_out, void *stream)
{
    using namespace pti;
    const char *mod = "B200 HiCOO MTTKRP (no allocation)";
    PTI_CHECK(ndims && mats_order && dev_mats && dev_out, PTIERR_VALUE_ERROR, mod, "null argument");
    PTI_CHECK(nmodes >= 2 && nmodes <= (uint32_t)kMaxModes, PTIERR_VALUE_ERROR, mod, "unsupported number of modes");
    PTI_CHECK(mode < nmodes, PTIERR_VALUE_ERROR, mod, "mode out of range");
    PTI_CHECK(sb_bits <= 8, PTIERR_VALUE_ERROR, mod, "sb_bits must be <= 8");
    PTI_CHECK(rank >= 1 && stride >= rank && stride % 4 == 0, PTIERR_SHAPE_MISMATCH, mod,
              "stride must be >= rank and a multiple of 4");
    const uint64_t ntiles = (nnz + kHiTile - 1) / kHiTile;
    PTI_CHECK(ntiles <= kNoAllocMaxTiles, PTIERR_VALUE_ERROR, mod,
              "more than 268,435,456 nonzeros: beyond the fixed scratch of this entry point");
    PTI_CHECK(nnz == 0 || (nb >= 1 && nb < 0xFFFFFFFFull && dev_bptr && dev_binds && dev_einds && dev_vals),
              PTIERR_VALUE_ERROR, mod, "missing HiCOO arrays");
    uint32_t seen = 0;
    for (uint32_t i = 0; i < nmodes; ++i) {
        PTI_CHECK(mats_order[i] < nmodes && !(seen >> mats_order[i] & 1u), PTIERR_VALUE_ERROR, mod,
                  "mats_order must be a permutation of the modes");
        seen |= 1u << mats_order[i];
    }
    PTI_CHECK(mats_order[0] == mode, PTIERR_VALUE_ERROR, mod, "mats_order[0] must equal mode");
    PTI_CHECK(((uintptr_t)dev_out & 15) == 0, PTIERR_VALUE_ERROR, mod, "output must be 16-byte aligned");
    for (uint32_t i = 1; i < nmodes; ++i)
        PTI_CHECK(dev_mats[mats_order[i]] && ((uintptr_t)dev_mats[mats_order[i]] & 15) == 0, PTIERR_VALUE_ERROR,
                  mod, "factors must be non-null and 16-byte aligned");

    cudaStream_t s = static_cast<cudaStream_t>(stream);
    NoAllocScratch sc;
    PTI_TRY(noalloc_scratch(sc, mod));
    PTI_CUDA(cudaMemsetAsync(dev_out, 0, (size_t)ndims[mode] * stride * sizeof(float), s), mod);
    PTI_CUDA(cudaMemsetAsync(sc.err, 0, sizeof(uint32_t), s), mod);
    if (nnz == 0) return 0;

    tile_block_kernel<<<ceil_div(nb, 256), 256, 0, s>>>(dev_bptr, nb, (uint32_t)ntiles, sc.tile_block);
    HicooArgs a{};
    a.nnz = nnz;
    a.nb = nb;
    a.nin = nmodes - 1;
    a.R = rank;
    a.stride = stride;
    a.sb = sb_bits;
    a.bptr = dev_bptr;
    a.tile_block = sc.tile_block;
    a.out_bind = dev_binds[mode];
    a.out_eind = dev_einds[mode];
    a.out_dim = ndims[mode];
    for (uint32_t i = 1; i < nmodes; ++i) {
        const uint32_t k = mats_order[i];
        a.in_bind[i - 1] = dev_binds[k];
        a.in_eind[i - 1] = dev_einds[k];
        a.in_dim[i - 1] = ndims[k];
        a.in_mat[i - 1] = dev_mats[k];
    }
    a.vals = dev_vals;
    a.out = dev_out;
    a.err = sc.err;
    launch_hicoo<float>(a, group_lanes(rank), (unsigned)ntiles, s);
    PTI_CUDA(cudaGetLastError(), mod);
    return 0;
}
