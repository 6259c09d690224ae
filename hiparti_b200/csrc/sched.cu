// sched.cu -- per-mode schedules and the output-privatised MTTKRP kernels.
//
// Problem.  With skewed (power-law) mode sizes a few output rows receive a
// large share of all nonzeros; adding every product straight into global
// memory serialises the atomics of such a row in one L2 slice.
//
// Schedule (built once per tensor and mode, kept in the device handle).
// HiCOO: the blocks are stably re-ordered by their block coordinate in the
// output mode, and the nonzeros of each block by their 8-bit output offset --
// the reference's per-mode kernel scheduler (kschr, src/sptensor/hicoo/
// convert.c:378-421) taken down to block granularity and materialised as a
// second HiCOO array set.  COO: the nonzeros are stably sorted by their
// output index.
//
// Kernel (one CTA per tile of kTile nonzeros).  The tile's element offsets and
// values are staged into shared memory with bulk (TMA) copies; block
// coordinates are loaded alongside and every nonzero is tagged with its block.
// For HiCOO the tile is then counting-sorted by output row in shared memory
// (at most 1024 >> sb block rows at a time), so each thread group walks a
// contiguous run of nonzeros ordered by output row, accumulates the rank-R
// Hadamard products in registers and adds a row into global memory once per
// run (16-byte vector atomics).  A hot row is thus added once per group that
// touches it instead of once per nonzero.
#include "kutil.cuh"
#include "primitives.cuh"
#include "tensor.cuh"
#include "tma.cuh"

namespace pti {

constexpr int kTile = 2048;        // nonzeros per CTA (COO kernel)
constexpr int kHiTile = kPlanTile; // nonzeros per CTA (HiCOO kernel)
constexpr int kHist = 2048;        // counting-sort buckets: (2048 >> sb) block rows per pass
constexpr int kSchedThreads = 256;
constexpr int kUnroll = 4;         // nonzeros in flight per thread group

uint32_t *err_word();
int ensure_err_word(cudaStream_t s);

struct SchedArgs {
    uint64_t nnz, nb;
    uint32_t R, stride, sb;
    const uint64_t *bptr;
    const uint32_t *tile_block;
    const uint32_t *out_bind;   // HiCOO: block coords of the output mode; COO: output indices
    const uint8_t *out_eind;
    uint32_t out_dim;
    const uint32_t *in_bind[kMaxModes - 1];  // HiCOO block coords / COO indices of operand modes
    const uint8_t *in_eind[kMaxModes - 1];
    uint32_t in_dim[kMaxModes - 1];
    const void *in_mat[kMaxModes - 1];
    const float *vals;
    float *out;
    uint32_t *err;
};

__device__ __forceinline__ uint32_t round16(uint32_t x) { return (x + 15u) & ~15u; }

// Words per packed nonzero record {output row, operand rows..., value},
// rounded up to 16 bytes.
template <int NIN>
struct Rec {
    static constexpr int words = ((NIN + 2 + 3) / 4) * 4;
};

// Columns of one operand row held by a lane: 4 (one float4 of FP32) or 8 (one
// 16-byte load of BF16).
template <int CPL, class FT>
struct RowPart {
    uint4 raw;
    __device__ __forceinline__ void load(const FT *row, uint32_t col)
    {
        if constexpr (CPL == 4 && sizeof(FT) == 4) {
            const float4 f = __ldg(reinterpret_cast<const float4 *>(row + col));
            raw = make_uint4(__float_as_uint(f.x), __float_as_uint(f.y), __float_as_uint(f.z), __float_as_uint(f.w));
        } else if constexpr (CPL == 8) {
            raw = __ldg(reinterpret_cast<const uint4 *>(row + col));
        } else {
            const uint2 r = __ldg(reinterpret_cast<const uint2 *>(row + col));
            raw = make_uint4(r.x, r.y, 0u, 0u);
        }
    }
    // column c (0 <= c < CPL) as FP32
    __device__ __forceinline__ float at(int c) const
    {
        const uint32_t w[4] = {raw.x, raw.y, raw.z, raw.w};
        if constexpr (sizeof(FT) == 4) {
            return __uint_as_float(w[c]);
        } else {
            const uint32_t h = w[c >> 1];
            return __uint_as_float((c & 1) ? (h & 0xFFFF0000u) : (h << 16));
        }
    }
};

// Walks records [j0, j1) (ordered by output row): gathers the operand rows,
// accumulates v * prod_k A_k[row_k] in registers, and adds the sum into the
// output once per run of equal output rows.
template <int G, int CPL, int U, int NIN, class FT>
__device__ __forceinline__ void process_records(const uint32_t *s_rec, uint32_t j0, uint32_t j1, uint32_t lane,
                                                const SchedArgs &a, const float *alt = nullptr)
{
    constexpr int RW = Rec<NIN>::words;
    const uint32_t col = lane * CPL;
    const bool active = col < a.R;
    float acc[CPL];
#pragma unroll
    for (int c = 0; c < CPL; ++c) acc[c] = 0.f;
    uint32_t cur = 0xFFFFFFFFu;
    auto flush = [&](uint32_t row) {
#pragma unroll
        for (int q = 0; q < CPL / 4; ++q)
            if (col + 4 * q < a.R)
                red_add4(a.out + (size_t)row * a.stride + col + 4 * q,
                         mask4(make_float4(acc[4 * q], acc[4 * q + 1], acc[4 * q + 2], acc[4 * q + 3]), col + 4 * q, a.R));
    };
    for (uint32_t j = j0; j < j1; j += U) {
        uint32_t orow[U];
        float val[U];
        RowPart<CPL, FT> f[U][NIN];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            orow[u] = 0xFFFFFFFFu;
            if (j + u < j1) {
                uint32_t w[RW];
#pragma unroll
                for (int q = 0; q < RW; q += 4) {
                    const uint4 r = *reinterpret_cast<const uint4 *>(s_rec + (size_t)(j + u) * RW + q);
                    w[q] = r.x; w[q + 1] = r.y; w[q + 2] = r.z; w[q + 3] = r.w;
                }
                orow[u] = w[0];
                val[u] = alt ? __ldg(alt + j + u) : __uint_as_float(w[1 + NIN]);
                if (orow[u] != 0xFFFFFFFFu && active) {
#pragma unroll
                    for (int k = 0; k < NIN; ++k)
                        f[u][k].load(static_cast<const FT *>(a.in_mat[k]) + (size_t)w[1 + k] * a.stride, col);
                }
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (orow[u] == 0xFFFFFFFFu) continue;
            if (orow[u] != cur) {
                if (cur != 0xFFFFFFFFu && active) flush(cur);
#pragma unroll
                for (int c = 0; c < CPL; ++c) acc[c] = 0.f;
                cur = orow[u];
            }
            if (active) {
#pragma unroll
                for (int c = 0; c < CPL; ++c) {
                    float p = val[u] * f[u][0].at(c);
#pragma unroll
                    for (int k = 1; k < NIN; ++k) p *= f[u][k].at(c);
                    acc[c] += p;
                }
            }
        }
    }
    if (cur != 0xFFFFFFFFu && active) flush(cur);
}

template <int NIN>
struct HiSmem {
    // byte offsets inside the dynamic shared memory of hicoo_sched_kernel
    static constexpr uint32_t val = 0;                                  // float[kHiTile]
    static constexpr uint32_t eout = val + 4 * kHiTile;                 // u8[kHiTile]
    static constexpr uint32_t ein = eout + kHiTile;                     // u8[NIN][kHiTile]
    static constexpr uint32_t blk = ein + NIN * kHiTile;                // u16[kHiTile]
    static constexpr uint32_t ord = blk + 2 * kHiTile;                  // u16[kHiTile]
    static constexpr uint32_t hist = ord + 2 * kHiTile;                 // u32[kHist]
    static constexpr uint32_t brow = hist + 4 * kHist;                  // u32[kHiTile + 4]
    static constexpr uint32_t bin = brow + 4 * (kHiTile + 4);           // u32[NIN][kHiTile + 4]
    static constexpr uint32_t total = bin + 4 * NIN * (kHiTile + 4);
};

template <int G, int CPL, class FT, int NIN>
__global__ void __launch_bounds__(kSchedThreads) hicoo_sched_kernel(SchedArgs a)
{
    using L = HiSmem<NIN>;
    constexpr int U = NIN <= 2 ? 4 : 2;  // nonzeros in flight per group
    extern __shared__ __align__(128) unsigned char sm[];
    __shared__ uint64_t mbar;
    __shared__ uint32_t s_scan[kSchedThreads / 32];
    float *s_val = reinterpret_cast<float *>(sm + L::val);
    uint8_t *s_eout = sm + L::eout;
    uint8_t *s_ein = sm + L::ein;
    uint16_t *s_blk = reinterpret_cast<uint16_t *>(sm + L::blk);
    uint16_t *s_ord = reinterpret_cast<uint16_t *>(sm + L::ord);
    uint32_t *s_hist = reinterpret_cast<uint32_t *>(sm + L::hist);
    uint32_t *s_brow = reinterpret_cast<uint32_t *>(sm + L::brow);
    uint32_t *s_bin = reinterpret_cast<uint32_t *>(sm + L::bin);
    const uint32_t tid = threadIdx.x;

    const uint64_t z0 = (uint64_t)blockIdx.x * kHiTile;
    const uint32_t n = (uint32_t)((a.nnz - z0) < (uint64_t)kHiTile ? (a.nnz - z0) : (uint64_t)kHiTile);
    const uint32_t b0 = a.tile_block[blockIdx.x];
    uint32_t nblk = a.tile_block[blockIdx.x + 1] - b0 + 1;
    if (nblk > kHiTile + 1) nblk = kHiTile + 1;
    if (b0 + (uint64_t)nblk > a.nb) nblk = (uint32_t)(a.nb - b0);

    // stage element offsets and values with bulk copies
    if (tid == 0) {
        mbar_init(&mbar, 1);
        mbar_fence_init();
    }
    __syncthreads();
    if (tid == 0) {
        const uint32_t be = round16(n), bv = round16(4 * n);
        mbar_arrive_expect_tx(&mbar, bv + (NIN + 1) * be);
        bulk_g2s(s_val, a.vals + z0, bv, &mbar);
        bulk_g2s(s_eout, a.out_eind + z0, be, &mbar);
#pragma unroll
        for (int k = 0; k < NIN; ++k) bulk_g2s(s_ein + k * kHiTile, a.in_eind[k] + z0, be, &mbar);
    }
    // block coordinates and the block of every nonzero, meanwhile
    for (uint32_t i = tid; i < nblk; i += kSchedThreads) {
        const uint64_t b = b0 + i;
        s_brow[i] = __ldg(a.out_bind + b);
#pragma unroll
        for (int k = 0; k < NIN; ++k) s_bin[k * (kHiTile + 4) + i] = __ldg(a.in_bind[k] + b) << a.sb;
        const uint64_t zs = max(__ldg(a.bptr + b), z0), ze = min(__ldg(a.bptr + b + 1), z0 + n);
        for (uint64_t z = zs; z < ze; ++z) s_blk[z - z0] = (uint16_t)i;
    }
    const bool ok = mbar_wait_bounded(&mbar, 0);
    if (!__syncthreads_and(ok)) {
        if (tid == 0) {
            atomicOr(a.err, 2u);
            mbar_wait_bounded(&mbar, 0);
        }
        return;
    }

    const uint32_t g = tid / G, lane = tid % G;
    constexpr uint32_t kGroups = kSchedThreads / G;
    const uint32_t col = lane * CPL;
    const bool active = col < a.R;
    const uint32_t span = (uint32_t)kHist >> a.sb;
    uint32_t zs = 0;
    while (zs < n) {
        // the pass covers nonzeros whose block row is < br0 + span
        const uint32_t br0 = s_brow[s_blk[zs]];
        uint32_t lo = zs + 1, hi = n;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (s_brow[s_blk[mid]] - br0 >= span) hi = mid;
            else lo = mid + 1;
        }
        const uint32_t ze = lo;
        for (uint32_t h = tid; h < (uint32_t)kHist; h += kSchedThreads) s_hist[h] = 0;
        __syncthreads();
        for (uint32_t z = zs + tid; z < ze; z += kSchedThreads)
            atomicAdd(&s_hist[((s_brow[s_blk[z]] - br0) << a.sb) | s_eout[z]], 1u);
        __syncthreads();
        {   // exclusive scan of the histogram (kHist = 256 threads x 8)
            constexpr int per = kHist / kSchedThreads;
            uint32_t v[per], sum = 0;
#pragma unroll
            for (int j = 0; j < per; ++j) {
                v[j] = s_hist[tid * per + j];
                sum += v[j];
            }
            uint32_t x = sum;
            const uint32_t l = tid & 31, w = tid >> 5;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
                if (l >= (uint32_t)o) x += y;
            }
            if (l == 31) s_scan[w] = x;
            __syncthreads();
            uint32_t wp = 0;
            for (uint32_t q = 0; q < w; ++q) wp += s_scan[q];
            uint32_t run = wp + x - sum + zs;
#pragma unroll
            for (int j = 0; j < per; ++j) {
                s_hist[tid * per + j] = run;
                run += v[j];
            }
        }
        __syncthreads();
        for (uint32_t z = zs + tid; z < ze; z += kSchedThreads) {
            const uint32_t pos = atomicAdd(&s_hist[((s_brow[s_blk[z]] - br0) << a.sb) | s_eout[z]], 1u);
            s_ord[pos] = (uint16_t)z;
        }
        __syncthreads();

        // each group: a contiguous run of the row-sorted nonzeros
        // an odd slice length puts the groups' first records on different shared-memory banks
        const uint32_t cnt = ze - zs, per = ((cnt + kGroups - 1) / kGroups) | 1u;
        const uint32_t j0 = min(zs + g * per, ze), j1 = min(j0 + per, ze);
        float acc[CPL];
#pragma unroll
        for (int c = 0; c < CPL; ++c) acc[c] = 0.f;
        uint32_t cur = 0xFFFFFFFFu;
        auto flush = [&](uint32_t row) {
#pragma unroll
            for (int q = 0; q < CPL / 4; ++q)
                if (col + 4 * q < a.R)
                    red_add4(a.out + (size_t)row * a.stride + col + 4 * q,
                             mask4(make_float4(acc[4 * q], acc[4 * q + 1], acc[4 * q + 2], acc[4 * q + 3]), col + 4 * q, a.R));
        };
        for (uint32_t j = j0; j < j1; j += U) {
            uint32_t orow[U];
            float v[U];
            RowPart<CPL, FT> f[U][NIN];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                orow[u] = 0xFFFFFFFFu;
                if (j + u >= j1) continue;
                const uint32_t z = s_ord[j + u], i = s_blk[z];
                const uint32_t o = (s_brow[i] << a.sb) + s_eout[z];
                v[u] = s_val[z];
                bool in_range = o < a.out_dim;
                uint32_t r[NIN];
#pragma unroll
                for (int k = 0; k < NIN; ++k) {
                    r[k] = s_bin[k * (kHiTile + 4) + i] + s_ein[k * kHiTile + z];
                    in_range = in_range && r[k] < a.in_dim[k];
                }
                if (!in_range) {
                    if (lane == 0) atomicOr(a.err, 1u);
                    continue;
                }
                orow[u] = o;
                if (active) {
#pragma unroll
                    for (int k = 0; k < NIN; ++k)
                        f[u][k].load(static_cast<const FT *>(a.in_mat[k]) + (size_t)r[k] * a.stride, col);
                }
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                if (orow[u] == 0xFFFFFFFFu) continue;
                if (orow[u] != cur) {
                    if (cur != 0xFFFFFFFFu && active) flush(cur);
#pragma unroll
                    for (int c = 0; c < CPL; ++c) acc[c] = 0.f;
                    cur = orow[u];
                }
                if (active) {
#pragma unroll
                    for (int c = 0; c < CPL; ++c) {
                        float p = v[u] * f[u][0].at(c);
#pragma unroll
                        for (int k = 1; k < NIN; ++k) p *= f[u][k].at(c);
                        acc[c] += p;
                    }
                }
            }
        }
        if (cur != 0xFFFFFFFFu && active) flush(cur);
        __syncthreads();
        zs = ze;
    }
}

// COO schedule: packed records sorted by output index; no sorting in the kernel.
template <int G, int CPL, int U, int MINB, class FT, int NIN>
__global__ void __launch_bounds__(kSchedThreads, MINB) coo_sched_kernel(SchedArgs a, const uint32_t *recs)
{
    constexpr int RW = Rec<NIN>::words;
    extern __shared__ __align__(128) unsigned char sm[];
    __shared__ uint64_t mbar;
    uint32_t *s_rec = reinterpret_cast<uint32_t *>(sm);
    const uint32_t tid = threadIdx.x;
    const uint64_t z0 = (uint64_t)blockIdx.x * kTile;
    const uint32_t n = (uint32_t)((a.nnz - z0) < (uint64_t)kTile ? (a.nnz - z0) : (uint64_t)kTile);
    if (tid == 0) {
        mbar_init(&mbar, 1);
        mbar_fence_init();
    }
    __syncthreads();
    if (tid == 0) {
        const uint32_t bytes = n * RW * 4;
        mbar_arrive_expect_tx(&mbar, bytes);
        bulk_g2s(s_rec, recs + z0 * RW, bytes, &mbar);
    }
    const bool ok = mbar_wait_bounded(&mbar, 0);
    if (!__syncthreads_and(ok)) {
        if (tid == 0) {
            atomicOr(a.err, 2u);
            mbar_wait_bounded(&mbar, 0);
        }
        return;
    }
    const uint32_t g = tid / G, lane = tid % G;
    constexpr uint32_t kGroups = kSchedThreads / G;
    const uint32_t per = ((n + kGroups - 1) / kGroups) | 1u;  // odd: groups start on different banks
    const uint32_t j0 = min(g * per, n), j1 = min(j0 + per, n);
    process_records<G, CPL, U, NIN, FT>(s_rec, j0, j1, lane, a, a.vals ? a.vals + z0 : nullptr);
}

// ---------------------------------------------------------------------------
// Schedule construction
// ---------------------------------------------------------------------------
__global__ void iota_keys_kernel(const uint32_t *src, uint64_t n, uint64_t *keys, uint32_t *vals)
{
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        keys[i] = src[i];
        vals[i] = (uint32_t)i;
    }
}

// COO packed records in sorted order: {out index, operand indices (modes in
// increasing order, skipping the output mode), value, 0...}.
struct PackArgs {
    uint32_t nin, rw;
    const uint32_t *out;
    const uint32_t *in[kMaxModes - 1];
    const float *vals;
};

__global__ void pack_records_kernel(PackArgs pa, const uint32_t *perm, uint64_t n, uint32_t *recs)
{
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t z = perm[j];
        uint32_t *r = recs + j * pa.rw;
        r[0] = pa.out[z];
        for (uint32_t k = 0; k < pa.nin; ++k) r[1 + k] = pa.in[k][z];
        r[1 + pa.nin] = __float_as_uint(pa.vals[z]);
        for (uint32_t k = pa.nin + 2; k < pa.rw; ++k) r[k] = 0;
    }
}

__global__ void block_of_nnz_kernel(const uint64_t *bptr, uint64_t nb, uint32_t *blk)
{
    for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += (uint64_t)gridDim.x * blockDim.x)
        for (uint64_t z = bptr[b]; z < bptr[b + 1]; ++z) blk[z] = (uint32_t)b;
}

__global__ void permuted_blocks_kernel(const uint32_t *perm, uint64_t nb, const uint64_t *bptr, uint32_t *size,
                                       uint32_t *inv)
{
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < nb; j += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t b = perm[j];
        size[j] = (uint32_t)(bptr[b + 1] - bptr[b]);
        inv[b] = (uint32_t)j;
    }
}

__global__ void nnz_keys_kernel(const uint32_t *blk, const uint32_t *inv, const uint8_t *eout, uint64_t n,
                                uint64_t *keys, uint32_t *vals)
{
    for (uint64_t z = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; z < n; z += (uint64_t)gridDim.x * blockDim.x) {
        keys[z] = ((uint64_t)inv[blk[z]] << 8) | eout[z];
        vals[z] = (uint32_t)z;
    }
}

template <class T>
__global__ void gather_kernel(const T *src, const uint32_t *perm, uint64_t n, T *dst)
{
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        dst[i] = src[perm[i]];
}

__global__ void tile_block_kernel_t(const uint64_t *bptr, uint64_t nb, uint32_t ntiles, uint32_t tile,
                                    uint32_t *tile_block)
{
    for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t zs = bptr[b], ze = bptr[b + 1];
        for (uint64_t t = (zs + tile - 1) / tile; t * tile < ze && t < ntiles; ++t) tile_block[t] = (uint32_t)b;
        if (b == nb - 1) tile_block[ntiles] = (uint32_t)b;
    }
}

struct SizeIn {
    const uint32_t *p;
    __device__ uint64_t operator()(uint64_t i) const { return p[i]; }
};
struct BptrOut {
    uint64_t *p;
    __device__ void operator()(uint64_t i, uint64_t prefix, uint64_t) const { p[i] = prefix; }
};

static uint32_t bits_for_count(uint64_t count)
{
    uint32_t b = 0;
    while (b < 64 && ((uint64_t)1 << b) < count) ++b;
    return b;
}

static unsigned grid_n(uint64_t n)
{
    return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, (uint64_t)sm_count() * 32));
}

int prepare_mode(ptiB200Tensor *t, uint32_t mode, cudaStream_t s)
{
    const char *mod = "B200 Prepare";
    PTI_CHECK(mode < t->nmodes, PTIERR_VALUE_ERROR, mod, "mode out of range");
    const uint32_t N = t->nmodes;
    const uint64_t n = t->nnz;
    PTI_CHECK(n < 0xFFFFFFFFull, PTIERR_VALUE_ERROR, mod, "too many nonzeros");
    if (n == 0) return 0;
    if (!t->hicoo) {
        CooModePlan &P = t->coo_plan[mode];
        if (P.ready) return 0;
        PTI_CHECK(N <= 4, PTIERR_VALUE_ERROR, mod, "COO schedules cover orders up to 4");
        DevBuf keys, perm;
        RadixScratch rs;
        PTI_CUDA(keys.alloc(padded(n * 8), s), mod);
        PTI_CUDA(perm.alloc(padded(n * 4), s), mod);
        PTI_TRY(rs.alloc(n, s));
        iota_keys_kernel<<<grid_n(n), 256, 0, s>>>(t->inds[mode].as<uint32_t>(), n, keys.as<uint64_t>(),
                                                   perm.as<uint32_t>());
        PTI_TRY(radix_sort_pairs(keys, perm, n, (int)bits_for_count(t->ndims[mode]), rs, s));
        const int RW = N <= 3 ? 4 : 8;
        PTI_CUDA(P.recs.alloc(padded(n * RW * 4), s), mod);
        PackArgs pa{};
        pa.nin = N - 1;
        pa.rw = RW;
        pa.out = t->inds[mode].as<uint32_t>();
        for (uint32_t k = 0, i = 0; k < N; ++k)
            if (k != mode) pa.in[i++] = t->inds[k].as<uint32_t>();
        pa.vals = t->vals.as<float>();
        pack_records_kernel<<<grid_n(n), 256, 0, s>>>(pa, perm.as<uint32_t>(), n, P.recs.as<uint32_t>());
        PTI_CUDA(cudaGetLastError(), mod);
        P.perm = std::move(perm);
        P.ready = true;
        return 0;
    }
    HicooModePlan &P = t->hicoo_plan[mode];
    if (P.ready) return 0;
    const uint64_t nb = t->nb;
    PTI_CHECK(t->sb <= 8, PTIERR_VALUE_ERROR, mod, "sb_bits must be <= 8");
    // 1. blocks by output-mode block coordinate (stable)
    DevBuf bkeys, bperm, inv, bsize;
    {
        RadixScratch rs;
        PTI_CUDA(bkeys.alloc(padded(nb * 8), s), mod);
        PTI_CUDA(bperm.alloc(padded(nb * 4), s), mod);
        PTI_TRY(rs.alloc(nb, s));
        iota_keys_kernel<<<grid_n(nb), 256, 0, s>>>(t->binds[mode].as<uint32_t>(), nb, bkeys.as<uint64_t>(),
                                                    bperm.as<uint32_t>());
        const uint64_t brows = ((uint64_t)t->ndims[mode] + ((uint64_t)1 << t->sb) - 1) >> t->sb;
        PTI_TRY(radix_sort_pairs(bkeys, bperm, nb, (int)bits_for_count(brows + 1), rs, s));
    }
    bkeys.reset();
    PTI_CUDA(inv.alloc(padded(nb * 4), s), mod);
    PTI_CUDA(bsize.alloc(padded(nb * 4), s), mod);
    permuted_blocks_kernel<<<grid_n(nb), 256, 0, s>>>(bperm.as<uint32_t>(), nb, t->bptr.as<uint64_t>(),
                                                      bsize.as<uint32_t>(), inv.as<uint32_t>());
    PTI_CUDA(P.bptr.alloc(padded((nb + 1) * 8), s), mod);
    {
        DevBuf tmp;
        PTI_CUDA(tmp.alloc(padded(scan_tmp_elems<uint64_t>(nb) * 8), s), mod);
        PTI_TRY((exclusive_scan<uint64_t>(SizeIn{bsize.as<uint32_t>()}, BptrOut{P.bptr.as<uint64_t>()}, nb,
                                          tmp.as<uint64_t>(), nullptr, s)));
        PTI_CUDA(cudaMemcpyAsync(P.bptr.as<uint64_t>() + nb, tmp.as<uint64_t>() + (nb + kScanTile - 1) / kScanTile,
                                 8, cudaMemcpyDeviceToDevice, s), mod);
    }
    for (uint32_t k = 0; k < N; ++k) {
        PTI_CUDA(P.binds[k].alloc(padded(nb * 4), s), mod);
        gather_kernel<uint32_t><<<grid_n(nb), 256, 0, s>>>(t->binds[k].as<uint32_t>(), bperm.as<uint32_t>(), nb,
                                                           P.binds[k].as<uint32_t>());
    }
    bsize.reset();
    bperm.reset();
    // 2. nonzeros: (new block, output offset), stable
    {
        DevBuf blk, zkeys, zperm;
        RadixScratch rs;
        PTI_CUDA(blk.alloc(padded(n * 4), s), mod);
        block_of_nnz_kernel<<<grid_n(nb), 256, 0, s>>>(t->bptr.as<uint64_t>(), nb, blk.as<uint32_t>());
        PTI_CUDA(zkeys.alloc(padded(n * 8), s), mod);
        PTI_CUDA(zperm.alloc(padded(n * 4), s), mod);
        nnz_keys_kernel<<<grid_n(n), 256, 0, s>>>(blk.as<uint32_t>(), inv.as<uint32_t>(),
                                                  t->einds[mode].as<uint8_t>(), n, zkeys.as<uint64_t>(),
                                                  zperm.as<uint32_t>());
        blk.reset();
        PTI_TRY(rs.alloc(n, s));
        PTI_TRY(radix_sort_pairs(zkeys, zperm, n, (int)bits_for_count(nb) + 8, rs, s));
        for (uint32_t k = 0; k < N; ++k) {
            PTI_CUDA(P.einds[k].alloc(padded(n), s), mod);
            gather_kernel<uint8_t><<<grid_n(n), 256, 0, s>>>(t->einds[k].as<uint8_t>(), zperm.as<uint32_t>(), n,
                                                             P.einds[k].as<uint8_t>());
        }
        PTI_CUDA(P.vals.alloc(padded(n * 4), s), mod);
        gather_kernel<float><<<grid_n(n), 256, 0, s>>>(t->vals.as<float>(), zperm.as<uint32_t>(), n,
                                                       P.vals.as<float>());
    }
    inv.reset();
    P.nb = nb;
    P.ntiles = (uint32_t)((n + kHiTile - 1) / kHiTile);
    PTI_CUDA(P.tile_block.alloc(padded(((size_t)P.ntiles + 1) * 4), s), mod);
    tile_block_kernel_t<<<grid_n(nb), 256, 0, s>>>(P.bptr.as<uint64_t>(), nb, P.ntiles, kHiTile,
                                                   P.tile_block.as<uint32_t>());
    PTI_CUDA(cudaGetLastError(), mod);
    P.ready = true;
    return 0;
}

// ---------------------------------------------------------------------------
// Launch
// ---------------------------------------------------------------------------
template <int G, int CPL, int U, class FT, int NIN>
static int launch_coo(const SchedArgs &a, const uint32_t *recs, unsigned ntiles, cudaStream_t s)
{
    const size_t smem = (size_t)kTile * Rec<NIN>::words * 4;
    auto k = coo_sched_kernel<G, CPL, U, 4, FT, NIN>;
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return PTIERR_CUDA_ERROR;
    k<<<ntiles, kSchedThreads, smem, s>>>(a, recs);
    return 0;
}

template <int G, int CPL, class FT, int NIN>
static int launch_hicoo(const SchedArgs &a, unsigned ntiles, cudaStream_t s)
{
    const size_t smem = HiSmem<NIN>::total;
    auto k = hicoo_sched_kernel<G, CPL, FT, NIN>;
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return PTIERR_CUDA_ERROR;
    k<<<ntiles, kSchedThreads, smem, s>>>(a);
    return 0;
}

// Lanes per nonzero: 4 columns per lane (FP32 factors, or BF16 factors that
// are not 16-byte addressable by rows) or 8 columns per lane (BF16 with a
// stride that is a multiple of 8); one column pass (R <= 128).
template <class FT, int NIN>
static int launch_r(bool hicoo, bool wide, const SchedArgs &a, const uint32_t *recs, unsigned ntiles, cudaStream_t s)
{
    const uint32_t R = a.R;
    if constexpr (sizeof(FT) == 2) {
        if (wide) {
            if (hicoo) {
                if (R <= 8) return launch_hicoo<1, 8, FT, NIN>(a, ntiles, s);
                if (R <= 16) return launch_hicoo<2, 8, FT, NIN>(a, ntiles, s);
                if (R <= 32) return launch_hicoo<4, 8, FT, NIN>(a, ntiles, s);
                if (R <= 64) return launch_hicoo<8, 8, FT, NIN>(a, ntiles, s);
                return launch_hicoo<16, 8, FT, NIN>(a, ntiles, s);
            }
            if (R <= 8) return launch_coo<1, 8, 2, FT, NIN>(a, recs, ntiles, s);
            if (R <= 16) return launch_coo<2, 8, 2, FT, NIN>(a, recs, ntiles, s);
            if (R <= 32) return launch_coo<4, 8, 2, FT, NIN>(a, recs, ntiles, s);
            if (R <= 64) return launch_coo<8, 8, 2, FT, NIN>(a, recs, ntiles, s);
            return launch_coo<16, 8, 2, FT, NIN>(a, recs, ntiles, s);
        }
    }
    if (hicoo) {
        if (R <= 4) return launch_hicoo<1, 4, FT, NIN>(a, ntiles, s);
        if (R <= 8) return launch_hicoo<2, 4, FT, NIN>(a, ntiles, s);
        if (R <= 16) return launch_hicoo<4, 4, FT, NIN>(a, ntiles, s);
        if (R <= 32) return launch_hicoo<8, 4, FT, NIN>(a, ntiles, s);
        if (R <= 64) return launch_hicoo<16, 4, FT, NIN>(a, ntiles, s);
        return launch_hicoo<32, 4, FT, NIN>(a, ntiles, s);
    }
    if (R <= 4) return launch_coo<1, 4, 3, FT, NIN>(a, recs, ntiles, s);
    if (R <= 8) return launch_coo<2, 4, 3, FT, NIN>(a, recs, ntiles, s);
    if (R <= 16) return launch_coo<4, 4, 3, FT, NIN>(a, recs, ntiles, s);
    if (R <= 32) return launch_coo<8, 4, 3, FT, NIN>(a, recs, ntiles, s);
    if (R <= 64) return launch_coo<16, 4, 2, FT, NIN>(a, recs, ntiles, s);
    return launch_coo<32, 4, 2, FT, NIN>(a, recs, ntiles, s);
}

template <class FT>
static int launch_n(int nin, bool hicoo, bool wide, const SchedArgs &a, const uint32_t *recs, unsigned ntiles,
                    cudaStream_t s)
{
    switch (nin) {
        case 1: return launch_r<FT, 1>(hicoo, wide, a, recs, ntiles, s);
        case 2: return launch_r<FT, 2>(hicoo, wide, a, recs, ntiles, s);
        default: return launch_r<FT, 3>(hicoo, wide, a, recs, ntiles, s);
    }
}

bool schedule_supported(const ptiB200Tensor *t, uint32_t R)
{
    return t->nmodes >= 2 && t->nmodes <= 4 && R >= 1 && R <= 128;
}

// Runs the scheduled kernel for `mode` (the schedule must be ready).  Output
// must already be zeroed.
int mttkrp_scheduled(ptiB200Tensor *t, const void *const *mats, int ft, uint32_t R, uint32_t stride,
                     const uint32_t *mats_order, uint32_t mode, float *out, cudaStream_t s,
                     const float *vals_override)
{
    const char *mod = "B200 MTTKRP";
    const uint32_t N = t->nmodes;
    PTI_TRY(ensure_err_word(s));
    SchedArgs a{};
    a.nnz = t->nnz;
    a.R = R;
    a.stride = stride;
    a.out_dim = t->ndims[mode];
    a.out = out;
    a.err = err_word();
    const uint32_t *recs = nullptr;
    unsigned ntiles;
    if (t->hicoo) {
        const HicooModePlan &P = t->hicoo_plan[mode];
        ntiles = P.ntiles;
        a.nb = P.nb;
        a.sb = t->sb;
        a.bptr = P.bptr.as<uint64_t>();
        a.tile_block = P.tile_block.as<uint32_t>();
        a.out_bind = P.binds[mode].as<uint32_t>();
        a.out_eind = P.einds[mode].as<uint8_t>();
        for (uint32_t i = 1; i < N; ++i) {
            const uint32_t k = mats_order[i];
            a.in_bind[i - 1] = P.binds[k].as<uint32_t>();
            a.in_eind[i - 1] = P.einds[k].as<uint8_t>();
            a.in_dim[i - 1] = t->ndims[k];
            a.in_mat[i - 1] = mats[k];
        }
        a.vals = P.vals.as<float>();
    } else {
        // records hold the operand modes in increasing order
        ntiles = (unsigned)((t->nnz + kTile - 1) / kTile);
        CooModePlan &P = t->coo_plan[mode];
        recs = P.recs.as<uint32_t>();
        if (vals_override) {  // substituted values, brought into record order
            if (!P.alt_vals.ptr) PTI_CUDA(P.alt_vals.alloc(padded(t->nnz * 4), s), mod);
            gather_kernel<float><<<grid_n(t->nnz), 256, 0, s>>>(vals_override, P.perm.as<uint32_t>(), t->nnz,
                                                                P.alt_vals.as<float>());
            a.vals = P.alt_vals.as<float>();
        }
        for (uint32_t k = 0, i = 0; k < N; ++k)
            if (k != mode) {
                a.in_dim[i] = t->ndims[k];
                a.in_mat[i] = mats[k];
                ++i;
            }
    }
    // BF16 rows are read 8 columns (16 bytes) per lane when every row start
    // is 16-byte aligned.
    bool wide = ft == PTI_B200_BF16 && stride % 8 == 0;
    for (uint32_t k = 0; k < N && wide; ++k)
        if (k != mode && ((uintptr_t)mats[k] & 15) != 0) wide = false;
    int r = ft == PTI_B200_F32 ? launch_n<float>((int)N - 1, t->hicoo, false, a, recs, ntiles, s)
                               : launch_n<__nv_bfloat16>((int)N - 1, t->hicoo, wide, a, recs, ntiles, s);
    PTI_CHECK(r == 0, r, mod, "kernel attribute setup failed");
    PTI_CUDA(cudaGetLastError(), mod);
    return 0;
}

}  // namespace pti
