// gradcp.cu -- the pieces of all-at-once gradient CP on a COO tensor:
//   model(z) = sum_r prod_k A_k[i_k(z), r]     (the CP model at each nonzero)
//   dL/dA_k  = MTTKRP_k(g)                     (g = dL/dmodel at the nonzeros)
// For the loss 0.5 * sum_z (x_z - model(z))^2, g = model - x, so the gradient
// of every factor is a per-mode MTTKRP of the residual; the Hadamard partials
// are recomputed by the MTTKRP kernels rather than stored per nonzero.
#include "kutil.cuh"
#include "tensor.cuh"
#include "tma.cuh"

namespace pti {

uint32_t *err_word(ptiB200Tensor *t);
int ensure_err_word(ptiB200Tensor *t, cudaStream_t s);

struct KVArgs {
    uint64_t nnz;
    uint32_t nmodes, R, stride;
    const uint32_t *inds[kMaxModes];
    const float *mats[kMaxModes];
    float *out;
};

// A group of G lanes per nonzero; each lane multiplies 4 columns across the
// modes and the group sums its lanes with shuffles.  A warp takes 32/G * U
// consecutive nonzeros per pass: their coordinates are read once, coalesced,
// by one lane each and handed to the groups with shuffles, and each group
// then has the rows of U nonzeros in flight.
template <int G, int U, int NM>
__global__ void __launch_bounds__(256) kruskal_values_kernel(KVArgs a)
{
    constexpr uint32_t kGroupsPerWarp = 32 / G;
    constexpr uint32_t kPer = kGroupsPerWarp * U;  // nonzeros per warp and pass (<= 32)
    static_assert(kPer <= 32, "one coordinate per lane");
    const uint32_t lane32 = threadIdx.x % 32, lane = lane32 % G, grp = lane32 / G;
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / 32;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) / 32;
    // the loop bound is uniform across a warp, so every lane reaches the shuffles
    for (uint64_t base = warp * kPer; base < a.nnz; base += nwarps * kPer) {
        uint32_t rows[U][NM];
        const uint64_t zt = base + lane32;
        const bool have = lane32 < kPer && zt < a.nnz;
        uint32_t mine[NM];
#pragma unroll
        for (int k = 0; k < NM; ++k) mine[k] = have && k < (int)a.nmodes ? __ldg(a.inds[k] + zt) : 0u;
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int k = 0; k < NM; ++k)
                rows[u][k] = k < (int)a.nmodes ? __shfl_sync(0xffffffffu, mine[k], grp * U + u) : 0u;
        float s[U];
#pragma unroll
        for (int u = 0; u < U; ++u) s[u] = 0.f;
        for (uint32_t col = lane * 4; col < a.R; col += 4 * G) {
            float4 p[U];
#pragma unroll
            for (int u = 0; u < U; ++u) p[u] = load4(a.mats[0] + (size_t)rows[u][0] * a.stride, col);
#pragma unroll
            for (int k = 1; k < NM; ++k)
                if (k < (int)a.nmodes) {
#pragma unroll
                    for (int u = 0; u < U; ++u)
                        p[u] = mul4(p[u], load4(a.mats[k] + (size_t)rows[u][k] * a.stride, col));
                }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                p[u] = mask4(p[u], col, a.R);
                s[u] += (p[u].x + p[u].y) + (p[u].z + p[u].w);
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int o = G / 2; o > 0; o >>= 1) s[u] += __shfl_xor_sync(0xffffffffu, s[u], o, G);
        if (lane == 0) {
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const uint64_t z = base + grp * U + u;
                if (z < a.nnz) a.out[z] = s[u];
            }
        }
    }
}

// The CP model over the mode-0 COO schedule of a 2- or 3-mode tensor (the
// schedule the residual MTTKRPs walk): records {mode-0 row, other rows,
// value} sorted by the mode-0 row, bulk-copied a tile at a time.  Runs of one
// mode-0 row keep that factor row in registers, so a nonzero gathers the
// other modes' rows only (2 instead of 3 for a 3-mode tensor).  Each value is
// written to its input position (the schedule's permutation).
constexpr uint32_t kKsTile = 2048;  // records per CTA
#ifndef PTI_KS_U
#define PTI_KS_U 3
#endif
// records in flight per lane group: 3 (64 registers, 4 CTAs per SM) measured
// a little faster than 2 (48 registers, 5 CTAs) on a 20M-nonzero tensor
constexpr int kKsU = PTI_KS_U;

struct KSArgs {
    uint64_t nnz;
    uint32_t R, stride;
    const uint32_t *recs;  // 4 words per record
    const uint32_t *perm;  // schedule position -> input nonzero
    const float *mats[3];
    float *out;
    uint32_t *err;
};

template <int G, int NIN>
__global__ void __launch_bounds__(256) kruskal_sched_kernel(KSArgs a)
{
    static_assert(NIN == 1 || NIN == 2, "records of 4 words hold up to 3 modes");
    __shared__ __align__(128) uint4 s_rec[kKsTile];
    __shared__ uint64_t mbar;
    const uint32_t tid = threadIdx.x;
    const uint64_t z0 = (uint64_t)blockIdx.x * kKsTile;
    const uint32_t n = (uint32_t)((a.nnz - z0) < kKsTile ? (a.nnz - z0) : kKsTile);
    if (tid == 0) {
        mbar_init(&mbar, 1);
        mbar_fence_init();
    }
    __syncthreads();
    if (tid == 0) {
        mbar_arrive_expect_tx(&mbar, 16 * n);
        bulk_g2s_ef(s_rec, a.recs + z0 * 4, 16 * n, &mbar);
    }
    const bool ok = mbar_wait_bounded(&mbar, 0);
    if (!__syncthreads_and(ok)) {
        if (tid == 0) {
            atomicOr(a.err, 2u);
            mbar_wait_bounded(&mbar, 0);  // the copy lands before the CTA's shared memory is released
        }
        return;
    }
    constexpr uint32_t kGroups = 256 / G;
    const uint32_t g = tid / G, lane = tid % G;
    // the same slice length for every group, so the warp's groups run the
    // same number of passes (the shuffles below need every lane)
    const uint32_t per = (n + kGroups - 1) / kGroups;
    const uint32_t j0 = min(g * per, n), j1 = min(j0 + per, n);
    const uint32_t col = lane * 4;
    const bool active = col < a.R;
    const uint32_t c0 = active ? col : 0u;  // inactive lanes read column 0 and are masked
    uint32_t cur = 0xFFFFFFFFu;
    float4 arow = make_float4(0.f, 0.f, 0.f, 0.f);
    for (uint32_t t = 0; t < per; t += kKsU) {
        uint4 r[kKsU];
        bool valid[kKsU];
#pragma unroll
        for (int u = 0; u < kKsU; ++u) {
            const uint32_t j = j0 + t + u;
            valid[u] = j < j1;
            r[u] = valid[u] ? s_rec[j] : make_uint4(0u, 0u, 0u, 0u);
        }
        float4 f[kKsU][NIN];
#pragma unroll
        for (int u = 0; u < kKsU; ++u) {
            const uint32_t rows[2] = {r[u].y, r[u].z};
#pragma unroll
            for (int k = 0; k < NIN; ++k) f[u][k] = load4(a.mats[1 + k] + (size_t)rows[k] * a.stride, c0);
        }
        // the mode-0 rows: the cached row while every record of the warp's
        // batch continues it, else one gather per record
        bool same = true;
#pragma unroll
        for (int u = 0; u < kKsU; ++u) same = same && (!valid[u] || r[u].x == cur);
        float4 fa[kKsU];
        if (__all_sync(0xffffffffu, same)) {
#pragma unroll
            for (int u = 0; u < kKsU; ++u) fa[u] = arow;
        } else {
#pragma unroll
            for (int u = 0; u < kKsU; ++u) fa[u] = load4(a.mats[0] + (size_t)r[u].x * a.stride, c0);
#pragma unroll
            for (int u = 0; u < kKsU; ++u)
                if (valid[u]) {
                    cur = r[u].x;
                    arow = fa[u];
                }
        }
        float s[kKsU];
#pragma unroll
        for (int u = 0; u < kKsU; ++u) {
            float4 p = fa[u];
#pragma unroll
            for (int k = 0; k < NIN; ++k) p = mul4(p, f[u][k]);
            p = mask4(p, col, a.R);
            s[u] = (p.x + p.y) + (p.z + p.w);
        }
#pragma unroll
        for (int u = 0; u < kKsU; ++u)
#pragma unroll
            for (int o = G / 2; o > 0; o >>= 1) s[u] += __shfl_xor_sync(0xffffffffu, s[u], o, G);
        if (lane == 0) {
#pragma unroll
            for (int u = 0; u < kKsU; ++u)
                if (valid[u]) a.out[__ldg(a.perm + z0 + j0 + t + u)] = s[u];
        }
    }
}

#ifndef PTI_KV_U
#define PTI_KV_U 2
#endif
// nonzeros in flight per group (32/G * U <= 32): on a 3-D tensor of 20M
// nonzeros at R = 64, 2 gave the fastest gradient (4 costs more registers
// than its extra rows in flight return)
template <int G>
constexpr int kv_u()
{
    return G < PTI_KV_U ? G : PTI_KV_U;
}

static int lanes_for(uint32_t R)
{
    uint32_t q = (R + 3) / 4;
    int g = 1;
    while ((uint32_t)g < q && g < 32) g *= 2;
    return g;
}

template <int NIN>
static int launch_ks(int G, const KSArgs &a, unsigned tiles, cudaStream_t s)
{
    switch (G) {
        case 1: kruskal_sched_kernel<1, NIN><<<tiles, 256, 0, s>>>(a); break;
        case 2: kruskal_sched_kernel<2, NIN><<<tiles, 256, 0, s>>>(a); break;
        case 4: kruskal_sched_kernel<4, NIN><<<tiles, 256, 0, s>>>(a); break;
        case 8: kruskal_sched_kernel<8, NIN><<<tiles, 256, 0, s>>>(a); break;
        case 16: kruskal_sched_kernel<16, NIN><<<tiles, 256, 0, s>>>(a); break;
        default: kruskal_sched_kernel<32, NIN><<<tiles, 256, 0, s>>>(a); break;
    }
    return 0;
}

template <int NM>
static int launch_kv(int G, const KVArgs &a, unsigned grid, cudaStream_t s)
{
    constexpr bool any = NM == kMaxModes;  // any order: one nonzero in flight per group
    switch (G) {
        case 1: kruskal_values_kernel<1, any ? 1 : kv_u<1>(), NM><<<grid, 256, 0, s>>>(a); break;
        case 2: kruskal_values_kernel<2, any ? 1 : kv_u<2>(), NM><<<grid, 256, 0, s>>>(a); break;
        case 4: kruskal_values_kernel<4, any ? 1 : kv_u<4>(), NM><<<grid, 256, 0, s>>>(a); break;
        case 8: kruskal_values_kernel<8, any ? 1 : kv_u<8>(), NM><<<grid, 256, 0, s>>>(a); break;
        case 16: kruskal_values_kernel<16, any ? 1 : kv_u<16>(), NM><<<grid, 256, 0, s>>>(a); break;
        default: kruskal_values_kernel<32, any ? 1 : kv_u<32>(), NM><<<grid, 256, 0, s>>>(a); break;
    }
    return 0;
}

}  // namespace pti

extern "C" {

int ptiB200KruskalValues(ptiB200Tensor *t, const float *const *dev_factors, ptiIndex rank, ptiIndex stride,
                         float *dev_out, void *stream)
{
    using namespace pti;
    const char *mod = "B200 Kruskal values";
    PTI_CHECK(t && dev_factors && dev_out, PTIERR_VALUE_ERROR, mod, "null argument");
    PTI_CHECK(!t->hicoo, PTIERR_VALUE_ERROR, mod, "needs a COO tensor");
    PTI_CHECK(rank >= 1 && stride >= rank && stride % 4 == 0, PTIERR_SHAPE_MISMATCH, mod,
              "stride must be >= rank and a multiple of 4");
    for (uint32_t k = 0; k < t->nmodes; ++k)
        PTI_CHECK(dev_factors[k] && ((uintptr_t)dev_factors[k] & 15) == 0, PTIERR_VALUE_ERROR, mod,
                  "factors must be non-null and 16-byte aligned");
    if (t->nnz == 0) return 0;
    KVArgs a{};
    a.nnz = t->nnz;
    a.nmodes = t->nmodes;
    a.R = rank;
    a.stride = stride;
    for (uint32_t k = 0; k < t->nmodes; ++k) {
        a.inds[k] = t->inds[k].as<uint32_t>();
        a.mats[k] = dev_factors[k];
    }
    a.out = dev_out;
    const int G = lanes_for(rank);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // 2- and 3-mode tensors up to rank 128: over the mode-0 schedule (built
    // here if no MTTKRP has built it yet)
    if ((t->nmodes == 2 || t->nmodes == 3) && rank <= 128 && t->nnz < 0xFFFFFFFFull) {
        PTI_TRY(prepare_mode(t, 0, st));
        PTI_TRY(ensure_err_word(t, st));
        KSArgs k{};
        k.nnz = t->nnz;
        k.R = rank;
        k.stride = stride;
        k.recs = t->coo_plan[0].recs.as<uint32_t>();
        k.perm = t->coo_plan[0].perm.as<uint32_t>();
        for (uint32_t m = 0; m < t->nmodes; ++m) k.mats[m] = dev_factors[m];
        k.out = dev_out;
        k.err = err_word(t);
        const unsigned tiles = (unsigned)((t->nnz + kKsTile - 1) / kKsTile);
        PTI_TRY(t->nmodes == 3 ? launch_ks<2>(G, k, tiles, st) : launch_ks<1>(G, k, tiles, st));
        PTI_CUDA(cudaGetLastError(), mod);
        return 0;
    }
    const unsigned grid = (unsigned)std::max<uint64_t>(
        1, std::min<uint64_t>((t->nnz * G + 255) / 256, (uint64_t)sm_count() * 16));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // 3- and 4-mode tensors: U nonzeros in flight per group; other orders one
    if (t->nmodes == 3) {
        PTI_TRY(launch_kv<3>(G, a, grid, s));
    } else if (t->nmodes == 4) {
        PTI_TRY(launch_kv<4>(G, a, grid, s));
    } else {
        PTI_TRY(launch_kv<kMaxModes>(G, a, grid, s));
    }
    PTI_CUDA(cudaGetLastError(), mod);
    return 0;
}

int ptiB200MTTKRPValues(ptiB200Tensor *t, const float *dev_vals, const void *const *dev_mats, int factor_type,
                        ptiIndex rank, ptiIndex stride, const ptiIndex *mats_order, ptiIndex mode, float *dev_out,
                        void *stream)
{
    PTI_CHECK(t && dev_vals && dev_mats && mats_order && dev_out, PTIERR_VALUE_ERROR, "B200 MTTKRP",
              "null argument");
    return pti::mttkrp_device(t, dev_mats, factor_type, rank, stride, mats_order, mode, dev_out,
                              static_cast<cudaStream_t>(stream), dev_vals);
}

}  // extern "C"
