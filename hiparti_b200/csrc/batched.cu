// batched.cu -- CPD-ALS of many small 3-D tensors at once (no counterpart in
// the reference, whose CPD drivers factor one tensor per call:
// src/sptensor/cpd.c:32-208, src/sptensor/hicoo/cpd.c).
//
// Every tensor of the batch is converted to HiCOO on the GPU and given the
// per-mode schedules of sched.cu (blocks ordered by output block row, cut into
// tiles of kPlanTile nonzeros).  One ALS iteration of the WHOLE batch is one
// launch of a persistent kernel whose CTAs pull tasks from a queue:
//
//   tile task  (b, m, t)  MTTKRP of tile t of tensor b's mode-m schedule into
//                         M_bm (as in sched.cu: bulk-copied tile already in
//                         output-row order, one vector atomic per row run and
//                         thread group)
//   dense task (b, m)     the mode-m ALS step of tensor b, in FP64:
//                         W = (G_a o G_b)^-1 (Cholesky; Gauss-Jordan fallback),
//                         A_bm = M_bm W, lambda (2-norm in iteration 0, else
//                         max(column max, 1)), A_bm /= lambda, BF16 copy,
//                         G_bm = A_bm^T A_bm, and after the last mode the fit
//                         (src/sptensor/cpd.c:90-147 for one tensor)
//
// The queue is ordered in waves -- all mode-0 tiles, all mode-0 dense steps,
// all mode-1 tiles, ... -- and a task waits (bounded) on per-tensor counters
// for the tasks it depends on.  Tasks are handed out in queue order and only
// depend on earlier tasks, so the earliest unfinished task always has its
// inputs complete and is held by a running CTA: the queue makes progress
// whatever the number of co-resident CTAs.
//
// Data written inside the launch (factors, M, Grams) is read with L2-coherent
// loads (ld.global.cg) after an acquire on the counter; static data (the
// schedules) uses the read-only path and bulk copies.
//
// The iteration (counter reset, persistent kernel, iteration-counter bump) is
// captured once per call in a CUDA graph and replayed; the kernel reads the
// iteration number from device memory, so one graph serves the BF16 and the
// closing FP32 iterations alike.
//
// An autotuner picks the HiCOO block size (sb_bits) and the columns per lane
// of the BF16 iterations (4 or 8, i.e. R/4 or R/8 threads per nonzero) by
// timing whole iterations of the batch, and caches the choice per batch shape.
#include <cuda_bf16.h>

#include <algorithm>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <tuple>

#include "kutil.cuh"
#include "spd.cuh"
#include "tensor.cuh"
#include "tma.cuh"

namespace pti {

constexpr int kBThreads = 256;
constexpr int kBMaxRank = 32;
constexpr int kRowPad = 40;                     // row stride (doubles) of the dense passes' row tiles
constexpr int kBTile = kPlanTile;
constexpr uint64_t kWaitNs = 2000000000ull;     // bound of every dependency wait: 2 s

// error bits of the batch's error word
constexpr uint32_t kErrRange = 1u, kErrCopy = 2u, kErrWait = 4u;

struct BatchPlan {        // the mode-m schedule of tensor b
    uint64_t nnz, nb;
    const uint16_t *lblk;             // block of each nonzero within its tile
    const uint32_t *tile_block;
    const uint32_t *out_bind;
    const uint32_t *in_bind[2];
    const uint8_t *out_eind;
    const uint8_t *in_eind[2];
    const float *vals;
    float *M;                         // MTTKRP output, dims[m] x stride
    const float *A32[2];              // operand factors (modes k != m, increasing)
    const __nv_bfloat16 *A16[2];
    uint32_t ntiles, sb, R, stride, out_dim, in_dim[2];
};

struct BatchTensor {
    float *A[3];                      // FP32 factors, dims[m] x stride
    __nv_bfloat16 *Ab[3];             // BF16 copies read by the MTTKRP in mixed mode
    float *M[3];
    double *G;                        // [3][R][R] Grams
    float *lambda;                    // [R]
    const double *normX2;             // ||X||^2
    uint32_t dims[3];
    uint32_t R, stride;
};

struct BatchArgs {
    const uint2 *tasks;               // x = (plan << 1) | dense, y = tile
    const BatchPlan *plans;           // [B*3], plan = b*3 + m
    const BatchTensor *tens;          // [B]
    uint32_t *ctrl;                   // [0] queue head, [1, 1+3B) tiles done, [1+3B, 1+4B) dense steps done
    const uint32_t *iter;             // iteration number (bumped after every launch)
    double *fits;                     // [B][niters]
    uint32_t *err;
    uint32_t ntasks, ntensors, niters, fp32_sweeps, cpl;
    int mixed;
    uint64_t wait_ns;                 // bound of every dependency wait
};

__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t *p)
{
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Waits until *p >= target.  Gives up (false) after wait_ns, after 2^28
// polls should the timer not advance, or as soon as another wait of the
// launch has given up (err holds kErrWait), so a failed launch ends within
// about one wait bound instead of one per task.
__device__ bool wait_at_least(const uint32_t *p, uint32_t target, const uint32_t *err, uint64_t wait_ns)
{
    if (ld_acquire(p) >= target) return true;
    const uint64_t t0 = global_ns();
    for (uint32_t i = 0; i < (1u << 28); ++i) {
        __nanosleep(64);
        if (ld_acquire(p) >= target) return true;
        if ((i & 255u) == 255u &&
            (global_ns() - t0 > wait_ns || (*(volatile const uint32_t *)err & kErrWait))) return false;
    }
    return false;
}

// CPL consecutive columns of a factor row, loaded through L2 (the factors
// change during the launch, so the non-coherent read-only path is not used).
template <int CPL, class FT>
struct Cols {
    static constexpr int kWords = CPL * (int)sizeof(FT) / 4;
    uint32_t w[kWords];
    __device__ __forceinline__ void load(const FT *row, uint32_t col)
    {
        const FT *p = row + col;
        if constexpr (kWords == 8) {
            const uint4 x = __ldcg(reinterpret_cast<const uint4 *>(p));
            const uint4 y = __ldcg(reinterpret_cast<const uint4 *>(p) + 1);
            w[0] = x.x; w[1] = x.y; w[2] = x.z; w[3] = x.w;
            w[4] = y.x; w[5] = y.y; w[6] = y.z; w[7] = y.w;
        } else if constexpr (kWords == 4) {
            const uint4 x = __ldcg(reinterpret_cast<const uint4 *>(p));
            w[0] = x.x; w[1] = x.y; w[2] = x.z; w[3] = x.w;
        } else {
            const uint2 x = __ldcg(reinterpret_cast<const uint2 *>(p));
            w[0] = x.x; w[1] = x.y;
        }
    }
    __device__ __forceinline__ float at(int c) const
    {
        if constexpr (sizeof(FT) == 4) {
            return __uint_as_float(w[c]);
        } else {
            const uint32_t h = w[c >> 1];
            return __uint_as_float((c & 1) ? (h & 0xFFFF0000u) : (h << 16));
        }
    }
};

// Shared-memory layout of a tile task (bytes).
struct TileSmem {
    static constexpr uint32_t val = 0;                          // float[kBTile]
    static constexpr uint32_t eout = val + 4 * kBTile;          // u8[kBTile]
    static constexpr uint32_t ein = eout + kBTile;              // u8[2][kBTile]
    static constexpr uint32_t blk = ein + 2 * kBTile;           // u16[kBTile]
    static constexpr uint32_t brow = blk + 2 * kBTile;          // u32[kBTile + 4]
    static constexpr uint32_t bin = brow + 4 * (kBTile + 4);    // u32[2][kBTile + 4]
    static constexpr uint32_t rec = bin + 8 * (kBTile + 4);     // u32[3][kBTile]: decoded output and operand rows
    static constexpr uint32_t total = rec + 12 * kBTile;
};

// Shared-memory layout of a dense task (doubles unless noted).
struct DenseSmem {
    static constexpr uint32_t RR = kBMaxRank * kBMaxRank;
    static constexpr uint32_t V = 0, L = V + 8 * RR, Li = L + 8 * RR, W = Li + 8 * RR, Gs = W + 8 * RR;
    static constexpr uint32_t Wf = Gs + 8 * RR;                 // double[8 k-steps][4 n-tiles][32 lanes]
    static constexpr uint32_t rows = Wf + 8 * RR;               // double[warps][8][kRowPad]
    static constexpr uint32_t colsq = rows + 8 * (kBThreads / 32) * 8 * kRowPad;  // double[32]
    static constexpr uint32_t red = colsq + 8 * kBMaxRank;      // double[kBThreads/32 + 1]
    static constexpr uint32_t lam = red + 8 * (kBThreads / 32 + 1);  // float[32]
    static constexpr uint32_t colmax = lam + 4 * kBMaxRank;     // int[32]
    static constexpr uint32_t total = colmax + 4 * kBMaxRank;
};

constexpr uint32_t kBatchSmem = TileSmem::total > DenseSmem::total ? TileSmem::total : DenseSmem::total;
static_assert(TileSmem::rec % 16 == 0 && kBatchSmem <= 76 * 1024, "three CTAs per SM must fit");

// D += A B for one 8x8x4 FP64 tensor-core tile (mma.sync m8n8k4): lane l holds
// A[l/4][l%4], B[l%4][l/4] and D[l/4][2(l%4)], D[l/4][2(l%4)+1].
__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

__device__ __forceinline__ uint32_t round16u(uint32_t x) { return (x + 15u) & ~15u; }

// One tile of a mode-m schedule: a group of 2^glog lanes x CPL columns per
// nonzero (the group size is chosen from the tensor's rank at run time, so a
// kernel holds one tile variant).  The schedule keeps each tile's nonzeros in
// output-row order, so a group walks a contiguous slice and adds a row into
// M once per run.  Returns false (uniformly over the CTA) if the tile's bulk
// copies did not complete within the wait bound.
template <int CPL, class FT>
__device__ bool tile_task(const BatchPlan *__restrict__ gp, uint32_t tile, unsigned char *sm, uint64_t *mbar,
                          uint32_t &phase, uint32_t *err)
{
    constexpr int U = 4;  // nonzeros in flight per group
    float *s_val = reinterpret_cast<float *>(sm + TileSmem::val);
    uint8_t *s_eout = sm + TileSmem::eout;
    uint8_t *s_ein = sm + TileSmem::ein;
    uint16_t *s_blk = reinterpret_cast<uint16_t *>(sm + TileSmem::blk);
    uint32_t *s_brow = reinterpret_cast<uint32_t *>(sm + TileSmem::brow);
    uint32_t *s_bin = reinterpret_cast<uint32_t *>(sm + TileSmem::bin);
    const uint32_t tid = threadIdx.x;

    const uint64_t nnz = gp->nnz, nb = gp->nb;
    const uint32_t sb = gp->sb, R = gp->R, stride = gp->stride, out_dim = gp->out_dim;
    const uint32_t in_dim0 = gp->in_dim[0], in_dim1 = gp->in_dim[1];
    const uint64_t z0 = (uint64_t)tile * kBTile;
    const uint32_t n = (uint32_t)((nnz - z0) < (uint64_t)kBTile ? (nnz - z0) : (uint64_t)kBTile);
    const uint32_t b0 = __ldg(gp->tile_block + tile);
    uint32_t nblk = __ldg(gp->tile_block + tile + 1) - b0 + 1;
    if (nblk > kBTile + 1) nblk = kBTile + 1;
    if (b0 + (uint64_t)nblk > nb) nblk = (uint32_t)(nb - b0);
    const uint32_t bo4 = b0 & 3u;  // block coordinates are copied from b0 rounded down to 16 bytes

    if (tid == 0) {
        const uint32_t be = round16u(n), bv = round16u(4 * n), bl = round16u(2 * n);
        const uint32_t bb = 4 * ((nblk + bo4 + 3) & ~3u);
        mbar_arrive_expect_tx(mbar, bv + 3 * be + bl + 3 * bb);
        bulk_g2s_ef(s_val, gp->vals + z0, bv, mbar);
        bulk_g2s_ef(s_eout, gp->out_eind + z0, be, mbar);
        bulk_g2s_ef(s_ein, gp->in_eind[0] + z0, be, mbar);
        bulk_g2s_ef(s_ein + kBTile, gp->in_eind[1] + z0, be, mbar);
        bulk_g2s_ef(s_blk, gp->lblk + z0, bl, mbar);
        bulk_g2s_ef(s_brow, gp->out_bind + (b0 - bo4), bb, mbar);
        bulk_g2s_ef(s_bin, gp->in_bind[0] + (b0 - bo4), bb, mbar);
        bulk_g2s_ef(s_bin + (kBTile + 4), gp->in_bind[1] + (b0 - bo4), bb, mbar);
    }
    const bool ok = mbar_wait_bounded(mbar, phase);
    if (!__syncthreads_and(ok)) {
        // Copies still in flight would land in the staging area of a later
        // task: wait once more (bounded) for this phase.  The caller then
        // stops issuing bulk copies in this CTA, so the barrier is never
        // re-armed while this phase may still be open.
        if (tid == 0) {
            atomicOr(err, kErrCopy);
            mbar_wait_bounded(mbar, phase);
        }
        return false;
    }
    phase ^= 1u;
    s_brow += bo4;
    s_bin += bo4;
    // decode every nonzero once: output row (or a marker for a bad
    // coordinate) and operand rows, into shared memory beside the tile
    uint32_t *s_ro = reinterpret_cast<uint32_t *>(sm + TileSmem::rec);
    uint32_t *s_r0 = s_ro + kBTile, *s_r1 = s_r0 + kBTile;
    for (uint32_t z = tid; z < n; z += kBThreads) {
        const uint32_t i = s_blk[z];
        const uint32_t o = (s_brow[i] << sb) + s_eout[z];
        const uint32_t r0 = (s_bin[i] << sb) + s_ein[z];
        const uint32_t r1 = (s_bin[(kBTile + 4) + i] << sb) + s_ein[kBTile + z];
        const bool ok_z = i < nblk && o < out_dim && r0 < in_dim0 && r1 < in_dim1;
        if (!ok_z) atomicOr(err, kErrRange);
        s_ro[z] = ok_z ? o : 0xFFFFFFFFu;
        s_r0[z] = r0;
        s_r1[z] = r1;
    }
    __syncthreads();

    const FT *mat0, *mat1;
    if constexpr (sizeof(FT) == 4) {
        mat0 = reinterpret_cast<const FT *>(gp->A32[0]);
        mat1 = reinterpret_cast<const FT *>(gp->A32[1]);
    } else {
        mat0 = reinterpret_cast<const FT *>(gp->A16[0]);
        mat1 = reinterpret_cast<const FT *>(gp->A16[1]);
    }
    float *out = gp->M;
    const uint32_t need = (R + CPL - 1) / CPL;
    const uint32_t glog = need <= 1 ? 0u : 32u - __clz(need - 1);
    const uint32_t g = tid >> glog, lane = tid & ((1u << glog) - 1u);
    const uint32_t kGroups = (uint32_t)kBThreads >> glog;
    const uint32_t col = lane * CPL;
    const bool active = col < R;
    // an odd slice length puts the groups' first nonzeros on different banks
    const uint32_t per = ((n + kGroups - 1) >> (8u - glog)) | 1u;
    const uint32_t j0 = min(g * per, n), j1 = min(j0 + per, n);
    float acc[CPL];
#pragma unroll
    for (int c = 0; c < CPL; ++c) acc[c] = 0.f;
    uint32_t cur = 0xFFFFFFFFu;
    auto flush = [&](uint32_t row) {
#pragma unroll
        for (int q = 0; q < CPL / 4; ++q)
            if (col + 4 * q < R)
                red_add4(out + (size_t)row * stride + col + 4 * q,
                         mask4(make_float4(acc[4 * q], acc[4 * q + 1], acc[4 * q + 2], acc[4 * q + 3]),
                               col + 4 * q, R));
    };
    for (uint32_t j = j0; j < j1; j += U) {
        uint32_t orow[U];
        float v[U];
        Cols<CPL, FT> f0[U], f1[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            orow[u] = 0xFFFFFFFFu;
            if (j + u >= j1) continue;
            const uint32_t z = j + u;
            orow[u] = s_ro[z];
            v[u] = s_val[z];
            if (orow[u] != 0xFFFFFFFFu && active) {
                f0[u].load(mat0 + (size_t)s_r0[z] * stride, col);
                f1[u].load(mat1 + (size_t)s_r1[z] * stride, col);
            }
        }
        auto add = [&](int u) {
            const float2 vv = make_float2(v[u], v[u]);
#pragma unroll
            for (int c = 0; c < CPL; c += 2) {
                float2 p;
                if constexpr (sizeof(FT) == 2) p = bf16x2_mul(f0[u].w[c >> 1], f1[u].w[c >> 1]);
                else p = __fmul2_rn(make_float2(f0[u].at(c), f0[u].at(c + 1)), make_float2(f1[u].at(c), f1[u].at(c + 1)));
                const float2 r = __ffma2_rn(p, vv, make_float2(acc[c], acc[c + 1]));
                acc[c] = r.x;
                acc[c + 1] = r.y;
            }
        };
        // every group of the warp still walking continues its row: no row
        // bookkeeping for this batch
        bool same = cur != 0xFFFFFFFFu;
#pragma unroll
        for (int u = 0; u < U; ++u) same = same && orow[u] == cur;
        if (__all_sync(__activemask(), same)) {
            if (active) {
#pragma unroll
                for (int u = 0; u < U; ++u) add(u);
            }
            continue;
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
            if (active) add(u);
        }
    }
    if (cur != 0xFFFFFFFFu && active) flush(cur);
    return true;
}

// Block-wide sum of one double per thread; the result is returned to every
// thread.  red holds kBThreads/32 + 1 doubles.
__device__ double block_sum(double x, double *red)
{
    const uint32_t tid = threadIdx.x;
    for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    __syncthreads();
    if ((tid & 31) == 0) red[tid >> 5] = x;
    __syncthreads();
    if (tid == 0) {
        double s = 0.0;
        for (int w = 0; w < kBThreads / 32; ++w) s += red[w];
        red[kBThreads / 32] = s;
    }
    __syncthreads();
    return red[kBThreads / 32];
}

// Accumulates G += v v^T for one row held one column per lane (lanes >= R hold
// 0): lane c keeps row c of G in g[].
__device__ __forceinline__ void gram_row(double (&g)[kBMaxRank], float v, uint32_t R)
{
#pragma unroll
    for (int k = 0; k < kBMaxRank; ++k) {
        if (k < (int)R) {
            const float vk = __shfl_sync(0xffffffffu, v, k);
            g[k] = fma((double)v, (double)vk, g[k]);
        }
    }
}

// The mode-m ALS step of one tensor (one CTA).  With gram_bf16 (the
// iterations whose MTTKRPs gather BF16 factors) the new Gram is formed from
// the BF16-rounded factor, the values those gathers read, so that the next
// steps' right-hand sides and normal matrices come from the same factors.
__device__ void dense_task(const BatchTensor *__restrict__ gt, uint32_t b, uint32_t m, uint32_t it,
                           const BatchArgs &a, unsigned char *sm, bool gram_bf16)
{
    double *V = reinterpret_cast<double *>(sm + DenseSmem::V);
    double *Lm = reinterpret_cast<double *>(sm + DenseSmem::L);
    double *Li = reinterpret_cast<double *>(sm + DenseSmem::Li);
    double *W = reinterpret_cast<double *>(sm + DenseSmem::W);
    double *Gs = reinterpret_cast<double *>(sm + DenseSmem::Gs);
    double *s_colsq = reinterpret_cast<double *>(sm + DenseSmem::colsq);
    double *s_red = reinterpret_cast<double *>(sm + DenseSmem::red);
    float *s_lam = reinterpret_cast<float *>(sm + DenseSmem::lam);
    int *s_colmax = reinterpret_cast<int *>(sm + DenseSmem::colmax);
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr uint32_t kWarps = kBThreads / 32;
    const uint32_t R = gt->R, stride = gt->stride, RR = R * R, I = gt->dims[m];
    double *G = gt->G;
    float *A = gt->A[m];
    const float *M = gt->M[m];
    __nv_bfloat16 *Ab = gt->Ab[m];
    const uint32_t ma = (m + 1) % 3, mb = (m + 2) % 3;

    for (uint32_t e = tid; e < RR; e += kBThreads) {
        V[e] = __ldcg(G + (size_t)ma * RR + e) * __ldcg(G + (size_t)mb * RR + e);
        Gs[e] = 0.0;
    }
    if (tid < kBMaxRank) {
        s_colsq[tid] = 0.0;
        s_colmax[tid] = 0;
    }
    __syncthreads();
    spd_inverse(V, Lm, Li, W, R);

    // B operands of pass 1 in fragment order: Wf[kt][nt][lane] = W[4kt + lane%4][8nt + lane/4]
    double *Wf = reinterpret_cast<double *>(sm + DenseSmem::Wf);
    for (uint32_t e = tid; e < 8 * 4 * 32; e += kBThreads) {
        const uint32_t l = e & 31, nt = (e >> 5) & 3, kt = e >> 7;
        const uint32_t k = 4 * kt + (l & 3), c = 8 * nt + (l >> 2);
        Wf[e] = (k < R && c < R) ? W[k * R + c] : 0.0;
    }
    __syncthreads();

    // The passes run on the FP64 tensor cores (mma.sync m8n8k4), one warp per
    // block of 8 rows; lane l is (g, t) = (l/4, l%4).
    const uint32_t g8 = lane >> 2, t4 = lane & 3;
    const uint32_t KT = (R + 3) / 4, NT = (R + 7) / 8;  // k-steps and 8-column tiles (NT * 8 == stride)
    const uint32_t nblk8 = (I + 7) / 8;
    const bool colok = lane < R;

    // pass 1: A = M W, with column sums of squares and maxima
    {
        double csq[8];
        float cmx[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            csq[j] = 0.0;
            cmx[j] = 0.f;
        }
        float anext[8];
        auto load_a = [&](uint32_t blk, float (&av)[8]) {
            const uint32_t row = blk * 8 + g8;
#pragma unroll
            for (int kt = 0; kt < 8; ++kt) {
                const uint32_t k = 4 * kt + t4;
                av[kt] = (blk < nblk8 && row < I && k < R) ? __ldcg(M + (size_t)row * stride + k) : 0.f;
            }
        };
        uint32_t blk = warp;
        load_a(blk, anext);
        for (; blk < nblk8; blk += kWarps) {
            float av[8];
#pragma unroll
            for (int kt = 0; kt < 8; ++kt) av[kt] = anext[kt];
            load_a(blk + kWarps, anext);
            double c[4][2];
#pragma unroll
            for (int nt = 0; nt < 4; ++nt) c[nt][0] = c[nt][1] = 0.0;
#pragma unroll
            for (int kt = 0; kt < 8; ++kt) {
                if (kt < (int)KT) {
                    const double a = (double)av[kt];
#pragma unroll
                    for (int nt = 0; nt < 4; ++nt)
                        if (nt < (int)NT) dmma(c[nt][0], c[nt][1], a, Wf[(kt * 4 + nt) * 32 + lane]);
                }
            }
            const uint32_t row = blk * 8 + g8;
#pragma unroll
            for (int nt = 0; nt < 4; ++nt) {
                if (nt >= (int)NT) break;
#pragma unroll
                for (int i = 0; i < 2; ++i) {
                    const uint32_t col = 8 * nt + 2 * t4 + i;
                    const float v = col < R ? (float)c[nt][i] : 0.f;
                    if (row < I) {
                        A[(size_t)row * stride + col] = v;
                        csq[2 * nt + i] += (double)v * (double)v;
                        cmx[2 * nt + i] = fmaxf(cmx[2 * nt + i], v);
                    }
                }
            }
        }
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
            if (nt >= (int)NT) break;
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const uint32_t col = 8 * nt + 2 * t4 + i;
                if (col < R) {
                    atomicAdd(&s_colsq[col], csq[2 * nt + i]);
                    atomicMax(&s_colmax[col], __float_as_int(cmx[2 * nt + i]));
                }
            }
        }
    }
    __syncthreads();
    // lambda: 2-norm in the first iteration (src/matrix/matrix.c:389-469),
    // max(column max, 1) afterwards (:472-553)
    const float lam = colok ? (it == 0 ? (float)sqrt(s_colsq[lane])
                                       : fmaxf(__int_as_float(s_colmax[lane]), 1.f))
                            : 1.f;
    if (warp == 0 && colok) s_lam[lane] = lam;

    // pass 2: A /= lambda, BF16 copy, <X, model> for the fit, and the Gram
    // A^T A on the tensor cores: the warp's 8 scaled rows go through a
    // shared-memory tile, each half (4 rows) is one k-step for the tiles
    // (p, q), p <= q, of the symmetric Gram.
    const bool last = m == 2;
    double inner = 0.0;
    {
        double *tile = reinterpret_cast<double *>(sm + DenseSmem::rows) + warp * (8 * kRowPad);
        double gacc[10][2];
#pragma unroll
        for (int j = 0; j < 10; ++j) gacc[j][0] = gacc[j][1] = 0.0;
        for (uint32_t blk = warp; blk < nblk8; blk += kWarps) {
            float v[8], mm[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const uint32_t row = blk * 8 + q;
                const bool here = colok && row < I;
                v[q] = here ? A[(size_t)row * stride + lane] : 0.f;
                mm[q] = here && last ? __ldcg(M + (size_t)row * stride + lane) : 0.f;
            }
            __syncwarp();
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const uint32_t row = blk * 8 + q;
                if (colok) v[q] = v[q] / lam;
                const __nv_bfloat16 h = __float2bfloat16_rn(colok ? v[q] : 0.f);
                // the value the next MTTKRPs gather (and the fit's model uses)
                const double used = gram_bf16 ? (double)__bfloat162float(h) : (double)v[q];
                if (colok && row < I) {
                    A[(size_t)row * stride + lane] = v[q];
                    if (last) inner += (double)lam * used * (double)mm[q];
                }
                if (a.mixed && lane < stride && row < I) Ab[(size_t)row * stride + lane] = h;
                tile[q * kRowPad + lane] = used;
            }
            __syncwarp();
#pragma unroll
            for (int ks = 0; ks < 2; ++ks) {
                double fr[4];
#pragma unroll
                for (int nt = 0; nt < 4; ++nt) fr[nt] = tile[(4 * ks + t4) * kRowPad + 8 * nt + g8];
                int j = 0;
#pragma unroll
                for (int pt = 0; pt < 4; ++pt)
#pragma unroll
                    for (int qt = pt; qt < 4; ++qt, ++j)
                        if (qt < (int)NT) dmma(gacc[j][0], gacc[j][1], fr[pt], fr[qt]);
            }
            __syncwarp();
        }
        // add the warp's tiles into the Gram: tile (p, q) holds G[8p + g][8q + 2t + i]
        int j = 0;
#pragma unroll
        for (int pt = 0; pt < 4; ++pt)
#pragma unroll
            for (int qt = pt; qt < 4; ++qt, ++j) {
                if (qt >= (int)NT) continue;
#pragma unroll
                for (int i = 0; i < 2; ++i) {
                    const uint32_t r = 8 * pt + g8, c = 8 * qt + 2 * t4 + i;
                    if (r < R && c < R) {
                        atomicAdd(&Gs[r * R + c], gacc[j][i]);
                        if (pt != qt) atomicAdd(&Gs[c * R + r], gacc[j][i]);
                    }
                }
            }
    }
    // zero the next mode's MTTKRP output (its tiles wait for this step)
    {
        const uint32_t mn = (m + 1) % 3;
        float4 *Mn = reinterpret_cast<float4 *>(gt->M[mn]);
        const size_t n4 = (size_t)gt->dims[mn] * stride / 4;
        for (size_t e = tid; e < n4; e += kBThreads) Mn[e] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    const double inner_all = last ? block_sum(inner, s_red) : 0.0;  // ends with a barrier
    __syncthreads();
    for (uint32_t e = tid; e < RR; e += kBThreads) G[(size_t)m * RR + e] = Gs[e];
    if (tid < R) gt->lambda[tid] = s_lam[tid];
    if (last) {
        // fit = 1 - sqrt(||X||^2 + |lambda^T (G_0 o G_1 o G_2) lambda| - 2 <X, model>) / ||X||
        // (src/ktensor/ktensor.c:77-99, with full symmetric Grams)
        double s = 0.0;
        for (uint32_t e = tid; e < RR; e += kBThreads)
            s += __ldcg(G + e) * __ldcg(G + RR + e) * Gs[e] * (double)s_lam[e / R] * (double)s_lam[e % R];
        const double norm_mats = fabs(block_sum(s, s_red));
        if (tid == 0) {
            const double nx = *gt->normX2;
            double residual = nx + norm_mats - 2.0 * inner_all;
            if (residual > 0.0) residual = sqrt(residual);
            a.fits[(size_t)b * a.niters + it] = 1.0 - residual / sqrt(nx);
        }
    }
}

// One ALS iteration of the batch; CPL columns per lane and factor type FT for
// the MTTKRP gathers (BF16 iterations and FP32 iterations launch different
// instantiations).
template <int CPL, class FT>
__global__ void __launch_bounds__(kBThreads, 2) batch_als_kernel(BatchArgs a)
{
    extern __shared__ __align__(128) unsigned char sm[];
    __shared__ uint64_t mbar;
    __shared__ uint32_t s_q;
    __shared__ int s_ok;
    __shared__ int s_copies_ok;  // 0 once a tile's bulk copies missed their wait bound
    const uint32_t tid = threadIdx.x;
    const uint32_t it = *a.iter;
    uint32_t *head = a.ctrl, *tiles_done = a.ctrl + 1, *dense_done = a.ctrl + 1 + 3 * a.ntensors;
    if (tid == 0) {
        mbar_init(&mbar, 1);
        mbar_fence_init();
        s_copies_ok = 1;
    }
    uint32_t phase = 0;
    __syncthreads();
    for (;;) {
        if (tid == 0) s_q = atomicAdd(head, 1u);
        __syncthreads();
        const uint32_t q = s_q;
        if (q >= a.ntasks) break;
        const uint2 task = __ldg(a.tasks + q);
        const bool dense = task.x & 1u;
        const uint32_t pid = task.x >> 1, b = pid / 3, m = pid % 3;
        if (tid == 0) {
            bool ok = wait_at_least(dense_done + b, m, a.err, a.wait_ns);
            if (ok && dense) ok = wait_at_least(tiles_done + pid, __ldg(&a.plans[pid].ntiles), a.err, a.wait_ns);
            __threadfence();
            if (!ok) atomicOr(a.err, kErrWait);
            s_ok = ok;
        }
        __syncthreads();
        if (s_ok) {
            if (dense) dense_task(a.tens + b, b, m, it, a, sm, sizeof(FT) == 2);
            else if (s_copies_ok && !tile_task<CPL, FT>(a.plans + pid, task.y, sm, &mbar, phase, a.err) && tid == 0)
                s_copies_ok = 0;  // read by the next task after the barrier below
        }
        // shared memory written by this task may next be filled by bulk copies
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            atomicAdd(dense ? dense_done + b : tiles_done + pid, 1u);
        }
    }
}

__global__ void bump_kernel(uint32_t *iter) { *iter += 1; }

// Grams of the current factors and their BF16 copies; one CTA per (tensor,
// mode).  With round_bf16 the Grams are of the BF16-rounded factors (the
// values the BF16 iterations gather, see dense_task).
__global__ void __launch_bounds__(kBThreads) batch_init_kernel(const BatchTensor *tens, int mixed, int round_bf16)
{
    __shared__ double Gs[kBMaxRank * kBMaxRank];
    const BatchTensor *gt = tens + blockIdx.x / 3;
    const uint32_t m = blockIdx.x % 3;
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t R = gt->R, stride = gt->stride, RR = R * R, I = gt->dims[m];
    const float *A = gt->A[m];
    __nv_bfloat16 *Ab = gt->Ab[m];
    for (uint32_t e = tid; e < RR; e += kBThreads) Gs[e] = 0.0;
    __syncthreads();
    double g[kBMaxRank];
#pragma unroll
    for (int k = 0; k < kBMaxRank; ++k) g[k] = 0.0;
    for (uint32_t i = warp; i < I; i += kBThreads / 32) {
        const size_t e = (size_t)i * stride + lane;
        const float v = lane < R ? A[e] : 0.f;
        const __nv_bfloat16 h = __float2bfloat16_rn(v);
        if (mixed && lane < stride) Ab[e] = h;
        gram_row(g, round_bf16 ? __bfloat162float(h) : v, R);
    }
    if (lane < R) {
#pragma unroll
        for (int k = 0; k < kBMaxRank; ++k)
            if (k < (int)R) atomicAdd(&Gs[lane * R + k], g[k]);
    }
    __syncthreads();
    for (uint32_t e = tid; e < RR; e += kBThreads) gt->G[(size_t)m * RR + e] = Gs[e];
}

// ||X||^2 of every tensor; one CTA per tensor.
__global__ void batch_norm_kernel(const float *const *vals, const uint64_t *nnz, double *out)
{
    __shared__ double red[kBThreads / 32 + 1];
    const float *v = vals[blockIdx.x];
    const uint64_t n = nnz[blockIdx.x];
    double s = 0.0;
    for (uint64_t i = threadIdx.x; i < n; i += kBThreads) s += (double)v[i] * (double)v[i];
    s = block_sum(s, red);
    if (threadIdx.x == 0) out[blockIdx.x] = s;
}

// Final lambda (src/matrix/matrix.c:556-572): every column of every factor is
// normalised and lambda takes the norms; one CTA per tensor.
__global__ void __launch_bounds__(kBThreads) batch_final_kernel(const BatchTensor *tens)
{
    __shared__ double s_sq[kBMaxRank];
    const BatchTensor *gt = tens + blockIdx.x;
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t R = gt->R, stride = gt->stride;
    for (uint32_t m = 0; m < 3; ++m) {
        float *A = gt->A[m];
        const uint32_t I = gt->dims[m];
        if (tid < kBMaxRank) s_sq[tid] = 0.0;
        __syncthreads();
        double sq = 0.0;
        for (uint32_t i = warp; i < I; i += kBThreads / 32)
            if (lane < R) {
                const double v = A[(size_t)i * stride + lane];
                sq += v * v;
            }
        if (lane < R) atomicAdd(&s_sq[lane], sq);
        __syncthreads();
        for (uint32_t i = warp; i < I; i += kBThreads / 32)
            if (lane < R) A[(size_t)i * stride + lane] /= (float)sqrt(s_sq[lane]);
        if (tid < R) gt->lambda[tid] *= (float)sqrt(s_sq[tid]);
        __syncthreads();
    }
}

struct CopyItem {
    const float *src;
    float *dst;
    uint64_t n;  // floats
};

// One CTA per item; 16-byte copies where both ends allow them.
__global__ void batch_copy_kernel(const CopyItem *items)
{
    const CopyItem c = items[blockIdx.x];
    if (((uintptr_t)c.src | (uintptr_t)c.dst) % 16 == 0 && c.n % 4 == 0) {
        const float4 *s = reinterpret_cast<const float4 *>(c.src);
        float4 *d = reinterpret_cast<float4 *>(c.dst);
        for (uint64_t i = threadIdx.x; i < c.n / 4; i += blockDim.x) d[i] = s[i];
    } else {
        for (uint64_t i = threadIdx.x; i < c.n; i += blockDim.x) c.dst[i] = c.src[i];
    }
}

// Fills the factor arena with values in [0.1, 1.1) from a hash (used to time
// autotuning candidates on a well-conditioned problem).
__global__ void batch_fill_kernel(float *A, uint64_t n)
{
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t x = i * 0x9E3779B97F4A7C15ull;
        x ^= x >> 31;
        x *= 0xBF58476D1CE4E5B9ull;
        x ^= x >> 29;
        A[i] = 0.1f + (float)(x >> 40) * (1.0f / 16777216.0f);
    }
}

}  // namespace pti

struct ptiB200Batch {
    uint32_t B = 0;
    int device = 0;
    cudaStream_t s = nullptr;
    std::vector<uint32_t> dims, R, stride;  // dims: [B][3]
    std::vector<uint64_t> nnz;
    std::vector<std::unique_ptr<ptiB200Tensor>> coo;  // device COO copies (kept while tuning)
    std::vector<std::unique_ptr<ptiB200Tensor>> hic;  // HiCOO tensors with their per-mode schedules
    int sb = 7, cpl = 4;
    float tune_ms = 0.f, setup_ms = 0.f;
    std::vector<size_t> off;   // element offset of factor (b, m) in the arenas
    std::vector<size_t> goff;  // Gram offset (doubles) of tensor b
    std::vector<size_t> loff;  // lambda offset (floats) of tensor b
    size_t elems = 0;
    pti::DevBuf A, Ab, M, G, lam, norm2, ctrl, misc, plans, tens, tasks, copies;
    uint32_t ntasks = 0;
};

namespace pti {
namespace {

const char *kMod = "B200 Batched CPD-ALS";

int batch_build_plans(ptiB200Batch *bt, int sb)
{
    cudaStream_t s = bt->s;
    const uint32_t B = bt->B;
    for (uint32_t b = 0; b < B; ++b) {
        bt->hic[b].reset();
        ptiB200Tensor *h = nullptr;
        PTI_TRY(ptiB200ConvertToHiCOO(&h, bt->coo[b].get(), (ptiElementIndex)sb, (ptiElementIndex)sb,
                                      (ptiElementIndex)sb, nullptr, nullptr, s));
        bt->hic[b].reset(h);
        for (uint32_t m = 0; m < 3; ++m) PTI_TRY(prepare_mode(h, m, s));
    }
    bt->sb = sb;
    std::vector<BatchPlan> hp(3 * (size_t)B);
    std::vector<uint32_t> ntiles(3 * (size_t)B);
    float *A = bt->A.as<float>();
    auto *Ab = bt->Ab.as<__nv_bfloat16>();
    float *M = bt->M.as<float>();
    for (uint32_t b = 0; b < B; ++b) {
        ptiB200Tensor *h = bt->hic[b].get();
        for (uint32_t m = 0; m < 3; ++m) {
            const HicooModePlan &P = h->hicoo_plan[m];
            BatchPlan p{};
            p.nnz = h->nnz;
            p.nb = P.nb;
            p.lblk = P.lblk.as<uint16_t>();
            p.tile_block = P.tile_block.as<uint32_t>();
            p.out_bind = P.binds[m].as<uint32_t>();
            p.out_eind = P.einds[m].as<uint8_t>();
            for (uint32_t k = 0, i = 0; k < 3; ++k) {
                if (k == m) continue;
                p.in_bind[i] = P.binds[k].as<uint32_t>();
                p.in_eind[i] = P.einds[k].as<uint8_t>();
                p.in_dim[i] = bt->dims[3 * b + k];
                p.A32[i] = A + bt->off[3 * b + k];
                p.A16[i] = Ab + bt->off[3 * b + k];
                ++i;
            }
            p.vals = P.vals.as<float>();
            p.M = M + bt->off[3 * b + m];
            p.ntiles = P.ntiles;
            p.sb = h->sb;
            p.R = bt->R[b];
            p.stride = bt->stride[b];
            p.out_dim = bt->dims[3 * b + m];
            hp[3 * b + m] = p;
            ntiles[3 * b + m] = P.ntiles;
        }
    }
    PTI_CUDA(bt->plans.alloc(padded(hp.size() * sizeof(BatchPlan)), s), kMod);
    PTI_CUDA(cudaMemcpyAsync(bt->plans.ptr, hp.data(), hp.size() * sizeof(BatchPlan), cudaMemcpyHostToDevice, s),
             kMod);

    // the queue: mode-0 tiles (largest tensors first), mode-0 dense steps
    // (costliest first), mode-1 tiles (tensors whose dense step ends first
    // first), ...
    std::vector<uint32_t> order(B);
    std::vector<uint2> tasks;
    auto dense_cost = [&](uint32_t b, uint32_t m) {
        return (uint64_t)bt->dims[3 * b + m] * bt->R[b] * bt->R[b];
    };
    for (uint32_t m = 0; m < 3; ++m) {
        std::iota(order.begin(), order.end(), 0u);
        if (m == 0)
            std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) { return bt->nnz[x] > bt->nnz[y]; });
        else
            std::stable_sort(order.begin(), order.end(),
                             [&](uint32_t x, uint32_t y) { return dense_cost(x, m - 1) < dense_cost(y, m - 1); });
        for (uint32_t b : order)
            for (uint32_t t = 0; t < ntiles[3 * b + m]; ++t) tasks.push_back(make_uint2((3 * b + m) << 1, t));
        std::iota(order.begin(), order.end(), 0u);
        std::stable_sort(order.begin(), order.end(),
                         [&](uint32_t x, uint32_t y) { return dense_cost(x, m) > dense_cost(y, m); });
        for (uint32_t b : order) tasks.push_back(make_uint2(((3 * b + m) << 1) | 1u, 0u));
    }
    bt->ntasks = (uint32_t)tasks.size();
    PTI_CUDA(bt->tasks.alloc(padded(tasks.size() * sizeof(uint2)), s), kMod);
    PTI_CUDA(cudaMemcpyAsync(bt->tasks.ptr, tasks.data(), tasks.size() * sizeof(uint2), cudaMemcpyHostToDevice, s),
             kMod);
    PTI_CUDA(cudaStreamSynchronize(s), kMod);
    return 0;
}

using BatchKernel = void (*)(BatchArgs);

// 8 columns per lane is one 16-byte load of BF16; FP32 iterations always use
// 4 columns (one 16-byte load) per lane.
BatchKernel batch_kernel(int cpl, bool bf16)
{
    if (!bf16) return batch_als_kernel<4, float>;
    return cpl == 8 ? batch_als_kernel<8, __nv_bfloat16> : batch_als_kernel<4, __nv_bfloat16>;
}

// Grid of the persistent kernel: as many CTAs as fit on the GPU at once, at
// most one per task.
int batch_grid(const ptiB200Batch *bt, BatchKernel k, uint32_t *grid)
{
    static std::once_flag once;
    static cudaError_t attr_err = cudaSuccess;
    std::call_once(once, [] {
        for (int cpl : {4, 8})
            for (bool bf16 : {false, true}) {
                const cudaError_t e = cudaFuncSetAttribute(batch_kernel(cpl, bf16),
                                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                           (int)kBatchSmem);
                if (e != cudaSuccess) attr_err = e;
            }
    });
    PTI_CUDA(attr_err, kMod);
    int per_sm = 0;
    PTI_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kBThreads, kBatchSmem), kMod);
    PTI_CHECK(per_sm >= 1, PTIERR_CUDA_ERROR, kMod, "batched kernel does not fit on an SM");
    *grid = (uint32_t)std::min<uint64_t>((uint64_t)per_sm * sm_count(), bt->ntasks);
    return 0;
}

// Captures one iteration (counter reset, persistent kernel, iteration bump).
int batch_capture(ptiB200Batch *bt, const BatchArgs &a, BatchKernel k, cudaGraphExec_t *exec)
{
    cudaStream_t s = bt->s;
    uint32_t grid = 0;
    PTI_TRY(batch_grid(bt, k, &grid));
    cudaGraph_t graph = nullptr;
    PTI_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), kMod);
    cudaMemsetAsync(bt->ctrl.ptr, 0, (1 + 4 * (size_t)bt->B) * 4, s);
    k<<<grid, kBThreads, kBatchSmem, s>>>(a);
    bump_kernel<<<1, 1, 0, s>>>(const_cast<uint32_t *>(a.iter));
    PTI_CUDA(cudaStreamEndCapture(s, &graph), kMod);
    const cudaError_t inst = cudaGraphInstantiate(exec, graph, 0);
    cudaGraphDestroy(graph);
    PTI_CUDA(inst, kMod);
    return 0;
}

// Runs `niters` ALS iterations from the factors in the arena (Grams and BF16
// copies already initialised): the BF16 iterations, then the FP32 ones, each
// phase a replay of its own captured graph.  fits (device, B x niters)
// receives the fits.  *ms: device time per iteration.
int batch_iterate(ptiB200Batch *bt, uint32_t niters, int mixed, uint32_t fp32_sweeps, int cpl, double *fits,
                  float *ms)
{
    cudaStream_t s = bt->s;
    uint32_t *misc = bt->misc.as<uint32_t>();  // [0] iteration, [1] error word
    PTI_CUDA(cudaMemsetAsync(misc, 0, 8, s), kMod);
    BatchArgs a{};
    a.tasks = bt->tasks.as<uint2>();
    a.plans = bt->plans.as<BatchPlan>();
    a.tens = bt->tens.as<BatchTensor>();
    a.ctrl = bt->ctrl.as<uint32_t>();
    a.iter = misc;
    a.fits = fits;
    a.err = misc + 1;
    a.ntasks = bt->ntasks;
    a.ntensors = bt->B;
    a.niters = niters;
    a.fp32_sweeps = fp32_sweeps;
    a.cpl = (uint32_t)cpl;
    a.mixed = mixed;
    a.wait_ns = kWaitNs;
    const uint32_t n16 = mixed && niters > fp32_sweeps ? niters - fp32_sweeps : 0, n32 = niters - n16;
    cudaGraphExec_t g16 = nullptr, g32 = nullptr;
    int r = 0;
    if (n16) r = batch_capture(bt, a, batch_kernel(cpl, true), &g16);
    if (!r && n32) r = batch_capture(bt, a, batch_kernel(cpl, false), &g32);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t lerr = cudaSuccess;
    float t = 0.f;
    if (!r) {
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, s);
        for (uint32_t i = 0; i < n16 && lerr == cudaSuccess; ++i) lerr = cudaGraphLaunch(g16, s);
        if (n16 && n32 && lerr == cudaSuccess) {  // the FP32 sweeps start from Grams of the FP32 factors
            batch_init_kernel<<<3 * bt->B, kBThreads, 0, s>>>(bt->tens.as<BatchTensor>(), mixed, 0);
            lerr = cudaGetLastError();
        }
        for (uint32_t i = 0; i < n32 && lerr == cudaSuccess; ++i) lerr = cudaGraphLaunch(g32, s);
        cudaEventRecord(e1, s);
        const cudaError_t serr = cudaStreamSynchronize(s);
        if (lerr == cudaSuccess) lerr = serr;
        cudaEventElapsedTime(&t, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
    if (g16) cudaGraphExecDestroy(g16);
    if (g32) cudaGraphExecDestroy(g32);
    if (r) return r;
    PTI_CUDA(lerr, kMod);
    if (ms) *ms = t / (float)niters;
    uint32_t err = 0;
    PTI_CUDA(cudaMemcpy(&err, misc + 1, 4, cudaMemcpyDeviceToHost), kMod);
    PTI_CHECK(!(err & kErrRange), PTIERR_VALUE_ERROR, kMod, "tensor coordinate out of range");
    PTI_CHECK(err == 0, PTIERR_CUDA_ERROR, kMod, "a work-queue or copy wait timed out");
    return 0;
}

// round_bf16: the first iterations gather BF16 factors (their Grams are of
// the rounded values)
int batch_init_factors(ptiB200Batch *bt, int mixed, int round_bf16)
{
    cudaStream_t s = bt->s;
    PTI_CUDA(cudaMemsetAsync(bt->M.ptr, 0, bt->elems * 4, s), kMod);
    batch_init_kernel<<<3 * bt->B, kBThreads, 0, s>>>(bt->tens.as<BatchTensor>(), mixed, round_bf16);
    PTI_CUDA(cudaGetLastError(), kMod);
    return 0;
}

struct TuneKey {
    uint32_t B;
    uint64_t nnz_sum, dims_sum, rank_sum;
    int device;
    bool operator<(const TuneKey &o) const
    {
        return std::tie(B, nnz_sum, dims_sum, rank_sum, device) <
               std::tie(o.B, o.nnz_sum, o.dims_sum, o.rank_sum, o.device);
    }
};
std::mutex g_tune_mu;
std::map<TuneKey, std::pair<int, int>> g_tuned;

}  // namespace
}  // namespace pti

extern "C" {

int ptiB200BatchCreate(ptiB200Batch **out, ptiIndex ntensors, const ptiIndex *ndims, const ptiNnzIndex *nnz,
                       const ptiIndex *const *dev_inds, const ptiValue *const *dev_vals, const ptiIndex *ranks,
                       int tune, void *stream)
{
    using namespace pti;
    PTI_CHECK(out && ndims && nnz && dev_inds && dev_vals && ranks, PTIERR_VALUE_ERROR, kMod, "null argument");
    PTI_CHECK(ntensors >= 1 && ntensors <= (1u << 24), PTIERR_VALUE_ERROR, kMod, "ntensors must be in [1, 2^24]");
    for (uint32_t b = 0; b < ntensors; ++b) {
        PTI_CHECK(nnz[b] >= 1 && nnz[b] < 0xFFFFFFFFull, PTIERR_VALUE_ERROR, kMod,
                  "every tensor needs between 1 and 2^32-2 nonzeros");
        PTI_CHECK(ranks[b] >= 1 && ranks[b] <= (uint32_t)kBMaxRank, PTIERR_VALUE_ERROR, kMod,
                  "ranks must be in [1, 32]");
        for (uint32_t m = 0; m < 3; ++m)
            PTI_CHECK(ndims[3 * b + m] >= 1, PTIERR_VALUE_ERROR, kMod, "empty mode");
        PTI_CHECK(dev_vals[b] && dev_inds[3 * b] && dev_inds[3 * b + 1] && dev_inds[3 * b + 2], PTIERR_VALUE_ERROR,
                  kMod, "null tensor array");
    }
    configure_pool_once();
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    auto bt = std::make_unique<ptiB200Batch>();
    cudaGetDevice(&bt->device);
    bt->s = sync_stream();
    cudaStream_t s = bt->s;
    {   // order after the caller's stream
        cudaEvent_t ev;
        PTI_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), kMod);
        cudaEventRecord(ev, static_cast<cudaStream_t>(stream));
        cudaStreamWaitEvent(s, ev, 0);
        cudaEventDestroy(ev);
    }
    cudaEventRecord(t0, s);
    const uint32_t B = ntensors;
    bt->B = B;
    bt->dims.assign(ndims, ndims + 3 * (size_t)B);
    bt->nnz.assign(nnz, nnz + B);
    bt->R.resize(B);
    bt->stride.resize(B);
    bt->coo.resize(B);
    bt->hic.resize(B);
    bt->off.resize(3 * (size_t)B);
    bt->goff.resize(B);
    bt->loff.resize(B);
    size_t elems = 0, gel = 0, lel = 0;
    for (uint32_t b = 0; b < B; ++b) {
        bt->R[b] = ranks[b];
        bt->stride[b] = ((ranks[b] + 7) / 8) * 8;
        for (uint32_t m = 0; m < 3; ++m) {
            bt->off[3 * b + m] = elems;
            elems += (size_t)bt->dims[3 * b + m] * bt->stride[b];
        }
        bt->goff[b] = gel;
        gel += 3 * (size_t)ranks[b] * ranks[b];
        bt->loff[b] = lel;
        lel += ((ranks[b] + 3) / 4) * 4;
    }
    bt->elems = elems;
    for (uint32_t b = 0; b < B; ++b) {
        ptiB200Tensor *t = nullptr;
        PTI_TRY(ptiB200TensorFromDeviceCOO(&t, 3, ndims + 3 * (size_t)b, nnz[b], dev_inds + 3 * (size_t)b,
                                           dev_vals[b], s));
        bt->coo[b].reset(t);
    }
    PTI_CUDA(bt->A.alloc(padded(elems * 4), s), kMod);
    PTI_CUDA(bt->Ab.alloc(padded(elems * 2), s), kMod);
    PTI_CUDA(bt->M.alloc(padded(elems * 4), s), kMod);
    PTI_CUDA(bt->G.alloc(padded(gel * 8), s), kMod);
    PTI_CUDA(bt->lam.alloc(padded(lel * 4), s), kMod);
    PTI_CUDA(bt->norm2.alloc(padded((size_t)B * 8), s), kMod);
    PTI_CUDA(bt->ctrl.alloc(padded((1 + 4 * (size_t)B) * 4), s), kMod);
    PTI_CUDA(bt->misc.alloc(64, s), kMod);
    {
        std::vector<BatchTensor> ht(B);
        for (uint32_t b = 0; b < B; ++b) {
            BatchTensor &T = ht[b];
            for (uint32_t m = 0; m < 3; ++m) {
                T.A[m] = bt->A.as<float>() + bt->off[3 * b + m];
                T.Ab[m] = bt->Ab.as<__nv_bfloat16>() + bt->off[3 * b + m];
                T.M[m] = bt->M.as<float>() + bt->off[3 * b + m];
                T.dims[m] = bt->dims[3 * b + m];
            }
            T.G = bt->G.as<double>() + bt->goff[b];
            T.lambda = bt->lam.as<float>() + bt->loff[b];
            T.normX2 = bt->norm2.as<double>() + b;
            T.R = bt->R[b];
            T.stride = bt->stride[b];
        }
        PTI_CUDA(bt->tens.alloc(padded(B * sizeof(BatchTensor)), s), kMod);
        PTI_CUDA(cudaMemcpyAsync(bt->tens.ptr, ht.data(), B * sizeof(BatchTensor), cudaMemcpyHostToDevice, s), kMod);
        std::vector<const float *> vp(B);
        for (uint32_t b = 0; b < B; ++b) vp[b] = bt->coo[b]->vals.as<float>();
        DevBuf dvp, dnnz;
        PTI_CUDA(dvp.alloc(padded(B * sizeof(void *)), s), kMod);
        PTI_CUDA(dnnz.alloc(padded(B * 8), s), kMod);
        PTI_CUDA(cudaMemcpyAsync(dvp.ptr, vp.data(), B * sizeof(void *), cudaMemcpyHostToDevice, s), kMod);
        PTI_CUDA(cudaMemcpyAsync(dnnz.ptr, bt->nnz.data(), B * 8, cudaMemcpyHostToDevice, s), kMod);
        batch_norm_kernel<<<B, kBThreads, 0, s>>>(dvp.as<const float *>(), dnnz.as<uint64_t>(),
                                                  bt->norm2.as<double>());
        PTI_CUDA(cudaGetLastError(), kMod);
        PTI_CUDA(cudaStreamSynchronize(s), kMod);
    }

    TuneKey key{B, 0, 0, 0, bt->device};
    for (uint32_t b = 0; b < B; ++b) {
        key.nnz_sum += bt->nnz[b];
        key.rank_sum += (uint64_t)bt->R[b] * (b + 1);
        for (uint32_t m = 0; m < 3; ++m) key.dims_sum += (uint64_t)bt->dims[3 * b + m] * (3 * b + m + 1);
    }
    int best_sb = 7, best_cpl = 4;
    bool cached = false;
    // HIPARTI_B200_BATCH_CONFIG="sb_bits,cols_per_lane" fixes the choice
    // (sb_bits in [4, 8], cols_per_lane 4 or 8) and skips the tuner.
    if (const char *env = std::getenv("HIPARTI_B200_BATCH_CONFIG")) {
        int e_sb = 0, e_cpl = 0;
        PTI_CHECK(std::sscanf(env, "%d,%d", &e_sb, &e_cpl) == 2 && e_sb >= 4 && e_sb <= 8 &&
                      (e_cpl == 4 || e_cpl == 8),
                  PTIERR_VALUE_ERROR, kMod, "HIPARTI_B200_BATCH_CONFIG must be \"sb_bits,cols_per_lane\"");
        best_sb = e_sb;
        best_cpl = e_cpl;
        cached = true;
    }
    if (!cached) {
        std::lock_guard<std::mutex> g(g_tune_mu);
        auto it = g_tuned.find(key);
        if (it != g_tuned.end()) {
            best_sb = it->second.first;
            best_cpl = it->second.second;
            cached = true;
        }
    }
    if (tune && !cached) {
        // time one BF16 and one FP32 iteration of the whole batch per candidate
        cudaEvent_t u0, u1;
        cudaEventCreate(&u0);
        cudaEventCreate(&u1);
        cudaEventRecord(u0, s);
        DevBuf fits;
        PTI_CUDA(fits.alloc(padded((size_t)B * 2 * 8), s), kMod);
        float best = 3.4e38f;
        const int sbs[] = {7, 6, 5, 4};
        for (int sb : sbs) {
            PTI_TRY(batch_build_plans(bt.get(), sb));
            for (int cpl : {4, 8}) {
                batch_fill_kernel<<<sm_count() * 4, 256, 0, s>>>(bt->A.as<float>(), elems);
                PTI_TRY(batch_init_factors(bt.get(), 1, 1));
                float ms = 0.f;
                PTI_TRY(batch_iterate(bt.get(), 2, 1, 1, cpl, fits.as<double>(), &ms));  // warm-up
                PTI_TRY(batch_iterate(bt.get(), 2, 1, 1, cpl, fits.as<double>(), &ms));
                if (ms < best) {
                    best = ms;
                    best_sb = sb;
                    best_cpl = cpl;
                }
            }
        }
        cudaEventRecord(u1, s);
        cudaEventSynchronize(u1);
        cudaEventElapsedTime(&bt->tune_ms, u0, u1);
        cudaEventDestroy(u0);
        cudaEventDestroy(u1);
        std::lock_guard<std::mutex> g(g_tune_mu);
        g_tuned[key] = {best_sb, best_cpl};
    }
    if (bt->sb != best_sb || !bt->hic[0]) PTI_TRY(batch_build_plans(bt.get(), best_sb));
    bt->cpl = best_cpl;
    for (auto &c : bt->coo) c.reset();
    cudaEventRecord(t1, s);
    PTI_CUDA(cudaEventSynchronize(t1), kMod);
    cudaEventElapsedTime(&bt->setup_ms, t0, t1);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    *out = bt.release();
    return 0;
}

int ptiB200BatchInfo(const ptiB200Batch *bt, int *sb_bits, int *cols_per_lane, float *tune_ms, float *setup_ms,
                     ptiNnzIndex *ntasks)
{
    PTI_CHECK(bt, PTIERR_VALUE_ERROR, pti::kMod, "null batch");
    if (sb_bits) *sb_bits = bt->sb;
    if (cols_per_lane) *cols_per_lane = bt->cpl;
    if (tune_ms) *tune_ms = bt->tune_ms;
    if (setup_ms) *setup_ms = bt->setup_ms;
    if (ntasks) *ntasks = bt->ntasks;
    return 0;
}

int ptiB200BatchWaitProbe(ptiB200Batch *bt, double wait_seconds)
{
    using namespace pti;
    PTI_CHECK(bt && bt->B >= 1, PTIERR_VALUE_ERROR, kMod, "empty batch");
    PTI_CHECK(wait_seconds > 0.0 && wait_seconds <= 2.0, PTIERR_VALUE_ERROR, kMod,
              "wait bound must be in (0, 2] seconds");
    cudaStream_t s = bt->s;
    // one task: the mode-1 dense step of tensor 0, which waits for the mode-0
    // dense step -- a task this queue does not hold, so the counter it waits
    // on stays 0 and the wait must give up after its bound
    DevBuf task;
    PTI_CUDA(task.alloc(64, s), kMod);
    const uint2 t = make_uint2((1u << 1) | 1u, 0u);
    PTI_CUDA(cudaMemcpyAsync(task.ptr, &t, sizeof t, cudaMemcpyHostToDevice, s), kMod);
    uint32_t *misc = bt->misc.as<uint32_t>();
    PTI_CUDA(cudaMemsetAsync(misc, 0, 8, s), kMod);
    PTI_CUDA(cudaMemsetAsync(bt->ctrl.ptr, 0, (1 + 4 * (size_t)bt->B) * 4, s), kMod);
    BatchArgs a{};
    a.tasks = task.as<uint2>();
    a.plans = bt->plans.as<BatchPlan>();
    a.tens = bt->tens.as<BatchTensor>();
    a.ctrl = bt->ctrl.as<uint32_t>();
    a.iter = misc;
    a.fits = nullptr;
    a.err = misc + 1;
    a.ntasks = 1;
    a.ntensors = bt->B;
    a.niters = 1;
    a.cpl = 4;
    a.wait_ns = (uint64_t)(wait_seconds * 1e9);
    uint32_t grid = 0;
    PTI_TRY(batch_grid(bt, batch_kernel(4, false), &grid));
    batch_kernel(4, false)<<<1, kBThreads, kBatchSmem, s>>>(a);
    PTI_CUDA(cudaGetLastError(), kMod);
    PTI_CUDA(cudaStreamSynchronize(s), kMod);
    uint32_t err = 0;
    PTI_CUDA(cudaMemcpy(&err, misc + 1, 4, cudaMemcpyDeviceToHost), kMod);
    PTI_CUDA(cudaMemsetAsync(misc, 0, 8, s), kMod);
    PTI_CHECK(err == 0, PTIERR_CUDA_ERROR, kMod, "a work-queue or copy wait timed out");
    return 0;
}

int ptiB200BatchCpdAls(ptiB200Batch *bt, ptiIndex niters, int precision, ptiIndex fp32_sweeps,
                       float *const *dev_factors, float *const *dev_lambda, double *fits, float *ms_per_iter,
                       void *stream)
{
    using namespace pti;
    PTI_CHECK(bt && dev_factors && dev_lambda, PTIERR_VALUE_ERROR, kMod, "null argument");
    PTI_CHECK(niters >= 1 && niters <= 1000000, PTIERR_VALUE_ERROR, kMod, "niters must be in [1, 10^6]");
    PTI_CHECK(precision == PTI_B200_F32 || precision == PTI_B200_BF16, PTIERR_VALUE_ERROR, kMod, "bad precision");
    const uint32_t B = bt->B;
    for (uint32_t i = 0; i < 3 * B; ++i)
        PTI_CHECK(dev_factors[i] && ((uintptr_t)dev_factors[i] & 15) == 0, PTIERR_VALUE_ERROR, kMod,
                  "factors must be non-null and 16-byte aligned");
    for (uint32_t b = 0; b < B; ++b) PTI_CHECK(dev_lambda[b], PTIERR_VALUE_ERROR, kMod, "null lambda");
    cudaStream_t s = bt->s;
    {
        cudaEvent_t ev;
        PTI_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), kMod);
        cudaEventRecord(ev, static_cast<cudaStream_t>(stream));
        cudaStreamWaitEvent(s, ev, 0);
        cudaEventDestroy(ev);
    }
    const int mixed = precision == PTI_B200_BF16;
    // factors in: caller's arrays -> arena
    std::vector<CopyItem> items(3 * (size_t)B);
    for (uint32_t b = 0; b < B; ++b)
        for (uint32_t m = 0; m < 3; ++m) {
            const size_t n = (size_t)bt->dims[3 * b + m] * bt->stride[b];
            items[3 * b + m] = CopyItem{dev_factors[3 * b + m], bt->A.as<float>() + bt->off[3 * b + m], n};
        }
    PTI_CUDA(bt->copies.alloc(padded(items.size() * sizeof(CopyItem)), s), kMod);
    PTI_CUDA(cudaMemcpyAsync(bt->copies.ptr, items.data(), 3 * (size_t)B * sizeof(CopyItem), cudaMemcpyHostToDevice,
                             s), kMod);
    batch_copy_kernel<<<3 * B, 256, 0, s>>>(bt->copies.as<CopyItem>());
    PTI_TRY(batch_init_factors(bt, mixed, mixed && niters > fp32_sweeps));
    DevBuf dfits;
    PTI_CUDA(dfits.alloc(padded((size_t)B * niters * 8), s), kMod);
    float ms = 0.f;
    PTI_TRY(batch_iterate(bt, niters, mixed, fp32_sweeps, bt->cpl, dfits.as<double>(), &ms));
    batch_final_kernel<<<B, kBThreads, 0, s>>>(bt->tens.as<BatchTensor>());
    // factors and lambda out: arena -> caller's arrays
    std::vector<CopyItem> outs(4 * (size_t)B);
    for (uint32_t b = 0; b < B; ++b) {
        for (uint32_t m = 0; m < 3; ++m)
            outs[3 * b + m] = CopyItem{bt->A.as<float>() + bt->off[3 * b + m], dev_factors[3 * b + m], items[3 * b + m].n};
        outs[3 * (size_t)B + b] = CopyItem{bt->lam.as<float>() + bt->loff[b], dev_lambda[b], bt->R[b]};
    }
    DevBuf out_items;
    PTI_CUDA(out_items.alloc(padded(outs.size() * sizeof(CopyItem)), s), kMod);
    PTI_CUDA(cudaMemcpyAsync(out_items.ptr, outs.data(), outs.size() * sizeof(CopyItem), cudaMemcpyHostToDevice, s),
             kMod);
    batch_copy_kernel<<<4 * B, 256, 0, s>>>(out_items.as<CopyItem>());
    PTI_CUDA(cudaGetLastError(), kMod);
    if (fits) PTI_CUDA(cudaMemcpyAsync(fits, dfits.ptr, (size_t)B * niters * 8, cudaMemcpyDeviceToHost, s), kMod);
    PTI_CUDA(cudaStreamSynchronize(s), kMod);
    if (ms_per_iter) *ms_per_iter = ms;
    return 0;
}

void ptiB200BatchFree(ptiB200Batch *bt)
{
    if (!bt) return;
    cudaStreamSynchronize(bt->s);
    delete bt;
}

}  // extern "C"
