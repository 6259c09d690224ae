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
// "coordinates changed" flags; the fiber structure is kept per mode.  Two
// kernels share the fibers, and in both every Y element is the same sequence
// of FP32 multiply-then-add steps as the reference's loop, so the result is
// bit-identical for tensors with distinct coordinates:
//   - ttm_short_kernel (R <= 32): one thread per fiber of at most kShortFiber
//     nonzeros, all R columns in registers, each factor row read as float4s.
//     Most fibers are short, and a thread per fiber keeps many fibers' load
//     chains in flight at once;
//   - ttm_kernel: a group of G lanes (G = 8, 16 or 32 by R) per fiber, each
//     lane CPL columns; the group loads G nonzeros at a time and walks them in
//     order.  It takes every fiber when R > 32;
//   - ttm_long_kernel and ttm_vlong_kernel (R <= 32): a warp, or for the
//     longest fibers a CTA whose warps compute the products while one warp
//     adds them, per fiber longer than kShortFiber.
#include <cerrno>

#include "primitives.cuh"
#include "tensor.cuh"
#include "tma.cuh"

namespace pti {
int ensure_err_word(ptiB200Tensor *t, cudaStream_t s);
uint32_t *err_word(ptiB200Tensor *t);
int take_device_error(ptiB200Tensor *t, cudaStream_t s, const char *mod);

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

constexpr uint32_t kShortFiber = 64;      // longest fiber a single thread takes
constexpr uint64_t kVLongFiber = 8192;    // longer fibers get a CTA each (ttm_vlong_kernel)

// Fibers longer than kShortFiber: up to kVLongFiber nonzeros from the front of
// `list` (count[0] of them), longer ones from the back (count[1]).
__global__ void long_fibers_k(const uint64_t *fptr, uint64_t nfib, uint32_t *list, unsigned long long *count)
{
    GRID_LOOP(f, nfib)
    {
        const uint64_t len = fptr[f + 1] - fptr[f];
        if (len > kVLongFiber) list[nfib - 1 - atomicAdd(count + 1, 1ull)] = (uint32_t)f;
        else if (len > kShortFiber) list[atomicAdd(count, 1ull)] = (uint32_t)f;
    }
}

// Length class of every fiber for the one-thread-per-fiber kernel: 0 for one
// nonzero, c for 2^(c-1) < length <= 2^c up to kShortFiber, 7 above.
__global__ void fiber_class_k(const uint64_t *fptr, uint64_t nfib, uint64_t *key, uint32_t *idx)
{
    GRID_LOOP(f, nfib)
    {
        const uint64_t len = fptr[f + 1] - fptr[f];
        key[f] = len > kShortFiber ? 7u : (len <= 1 ? 0u : 64u - __clzll(len - 1));
        idx[f] = (uint32_t)f;
    }
}

// {fiber, length, first nonzero} of the fibers in `order`, for the kernel below.
__global__ void pack_short_k(const uint64_t *fptr, const uint32_t *order, uint64_t n, uint4 *fibs)
{
    GRID_LOOP(i, n)
    {
        const uint32_t f = order[i];
        const uint64_t b = fptr[f];
        fibs[i] = make_uint4(f, (uint32_t)(fptr[f + 1] - b), (uint32_t)b, (uint32_t)(b >> 32));
    }
}

// One thread per short fiber, NC4 float4 column chunks (R <= 4 * NC4 <= 32).
// The fibers come packed in order of their length class (so that a warp's
// lanes walk fibers of similar lengths and finish together), each with its
// first nonzero, so a thread starts from one coalesced 16-byte load.
// U rows and Y rows are 16-byte aligned (ldu, ldy multiples of 4).
template <int NC4>
__global__ void __launch_bounds__(256) ttm_short_kernel(const uint4 *__restrict__ fibs, uint64_t nshort,
                                                        const uint32_t *__restrict__ sind,
                                                        const float *__restrict__ sval,
                                                        const float *__restrict__ U, uint32_t ldu,
                                                        float *__restrict__ Y, uint32_t ldy, uint32_t R)
{
    GRID_LOOP(i, nshort)
    {
        const uint4 fb = fibs[i];  // {fiber, length, first nonzero (64-bit)}
        const uint64_t f = fb.x;
        const uint64_t b = (uint64_t)fb.z | (uint64_t)fb.w << 32, e = b + fb.y;
        float4 acc[NC4];
#pragma unroll
        for (int c = 0; c < NC4; ++c) acc[c] = make_float4(0.f, 0.f, 0.f, 0.f);
        uint32_t r = sind[b];
        float x = sval[b];
        for (uint64_t j = b; j < e; ++j) {
            // the next nonzero's index and value load while this one is added
            const uint32_t rn = j + 1 < e ? sind[j + 1] : 0u;
            const float xn = j + 1 < e ? sval[j + 1] : 0.f;
            const float4 *u = reinterpret_cast<const float4 *>(U + (size_t)r * ldu);
#pragma unroll
            for (int c = 0; c < NC4; ++c) {
                const float4 v = __ldg(u + c);
                acc[c].x = __fadd_rn(acc[c].x, __fmul_rn(x, v.x));
                acc[c].y = __fadd_rn(acc[c].y, __fmul_rn(x, v.y));
                acc[c].z = __fadd_rn(acc[c].z, __fmul_rn(x, v.z));
                acc[c].w = __fadd_rn(acc[c].w, __fmul_rn(x, v.w));
            }
            r = rn;
            x = xn;
        }
        float4 *y = reinterpret_cast<float4 *>(Y + (size_t)f * ldy);
#pragma unroll
        for (int c = 0; c < NC4; ++c) {
            float4 v = acc[c];
            // columns at or beyond R (the U pad is not read as data): zero
            if (4 * c + 0 >= (int)R) v.x = 0.f;
            if (4 * c + 1 >= (int)R) v.y = 0.f;
            if (4 * c + 2 >= (int)R) v.z = 0.f;
            if (4 * c + 3 >= (int)R) v.w = 0.f;
            y[c] = v;
        }
        for (uint32_t k = 4 * NC4; k < ldy; k += 4) y[k / 4] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
}

// Long fibers (R <= 32, U rows 16-byte aligned): each warp takes fibers
// list[blockIdx.x], list[blockIdx.x + gridDim.x], ... and walks them as one
// stream of groups of 32 nonzeros (a fiber's last group may be shorter), lane
// l summing column l of the current fiber.  Two cp.async stages run ahead of
// the sums (lane t copying element t of a group):
//   iteration g  copies the indices and values of stream group g + D into rings,
//                copies the factor rows of stream group g (the indices landed
//                D iterations ago) into the row ring,
//                sums stream group g - D (its rows landed), and at the last
//                group of a fiber writes the fiber's row of Y,
// so 32 D rows are in flight across fiber boundaries, and the pipeline fills
// and drains once per warp rather than once per fiber, while every column is
// summed in the reference's order.  One cp.async.wait_group D-1 at the top of
// each iteration covers both stages: everything committed at iteration g - D
// or earlier has landed.  Dynamic shared memory: row ring (D+1) x 32 x W
// floats (W = R rounded up to 4), index and value rings 2D+2 slots of 32.
constexpr int kLongD = 6;
constexpr int kLongRowSlots = kLongD + 1;
constexpr int kLongIdxSlots = 2 * kLongD + 2;

inline size_t long_smem_bytes(uint32_t W)
{
    return (size_t)kLongRowSlots * 32 * W * 4 + (size_t)kLongIdxSlots * 32 * 8;
}

// Position in a warp's stream of groups: fiber list[i], group k of its ng.
struct GroupCursor {
    uint64_t i, f, b, e, k, ng;
    bool live;
    __device__ __forceinline__ void fiber(const uint64_t *fptr, const uint32_t *list, uint64_t nlong)
    {
        live = i < nlong;
        if (!live) return;
        f = list[i];
        b = fptr[f];
        e = fptr[f + 1];
        ng = (e - b + 31) / 32;
        k = 0;
    }
    __device__ __forceinline__ void next(const uint64_t *fptr, const uint32_t *list, uint64_t nlong)
    {
        if (++k == ng) {
            i += gridDim.x;
            fiber(fptr, list, nlong);
        }
    }
    __device__ __forceinline__ uint64_t first() const { return b + 32 * k; }  // first nonzero of the group
};

__global__ void __launch_bounds__(32) ttm_long_kernel(const uint64_t *__restrict__ fptr,
                                                      const uint32_t *__restrict__ list, uint64_t nlong,
                                                      const uint32_t *__restrict__ sind,
                                                      const float *__restrict__ sval, const float *__restrict__ U,
                                                      uint32_t ldu, uint32_t R, uint32_t W, float *__restrict__ Y,
                                                      uint32_t ldy)
{
    extern __shared__ __align__(16) float ring[];
    float *su = ring;                                                    // [slot][32][W]
    uint32_t *si = reinterpret_cast<uint32_t *>(su + (size_t)kLongRowSlots * 32 * W);  // [slot][32]
    float *sx = reinterpret_cast<float *>(si + kLongIdxSlots * 32);      // [slot][32]
    const int lane = threadIdx.x;
    auto cp4 = [](void *dst, const void *src) {
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
                     "l"(src)
                     : "memory");
    };
    // cursors of the three stages: sums (group g - D), rows (g), indices (g + D)
    GroupCursor cs{blockIdx.x}, cr{blockIdx.x}, ci{blockIdx.x};
    cs.fiber(fptr, list, nlong);
    cr.fiber(fptr, list, nlong);
    ci.fiber(fptr, list, nlong);
    float acc = 0.f;
    // ring slots of stream group g: row slot g mod (D+1), index slot g mod (2D+2)
    uint32_t r13 = kLongRowSlots - kLongD % kLongRowSlots, r26 = kLongIdxSlots - kLongD;  // g = -D
    auto wrap = [](uint32_t x, uint32_t n) { return x >= n ? x - n : x; };
    for (int64_t g = -kLongD; cs.live; ++g) {
        asm volatile("cp.async.wait_group %0;\n" ::"n"(kLongD - 1) : "memory");
        __syncwarp();
        if (g >= kLongD) {  // sum stream group g - D
            const uint64_t j0 = cs.first();
            const int cnt = (cs.e - j0) < 32 ? (int)(cs.e - j0) : 32;
            // slots of g - D: (D+1) - D = 1 row slot ahead, 2D+2 - D index slots ahead
            const float *rows = su + (size_t)wrap(r13 + 1, kLongRowSlots) * 32 * W;
            const float *xs = sx + wrap(r26 + (kLongIdxSlots - kLongD), kLongIdxSlots) * 32;
            if ((uint32_t)lane < R) {
#pragma unroll 8
                for (int t = 0; t < cnt; ++t) acc = __fadd_rn(acc, __fmul_rn(xs[t], rows[(size_t)t * W + lane]));
            }
            if (cs.k + 1 == cs.ng) {  // the fiber's last group: its row of Y
                float *y = Y + (size_t)cs.f * ldy;
                if ((uint32_t)lane < R) y[lane] = acc;
                for (uint32_t k = R + lane; k < ldy; k += 32) y[k] = 0.f;
                acc = 0.f;
            }
            cs.next(fptr, list, nlong);
        }
        if (g >= 0 && cr.live) {  // rows of stream group g
            const uint64_t mine = cr.first() + lane;
            if (mine < cr.e) {
                const uint32_t r = si[r26 * 32 + lane];  // this lane's own copy
                const float *src = U + (size_t)r * ldu;
                float *dst = su + (size_t)r13 * 32 * W + (size_t)lane * W;
                for (uint32_t q = 0; q < W; q += 4) {
                    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n"
                                 ::"r"((unsigned)__cvta_generic_to_shared(dst + q)), "l"(src + q)
                                 : "memory");
                }
            }
            cr.next(fptr, list, nlong);
        }
        if (ci.live) {  // indices and values of stream group g + D
            const uint64_t mine = ci.first() + lane;
            if (mine < ci.e) {
                const uint32_t slot = wrap(r26 + kLongD, kLongIdxSlots) * 32 + lane;  // slot of g + D
                cp4(si + slot, sind + mine);
                cp4(sx + slot, sval + mine);
            }
            ci.next(fptr, list, nlong);
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
        __syncwarp();  // the slots read above are refilled in later iterations
        r13 = wrap(r13 + 1, kLongRowSlots);
        r26 = wrap(r26 + 1, kLongIdxSlots);
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// The longest fibers (more than kVLongFiber nonzeros; R <= 32, U rows
// 16-byte aligned): one CTA of kVWarps warps per fiber.  The products
// x_j * U[i_j, c] do not depend on one another, so warps 1 .. kVWarps-1
// compute them, rounded to FP32 as the reference rounds them, into shared
// memory, chunk by chunk of kVChunk nonzeros, and warp 0 adds the chunks in
// fiber order, lane c summing column c.  Every column is then the reference's
// sequence of FP32 additions, and only that chain of dependent additions is
// serial: the factor-row gathers of up to kVWarps-1 chunks run ahead of it.
// Chunk q of the CTA's running count belongs to producer warp 1 + q % P
// (P = kVWarps - 1) and its slot q % P, as use q / P of that slot: each slot
// is filled by one warp in order and emptied by warp 0 in order, so its
// "full" mbarrier (32 arrivals, the producer's lanes) and "empty" mbarrier
// (32 arrivals, warp 0's lanes) are never more than one phase apart, and the
// parity waits are exact.  Every wait is bounded by a deadline on
// %globaltimer (kVWaitNs each); a warp that gives up sets bit 2 of the error
// word and a shared abort flag that ends the other warps' waits, and the CTA
// stops.
constexpr int kVWarps = 16;
constexpr int kVSlots = kVWarps - 1;
constexpr int kVChunk = 64;
constexpr uint64_t kVWaitNs = 2000000000ull;  // 2 s

inline size_t vlong_smem_bytes(uint32_t W) { return (size_t)kVSlots * kVChunk * W * 4; }

__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_arrive_cta(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// true once the phase of `bar` with parity `parity` has completed; false if
// `abort` is set or kVWaitNs pass first
__device__ __forceinline__ bool vwait(uint64_t *bar, uint32_t parity, const volatile int *abort)
{
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t deadline = global_ns() + kVWaitNs;
    for (uint32_t i = 0;; ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        if (*abort) return false;
        if ((i & 255u) == 255u && global_ns() > deadline) return false;
    }
}

__global__ void __launch_bounds__(kVWarps * 32) ttm_vlong_kernel(const uint64_t *__restrict__ fptr,
                                                                 const uint32_t *__restrict__ list, uint64_t nvl,
                                                                 const uint32_t *__restrict__ sind,
                                                                 const float *__restrict__ sval,
                                                                 const float *__restrict__ U, uint32_t ldu, uint32_t R,
                                                                 uint32_t W, float *__restrict__ Y, uint32_t ldy,
                                                                 uint32_t *err)
{
    extern __shared__ __align__(16) float vring[];  // [kVSlots][kVChunk][W]
    __shared__ uint64_t full[kVSlots], empty[kVSlots];
    __shared__ int abort_flag;
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    if (threadIdx.x == 0) {
        for (int k = 0; k < kVSlots; ++k) {
            mbar_init(&full[k], 32);
            mbar_init(&empty[k], 32);
        }
        abort_flag = 0;
        mbar_fence_init();
    }
    __syncthreads();
    auto give_up = [&]() {
        if (lane == 0) {
            atomicOr(err, 2u);
            abort_flag = 1;
        }
    };
    uint64_t q0 = 0;  // chunks of the CTA's earlier fibers
    for (uint64_t i = blockIdx.x; i < nvl; i += gridDim.x) {
        const uint64_t f = list[i];
        const uint64_t b = fptr[f], e = fptr[f + 1];
        const uint64_t nq = (e - b + kVChunk - 1) / kVChunk;
        if (warp == 0) {
            float acc = 0.f;
            uint32_t slot = (uint32_t)(q0 % kVSlots), parity = (uint32_t)(q0 / kVSlots) & 1u;  // of chunk q0 + q
            for (uint64_t q = 0; q < nq; ++q) {
                if (q) {
                    if (++slot == kVSlots) {
                        slot = 0;
                        parity ^= 1u;
                    }
                }
                if (!vwait(&full[slot], parity, &abort_flag)) {
                    give_up();
                    return;
                }
                const uint64_t j0 = b + q * kVChunk;
                const int cnt = (e - j0) < (uint64_t)kVChunk ? (int)(e - j0) : kVChunk;
                const float *src = vring + (size_t)slot * kVChunk * W + lane;
                if ((uint32_t)lane < R) {
                    if (cnt == kVChunk) {
                        // straight-line: the loads of the next 16 products are
                        // in flight while the current 16 are added
                        float v[16], nv[16];
#pragma unroll
                        for (int t = 0; t < 16; ++t) v[t] = src[(size_t)t * W];
#pragma unroll
                        for (int t0 = 0; t0 < kVChunk; t0 += 16) {
                            if (t0 + 16 < kVChunk) {
#pragma unroll
                                for (int t = 0; t < 16; ++t) nv[t] = src[(size_t)(t0 + 16 + t) * W];
                            }
#pragma unroll
                            for (int t = 0; t < 16; ++t) acc = __fadd_rn(acc, v[t]);
#pragma unroll
                            for (int t = 0; t < 16; ++t) v[t] = nv[t];
                        }
                    } else {
                        for (int t = 0; t < cnt; ++t) acc = __fadd_rn(acc, src[(size_t)t * W]);
                    }
                }
                mbar_arrive_cta(&empty[slot]);
            }
            float *y = Y + (size_t)f * ldy;
            if ((uint32_t)lane < R) y[lane] = acc;
            for (uint32_t k = R + lane; k < ldy; k += 32) y[k] = 0.f;
        } else {
            const uint64_t pw = (uint64_t)warp - 1;  // this warp's slot
            const uint64_t qf = (pw + kVSlots - q0 % kVSlots) % kVSlots;  // its first chunk of the fiber
            uint32_t parity = (uint32_t)((q0 + qf) / kVSlots) & 1u;      // use (q0 + q) / kVSlots of the slot
            for (uint64_t q = qf; q < nq; q += kVSlots, parity ^= 1u) {
                // the slot's previous chunk has been added (a fresh barrier
                // passes the wait on the phase before its first at once)
                if (!vwait(&empty[pw], parity ^ 1u, &abort_flag)) {
                    give_up();
                    return;
                }
                const uint64_t j0 = b + q * kVChunk;
                const int cnt = (e - j0) < (uint64_t)kVChunk ? (int)(e - j0) : kVChunk;
                float *dst = vring + (size_t)pw * kVChunk * W;
                static_assert(kVChunk == 64, "two nonzeros per lane");
                // both nonzeros' indices, then both rows, are in flight together
                const bool h0 = lane < cnt, h1 = lane + 32 < cnt;
                const uint32_t k0 = h0 ? sind[j0 + lane] : 0u, k1 = h1 ? sind[j0 + lane + 32] : 0u;
                const float x0 = h0 ? sval[j0 + lane] : 0.f, x1 = h1 ? sval[j0 + lane + 32] : 0.f;
                const float4 *u0 = reinterpret_cast<const float4 *>(U + (size_t)k0 * ldu);
                const float4 *u1 = reinterpret_cast<const float4 *>(U + (size_t)k1 * ldu);
                float4 *d0 = reinterpret_cast<float4 *>(dst + (size_t)lane * W);
                float4 *d1 = reinterpret_cast<float4 *>(dst + (size_t)(lane + 32) * W);
                float4 v0[8], v1[8];  // W <= 32: at most 8 float4 per row
#pragma unroll
                for (uint32_t c = 0; c < 8; ++c) {
                    v0[c] = h0 && c < W / 4 ? __ldg(u0 + c) : make_float4(0.f, 0.f, 0.f, 0.f);
                    v1[c] = h1 && c < W / 4 ? __ldg(u1 + c) : make_float4(0.f, 0.f, 0.f, 0.f);
                }
#pragma unroll
                for (uint32_t c = 0; c < 8; ++c) {
                    if (h0 && c < W / 4)
                        d0[c] = make_float4(__fmul_rn(x0, v0[c].x), __fmul_rn(x0, v0[c].y), __fmul_rn(x0, v0[c].z),
                                            __fmul_rn(x0, v0[c].w));
                    if (h1 && c < W / 4)
                        d1[c] = make_float4(__fmul_rn(x1, v1[c].x), __fmul_rn(x1, v1[c].y), __fmul_rn(x1, v1[c].z),
                                            __fmul_rn(x1, v1[c].w));
                }
                mbar_arrive_cta(&full[pw]);
            }
        }
        q0 += nq;
    }
}

// One group of G lanes per fiber; lane l of the group owns columns
// l, l + G, ..., l + (CPL-1) G.  Pad columns [R, ldy) are written as zero.
// With `list`, the groups take the fibers list[0 .. nfib) instead of 0 .. nfib.
template <int CPL>
__global__ void __launch_bounds__(256) ttm_kernel(const uint64_t *__restrict__ fptr, uint64_t nfib,
                                                  const uint32_t *__restrict__ list,
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
    for (uint64_t i = g0; i < nfib; i += groups) {
        const uint64_t f = list ? list[i] : i;
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
    // fibers too long for one thread each (their order in the list is free:
    // every fiber is computed on its own)
    DevBuf cnt;
    PTI_CUDA(cnt.alloc(padded(16), s), mod);
    PTI_CUDA(cudaMemsetAsync(cnt.ptr, 0, 16, s), mod);
    PTI_CUDA(P.long_fibers.alloc(padded(nfib * 4), s), mod);
    unsigned long long nlong[2] = {0, 0};
    if (nfib) {
        long_fibers_k<<<grid_t(nfib), 256, 0, s>>>(P.fptr.as<uint64_t>(), nfib, P.long_fibers.as<uint32_t>(),
                                                  cnt.as<unsigned long long>());
        PTI_CUDA(cudaMemcpyAsync(nlong, cnt.ptr, 16, cudaMemcpyDeviceToHost, s), mod);
        PTI_CUDA(cudaStreamSynchronize(s), mod);
    }
    PTI_CUDA(cudaGetLastError(), mod);
    P.nfib = nfib;
    P.nlong = nlong[0];
    P.nvlong = nlong[1];
    // the fibers one thread takes, by length class (a stable sort of the
    // classes, so fibers of one class stay in fiber order)
    P.nshort = nfib - P.nlong - P.nvlong;
    if (P.nshort) {
        DevBuf keys, order;
        RadixScratch rs;
        PTI_CUDA(keys.alloc(padded(nfib * 8), s), mod);
        PTI_CUDA(order.alloc(padded(nfib * 4), s), mod);
        PTI_TRY(rs.alloc(nfib, s));
        fiber_class_k<<<grid_t(nfib), 256, 0, s>>>(P.fptr.as<uint64_t>(), nfib, keys.as<uint64_t>(),
                                                    order.as<uint32_t>());
        PTI_TRY(radix_sort_pairs(keys, order, nfib, 3, rs, s));
        PTI_CUDA(P.short_fibs.alloc(padded(P.nshort * 16), s), mod);
        pack_short_k<<<grid_t(P.nshort), 256, 0, s>>>(P.fptr.as<uint64_t>(), order.as<uint32_t>(), P.nshort,
                                                       P.short_fibs.as<uint4>());
        PTI_CUDA(cudaStreamSynchronize(s), mod);
    }
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
    const uint64_t *fp = P.fptr.as<uint64_t>();
    const uint32_t *si = P.sind.as<uint32_t>();
    const float *sv = P.sval.as<float>();
    const uint32_t nc4 = (R + 3) / 4;
    // thread per short fiber: R <= 32, float4 rows (ldu, ldy multiples of 4
    // and at least 4 * nc4, both arrays 16-byte aligned)
    const bool short_path = R <= 32 && ldu % 4 == 0 && ldy % 4 == 0 && ldu >= 4 * nc4 && ldy >= 4 * nc4 &&
                            reinterpret_cast<uintptr_t>(U) % 16 == 0 && reinterpret_cast<uintptr_t>(Y) % 16 == 0;
    uint64_t ngroup = P.nfib;
    const uint32_t *list = nullptr;
    cudaEvent_t ev[1] = {nullptr};
    bool joined = true;
    cudaEvent_t ev_vl = nullptr, ev_l = nullptr;
    if (short_path && (P.nlong || P.nvlong)) {
        // the long fibers run beside the short ones: the longest (whose serial
        // sums are the longest chains) on one side stream, the others on a
        // second, so that neither waits for the other
        const uint32_t W = 4 * nc4;
        PTI_CUDA(cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming), mod);
        PTI_CUDA(cudaEventRecord(ev[0], s), mod);
        if (P.nvlong) {
            cudaStream_t s2 = side_stream(0);
            PTI_CUDA(cudaStreamWaitEvent(s2, ev[0], 0), mod);
            PTI_TRY(ensure_err_word(t, s2));
            const size_t smem = vlong_smem_bytes(W);
            PTI_CUDA(cudaFuncSetAttribute(ttm_vlong_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                     mod);
            const unsigned grid = (unsigned)std::min<uint64_t>(P.nvlong, (uint64_t)sms * 2);
            ttm_vlong_kernel<<<grid, kVWarps * 32, smem, s2>>>(fp, P.long_fibers.as<uint32_t>() + (P.nfib - P.nvlong),
                                                               P.nvlong, si, sv, U, ldu, R, W, Y, ldy, err_word(t));
            PTI_CUDA(cudaGetLastError(), mod);
            PTI_CUDA(cudaEventCreateWithFlags(&ev_vl, cudaEventDisableTiming), mod);
            PTI_CUDA(cudaEventRecord(ev_vl, s2), mod);
        }
        if (P.nlong) {
            cudaStream_t s3 = side_stream(1);
            PTI_CUDA(cudaStreamWaitEvent(s3, ev[0], 0), mod);
            const size_t smem = long_smem_bytes(W);
            PTI_CUDA(cudaFuncSetAttribute(ttm_long_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                     mod);
            const unsigned grid = (unsigned)std::min<uint64_t>(P.nlong, (uint64_t)sms * 8);
            ttm_long_kernel<<<grid, 32, smem, s3>>>(fp, P.long_fibers.as<uint32_t>(), P.nlong, si, sv, U, ldu, R, W,
                                                    Y, ldy);
            PTI_CUDA(cudaGetLastError(), mod);
            PTI_CUDA(cudaEventCreateWithFlags(&ev_l, cudaEventDisableTiming), mod);
            PTI_CUDA(cudaEventRecord(ev_l, s3), mod);
        }
        joined = false;
    }
    if (short_path) {
        // a thread per fiber and as many CTAs as that takes: CTAs finish in
        // turn, so the long-fiber kernels beside this one find room
        const unsigned g = (unsigned)std::max<uint64_t>(1, (P.nshort + 255) / 256);
        const uint4 *sf = P.short_fibs.as<uint4>();
        const uint64_t ns = P.nshort;
        if (ns) switch (nc4) {
        case 1: ttm_short_kernel<1><<<g, 256, 0, s>>>(sf, ns, si, sv, U, ldu, Y, ldy, R); break;
        case 2: ttm_short_kernel<2><<<g, 256, 0, s>>>(sf, ns, si, sv, U, ldu, Y, ldy, R); break;
        case 3: ttm_short_kernel<3><<<g, 256, 0, s>>>(sf, ns, si, sv, U, ldu, Y, ldy, R); break;
        case 4: ttm_short_kernel<4><<<g, 256, 0, s>>>(sf, ns, si, sv, U, ldu, Y, ldy, R); break;
        case 5: ttm_short_kernel<5><<<g, 256, 0, s>>>(sf, ns, si, sv, U, ldu, Y, ldy, R); break;
        case 6: ttm_short_kernel<6><<<g, 256, 0, s>>>(sf, ns, si, sv, U, ldu, Y, ldy, R); break;
        case 7: ttm_short_kernel<7><<<g, 256, 0, s>>>(sf, ns, si, sv, U, ldu, Y, ldy, R); break;
        default: ttm_short_kernel<8><<<g, 256, 0, s>>>(sf, ns, si, sv, U, ldu, Y, ldy, R); break;
        }
        ngroup = 0;  // the long fibers are on the second stream
    }
    if (!joined) {  // `s` continues once the long fibers are done too
        if (ev_vl) PTI_CUDA(cudaStreamWaitEvent(s, ev_vl, 0), mod);
        if (ev_l) PTI_CUDA(cudaStreamWaitEvent(s, ev_l, 0), mod);
        cudaEventDestroy(ev[0]);
        if (ev_vl) cudaEventDestroy(ev_vl);
        if (ev_l) cudaEventDestroy(ev_l);
    }
    if (ngroup) {
        const int G = R > 16 ? 32 : (R > 8 ? 16 : 8);
        const int cpl = (int)((R + G - 1) / G);
        const unsigned per_cta = 256 / G;
        const unsigned grid =
            (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((ngroup + per_cta - 1) / per_cta, (uint64_t)sms * 16));
        if (cpl <= 1) ttm_kernel<1><<<grid, 256, 0, s>>>(fp, ngroup, list, si, sv, U, ldu, R, Y, ldy, G);
        else if (cpl <= 2) ttm_kernel<2><<<grid, 256, 0, s>>>(fp, ngroup, list, si, sv, U, ldu, R, Y, ldy, G);
        else if (cpl <= 4) ttm_kernel<4><<<grid, 256, 0, s>>>(fp, ngroup, list, si, sv, U, ldu, R, Y, ldy, G);
        else ttm_kernel<8><<<grid, 256, 0, s>>>(fp, ngroup, list, si, sv, U, ldu, R, Y, ldy, G);
    }
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
    return take_device_error(&t, s, mod);
}

// ---------------------------------------------------------------------------
// Semi-sparse -> sparse (src/sptensor/fromssp.c:32-84)
// ---------------------------------------------------------------------------
// An entry survives if it is NaN, infinite, or a normal number outside
// (-epsilon, epsilon); zeros and subnormals are dropped.
__device__ __forceinline__ bool ssp_keep(float v, float eps)
{
    const uint32_t e = (__float_as_uint(v) >> 23) & 0xFFu;
    if (e == 0xFFu) return true;
    if (e == 0u) return false;
    return !(v < eps && v > -eps);
}

struct SspArgs {
    const float *vals;   // nfib x stride
    uint32_t width, stride, mode, nmodes;
    float eps;
    const uint32_t *finds[kMaxModes];
    uint32_t *oinds[kMaxModes];
    float *ovals;
};
struct SspIn {
    SspArgs a;
    __device__ uint64_t operator()(uint64_t i) const
    {
        const uint64_t f = i / a.width, j = i - f * a.width;
        return ssp_keep(a.vals[f * a.stride + j], a.eps) ? 1 : 0;
    }
};
struct SspOut {
    SspArgs a;
    __device__ void operator()(uint64_t i, uint64_t prefix, uint64_t keep) const
    {
        if (!keep) return;
        const uint64_t f = i / a.width, j = i - f * a.width;
        for (uint32_t m = 0; m < a.nmodes; ++m) a.oinds[m][prefix] = m == a.mode ? (uint32_t)j : a.finds[m][f];
        a.ovals[prefix] = a.vals[f * a.stride + j];
    }
};

__global__ void permute_u32_t(const uint32_t *src, const uint32_t *perm, uint64_t n, uint32_t *dst)
{
    GRID_LOOP(i, n) dst[i] = src[perm[i]];
}
__global__ void permute_f32_t(const float *src, const uint32_t *perm, uint64_t n, float *dst)
{
    GRID_LOOP(i, n) dst[i] = src[perm[i]];
}

// Semi-sparse TTM (src/ssptensor/mmul.c:29-92): Y[i, k] = sum over r of
// X[i, r] * U[r, k] for every fiber i, r in order, FP32 multiply-then-add.
// One thread per (fiber, column), columns fastest so U rows are read together.
__global__ void ssp_ttm_kernel(const float *__restrict__ X, uint32_t xs, const float *__restrict__ U, uint32_t us,
                               uint32_t I, uint32_t R, uint64_t nfib, float *__restrict__ Y, uint32_t ys)
{
    GRID_LOOP(e, nfib * ys)
    {
        const uint64_t i = e / ys;
        const uint32_t k = (uint32_t)(e - i * ys);
        float acc = 0.f;
        if (k < R) {
            const float *x = X + i * xs;
            for (uint32_t r = 0; r < I; ++r) acc = __fadd_rn(acc, __fmul_rn(x[r], __ldg(U + (size_t)r * us + k)));
        }
        Y[e] = acc;
    }
}

int ssp_ttm(ptiSemiSparseTensor *Y, const ptiSemiSparseTensor *X, const ptiMatrix *U, uint32_t mode)
{
    const char *mod = "SspTns * Mtx";
    PTI_CHECK(Y && X && U, PTIERR_VALUE_ERROR, mod, "null argument");
    PTI_CHECK(mode < X->nmodes && X->ndims[mode] == U->nrows, PTIERR_SHAPE_MISMATCH, mod, "shape mismatch");
    const uint32_t N = X->nmodes, I = U->nrows, R = U->ncols;
    PTI_CHECK(I <= X->stride || X->nnz == 0, PTIERR_SHAPE_MISMATCH, mod, "fibers shorter than U's rows");
    PTI_CHECK(U->stride >= R, PTIERR_SHAPE_MISMATCH, mod, "U's stride below its column count");
    std::vector<ptiIndex> nd(X->ndims, X->ndims + N);
    nd[mode] = R;
    PTI_TRY(ptiNewSemiSparseTensor(Y, N, mode, nd.data()));
    const uint64_t nfib = X->nnz;
    const uint32_t ys = Y->stride;
    for (uint32_t m = 0; m < N; ++m) {
        if (m == mode) continue;
        std::free(Y->inds[m].data);
        const uint64_t len = X->inds[m].len;
        Y->inds[m].len = Y->inds[m].cap = len;
        Y->inds[m].data = static_cast<ptiIndex *>(std::malloc((len ? len : 1) * sizeof(ptiIndex)));
        PTI_CHECK(Y->inds[m].data, PTIERR_OS_ERROR + ENOMEM, mod, "out of memory");
        if (len) std::memcpy(Y->inds[m].data, X->inds[m].data, len * sizeof(ptiIndex));
    }
    ptiFreeMatrix(&Y->values);
    PTI_TRY(ptiNewMatrix(&Y->values, (ptiIndex)nfib, ys));
    Y->nnz = nfib;
    if (!nfib) return 0;
    cudaStream_t s = sync_stream();
    DevBuf dx, du, dy;
    PTI_CUDA(dx.alloc(padded(nfib * X->stride * 4), s), mod);
    PTI_CUDA(du.alloc(padded((size_t)I * U->stride * 4), s), mod);
    PTI_CUDA(dy.alloc(padded(nfib * ys * 4), s), mod);
    PTI_CUDA(cudaMemcpyAsync(dx.ptr, X->values.values, nfib * X->stride * 4, cudaMemcpyHostToDevice, s), mod);
    if (I) PTI_CUDA(cudaMemcpyAsync(du.ptr, U->values, (size_t)I * U->stride * 4, cudaMemcpyHostToDevice, s), mod);
    ssp_ttm_kernel<<<grid_t(nfib * ys), 256, 0, s>>>(dx.as<float>(), X->stride, du.as<float>(), U->stride, I, R, nfib,
                                                     dy.as<float>(), ys);
    PTI_CUDA(cudaGetLastError(), mod);
    PTI_CUDA(cudaMemcpyAsync(Y->values.values, dy.ptr, nfib * ys * 4, cudaMemcpyDeviceToHost, s), mod);
    PTI_CUDA(cudaStreamSynchronize(s), mod);
    return 0;
}

int ssp_to_sparse(ptiSparseTensor *dest, const ptiSemiSparseTensor *src, float eps)
{
    const char *mod = "SspTns -> SpTns";
    PTI_CHECK(dest && src, PTIERR_VALUE_ERROR, mod, "null argument");
    const uint32_t N = src->nmodes, mode = src->mode;
    PTI_CHECK(N >= 2 && N <= (uint32_t)kMaxModes && mode < N, PTIERR_VALUE_ERROR, mod, "bad semi-sparse tensor");
    const uint64_t nfib = src->nnz;
    const uint32_t width = src->ndims[mode], stride = src->stride;
    PTI_CHECK(width <= stride, PTIERR_SHAPE_MISMATCH, mod, "stride below the dense mode's size");
    const uint64_t cells = nfib * width;
    PTI_CHECK(cells < 0xFFFFFFFFull, PTIERR_VALUE_ERROR, mod, "too many entries");
    cudaStream_t s = sync_stream();
    DevBuf dv, df[kMaxModes], oi[kMaxModes], ov, tmp;
    PTI_CUDA(dv.alloc(padded(nfib * stride * 4), s), mod);
    if (nfib) PTI_CUDA(cudaMemcpyAsync(dv.ptr, src->values.values, nfib * stride * 4, cudaMemcpyHostToDevice, s), mod);
    SspArgs a{};
    a.vals = dv.as<float>();
    a.width = width;
    a.stride = stride;
    a.mode = mode;
    a.nmodes = N;
    a.eps = eps;
    for (uint32_t m = 0; m < N; ++m) {
        PTI_CUDA(oi[m].alloc(padded(cells * 4), s), mod);
        a.oinds[m] = oi[m].as<uint32_t>();
        if (m == mode) continue;
        PTI_CUDA(df[m].alloc(padded(nfib * 4), s), mod);
        if (nfib) PTI_CUDA(cudaMemcpyAsync(df[m].ptr, src->inds[m].data, nfib * 4, cudaMemcpyHostToDevice, s), mod);
        a.finds[m] = df[m].as<uint32_t>();
    }
    PTI_CUDA(ov.alloc(padded(cells * 4), s), mod);
    a.ovals = ov.as<float>();
    uint64_t nnz = 0;
    if (cells) {
        PTI_CUDA(tmp.alloc(padded(scan_tmp_elems<uint64_t>(cells) * 8), s), mod);
        PTI_TRY((exclusive_scan<uint64_t>(SspIn{a}, SspOut{a}, cells, tmp.as<uint64_t>(), &nnz, s)));
    }
    // ptiSparseTensorSortIndex(dest, 1, 1): lexicographic, mode 0 first
    DevBuf perm, key, si[kMaxModes], sv;
    RadixScratch sc;
    if (nnz > 1) {
        PTI_CUDA(perm.alloc(padded(nnz * 4), s), mod);
        PTI_CUDA(key.alloc(padded(nnz * 8), s), mod);
        PTI_TRY(sc.alloc(nnz, s));
        iota_t<<<grid_t(nnz), 256, 0, s>>>(perm.as<uint32_t>(), nnz);
        for (int m = (int)N - 1; m >= 0; --m) {
            gather_key_t<<<grid_t(nnz), 256, 0, s>>>(oi[m].as<uint32_t>(), perm.as<uint32_t>(), nnz,
                                                    key.as<uint64_t>());
            const uint32_t d = src->ndims[m];
            PTI_TRY(radix_sort_pairs(key, perm, nnz, ((bits_t(d ? d - 1 : 0) + 7) / 8) * 8, sc, s));
        }
        for (uint32_t m = 0; m < N; ++m) {
            PTI_CUDA(si[m].alloc(padded(nnz * 4), s), mod);
            permute_u32_t<<<grid_t(nnz), 256, 0, s>>>(oi[m].as<uint32_t>(), perm.as<uint32_t>(), nnz,
                                                     si[m].as<uint32_t>());
            oi[m].swap(si[m]);
        }
        PTI_CUDA(sv.alloc(padded(nnz * 4), s), mod);
        permute_f32_t<<<grid_t(nnz), 256, 0, s>>>(ov.as<float>(), perm.as<uint32_t>(), nnz, sv.as<float>());
        ov.swap(sv);
        PTI_CUDA(cudaGetLastError(), mod);
    }
    PTI_TRY(ptiNewSparseTensor(dest, N, src->ndims));
    dest->nnz = nnz;
    for (uint32_t m = 0; m < N; ++m) {
        std::free(dest->inds[m].data);
        dest->inds[m].len = dest->inds[m].cap = nnz;
        dest->inds[m].data = static_cast<ptiIndex *>(std::malloc((nnz ? nnz : 1) * sizeof(ptiIndex)));
        PTI_CHECK(dest->inds[m].data, PTIERR_OS_ERROR + ENOMEM, mod, "out of memory");
        if (nnz) PTI_CUDA(cudaMemcpyAsync(dest->inds[m].data, oi[m].ptr, nnz * 4, cudaMemcpyDeviceToHost, s), mod);
    }
    std::free(dest->values.data);
    dest->values.len = dest->values.cap = nnz;
    dest->values.data = static_cast<ptiValue *>(std::malloc((nnz ? nnz : 1) * sizeof(ptiValue)));
    PTI_CHECK(dest->values.data, PTIERR_OS_ERROR + ENOMEM, mod, "out of memory");
    if (nnz) PTI_CUDA(cudaMemcpyAsync(dest->values.data, ov.ptr, nnz * 4, cudaMemcpyDeviceToHost, s), mod);
    PTI_CUDA(cudaStreamSynchronize(s), mod);
    return 0;
}

}  // namespace
}  // namespace pti

extern "C" {

// include/includes/ssptensors.h:49-50, src/ssptensor/mmul.c:29-92 and
// mmul_cuda.cu:46-: the semi-sparse TTM, both variants on the GPU.
int ptiSemiSparseTensorMulMatrix(ptiSemiSparseTensor *Y, const ptiSemiSparseTensor *X, const ptiMatrix *U,
                                 ptiIndex mode)
{
    return pti::ssp_ttm(Y, X, U, mode);
}
int ptiCudaSemiSparseTensorMulMatrix(ptiSemiSparseTensor *Y, const ptiSemiSparseTensor *X, const ptiMatrix *U,
                                     ptiIndex mode)
{
    return pti::ssp_ttm(Y, X, U, mode);
}

// include/includes/ssptensors.h:26, src/sptensor/fromssp.c:32-84, computed on
// the GPU.  epsilon >= 0 (the reference asserts epsilon > 0; with 0 it keeps
// every normal, infinite and NaN entry, as a build without asserts does).
int ptiSemiSparseTensorToSparseTensor(ptiSparseTensor *dest, const ptiSemiSparseTensor *src, ptiValue epsilon)
{
    PTI_CHECK(epsilon >= 0.f, PTIERR_VALUE_ERROR, "SspTns -> SpTns", "epsilon must not be negative");
    return pti::ssp_to_sparse(dest, src, epsilon);
}

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
