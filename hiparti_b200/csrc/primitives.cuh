// primitives.cuh -- device-wide exclusive scan and a stable LSD radix sort of
// (64-bit key, 32-bit value) pairs, written for the COO->HiCOO conversion and
// the per-mode schedules.  Both are plain multi-kernel algorithms:
//   scan:  tile reduce -> single-CTA scan of tile sums -> tile rescan + add
//   sort:  per 8-bit digit: tile histograms -> scan (digit-major) -> stable
//          scatter, ranking equal digits within a warp with __match_any_sync
//          and across warps/rounds through shared-memory counters.
#pragma once
#include "common.cuh"

namespace pti {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

template <class T>
__device__ __forceinline__ T block_exclusive_scan(T v, T *s_warp, T &total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        T w = lane < (int)(blockDim.x >> 5) ? s_warp[lane] : T(0);
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            T y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < (int)(blockDim.x >> 5)) s_warp[lane] = w;
    }
    __syncthreads();
    T warp_prefix = warp ? s_warp[warp - 1] : T(0);
    total = s_warp[(blockDim.x >> 5) - 1];
    __syncthreads();
    return warp_prefix + x - v;
}

template <class T, class In>
__global__ void __launch_bounds__(kScanThreads) scan_reduce_kernel(In in, uint64_t n, T *tile_sums)
{
    __shared__ T s_warp[32];
    const uint64_t base = (uint64_t)blockIdx.x * kScanTile + (uint64_t)threadIdx.x * kScanItems;
    T sum = 0;
#pragma unroll
    for (int j = 0; j < kScanItems; ++j)
        if (base + j < n) sum += in(base + j);
    T total;
    block_exclusive_scan<T>(sum, s_warp, total);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

// Exclusive scan of tile sums by one CTA; writes the grand total at [ntiles].
template <class T>
__global__ void __launch_bounds__(1024) scan_tiles_kernel(T *sums, uint64_t ntiles)
{
    __shared__ T s_warp[32];
    T carry = 0;
    for (uint64_t b = 0; b < ntiles; b += 1024) {
        uint64_t i = b + threadIdx.x;
        T v = i < ntiles ? sums[i] : T(0);
        T total;
        T ex = block_exclusive_scan<T>(v, s_warp, total);
        if (i < ntiles) sums[i] = carry + ex;
        carry += total;
    }
    if (threadIdx.x == 0) sums[ntiles] = carry;
}

template <class T, class In, class Out>
__global__ void __launch_bounds__(kScanThreads) scan_apply_kernel(In in, uint64_t n, const T *tile_off, Out out)
{
    __shared__ T s_warp[32];
    const uint64_t base = (uint64_t)blockIdx.x * kScanTile + (uint64_t)threadIdx.x * kScanItems;
    T v[kScanItems];
    T sum = 0;
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
        v[j] = base + j < n ? in(base + j) : T(0);
        sum += v[j];
    }
    T total;
    T run = block_exclusive_scan<T>(sum, s_warp, total) + tile_off[blockIdx.x];
#pragma unroll
    for (int j = 0; j < kScanItems; ++j)
        if (base + j < n) {
            out(base + j, run, v[j]);
            run += v[j];
        }
}

// Exclusive scan: calls out(i, prefix_i, in(i)) for every i; returns the total
// through *total_host (synchronous copy) if non-null.  `tmp` must hold
// ceil(n / kScanTile) + 1 elements of T.
template <class T, class In, class Out>
int exclusive_scan(In in, Out out, uint64_t n, T *tmp, T *total_host, cudaStream_t s)
{
    const char *mod = "B200 scan";
    uint64_t ntiles = (n + kScanTile - 1) / kScanTile;
    if (ntiles == 0) {
        if (total_host) *total_host = 0;
        return 0;
    }
    scan_reduce_kernel<T, In><<<(unsigned)ntiles, kScanThreads, 0, s>>>(in, n, tmp);
    scan_tiles_kernel<T><<<1, 1024, 0, s>>>(tmp, ntiles);
    scan_apply_kernel<T, In, Out><<<(unsigned)ntiles, kScanThreads, 0, s>>>(in, n, tmp, out);
    PTI_CUDA(cudaGetLastError(), mod);
    if (total_host) {
        PTI_CUDA(cudaMemcpyAsync(total_host, tmp + ntiles, sizeof(T), cudaMemcpyDeviceToHost, s), mod);
        PTI_CUDA(cudaStreamSynchronize(s), mod);
    }
    return 0;
}

template <class T>
inline size_t scan_tmp_elems(uint64_t n) { return (n + kScanTile - 1) / kScanTile + 1; }

// ---------------------------------------------------------------------------
// Radix sort
// ---------------------------------------------------------------------------
constexpr int kSortThreads = 256;
constexpr int kSortRounds = 16;
constexpr int kSortTile = kSortThreads * kSortRounds;  // keys per CTA, striped
constexpr int kSortWarps = kSortThreads / 32;

static __global__ void __launch_bounds__(kSortThreads) radix_hist_kernel(const uint64_t *keys, uint64_t n, int shift,
                                                                  uint32_t ntiles, uint32_t *hist)
{
    __shared__ uint32_t s_hist[256];
    s_hist[threadIdx.x] = 0;
    __syncthreads();
    const uint64_t base = (uint64_t)blockIdx.x * kSortTile;
    for (int r = 0; r < kSortRounds; ++r) {
        uint64_t i = base + (uint64_t)r * kSortThreads + threadIdx.x;
        if (i < n) atomicAdd(&s_hist[(keys[i] >> shift) & 0xFF], 1u);
    }
    __syncthreads();
    hist[(uint64_t)threadIdx.x * ntiles + blockIdx.x] = s_hist[threadIdx.x];
}

static __global__ void __launch_bounds__(kSortThreads) radix_scatter_kernel(const uint64_t *keys_in, const uint32_t *vals_in,
                                                                     uint64_t n, int shift, uint32_t ntiles,
                                                                     const uint32_t *offsets, uint64_t *keys_out,
                                                                     uint32_t *vals_out)
{
    __shared__ uint32_t s_base[256];
    __shared__ uint32_t s_cnt[kSortWarps][256];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    s_base[threadIdx.x] = offsets[(uint64_t)threadIdx.x * ntiles + blockIdx.x];
    for (int w = 0; w < kSortWarps; ++w) s_cnt[w][threadIdx.x] = 0;
    __syncthreads();
    const uint64_t base = (uint64_t)blockIdx.x * kSortTile;
    const uint32_t lt_mask = (1u << lane) - 1u;
    for (int r = 0; r < kSortRounds; ++r) {
        const uint64_t i = base + (uint64_t)r * kSortThreads + threadIdx.x;
        const bool valid = i < n;
        uint64_t key = valid ? keys_in[i] : 0;
        uint32_t val = valid ? vals_in[i] : 0;
        const uint32_t digit = valid ? (uint32_t)((key >> shift) & 0xFF) : 0x100u;
        const uint32_t peers = __match_any_sync(0xffffffffu, digit);
        const uint32_t rank = __popc(peers & lt_mask);
        if (valid && rank == 0) s_cnt[warp][digit] = __popc(peers);
        __syncthreads();
        {   // thread d turns this round's per-warp counts of digit d into offsets
            const int d = threadIdx.x;
            uint32_t run = s_base[d];
            for (int w = 0; w < kSortWarps; ++w) {
                uint32_t c = s_cnt[w][d];
                s_cnt[w][d] = run;
                run += c;
            }
            s_base[d] = run;
        }
        __syncthreads();
        if (valid) {
            uint32_t pos = s_cnt[warp][digit] + rank;
            keys_out[pos] = key;
            vals_out[pos] = val;
        }
        __syncthreads();
        for (int w = 0; w < kSortWarps; ++w) s_cnt[w][threadIdx.x] = 0;
        __syncthreads();
    }
}

// Stable LSD sort of (keys, vals) on bits [0, nbits) of the keys.  The result
// ends in (keys, vals); (keys_alt, vals_alt) are scratch of the same size.
// hist must hold 256 * ceil(n / kSortTile) + scan_tmp elements (u32).
struct RadixScratch {
    DevBuf keys_alt, vals_alt, hist, scan_tmp;
    int alloc(uint64_t n, cudaStream_t s)
    {
        const char *mod = "B200 sort";
        uint64_t ntiles = (n + kSortTile - 1) / kSortTile;
        PTI_CUDA(keys_alt.alloc(padded(n * 8), s), mod);
        PTI_CUDA(vals_alt.alloc(padded(n * 4), s), mod);
        PTI_CUDA(hist.alloc(padded(256 * ntiles * 4), s), mod);
        PTI_CUDA(scan_tmp.alloc(padded(scan_tmp_elems<uint32_t>(256 * ntiles) * 4), s), mod);
        return 0;
    }
};

struct HistIn {
    const uint32_t *h;
    __device__ uint32_t operator()(uint64_t i) const { return h[i]; }
};
struct HistOut {
    uint32_t *h;
    __device__ void operator()(uint64_t i, uint32_t prefix, uint32_t) const { h[i] = prefix; }
};

// Sorts (keys, vals) in place (the buffers may be exchanged with the
// scratch ones, so callers must re-read keys.ptr / vals.ptr afterwards).
inline int radix_sort_pairs(DevBuf &keys, DevBuf &vals, uint64_t n, int nbits, RadixScratch &sc,
                            cudaStream_t s)
{
    const char *mod = "B200 sort";
    if (n <= 1 || nbits <= 0) return 0;
    PTI_CHECK(n < 0xFFFFFFFFull, PTIERR_VALUE_ERROR, mod, "too many keys");
    uint32_t ntiles = (uint32_t)((n + kSortTile - 1) / kSortTile);
    uint32_t *hist = sc.hist.as<uint32_t>();
    bool flipped = false;
    for (int shift = 0; shift < nbits; shift += 8) {
        const uint64_t *kin = flipped ? sc.keys_alt.as<uint64_t>() : keys.as<uint64_t>();
        const uint32_t *vin = flipped ? sc.vals_alt.as<uint32_t>() : vals.as<uint32_t>();
        uint64_t *kout = flipped ? keys.as<uint64_t>() : sc.keys_alt.as<uint64_t>();
        uint32_t *vout = flipped ? vals.as<uint32_t>() : sc.vals_alt.as<uint32_t>();
        radix_hist_kernel<<<ntiles, kSortThreads, 0, s>>>(kin, n, shift, ntiles, hist);
        PTI_TRY((exclusive_scan<uint32_t>(HistIn{hist}, HistOut{hist}, 256ull * ntiles,
                                          sc.scan_tmp.as<uint32_t>(), nullptr, s)));
        radix_scatter_kernel<<<ntiles, kSortThreads, 0, s>>>(kin, vin, n, shift, ntiles, hist, kout, vout);
        PTI_CUDA(cudaGetLastError(), mod);
        flipped = !flipped;
    }
    if (flipped) {
        keys.swap(sc.keys_alt);
        vals.swap(sc.vals_alt);
    }
    return 0;
}

}  // namespace pti
