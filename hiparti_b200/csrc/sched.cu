// sched.cu -- per-mode schedules and the output-privatised MTTKRP kernels.
//
// Problem.  With skewed (power-law) mode sizes a few output rows receive a
// large share of all nonzeros; adding every product straight into global
// memory serialises the atomics of such a row in one L2 slice.
//
// Schedule (built once per tensor and mode, kept in the device handle).
// HiCOO: the blocks are stably re-ordered by their block coordinate in the
// output mode -- the reference's per-mode kernel scheduler (kschr,
// src/sptensor/hicoo/convert.c:378-421) taken down to block granularity --
// and the nonzeros follow their blocks; the nonzeros are then cut into tiles
// of kPlanTile and re-ordered by output row inside each tile, each keeping its
// 8-bit element offsets and the index of its block among the tile's blocks.
// COO: the nonzeros are stably sorted by their output index and packed as
// records {output index, operand indices, value}.
//
// Kernels (one CTA per tile).  The tile is staged into shared memory with
// bulk (TMA) copies.  Its nonzeros are in output-row order, so each thread
// group walks a contiguous slice, gathers the operand rows with 16-byte
// loads, accumulates the rank-R Hadamard products in registers and adds a row
// into global memory once per run of equal rows (16-byte vector atomics); a
// row shared by neighbouring groups is merged in shared memory first, so a hot
// row costs one global add per tile instead of one per nonzero.
#include <type_traits>

#include "kutil.cuh"
#include "primitives.cuh"
#include "tensor.cuh"
#include "tma.cuh"

namespace pti {

constexpr int kTile = 2048;        // nonzeros per CTA (COO kernel)
constexpr int kHiTile = kPlanTile; // nonzeros per CTA (HiCOO kernel)
constexpr int kSchedThreads = 256;

uint32_t *err_word(ptiB200Tensor *t);
int ensure_err_word(ptiB200Tensor *t, cudaStream_t s);

struct SchedArgs {
    uint64_t nnz, nb;
    uint32_t R, stride, sb;
    const uint16_t *lblk;       // HiCOO: block of each nonzero within its tile
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
    const uint4 *bquad;         // HiCOO 4-D: per block {output, operand 0, 1, 2} block coordinates
    const uint4 *recs;          // HiCOO: decoded records of the schedule (HicooModePlan::recs)
    const float *rvals;         // HiCOO 4-D: their values
};


__device__ __forceinline__ uint32_t round16(uint32_t x) { return (x + 15u) & ~15u; }

// Words per packed nonzero record {output row, operand rows..., value},
// rounded up to 16 bytes.
template <int NIN>
struct Rec {
    static constexpr int words = ((NIN + 2 + 3) / 4) * 4;
};

// Columns of one operand row held by a lane: CPL consecutive columns, loaded
// with 8- or 16-byte loads (4 FP32 columns = one 16-byte load, 8 FP32 = two,
// 8 BF16 = one, 4 BF16 = one 8-byte load).
template <int CPL, class FT>
struct RowPart {
    static constexpr int kWords = CPL * (int)sizeof(FT) / 4;
    static_assert(kWords == 2 || kWords % 4 == 0, "8- or 16-byte loads");
    uint32_t w[kWords];
    __device__ __forceinline__ void load(const FT *row, uint32_t col)
    {
        const FT *p = row + col;
        if constexpr (kWords == 2) {
            const uint2 r = __ldg(reinterpret_cast<const uint2 *>(p));
            w[0] = r.x;
            w[1] = r.y;
        } else {
#pragma unroll
            for (int q = 0; q < kWords / 4; ++q) {
                const uint4 r = __ldg(reinterpret_cast<const uint4 *>(p) + q);
                w[4 * q] = r.x;
                w[4 * q + 1] = r.y;
                w[4 * q + 2] = r.z;
                w[4 * q + 3] = r.w;
            }
        }
    }
    // 32-bit word i of the loaded columns
    __device__ __forceinline__ uint32_t word(int i) const { return w[i]; }
    // column c (0 <= c < CPL) as FP32
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

// acc[c] += v * prod_k f[k][c] for the CPL columns of a lane, with packed
// FP32x2 arithmetic; BF16 rows multiply their first two factors exactly in
// FP32 without unpacking them.
template <int CPL, class FT, int NIN>
__device__ __forceinline__ void accumulate(float *acc, const RowPart<CPL, FT> (&f)[NIN], float v)
{
    const float2 vv = make_float2(v, v);
#pragma unroll
    for (int c = 0; c < CPL; c += 2) {
        float2 p;
        if constexpr (sizeof(FT) == 2 && NIN >= 2) {
            p = bf16x2_mul(f[0].word(c >> 1), f[1].word(c >> 1));
#pragma unroll
            for (int k = 2; k < NIN; ++k) p = __fmul2_rn(p, make_float2(f[k].at(c), f[k].at(c + 1)));
        } else {
            p = make_float2(f[0].at(c), f[0].at(c + 1));
#pragma unroll
            for (int k = 1; k < NIN; ++k) p = __fmul2_rn(p, make_float2(f[k].at(c), f[k].at(c + 1)));
        }
        const float2 r = __ffma2_rn(p, vv, make_float2(acc[c], acc[c + 1]));
        acc[c] = r.x;
        acc[c + 1] = r.y;
    }
}

constexpr uint32_t kNoRow = 0xFFFFFFFFu;

// Row runs of one thread group.  Products arrive in output-row order; a run
// that ends is added into the output with one vector atomic per 4 columns,
// except the runs a group shares with its neighbours in the CTA: the run that
// continues the previous group's last row is parked in the group's merge slot
// (shared memory), and the run that continues into the next group stays in
// registers until merge(), where the group that started the row adds the
// parked parts and writes the row once.  A row that fills many slices of a
// tile (a hot row of a power-law mode) is so written once per tile instead of
// once per group.
template <int CPL>
struct RunWriter {
    float acc[CPL];
    uint32_t cur = kNoRow;
    bool in_first = true, first_shared, last_shared, active;
    uint32_t col;
    float *slot;  // this lane's CPL floats of the group's merge slot

    __device__ __forceinline__ RunWriter(bool fs, bool ls, uint32_t col_, bool active_, float *slot_)
        : first_shared(fs), last_shared(ls), active(active_), col(col_), slot(slot_)
    {
#pragma unroll
        for (int c = 0; c < CPL; ++c) acc[c] = 0.f;
    }
    __device__ __forceinline__ void flush(const SchedArgs &a)
    {
        if (!active) return;
#pragma unroll
        for (int q = 0; q < CPL / 4; ++q)
            if (col + 4 * q < a.R)
                red_add4(a.out + (size_t)cur * a.stride + col + 4 * q,
                         mask4(make_float4(acc[4 * q], acc[4 * q + 1], acc[4 * q + 2], acc[4 * q + 3]),
                               col + 4 * q, a.R));
    }
    __device__ __forceinline__ void park()
    {
#pragma unroll
        for (int c = 0; c < CPL; ++c) slot[c] = acc[c];
    }
    // a product for `row` follows
    __device__ __forceinline__ void start(uint32_t row, const SchedArgs &a)
    {
        if (row == cur) return;
        if (cur != kNoRow) {
            if (in_first && first_shared) park();
            else flush(a);
            in_first = false;
        }
#pragma unroll
        for (int c = 0; c < CPL; ++c) acc[c] = 0.f;
        cur = row;
    }
    // after the slice: true if this group owns a row that continues into the
    // next group (merge() after a barrier)
    __device__ __forceinline__ bool finish(const SchedArgs &a)
    {
        if (cur == kNoRow) return false;
        if (in_first && first_shared) {
            park();
            return false;
        }
        if (last_shared) return true;
        flush(a);
        return false;
    }
    // adds the parked parts of the following groups that continue row `cur`
    // and writes the row
    template <int G>
    __device__ __forceinline__ void merge(const SchedArgs &a, const float *slots, const uint32_t *slot_row,
                                          const uint8_t *slot_whole, uint32_t g, uint32_t lane, uint32_t ngroups)
    {
        for (uint32_t h = g + 1; h < ngroups; ++h) {
            if (slot_row[h] != cur) break;
            const float *p = slots + ((size_t)h * G + lane) * CPL;
#pragma unroll
            for (int c = 0; c < CPL; ++c) acc[c] += p[c];
            if (!slot_whole[h]) break;
        }
        flush(a);
    }
};

// True when every record of the batch, in every group of the warp still
// walking, continues its group's current output row: the batch then needs no
// row bookkeeping (what RunWriter::start would do for each record is nothing).
// Deciding for the whole warp keeps its groups on one path.
template <int U>
__device__ __forceinline__ bool same_row_batch(const uint32_t (&orow)[U], uint32_t cur)
{
    bool same = cur != kNoRow;
#pragma unroll
    for (int u = 0; u < U; ++u) same = same && orow[u] == cur;
    return __all_sync(__activemask(), same);
}

// Walks records [j0, j1) (ordered by output row) of a tile whose records are
// s_rec[0, n): gathers the operand rows and accumulates v * prod_k A_k[row_k]
// in registers, one output row run at a time (RunWriter).
template <int G, int CPL, int U, int NIN, class FT>
__device__ __forceinline__ void process_records(const uint32_t *s_rec, uint32_t n, uint32_t j0, uint32_t j1,
                                                uint32_t g, uint32_t lane, const SchedArgs &a, const float *alt,
                                                float *s_slots, uint32_t *s_slot_row, uint8_t *s_slot_whole)
{
    constexpr int RW = Rec<NIN>::words;
    constexpr uint32_t kGroups = kSchedThreads / G;
    const uint32_t col = lane * CPL;
    const bool active = col < a.R;
    bool first_shared = false, last_shared = false;
    if (j0 < j1) {
        const uint32_t rf = s_rec[(size_t)j0 * RW], rl = s_rec[(size_t)(j1 - 1) * RW];
        first_shared = j0 > 0 && s_rec[(size_t)(j0 - 1) * RW] == rf;
        last_shared = j1 < n && s_rec[(size_t)j1 * RW] == rl;
        if (lane == 0) {
            s_slot_row[g] = first_shared ? rf : kNoRow;
            s_slot_whole[g] = rf == rl;
        }
    } else if (lane == 0) {
        s_slot_row[g] = kNoRow;
        s_slot_whole[g] = 0;
    }
    RunWriter<CPL> w(first_shared, last_shared, col, active, s_slots + ((size_t)g * G + lane) * CPL);
    const FT *base[NIN];  // this lane's columns of each operand factor
#pragma unroll
    for (int k = 0; k < NIN; ++k) base[k] = static_cast<const FT *>(a.in_mat[k]) + col;
    // full batches of U records without per-record bounds tests, then one
    // partial batch
    auto batch = [&](uint32_t j, auto check) {
        constexpr bool CHECK = decltype(check)::value;
        uint32_t orow[U];
        float val[U];
        RowPart<CPL, FT> f[U][NIN];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            orow[u] = kNoRow;
            if (!CHECK || j + u < j1) {
                uint32_t wd[RW];
#pragma unroll
                for (int q = 0; q < RW; q += 4) {
                    const uint4 r = *reinterpret_cast<const uint4 *>(s_rec + (size_t)(j + u) * RW + q);
                    wd[q] = r.x; wd[q + 1] = r.y; wd[q + 2] = r.z; wd[q + 3] = r.w;
                }
                orow[u] = wd[0];
                val[u] = alt ? __ldg(alt + j + u) : __uint_as_float(wd[1 + NIN]);
                if (orow[u] != kNoRow && active) {
#pragma unroll
                    for (int k = 0; k < NIN; ++k) f[u][k].load(base[k] + (size_t)wd[1 + k] * a.stride, 0);
                }
            }
        }
        if (same_row_batch<U>(orow, w.cur)) {  // no row bookkeeping
            if (active) {
#pragma unroll
                for (int u = 0; u < U; ++u) accumulate<CPL, FT, NIN>(w.acc, f[u], val[u]);
            }
            return;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (orow[u] == kNoRow) continue;
            w.start(orow[u], a);
            if (active) accumulate<CPL, FT, NIN>(w.acc, f[u], val[u]);
        }
    };
    uint32_t j = j0;
    for (; j + U <= j1; j += U) batch(j, std::false_type{});
    if (j < j1) batch(j, std::true_type{});
    const bool owner = w.finish(a);
    __syncthreads();
    if (owner) w.template merge<G>(a, s_slots, s_slot_row, s_slot_whole, g, lane, kGroups);
}

// Walks records [j0, j1) of a tile whose n records s_rec ({output row,
// operand rows, value or third operand row}) are in output-row order and
// accumulates v * prod_k A_k[row_k] one row run at a time.  Every
// record is walkable: the decode gave a record with a bad coordinate value 0
// and operand offsets 0, and an output row kNoRow only where its own row is
// out of range (such records sort after every valid row), so the rows of a
// slice never decrease and a batch whose last record continues the current
// row lies wholly in that row.  The batch loop is therefore one compare and
// one warp vote per U records; a row change falls to the per-record path.
// Runs shared with neighbouring groups are merged as RunWriter does.
template <int G, int CPL, int U, class FT, int NIN>
__device__ __forceinline__ void walk_rows(const uint4 *s_rec, const float *s_v3, uint32_t n, uint32_t j0,
                                          uint32_t j1, uint32_t g, uint32_t lane, const SchedArgs &a,
                                          float *s_slots, uint32_t *s_slot_row, uint8_t *s_slot_whole)
{
    constexpr uint32_t kGroups = kSchedThreads / G;
    const uint32_t col = lane * CPL;
    const bool active = col < a.R;
    bool first_shared = false, last_shared = false;
    uint32_t cur = kNoRow;
    if (j0 < j1) {
        const uint32_t rl = s_rec[j1 - 1].x;
        cur = s_rec[j0].x;
        first_shared = j0 > 0 && s_rec[j0 - 1].x == cur;
        last_shared = j1 < n && s_rec[j1].x == rl;
        if (lane == 0) {
            s_slot_row[g] = first_shared ? cur : kNoRow;
            s_slot_whole[g] = cur == rl;
        }
    } else if (lane == 0) {
        s_slot_row[g] = kNoRow;
        s_slot_whole[g] = 0;
    }
    float *slot = s_slots + ((size_t)g * G + lane) * CPL;
    // inactive lanes (col >= R) read column 0 and never write
    const FT *base[NIN];
#pragma unroll
    for (int k = 0; k < NIN; ++k) base[k] = static_cast<const FT *>(a.in_mat[k]) + (active ? col : 0u);
    const uint32_t stride = a.stride;
    float acc[CPL];
#pragma unroll
    for (int c = 0; c < CPL; ++c) acc[c] = 0.f;
    bool in_first = true;
    auto flush = [&]() {
#pragma unroll
        for (int q = 0; q < CPL / 4; ++q)
            if (col + 4 * q < a.R)
                red_add4(a.out + (size_t)cur * a.stride + col + 4 * q,
                         mask4(make_float4(acc[4 * q], acc[4 * q + 1], acc[4 * q + 2], acc[4 * q + 3]),
                               col + 4 * q, a.R));
    };
    // the run of `cur` ends before the slice does
    auto end_run = [&]() {
        if (in_first && first_shared) {
#pragma unroll
            for (int c = 0; c < CPL; ++c) slot[c] = acc[c];
        } else if (cur != kNoRow && active) {
            flush();
        }
        in_first = false;
#pragma unroll
        for (int c = 0; c < CPL; ++c) acc[c] = 0.f;
    };
    auto value = [&](const uint4 &r, uint32_t j) {
        return NIN == 3 ? s_v3[j] : __uint_as_float(NIN == 2 ? r.w : r.z);
    };
    uint32_t j = j0;
    for (; j + U <= j1; j += U) {
        uint4 r[U];
        RowPart<CPL, FT> f[U][NIN];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            r[u] = s_rec[j + u];
            const uint32_t rr[3] = {r[u].y, r[u].z, r[u].w};
#pragma unroll
            for (int k = 0; k < NIN; ++k) f[u][k].load(base[k] + (size_t)rr[k] * stride, 0);
        }
        if (__all_sync(__activemask(), r[U - 1].x == cur)) {
#pragma unroll
            for (int u = 0; u < U; ++u) accumulate<CPL, FT, NIN>(acc, f[u], value(r[u], j + u));
            continue;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (r[u].x != cur) {
                end_run();
                cur = r[u].x;
            }
            accumulate<CPL, FT, NIN>(acc, f[u], value(r[u], j + u));
        }
    }
    for (; j < j1; ++j) {
        const uint4 r = s_rec[j];
        const uint32_t rr[3] = {r.y, r.z, r.w};
        RowPart<CPL, FT> f[NIN];
#pragma unroll
        for (int k = 0; k < NIN; ++k) f[k].load(base[k] + (size_t)rr[k] * stride, 0);
        if (r.x != cur) {
            end_run();
            cur = r.x;
        }
        accumulate<CPL, FT, NIN>(acc, f, value(r, j));
    }
    // the slice's last run: parked if it is also the first and shared with the
    // previous group, kept for merging if it continues into the next group
    bool owner = false;
    if (cur != kNoRow) {
        if (in_first && first_shared) {
#pragma unroll
            for (int c = 0; c < CPL; ++c) slot[c] = acc[c];
        } else if (last_shared) {
            owner = true;
        } else if (active) {
            flush();
        }
    }
    __syncthreads();
    if (owner) {
        for (uint32_t h = g + 1; h < kGroups; ++h) {
            if (s_slot_row[h] != cur) break;
            const float *p = s_slots + ((size_t)h * G + lane) * CPL;
#pragma unroll
            for (int c = 0; c < CPL; ++c) acc[c] += p[c];
            if (!s_slot_whole[h]) break;
        }
        if (active) flush();
    }
}

template <int NIN, int CPL>
struct HiSmem {
    // byte offsets inside the dynamic shared memory of hicoo_sched_kernel
    static constexpr uint32_t val = 0;                                  // float[kHiTile]
    static constexpr uint32_t eout = val + 4 * kHiTile;                 // u8[kHiTile]
    static constexpr uint32_t ein = eout + kHiTile;                     // u8[NIN][kHiTile]
    static constexpr uint32_t blk = ein + NIN * kHiTile;                // u16[kHiTile]
    static constexpr uint32_t brow = blk + 2 * kHiTile;                 // u32[kHiTile + 4]
    static constexpr uint32_t bin = brow + 4 * (kHiTile + 4);           // u32[NIN][kHiTile + 4]
    static constexpr uint32_t staged = bin + 4 * NIN * (kHiTile + 4);   // end of the staged tile
    // decoded records, written over the staged arrays once they are read
    static constexpr uint32_t rec = 0;                                  // uint4[kHiTile]
    static constexpr uint32_t rval = rec + 16 * kHiTile;                // float[kHiTile] (4-D only)
    // FP32 rows (CPL 4): the groups' merge slots follow the records, over
    // the staged tile (they are first written during the walk, after the
    // decode), which lets one more CTA share an SM.  BF16 rows (CPL 8) keep
    // them after the tile: their walk is bound by L1 wavefronts, and the
    // extra CTA's shared memory comes out of the L1 that caches the rows.
    static constexpr uint32_t slots =
        CPL == 4 ? rval + (NIN == 3 ? 4 * kHiTile : 0) : staged;  // float[kSchedThreads * CPL]
    static constexpr uint32_t slots_end = slots + 4 * kSchedThreads * CPL;
    static constexpr uint32_t total = staged > slots_end ? staged : slots_end;
    static_assert(slots <= staged, "records must fit over the staged tile");
};

// HiCOO schedule, one CTA per tile of kHiTile nonzeros.  The tile's nonzeros
// (8-bit element offsets, values, block index within the tile) and its blocks'
// coordinates are staged into shared memory with bulk copies; the nonzeros
// are already in output-row order (the schedule sorted each tile), so every
// thread group walks a contiguous slice: a lane decodes one nonzero's output
// and operand rows from its block coordinates and offsets, the group shares
// them by shuffles, gathers the operand rows and accumulates row runs.
// Records in flight per thread group of the 3-D FP32 walk, and the CTAs per
// SM the compiler is asked to fit (0: no register cap): compile-time choices.
#ifndef PTI_HICOO_U
#define PTI_HICOO_U 2
#endif
#ifndef PTI_HICOO_MINB
#define PTI_HICOO_MINB 0
#endif

template <int G, int CPL, int U, class FT, int NIN>
__global__ void __launch_bounds__(kSchedThreads, PTI_HICOO_MINB) hicoo_sched_kernel(SchedArgs a)
{
    using L = HiSmem<NIN, CPL>;
    extern __shared__ __align__(128) unsigned char sm[];
    __shared__ uint64_t mbar;
    __shared__ uint32_t s_slot_row[kSchedThreads];
    __shared__ uint8_t s_slot_whole[kSchedThreads];
    float *s_val = reinterpret_cast<float *>(sm + L::val);
    uint8_t *s_eout = sm + L::eout;
    uint8_t *s_ein = sm + L::ein;
    uint16_t *s_blk = reinterpret_cast<uint16_t *>(sm + L::blk);
    uint32_t *s_brow = reinterpret_cast<uint32_t *>(sm + L::brow);
    uint32_t *s_bin = reinterpret_cast<uint32_t *>(sm + L::bin);
    float *s_slots = reinterpret_cast<float *>(sm + L::slots);
    const uint32_t tid = threadIdx.x;

    const uint64_t z0 = (uint64_t)blockIdx.x * kHiTile;
    const uint32_t n = (uint32_t)((a.nnz - z0) < (uint64_t)kHiTile ? (a.nnz - z0) : (uint64_t)kHiTile);
    const uint32_t b0 = a.tile_block[blockIdx.x];
    uint32_t nblk = a.tile_block[blockIdx.x + 1] - b0 + 1;
    if (nblk > kHiTile + 1) nblk = kHiTile + 1;
    if (b0 + (uint64_t)nblk > a.nb) nblk = (uint32_t)(a.nb - b0);

    // Stage the tile with bulk copies.  A bulk copy starts on 16 bytes, so the
    // block coordinates are copied from b0 rounded down to 4 entries.
    const uint32_t bo4 = b0 & 3u;
    if (tid == 0) {
        mbar_init(&mbar, 1);
        mbar_fence_init();
    }
    __syncthreads();
    // 4-D: the blocks' four coordinates come as one 16-byte record each, so a
    // nonzero's decode reads them with one shared-memory load
    const uint4 *s_bq = reinterpret_cast<const uint4 *>(sm + L::brow);
    if (tid == 0) {
        const uint32_t be = round16(n), bv = round16(4 * n), bl = round16(2 * n);
        const uint32_t bb = 4 * ((nblk + bo4 + 3) & ~3u);
        const uint32_t bq = 16 * nblk;
        mbar_arrive_expect_tx(&mbar, bv + (NIN + 1) * be + bl + (NIN == 3 ? bq : (NIN + 1) * bb));
        bulk_g2s_ef(s_val, a.vals + z0, bv, &mbar);
        bulk_g2s_ef(s_eout, a.out_eind + z0, be, &mbar);
#pragma unroll
        for (int k = 0; k < NIN; ++k) bulk_g2s_ef(s_ein + k * kHiTile, a.in_eind[k] + z0, be, &mbar);
        bulk_g2s_ef(s_blk, a.lblk + z0, bl, &mbar);
        if constexpr (NIN == 3) {
            bulk_g2s_ef(sm + L::brow, a.bquad + b0, bq, &mbar);
        } else {
            bulk_g2s_ef(s_brow, a.out_bind + (b0 - bo4), bb, &mbar);
#pragma unroll
            for (int k = 0; k < NIN; ++k)
                bulk_g2s_ef(s_bin + k * (kHiTile + 4), a.in_bind[k] + (b0 - bo4), bb, &mbar);
        }
    }
    const bool ok = mbar_wait_bounded(&mbar, 0);
    if (!__syncthreads_and(ok)) {
        if (tid == 0) {
            atomicOr(a.err, 2u);
            mbar_wait_bounded(&mbar, 0);
        }
        return;
    }
    s_brow += bo4;  // block i of the tile is entry i + bo4 of the staged coordinates
    s_bin += bo4;

    // Decode every nonzero once into a 16-byte record {output row, operand
    // row offsets (row x stride)} (the value in the last free word, or beside
    // the records for 4-D), written over the staged arrays once they have all
    // been read.  A nonzero with a coordinate out of range sets the error
    // word and becomes a record that adds nothing (value 0, operand rows 0);
    // its output row is kept if that is valid, else it is kNoRow, which sorts
    // where the schedule put it (after every valid row of the tile).
    constexpr int PER = kHiTile / kSchedThreads;
    {
        uint4 rec[PER];
        float vv[PER];
#pragma unroll
        for (int p = 0; p < PER; ++p) {
            const uint32_t z = tid + p * kSchedThreads;
            rec[p] = make_uint4(kNoRow, 0u, 0u, 0u);
            vv[p] = 0.f;
            if (z < n) {
                const uint32_t i0 = s_blk[z];
                const bool ok_b = i0 < nblk;
                const uint32_t i = ok_b ? i0 : 0u;
                uint32_t bo, bi[3];
                if constexpr (NIN == 3) {
                    const uint4 q = s_bq[i];
                    bo = q.x;
                    bi[0] = q.y;
                    bi[1] = q.z;
                    bi[2] = q.w;
                } else {
                    bo = s_brow[i];
#pragma unroll
                    for (int k = 0; k < NIN; ++k) bi[k] = s_bin[k * (kHiTile + 4) + i];
                }
                const uint64_t o = ((uint64_t)bo << a.sb) + s_eout[z];
                const bool ok_o = ok_b && o < a.out_dim;
                uint32_t r[3] = {0u, 0u, 0u};
                bool ok_in = true;
#pragma unroll
                for (int k = 0; k < NIN; ++k) {
                    const uint64_t rk = ((uint64_t)bi[k] << a.sb) + s_ein[k * kHiTile + z];
                    ok_in = ok_in && rk < a.in_dim[k];
                    r[k] = (uint32_t)rk;
                }
#pragma unroll
                for (int k = 0; k < NIN; ++k) r[k] = ok_in ? r[k] : 0u;
                vv[p] = ok_o && ok_in ? s_val[z] : 0.f;
                if (NIN == 1) r[1] = __float_as_uint(vv[p]);
                if (NIN == 2) r[2] = __float_as_uint(vv[p]);
                rec[p] = make_uint4(ok_o ? (uint32_t)o : kNoRow, r[0], r[1], r[2]);
                if (!(ok_o && ok_in)) atomicOr(a.err, 1u);
            }
        }
        __syncthreads();
        uint4 *s_rec_w = reinterpret_cast<uint4 *>(sm + L::rec);
        float *s_v3_w = reinterpret_cast<float *>(sm + L::rval);
#pragma unroll
        for (int p = 0; p < PER; ++p) {
            const uint32_t z = tid + p * kSchedThreads;
            if (z < n) {
                s_rec_w[z] = rec[p];
                if (NIN == 3) s_v3_w[z] = vv[p];
            }
        }
    }
    __syncthreads();
    const uint4 *s_rec = reinterpret_cast<const uint4 *>(sm + L::rec);
    const float *s_v3 = reinterpret_cast<const float *>(sm + L::rval);

    const uint32_t g = tid / G, lane = tid % G;
    constexpr uint32_t kGroups = kSchedThreads / G;
    // an odd slice length puts the groups' first records on different shared-memory banks
    const uint32_t per = ((n + kGroups - 1) / kGroups) | 1u;
    const uint32_t j0 = min(g * per, n), j1 = min(j0 + per, n);
    walk_rows<G, CPL, U, FT, NIN>(s_rec, s_v3, n, j0, j1, g, lane, a, s_slots, s_slot_row, s_slot_whole);
}

template <int NIN, int CPL>
struct RecSmem {
    // byte offsets inside the dynamic shared memory of hicoo_rec_kernel
    static constexpr uint32_t rec = 0;                                 // uint4[kHiTile]
    static constexpr uint32_t rval = rec + 16 * kHiTile;               // float[kHiTile] (4-D only)
    static constexpr uint32_t slots = rval + (NIN == 3 ? 4 * kHiTile : 0);  // float[kSchedThreads * CPL]
    static constexpr uint32_t total = slots + 4 * kSchedThreads * CPL;
};

// HiCOO schedule, one CTA per tile of kHiTile nonzeros whose records the
// schedule already holds decoded (HicooModePlan::recs, in output-row order
// within the tile): one bulk copy stages them (and the 4-D values), then the
// thread groups walk contiguous slices (walk_rows).
template <int G, int CPL, int U, class FT, int NIN>
__global__ void __launch_bounds__(kSchedThreads, PTI_HICOO_MINB) hicoo_rec_kernel(SchedArgs a)
{
    using L = RecSmem<NIN, CPL>;
    extern __shared__ __align__(128) unsigned char sm[];
    __shared__ uint64_t mbar;
    __shared__ uint32_t s_slot_row[kSchedThreads];
    __shared__ uint8_t s_slot_whole[kSchedThreads];
    uint4 *s_rec = reinterpret_cast<uint4 *>(sm + L::rec);
    float *s_v3 = reinterpret_cast<float *>(sm + L::rval);
    float *s_slots = reinterpret_cast<float *>(sm + L::slots);
    const uint32_t tid = threadIdx.x;
    const uint64_t z0 = (uint64_t)blockIdx.x * kHiTile;
    const uint32_t n = (uint32_t)((a.nnz - z0) < (uint64_t)kHiTile ? (a.nnz - z0) : (uint64_t)kHiTile);
    if (tid == 0) {
        mbar_init(&mbar, 1);
        mbar_fence_init();
    }
    __syncthreads();
    if (tid == 0) {
        const uint32_t bv = NIN == 3 ? round16(4 * n) : 0u;
        mbar_arrive_expect_tx(&mbar, 16 * n + bv);
        bulk_g2s_ef(s_rec, a.recs + z0, 16 * n, &mbar);
        if constexpr (NIN == 3) bulk_g2s_ef(s_v3, a.rvals + z0, bv, &mbar);
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
    // an odd slice length puts the groups' first records on different shared-memory banks
    const uint32_t per = ((n + kGroups - 1) / kGroups) | 1u;
    const uint32_t j0 = min(g * per, n), j1 = min(j0 + per, n);
    walk_rows<G, CPL, U, FT, NIN>(s_rec, s_v3, n, j0, j1, g, lane, a, s_slots, s_slot_row, s_slot_whole);
}

// Decodes a HiCOO schedule into records (HicooModePlan::recs): the nonzero at
// schedule position j lies in block tile_block[j / kHiTile] + lblk[j] of the
// schedule's block order.  Operands in increasing mode order.
struct RecBuildArgs {
    uint64_t n, nb;
    uint32_t nin, sb;
    const uint16_t *lblk;
    const uint32_t *tile_block;
    const uint32_t *out_bind;
    const uint8_t *out_eind;
    uint32_t out_dim;
    const uint32_t *in_bind[3];
    const uint8_t *in_eind[3];
    uint32_t in_dim[3];
    const float *vals;
    uint4 *recs;
    float *rvals;
    uint32_t *err;
};

__global__ void build_records_kernel(RecBuildArgs r)
{
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < r.n; j += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b0 = (uint64_t)r.tile_block[j / kHiTile] + r.lblk[j];
        const bool ok_b = b0 < r.nb;
        const uint64_t b = ok_b ? b0 : 0;
        const uint64_t o = ((uint64_t)r.out_bind[b] << r.sb) + r.out_eind[j];
        const bool ok_o = ok_b && o < r.out_dim;
        uint32_t row[3] = {0u, 0u, 0u};
        bool ok_in = true;
        for (uint32_t k = 0; k < r.nin; ++k) {
            const uint64_t rk = ((uint64_t)r.in_bind[k][b] << r.sb) + r.in_eind[k][j];
            ok_in = ok_in && rk < r.in_dim[k];
            row[k] = (uint32_t)rk;
        }
        if (!ok_in) row[0] = row[1] = row[2] = 0u;
        const float v = ok_o && ok_in ? r.vals[j] : 0.f;
        uint4 rec = make_uint4(ok_o ? (uint32_t)o : kNoRow, row[0], row[1], row[2]);
        if (r.nin == 1) rec.z = __float_as_uint(v);
        if (r.nin == 2) rec.w = __float_as_uint(v);
        if (r.nin == 3) r.rvals[j] = v;
        r.recs[j] = rec;
        if (!(ok_o && ok_in)) atomicOr(r.err, 1u);
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
        bulk_g2s_ef(s_rec, recs + z0 * RW, bytes, &mbar);
    }
    const bool ok = mbar_wait_bounded(&mbar, 0);
    if (!__syncthreads_and(ok)) {
        if (tid == 0) {
            atomicOr(a.err, 2u);
            mbar_wait_bounded(&mbar, 0);
        }
        return;
    }
    __shared__ uint32_t s_slot_row[kSchedThreads];
    __shared__ uint8_t s_slot_whole[kSchedThreads];
    float *s_slots = reinterpret_cast<float *>(sm + (size_t)kTile * RW * 4);  // [groups][G][CPL]
    const uint32_t g = tid / G, lane = tid % G;
    constexpr uint32_t kGroups = kSchedThreads / G;
    const uint32_t per = ((n + kGroups - 1) / kGroups) | 1u;  // odd: groups start on different banks
    const uint32_t j0 = min(g * per, n), j1 = min(j0 + per, n);
    process_records<G, CPL, U, NIN, FT>(s_rec, n, j0, j1, g, lane, a, a.vals ? a.vals + z0 : nullptr, s_slots,
                                        s_slot_row, s_slot_whole);
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

// 4-D schedules: each block's coordinates as one record {output mode,
// operand modes in increasing order}.
__global__ void pack_bquad_kernel(const uint32_t *bo, const uint32_t *b0, const uint32_t *b1, const uint32_t *b2,
                                  uint64_t nb, uint4 *q)
{
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += (uint64_t)gridDim.x * blockDim.x)
        q[i] = make_uint4(bo[i], b0[i], b1[i], b2[i]);
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

// Position of every nonzero in block order (blocks in their new order, the
// nonzeros of a block in their stored order): order[pos] = z.
__global__ void block_order_kernel(const uint32_t *blk, const uint32_t *inv, const uint64_t *bptr,
                                   const uint64_t *nbptr, uint64_t n, uint32_t *order)
{
    for (uint64_t z = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; z < n; z += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t b = blk[z];
        order[nbptr[inv[b]] + (z - bptr[b])] = (uint32_t)z;
    }
}

// One CTA per tile of the block order: stable sort of the tile's nonzeros by
// output row (a bitonic sort of (row, position) pairs in shared memory).
__global__ void __launch_bounds__(256) tile_sort_kernel(const uint32_t *order, uint64_t n, const uint32_t *blk,
                                                        const uint32_t *bout, const uint8_t *eout, uint32_t sb,
                                                        uint32_t *sorted)
{
    constexpr uint32_t T = kHiTile;
    static_assert((T & (T - 1)) == 0 && T <= 4096, "tile must be a power of two of at most 4096");
    __shared__ uint64_t key[T];
    const uint64_t z0 = (uint64_t)blockIdx.x * T;
    const uint32_t cnt = (uint32_t)((n - z0) < T ? (n - z0) : T);
    for (uint32_t i = threadIdx.x; i < T; i += blockDim.x) {
        if (i < cnt) {
            const uint32_t z = order[z0 + i];
            const uint64_t row = ((uint64_t)bout[blk[z]] << sb) + eout[z];
            key[i] = (row << 12) | i;
        } else {
            key[i] = ~0ull;  // padding sorts last
        }
    }
    __syncthreads();
    for (uint32_t k = 2; k <= T; k <<= 1)
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t i = threadIdx.x; i < T; i += blockDim.x) {
                const uint32_t ixj = i ^ j;
                if (ixj > i) {
                    const uint64_t x = key[i], y = key[ixj];
                    if ((x > y) == ((i & k) == 0)) {
                        key[i] = y;
                        key[ixj] = x;
                    }
                }
            }
            __syncthreads();
        }
    for (uint32_t i = threadIdx.x; i < cnt; i += blockDim.x) sorted[z0 + i] = order[z0 + (uint32_t)(key[i] & 4095u)];
}

// Block of the nonzero at position j, counted from the first block of its tile.
__global__ void local_block_kernel(const uint32_t *order, uint64_t n, const uint32_t *blk, const uint32_t *inv,
                                   const uint32_t *tile_block, uint16_t *lblk)
{
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (uint64_t)gridDim.x * blockDim.x)
        lblk[j] = (uint16_t)(inv[blk[order[j]]] - tile_block[j / kHiTile]);
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

int prepare_mode(ptiB200Tensor *t, uint32_t mode, cudaStream_t s, const Arrivals *arr)
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
    DevBuf bkeys, bperm, inv, bsize, nbptr;
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
    PTI_CUDA(nbptr.alloc(padded((nb + 1) * 8), s), mod);
    {
        DevBuf tmp;
        PTI_CUDA(tmp.alloc(padded(scan_tmp_elems<uint64_t>(nb) * 8), s), mod);
        PTI_TRY((exclusive_scan<uint64_t>(SizeIn{bsize.as<uint32_t>()}, BptrOut{nbptr.as<uint64_t>()}, nb,
                                          tmp.as<uint64_t>(), nullptr, s)));
        PTI_CUDA(cudaMemcpyAsync(nbptr.as<uint64_t>() + nb, tmp.as<uint64_t>() + (nb + kScanTile - 1) / kScanTile,
                                 8, cudaMemcpyDeviceToDevice, s), mod);
    }
    bsize.reset();
    P.nb = nb;
    P.ntiles = (uint32_t)((n + kHiTile - 1) / kHiTile);
    PTI_CUDA(P.tile_block.alloc(padded(((size_t)P.ntiles + 1) * 4), s), mod);
    tile_block_kernel_t<<<grid_n(nb), 256, 0, s>>>(nbptr.as<uint64_t>(), nb, P.ntiles, kHiTile,
                                                   P.tile_block.as<uint32_t>());
    {
        // 2. nonzeros in block order (blocks in their new order), then 3. inside
        // each tile of that order by output row
        DevBuf blk, border, order;
        PTI_CUDA(blk.alloc(padded(n * 4), s), mod);
        block_of_nnz_kernel<<<grid_n(nb), 256, 0, s>>>(t->bptr.as<uint64_t>(), nb, blk.as<uint32_t>());
        PTI_CUDA(border.alloc(padded(n * 4), s), mod);
        block_order_kernel<<<grid_n(n), 256, 0, s>>>(blk.as<uint32_t>(), inv.as<uint32_t>(), t->bptr.as<uint64_t>(),
                                                     nbptr.as<uint64_t>(), n, border.as<uint32_t>());
        PTI_CUDA(order.alloc(padded(n * 4), s), mod);
        tile_sort_kernel<<<P.ntiles, 256, 0, s>>>(border.as<uint32_t>(), n, blk.as<uint32_t>(),
                                                  t->binds[mode].as<uint32_t>(), t->einds[mode].as<uint8_t>(), t->sb,
                                                  order.as<uint32_t>());
        border.reset();
        // 4. everything up to here read only bptr and the output mode's arrays;
        // the gathers below read every array, each after its own arrival
        // (with `arr`), in the order the arrays arrive: the output mode's,
        // the values, then the other modes
        PTI_CUDA(P.lblk.alloc(padded(n * 2), s), mod);
        local_block_kernel<<<grid_n(n), 256, 0, s>>>(order.as<uint32_t>(), n, blk.as<uint32_t>(), inv.as<uint32_t>(),
                                                     P.tile_block.as<uint32_t>(), P.lblk.as<uint16_t>());
        auto wait = [&](cudaEvent_t ev) -> int {
            if (ev) PTI_CUDA(cudaStreamWaitEvent(s, ev, 0), mod);
            return 0;
        };
        auto gather_mode = [&](uint32_t k) -> int {
            if (arr) PTI_TRY(wait(arr->mode[k]));
            PTI_CUDA(P.binds[k].alloc(padded(nb * 4), s), mod);
            gather_kernel<uint32_t><<<grid_n(nb), 256, 0, s>>>(t->binds[k].as<uint32_t>(), bperm.as<uint32_t>(), nb,
                                                               P.binds[k].as<uint32_t>());
            PTI_CUDA(P.einds[k].alloc(padded(n), s), mod);
            gather_kernel<uint8_t><<<grid_n(n), 256, 0, s>>>(t->einds[k].as<uint8_t>(), order.as<uint32_t>(), n,
                                                             P.einds[k].as<uint8_t>());
            return 0;
        };
        PTI_TRY(gather_mode(mode));
        if (arr) PTI_TRY(wait(arr->vals));
        PTI_CUDA(P.vals.alloc(padded(n * 4), s), mod);
        gather_kernel<float><<<grid_n(n), 256, 0, s>>>(t->vals.as<float>(), order.as<uint32_t>(), n,
                                                       P.vals.as<float>());
        for (uint32_t k = 0; k < N; ++k)
            if (k != mode) PTI_TRY(gather_mode(k));
        bperm.reset();
        if (N == 4) {
            uint32_t o[3], c = 0;
            for (uint32_t k = 0; k < N; ++k)
                if (k != mode) o[c++] = k;
            PTI_CUDA(P.bquad.alloc(padded(nb * 16), s), mod);
            pack_bquad_kernel<<<grid_n(nb), 256, 0, s>>>(P.binds[mode].as<uint32_t>(), P.binds[o[0]].as<uint32_t>(),
                                                         P.binds[o[1]].as<uint32_t>(), P.binds[o[2]].as<uint32_t>(),
                                                         nb, P.bquad.as<uint4>());
        }
        // 5. the decoded records the MTTKRP kernel stages
        PTI_TRY(ensure_err_word(t, s));
        PTI_CUDA(P.recs.alloc(padded(n * 16), s), mod);
        if (N == 4) PTI_CUDA(P.rvals.alloc(padded(n * 4), s), mod);
        RecBuildArgs ra{};
        ra.n = n;
        ra.nb = nb;
        ra.nin = N - 1;
        ra.sb = t->sb;
        ra.lblk = P.lblk.as<uint16_t>();
        ra.tile_block = P.tile_block.as<uint32_t>();
        ra.out_bind = P.binds[mode].as<uint32_t>();
        ra.out_eind = P.einds[mode].as<uint8_t>();
        ra.out_dim = t->ndims[mode];
        for (uint32_t k = 0, i = 0; k < N; ++k)
            if (k != mode) {
                ra.in_bind[i] = P.binds[k].as<uint32_t>();
                ra.in_eind[i] = P.einds[k].as<uint8_t>();
                ra.in_dim[i] = t->ndims[k];
                ++i;
            }
        ra.vals = P.vals.as<float>();
        ra.recs = P.recs.as<uint4>();
        ra.rvals = N == 4 ? P.rvals.as<float>() : nullptr;
        ra.err = err_word(t);
        build_records_kernel<<<grid_n(n), 256, 0, s>>>(ra);
    }
    inv.reset();
    PTI_CUDA(cudaGetLastError(), mod);
    P.ready = true;
    return 0;
}

// ---------------------------------------------------------------------------
// Launch
// ---------------------------------------------------------------------------
// Records in flight per group of the COO walk (FP32, R <= 32) and the CTAs
// per SM its register budget is set for: compile-time choices.
#ifndef PTI_COO_U
#define PTI_COO_U 3
#endif
// ... and for 33 <= R <= 64 (3 fit the same 64-register budget as 2)
#ifndef PTI_COO_U64
#define PTI_COO_U64 3
#endif
#ifndef PTI_COO_MINB
#define PTI_COO_MINB 4
#endif

template <int G, int CPL, int U, class FT, int NIN>
static int launch_coo(const SchedArgs &a, const uint32_t *recs, unsigned ntiles, cudaStream_t s)
{
    const size_t smem = (size_t)kTile * Rec<NIN>::words * 4 + (size_t)kSchedThreads * CPL * 4;
    constexpr int UU = NIN == 3 && U > 2 ? 2 : U;  // 4-D records hold more registers per nonzero
    auto k = coo_sched_kernel<G, CPL, UU, PTI_COO_MINB, FT, NIN>;
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return PTIERR_CUDA_ERROR;
    k<<<ntiles, kSchedThreads, smem, s>>>(a, recs);
    return 0;
}

// Which HiCOO kernel runs (a compile-time choice): 0 decodes every tile from
// the staged HiCOO arrays (hicoo_sched_kernel), 2 stages the schedule's
// decoded records (hicoo_rec_kernel), 1 takes the records for 4-D tensors and
// for BF16 factors and decodes 3-D FP32 tiles.
#ifndef PTI_REC_POLICY
#define PTI_REC_POLICY 1
#endif
// CTAs per SM the BF16 record kernels are held to (0: no limit).  Their walk
// is bound by the L1 data pipe and feeds on the L1 that a further CTA's
// shared memory would take.
#ifndef PTI_REC_BF16_CTAS
#define PTI_REC_BF16_CTAS 3
#endif

template <class FT, int NIN>
constexpr bool use_records()
{
    return PTI_REC_POLICY == 2 || (PTI_REC_POLICY == 1 && (NIN == 3 || sizeof(FT) == 2));
}

template <int G, int CPL, class FT, int NIN>
static int launch_hicoo(const SchedArgs &a, unsigned ntiles, cudaStream_t s)
{
    constexpr int U = NIN == 3 || CPL == 8 ? 2 : PTI_HICOO_U;  // nonzeros in flight per group
    size_t smem;
    void (*k)(SchedArgs);
    if constexpr (use_records<FT, NIN>()) {
        smem = RecSmem<NIN, CPL>::total;
        if (sizeof(FT) == 2 && PTI_REC_BF16_CTAS > 0) {
            // more dynamic shared memory than 1/(n+1) of the SM's 228 KB (with
            // the static part and the 1 KB the runtime keeps per CTA)
            const size_t cap = 233472 / (PTI_REC_BF16_CTAS + 1) - 1408 - 1024 + 16;
            smem = smem > cap ? smem : cap;
        }
        k = hicoo_rec_kernel<G, CPL, U, FT, NIN>;
    } else {
        smem = HiSmem<NIN, CPL>::total;
        k = hicoo_sched_kernel<G, CPL, U, FT, NIN>;
    }
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
    if (R <= 4) return launch_coo<1, 4, PTI_COO_U, FT, NIN>(a, recs, ntiles, s);
    if (R <= 8) return launch_coo<2, 4, PTI_COO_U, FT, NIN>(a, recs, ntiles, s);
    if (R <= 16) return launch_coo<4, 4, PTI_COO_U, FT, NIN>(a, recs, ntiles, s);
    if (R <= 32) return launch_coo<8, 4, PTI_COO_U, FT, NIN>(a, recs, ntiles, s);
    if (R <= 64) return launch_coo<16, 4, PTI_COO_U64, FT, NIN>(a, recs, ntiles, s);
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

bool schedule_supported(const ptiB200Tensor *t, uint32_t R, uint32_t stride)
{
    if (!(t->nmodes >= 2 && t->nmodes <= 4 && R >= 1 && R <= 128)) return false;
    // the HiCOO kernel addresses factor rows by 32-bit element offsets
    if (t->hicoo)
        for (uint32_t m = 0; m < t->nmodes; ++m)
            if ((uint64_t)t->ndims[m] * stride >= ((uint64_t)1 << 32)) return false;
    return true;
}

// Runs the scheduled kernel for `mode` (the schedule must be ready).  Output
// must already be zeroed.
int mttkrp_scheduled(ptiB200Tensor *t, const void *const *mats, int ft, uint32_t R, uint32_t stride,
                     const uint32_t *mats_order, uint32_t mode, float *out, cudaStream_t s,
                     const float *vals_override)
{
    const char *mod = "B200 MTTKRP";
    const uint32_t N = t->nmodes;
    PTI_TRY(ensure_err_word(t, s));
    SchedArgs a{};
    a.nnz = t->nnz;
    a.R = R;
    a.stride = stride;
    a.out_dim = t->ndims[mode];
    a.out = out;
    a.err = err_word(t);
    const uint32_t *recs = nullptr;
    unsigned ntiles;
    if (t->hicoo) {
        const HicooModePlan &P = t->hicoo_plan[mode];
        ntiles = P.ntiles;
        a.nb = P.nb;
        a.sb = t->sb;
        a.lblk = P.lblk.as<uint16_t>();
        a.tile_block = P.tile_block.as<uint32_t>();
        a.out_bind = P.binds[mode].as<uint32_t>();
        a.out_eind = P.einds[mode].as<uint8_t>();
        // the operands in increasing mode order: the order of the decoded
        // records and of the 4-D block records (a product of two factors does
        // not depend on the order, of three only in its FP32 rounding)
        (void)mats_order;
        for (uint32_t i = 0, k = 0; k < N; ++k)
            if (k != mode) {
                a.in_bind[i] = P.binds[k].as<uint32_t>();
                a.in_eind[i] = P.einds[k].as<uint8_t>();
                a.in_dim[i] = t->ndims[k];
                a.in_mat[i] = mats[k];
                ++i;
            }
        a.bquad = N == 4 ? P.bquad.as<uint4>() : nullptr;
        a.vals = P.vals.as<float>();
        a.recs = P.recs.as<uint4>();
        a.rvals = P.rvals.as<float>();
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
