// tensor.cuh -- the device-resident tensor behind a ptiB200Tensor handle.
#pragma once
#include "common.cuh"

#include <array>
#include <memory>

namespace pti {

constexpr int kMaxModes = 8;

// Nonzeros per tile of a per-mode HiCOO schedule (HicooModePlan::tile_block);
// a power of two of at most 4096 (a compile-time choice, -DPTI_PLAN_TILE).
#ifndef PTI_PLAN_TILE
#define PTI_PLAN_TILE 2048
#endif
constexpr int kPlanTile = PTI_PLAN_TILE;

// Per-mode schedule of a HiCOO tensor.  The blocks are re-ordered by their
// block coordinate in the output mode (a materialised form of the reference's
// per-mode kernel scheduler kschr, src/sptensor/hicoo/convert.c:378-421) and
// the nonzeros follow their blocks; the nonzeros are then cut into tiles of
// kPlanTile, and inside each tile re-ordered by output row.  A nonzero keeps
// its HiCOO encoding -- 8-bit element offsets per mode, plus the index of its
// block among the tile's blocks (tile t covers blocks tile_block[t] ..
// tile_block[t+1] of binds) -- so a tile is staged as it is and decoded
// without sorting.
struct HicooModePlan {
    bool ready = false;
    uint64_t nb = 0;
    std::array<DevBuf, kMaxModes> binds;  // uint32 [nb]: block coordinates, blocks in output order
    std::array<DevBuf, kMaxModes> einds;  // uint8  [nnz]: element offsets, tile-local row order
    DevBuf vals;                          // float  [nnz]
    DevBuf lblk;                          // uint16 [nnz]: block of the nonzero - tile_block[tile]
    DevBuf tile_block;                    // uint32 [ntiles+1]: first block of each tile
    uint32_t ntiles = 0;
    DevBuf bquad;                         // 4-D: uint4 [nb], {output, operands in increasing mode order}
    // The same nonzeros decoded, in schedule order: {output row, operand
    // rows in increasing mode order, value bits (3-D) or the third operand
    // row (4-D)}, with the 4-D values beside them.  A coordinate out of range
    // decodes to a record that adds nothing (value 0, operand rows 0; output
    // row kNoRow when the output coordinate is the bad one).
    DevBuf recs;                          // uint4 [nnz]
    DevBuf rvals;                         // float [nnz], 4-D only
};

// Per-mode schedule of a COO tensor: nonzeros sorted by the output-mode index,
// packed as 16- or 32-byte records {out index, operand indices, value}.
struct CooModePlan {
    bool ready = false;
    DevBuf recs;                          // uint32 [nnz][4 or 8]
    DevBuf perm;                          // uint32 [nnz]: record j holds input nonzero perm[j]
    DevBuf alt_vals;                      // float [nnz]: caller-supplied values in record order
};

// Fibers of a COO tensor along one mode (TTM / TTV): the nonzeros sorted by
// the other modes with the mode last, cut where any other mode changes.
struct FiberPlan {
    bool ready = false;
    uint64_t nfib = 0;
    DevBuf fptr;                           // uint64 [nfib+1]: first nonzero of each fiber
    std::array<DevBuf, kMaxModes> finds;   // uint32 [nfib]: the fiber's coordinate in every other mode
    DevBuf sind;                           // uint32 [nnz]: the mode's index, fiber order
    DevBuf sval;                           // float  [nnz]: values, fiber order
    DevBuf perm;                           // uint32 [nnz]: fiber-order position -> input nonzero
    uint64_t nlong = 0;                    // fibers longer than one thread takes, up to the CTA limit
    uint64_t nvlong = 0;                   // fibers longer than that, one CTA each
    uint64_t nshort = 0;                   // fibers one thread takes
    DevBuf short_fibs;                     // uint4 [nshort]: {fiber, length, first nonzero} by length class
    DevBuf long_fibers;                    // uint32 [nfib]: the nlong fibers from the front, the nvlong from the back
};

}  // namespace pti

struct ptiB200Tensor {
    bool hicoo = false;
    uint32_t nmodes = 0;
    std::vector<uint32_t> ndims;
    uint64_t nnz = 0;
    int device = 0;

    // COO storage (also kept for HiCOO tensors built on the device from COO)
    std::array<pti::DevBuf, pti::kMaxModes> inds;  // uint32 [nnz]
    pti::DevBuf vals;                              // float  [nnz]

    // HiCOO storage
    uint64_t nb = 0;
    uint8_t sb = 0, sk = 0, sc = 0;
    pti::DevBuf bptr;                                // uint64 [nb+1]
    std::array<pti::DevBuf, pti::kMaxModes> binds;   // uint32 [nb]
    std::array<pti::DevBuf, pti::kMaxModes> einds;   // uint8  [nnz]
    pti::DevBuf tile_block;                          // first block of each nnz tile
    uint32_t ntiles = 0;

    pti::DevBuf err;  // uint32: device error word of this tensor's kernels

    std::array<pti::CooModePlan, pti::kMaxModes> coo_plan;
    std::array<pti::HicooModePlan, pti::kMaxModes> hicoo_plan;
    std::array<pti::FiberPlan, pti::kMaxModes> fiber_plan;
};

namespace pti {

// Events marking when a HiCOO tensor's arrays reach the device, for a
// schedule built while its copies still run (the drop-in HiCOO MTTKRP): each
// gather of the schedule waits only for its own array.  A null event means
// the array is already ordered before the caller's stream.
struct Arrivals {
    cudaEvent_t mode[kMaxModes] = {};  // binds[m] and einds[m]
    cudaEvent_t vals = nullptr;
    cudaEvent_t all = nullptr;         // everything the kernel reads, the factors included
};

int upload_coo(ptiB200Tensor *t, const ptiSparseTensor *X, cudaStream_t s);
// Checks every index of a device COO tensor against the mode sizes.
int check_coo_ranges(ptiB200Tensor *t, cudaStream_t s);
// Reads a .tns/.coo/.bin file into t's COO arrays on the GPU (ingest.cu);
// `text` (may be NULL) receives whether the text parser ran.  Synchronous.
int ingest_file(ptiB200Tensor *t, uint32_t start_index, const char *fname, bool *text, cudaStream_t s);
// Sorts t's nonzeros by coordinate and merges repeated coordinates.
int dedupe_coo(ptiB200Tensor *t, cudaStream_t s);
// With s2, the arrays that mode first_mode's schedule does not need first
// (the values, the other modes' coordinates and offsets) are copied on s2,
// and the events of `arr` (created by the caller) are recorded on s2 as they
// land.
int upload_hicoo(ptiB200Tensor *t, const ptiSparseTensorHiCOO *H, cudaStream_t s, int first_mode = -1,
                 cudaStream_t s2 = nullptr, Arrivals *arr = nullptr);

// MTTKRP launchers; factors are device pointers (element type ft), out is FP32.
// vals_override (optional): nnz values in the tensor's input order that replace
// its own values (COO tensors only).
// arr (optional): arrival events of the tensor's arrays and the factors; the
// schedule build and the kernel wait for each only where they read it.
int mttkrp_device(ptiB200Tensor *t, const void *const *mats, int ft, uint32_t R, uint32_t stride,
                  const uint32_t *mats_order, uint32_t mode, float *out, cudaStream_t s,
                  const float *vals_override = nullptr, const Arrivals *arr = nullptr);
int prepare_mode(ptiB200Tensor *t, uint32_t mode, cudaStream_t s, const Arrivals *arr = nullptr);

// Host-struct MTTKRP used by the reference entry points.
int mttkrp_host_coo(const ptiSparseTensor *X, ptiMatrix **mats, const ptiIndex *mats_order,
                    ptiIndex mode);
int mttkrp_host_hicoo(const ptiSparseTensorHiCOO *H, ptiMatrix **mats, const ptiIndex *mats_order,
                      ptiIndex mode);

}  // namespace pti
