// renumber.cu -- Lexi-order index renumbering on the GPU.
//
// The reference's Lexi-order (src/sptensor/renumber.c:26-92 and :403-520,
// lexOrderThem at :93-225) renumbers the indices of one mode at a time: the
// tensor is matricised with the other modes' coordinate tuples as rows
// (numbered in lexicographic order of the tuples, mode_order = the other modes
// ascending) and the mode's indices as columns, and the columns are put in
// the order that partition refinement over the rows in sequence produces.
// That order is the lexicographic order of the columns' sorted row lists in
// which, at the first row where two columns differ, the column present in the
// row comes first (so a list comes before its own prefixes, and indices with
// no nonzeros come last).  Every mode is renumbered in turn, `iterations`
// times, each pass seeing the other modes' latest numbering.
//
// Here the row lists are compared by prefix doubling, as in suffix-array
// construction: rank_0(p) is the row at list position p; rank_{k+1}(p) is the
// rank of the pair (rank_k(p), rank_k(p + 2^k)), with positions past the end
// of p's list ranking above everything.  After ceil(log2(longest list))
// rounds, the rank at a list's first position is the rank of the whole list.
// Every round is one stable radix sort of the nnz pairs.  Columns with equal
// lists keep their current relative order; the reference leaves those in the
// order of its last shared row, which its (unstable) quicksort decides, so
// the two agree exactly whenever no two indices of a mode have the same row
// list.
//
// The reference has two drivers of this ordering: orderit
// (src/sptensor/orderit.c:121-208), whose quicksort of the nonzeros by the
// other modes is correct, and ptiIndexRenumber (renumber.c:26-92), whose
// except-one-mode sort (pti_QuickSortIndexExceptSingleMode, sort.c:1500-1566)
// ends in an insertion sort that keeps comparing a fixed slot while the
// element it inserts moves away.  That sort leaves the nonzeros unsorted, so
// rows are split and its result depends on the order of the nonzeros.  Both
// entry points here compute orderit's ordering.
#include "primitives.cuh"
#include "tensor.cuh"

namespace pti {
namespace {

unsigned grid_n(uint64_t n)
{
    return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, (uint64_t)sm_count() * 8));
}

#define GRID_LOOP(i, n) \
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += (uint64_t)gridDim.x * blockDim.x)

__global__ void iota_k(uint32_t *v, uint64_t n) { GRID_LOOP(i, n) v[i] = (uint32_t)i; }

__global__ void gather_key_k(const uint32_t *ind, const uint32_t *perm, uint64_t n, uint64_t *key)
{
    GRID_LOOP(i, n) key[i] = ind[perm[i]];
}

// Rows of the matricisation: in nonzero order `perm` (sorted by the other
// modes, then the column), a new row starts where any other mode changes.
struct RowArgs {
    uint32_t nmodes, mode;
    const uint32_t *inds[kMaxModes];
    const uint32_t *perm;
};
struct RowHeadIn {
    RowArgs a;
    __device__ uint32_t operator()(uint64_t i) const
    {
        if (i == 0) return 0;
        const uint32_t p = a.perm[i], q = a.perm[i - 1];
        for (uint32_t m = 0; m < a.nmodes; ++m)
            if (m != a.mode && a.inds[m][p] != a.inds[m][q]) return 1;
        return 0;
    }
};
// row id of sorted position i = number of row starts before or at i (minus the first)
struct RowOut {
    RowArgs a;
    uint64_t *col_key;  // column of position i (sort key for the column-major pass)
    uint32_t *row;      // row of position i
    __device__ void operator()(uint64_t i, uint32_t prefix, uint32_t head) const
    {
        row[i] = prefix + head;
        col_key[i] = a.inds[a.mode][a.perm[i]];
    }
};

// After the column-major sort (col_key ascending, rows ascending inside):
// list start and end of every column, and the longest list.
__global__ void list_bounds_k(const uint64_t *col, uint64_t n, uint32_t *start, uint32_t *end, unsigned *maxlen)
{
    GRID_LOOP(p, n)
    {
        const uint32_t c = (uint32_t)col[p];
        if (p == 0 || col[p - 1] != c) start[c] = (uint32_t)p;
        if (p + 1 == n || col[p + 1] != c) end[c] = (uint32_t)(p + 1);
    }
    (void)maxlen;
}
__global__ void list_len_k(const uint32_t *start, const uint32_t *end, uint32_t ncols, unsigned *maxlen)
{
    unsigned mx = 0;
    GRID_LOOP(c, ncols) if (end[c] > start[c]) mx = max(mx, end[c] - start[c]);
    for (int o = 16; o; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0 && mx) atomicMax(maxlen, mx);
}

// pair key of position p: rank(p) in the high bits, rank(p + h) (or INF past
// the end of p's list) in the low b bits
__global__ void pair_key_k(const uint32_t *rank, const uint64_t *col, const uint32_t *end, uint64_t n, uint64_t h,
                           int b, uint32_t inf, uint64_t *key)
{
    GRID_LOOP(p, n)
    {
        const uint32_t e = end[(uint32_t)col[p]];
        const uint32_t second = p + h < e ? rank[p + h] : inf;
        key[p] = ((uint64_t)rank[p] << b) | second;
    }
}

struct PairHeadIn {
    const uint64_t *key;
    __device__ uint32_t operator()(uint64_t i) const { return i == 0 ? 0 : (key[i] != key[i - 1] ? 1 : 0); }
};
struct RankOut {
    const uint32_t *pos;
    uint32_t *rank;
    __device__ void operator()(uint64_t i, uint32_t prefix, uint32_t head) const { rank[pos[i]] = prefix + head; }
};

// column key: rank of its whole list, or `inf` for an index with no nonzeros
__global__ void col_key_k(const uint32_t *rank, const uint32_t *start, const uint32_t *end, uint32_t ncols,
                          uint32_t inf, uint64_t *key)
{
    GRID_LOOP(c, ncols) key[c] = end[c] > start[c] ? rank[start[c]] : inf;
}

// order[newpos] = old column; inv[old] = newpos; org'[newpos] = org[old]
__global__ void apply_order_k(const uint32_t *order, uint32_t ncols, const uint32_t *org, uint32_t *inv,
                              uint32_t *org_new)
{
    GRID_LOOP(i, ncols)
    {
        inv[order[i]] = (uint32_t)i;
        org_new[i] = org[order[i]];
    }
}

__global__ void remap_k(uint32_t *ind, const uint32_t *inv, uint64_t n) { GRID_LOOP(i, n) ind[i] = inv[ind[i]]; }

__global__ void final_map_k(const uint32_t *org, uint32_t ncols, uint32_t *map)
{
    GRID_LOOP(i, ncols) map[org[i]] = (uint32_t)i;
}

int bits_of(uint64_t maxval)
{
    int b = 0;
    while (b < 64 && (maxval >> b)) ++b;
    return b;
}

// One Lexi-order pass over `mode`: renumbers inds[mode] in place and
// composes org (current index -> original index).
int lexi_order_mode(uint32_t N, const std::vector<uint32_t> &ndims, uint64_t nnz, uint32_t *const *inds,
                    uint32_t mode, DevBuf &org, cudaStream_t s)
{
    const char *mod = "B200 Renumber";
    const uint32_t ncols = ndims[mode];
    if (ncols == 0) return 0;
    DevBuf perm, key, row, colk, start, end, rank, pos, tmp, scal, order, inv, org_new;
    RadixScratch sc;
    const uint64_t n = nnz;
    // radix_sort_pairs exchanges its buffers with the scratch ones, so every
    // buffer it sorts has room for the longest sort (n or ncols elements)
    const uint64_t M = std::max<uint64_t>(n, ncols);
    PTI_CUDA(perm.alloc(padded(M * 4), s), mod);
    PTI_CUDA(key.alloc(padded(M * 8), s), mod);
    PTI_CUDA(row.alloc(padded(M * 4), s), mod);
    PTI_CUDA(colk.alloc(padded(M * 8), s), mod);
    PTI_CUDA(pos.alloc(padded(M * 4), s), mod);
    PTI_CUDA(order.alloc(padded(M * 4), s), mod);
    PTI_CUDA(start.alloc(padded((uint64_t)ncols * 4), s), mod);
    PTI_CUDA(end.alloc(padded((uint64_t)ncols * 4), s), mod);
    PTI_CUDA(tmp.alloc(padded(scan_tmp_elems<uint32_t>(std::max<uint64_t>(n, 1)) * 4), s), mod);
    PTI_CUDA(scal.alloc(padded(16), s), mod);
    PTI_TRY(sc.alloc(M, s));

    if (n) {
        // 1. nonzeros sorted by the other modes (mode_order ascending, the
        //    first most significant), then by the column: LSD, stable
        iota_k<<<grid_n(n), 256, 0, s>>>(perm.as<uint32_t>(), n);
        for (int m = (int)N; m >= 0; --m) {
            const uint32_t mm = m == (int)N ? mode : (uint32_t)m;  // the column first
            if (m != (int)N && mm == mode) continue;
            gather_key_k<<<grid_n(n), 256, 0, s>>>(inds[mm], perm.as<uint32_t>(), n, key.as<uint64_t>());
            PTI_TRY(radix_sort_pairs(key, perm, n, ((bits_of(ndims[mm] ? ndims[mm] - 1 : 0) + 7) / 8) * 8, sc, s));
        }
        // 2. row ids, and each position's column
        RowArgs ra;
        ra.nmodes = N;
        ra.mode = mode;
        for (uint32_t m = 0; m < N; ++m) ra.inds[m] = inds[m];
        ra.perm = perm.as<uint32_t>();
        PTI_TRY((exclusive_scan<uint32_t>(RowHeadIn{ra}, RowOut{ra, colk.as<uint64_t>(), row.as<uint32_t>()}, n,
                                          tmp.as<uint32_t>(), nullptr, s)));
        // 3. column-major: stable sort by column keeps rows ascending in each list
        PTI_TRY(radix_sort_pairs(colk, row, n, ((bits_of(ncols - 1) + 7) / 8) * 8, sc, s));
    }
    PTI_CUDA(cudaMemsetAsync(start.ptr, 0, (size_t)ncols * 4, s), mod);
    PTI_CUDA(cudaMemsetAsync(end.ptr, 0, (size_t)ncols * 4, s), mod);
    PTI_CUDA(cudaMemsetAsync(scal.ptr, 0, 16, s), mod);
    unsigned maxlen = 0;
    if (n) {
        list_bounds_k<<<grid_n(n), 256, 0, s>>>(colk.as<uint64_t>(), n, start.as<uint32_t>(), end.as<uint32_t>(),
                                                 nullptr);
        list_len_k<<<grid_n(ncols), 256, 0, s>>>(start.as<uint32_t>(), end.as<uint32_t>(), ncols,
                                                 scal.as<unsigned>());
        PTI_CUDA(cudaMemcpyAsync(&maxlen, scal.ptr, 4, cudaMemcpyDeviceToHost, s), mod);
        PTI_CUDA(cudaStreamSynchronize(s), mod);
    }
    // 4. prefix doubling over the lists; rank starts as the row id
    const uint32_t inf = (uint32_t)std::min<uint64_t>(n, 0xFFFFFFFEull);  // ranks and rows are < n
    const int b = bits_of(inf);
    if (n) {
        rank.swap(row);  // rank_0 = row at each position
        for (uint64_t h = 1; h < maxlen; h <<= 1) {
            pair_key_k<<<grid_n(n), 256, 0, s>>>(rank.as<uint32_t>(), colk.as<uint64_t>(), end.as<uint32_t>(), n, h,
                                                 b, inf, key.as<uint64_t>());
            iota_k<<<grid_n(n), 256, 0, s>>>(pos.as<uint32_t>(), n);
            PTI_TRY(radix_sort_pairs(key, pos, n, ((2 * b + 7) / 8) * 8, sc, s));
            PTI_TRY((exclusive_scan<uint32_t>(PairHeadIn{key.as<uint64_t>()}, RankOut{pos.as<uint32_t>(),
                                              rank.as<uint32_t>()}, n, tmp.as<uint32_t>(), nullptr, s)));
        }
    }
    // 5. columns by (rank of their list, current index); no list ranks last
    PTI_CUDA(inv.alloc(padded((uint64_t)ncols * 4), s), mod);
    PTI_CUDA(org_new.alloc(padded((uint64_t)ncols * 4), s), mod);
    col_key_k<<<grid_n(ncols), 256, 0, s>>>(n ? rank.as<uint32_t>() : nullptr, start.as<uint32_t>(),
                                            end.as<uint32_t>(), ncols, inf + 1, key.as<uint64_t>());
    iota_k<<<grid_n(ncols), 256, 0, s>>>(order.as<uint32_t>(), ncols);
    PTI_TRY(radix_sort_pairs(key, order, ncols, ((bits_of((uint64_t)inf + 1) + 7) / 8) * 8, sc, s));
    apply_order_k<<<grid_n(ncols), 256, 0, s>>>(order.as<uint32_t>(), ncols, org.as<uint32_t>(), inv.as<uint32_t>(),
                                                 org_new.as<uint32_t>());
    if (n) remap_k<<<grid_n(n), 256, 0, s>>>(inds[mode], inv.as<uint32_t>(), n);
    PTI_CUDA(cudaGetLastError(), mod);
    org.swap(org_new);
    return 0;
}

// ---------------------------------------------------------------------------
// BFS-like renumbering (renumber == 2): src/sptensor/renumber.c:534-839.
//
// The tensor is a hypergraph with a vertex per index of every mode and a
// hyperedge per nonzero.  Mode by mode, the mode's vertices are taken from a
// binary max-heap on a key (all 0 at first); on equal keys the heap prefers
// the smaller degree when it sifts down and the larger degree when it sifts
// up, as the reference's heapify and heapIncreaseKey do (:644-701).  The
// vertex taken gets the next new index; every vertex of its hyperedges not
// yet visited in this mode's pass is visited, and each hyperedge of that
// vertex raises by one the key of its own vertex in the mode, if that vertex
// is still in the heap.  Every vertex starts unvisited: the reference reads
// the visit marks of other modes' vertices before it ever writes them
// (renumber.c:768), so its own result depends on leftover heap memory and is
// not reproducible; this is the reading under which the loop is the
// maximum-cardinality search it describes.
//
// The vertex -> hyperedge lists are built on the GPU (a stable sort of the
// nonzero ids by each mode's index).  The walk itself is a priority queue
// whose every step depends on the keys the previous steps raised, so it runs
// on the host, one heap operation at a time.
// ---------------------------------------------------------------------------
__global__ void widen_k(const uint32_t *src, uint64_t n, uint64_t *dst) { GRID_LOOP(i, n) dst[i] = src[i]; }

// off[c] = number of keys below c, for c in [0, ncols]
__global__ void lower_bound_k(const uint64_t *key, uint64_t n, uint32_t ncols, uint64_t *off)
{
    GRID_LOOP(c, (uint64_t)ncols + 1)
    {
        uint64_t lo = 0, hi = n;
        while (lo < hi) {
            const uint64_t mid = (lo + hi) >> 1;
            if (key[mid] < c) lo = mid + 1;
            else hi = mid;
        }
        off[c] = lo;
    }
}

// Per mode: the nonzeros of every index, in increasing nonzero order.
struct VertexLists {
    std::vector<std::vector<uint32_t>> edges;  // [mode][nnz]
    std::vector<std::vector<uint64_t>> off;    // [mode][ndims + 1]
};

int vertex_lists(uint32_t N, const uint32_t *ndims, uint64_t nnz, const uint32_t *const *host_inds, VertexLists &vl,
                 cudaStream_t s)
{
    const char *mod = "B200 BFS-like renumbering";
    PTI_CHECK(nnz < 0xFFFFFFFFull, PTIERR_VALUE_ERROR, mod, "too many nonzeros");
    vl.edges.assign(N, {});
    vl.off.assign(N, {});
    uint32_t maxd = 0;
    for (uint32_t m = 0; m < N; ++m) maxd = std::max(maxd, ndims[m]);
    DevBuf ind, keys, vals, off;
    RadixScratch sc;
    if (nnz) {
        PTI_CUDA(ind.alloc(padded(nnz * 4), s), mod);
        PTI_CUDA(keys.alloc(padded(nnz * 8), s), mod);
        PTI_CUDA(vals.alloc(padded(nnz * 4), s), mod);
        PTI_TRY(sc.alloc(nnz, s));
    }
    PTI_CUDA(off.alloc(padded(((uint64_t)maxd + 1) * 8), s), mod);
    for (uint32_t m = 0; m < N; ++m) {
        vl.edges[m].resize(nnz);
        vl.off[m].assign((size_t)ndims[m] + 1, 0);
        if (!nnz) continue;
        PTI_CUDA(cudaMemcpyAsync(ind.ptr, host_inds[m], nnz * 4, cudaMemcpyHostToDevice, s), mod);
        widen_k<<<grid_n(nnz), 256, 0, s>>>(ind.as<uint32_t>(), nnz, keys.as<uint64_t>());
        iota_k<<<grid_n(nnz), 256, 0, s>>>(vals.as<uint32_t>(), nnz);
        PTI_TRY(radix_sort_pairs(keys, vals, nnz, ((bits_of(ndims[m] ? ndims[m] - 1 : 0) + 7) / 8) * 8, sc, s));
        lower_bound_k<<<grid_n((uint64_t)ndims[m] + 1), 256, 0, s>>>(keys.as<uint64_t>(), nnz, ndims[m],
                                                                     off.as<uint64_t>());
        PTI_CUDA(cudaGetLastError(), mod);
        PTI_CUDA(cudaMemcpyAsync(vl.edges[m].data(), vals.ptr, nnz * 4, cudaMemcpyDeviceToHost, s), mod);
        PTI_CUDA(cudaMemcpyAsync(vl.off[m].data(), off.ptr, ((size_t)ndims[m] + 1) * 8, cudaMemcpyDeviceToHost, s),
                 mod);
        PTI_CUDA(cudaStreamSynchronize(s), mod);
    }
    return 0;
}

// The heap of one mode's pass: slots 1..size hold vertices; pos[v] is v's
// slot (0 once taken).
struct BfsHeap {
    std::vector<uint32_t> slot, pos;
    std::vector<uint64_t> key;
    const uint64_t *off;  // degree(v) = off[v+1] - off[v]
    uint32_t size = 0;
    uint64_t deg(uint32_t v) const { return off[v + 1] - off[v]; }
    // the reference's sift-down preference: larger key, then smaller degree
    bool above_down(uint32_t a, uint32_t b) const
    {
        return key[a] > key[b] || (key[a] == key[b] && deg(a) < deg(b));
    }
    void down(uint32_t j)
    {
        while (j <= size / 2) {
            const uint32_t l = 2 * j, r = 2 * j + 1;
            uint32_t big = above_down(slot[l], slot[j]) ? l : j;
            if (r <= size && above_down(slot[r], slot[big])) big = r;
            if (big == j) break;
            std::swap(slot[big], slot[j]);
            pos[slot[big]] = big;
            pos[slot[j]] = j;
            j = big;
        }
    }
    // raises v's key by one and sifts it up (larger key, then larger degree)
    void raise(uint32_t v)
    {
        uint32_t i = pos[v];
        if (i == 0 || i > size) return;
        key[v] += 1;
        while (i > 1) {
            const uint32_t p = slot[i >> 1];
            if (!(key[v] > key[p] || (key[v] == key[p] && deg(v) > deg(p)))) break;
            slot[i] = p;
            pos[p] = i;
            i >>= 1;
        }
        slot[i] = v;
        pos[v] = i;
    }
    uint32_t take()
    {
        const uint32_t v = slot[1];
        slot[1] = slot[size];
        pos[slot[1]] = 1;
        --size;
        pos[v] = 0;
        down(1);
        return v;
    }
};

int bfs_like(uint32_t N, const uint32_t *ndims, uint64_t nnz, const uint32_t *const *host_inds, uint32_t **newIndices,
             cudaStream_t s)
{
    VertexLists vl;
    PTI_TRY(vertex_lists(N, ndims, nnz, host_inds, vl, s));
    std::vector<std::vector<uint8_t>> visited(N);
    for (uint32_t d = 0; d < N; ++d) {
        const uint32_t n = ndims[d];
        if (n == 0) continue;
        BfsHeap H;
        H.off = vl.off[d].data();
        H.slot.resize((size_t)n + 1);
        H.pos.resize(n);
        H.key.assign(n, 0);
        for (uint32_t v = 0; v < n; ++v) {
            H.slot[v + 1] = v;
            H.pos[v] = v + 1;
        }
        H.size = n;
        for (uint32_t j = n / 2; j >= 1; --j) H.down(j);
        for (uint32_t m = 0; m < N; ++m) visited[m].assign(m == d ? 0 : ndims[m], 0);
        const uint32_t *mine = host_inds[d];
        for (uint32_t t = 0; t < n; ++t) {
            const uint32_t v = H.take();
            newIndices[d][v] = t;
            for (uint64_t j = vl.off[d][v]; j < vl.off[d][v + 1]; ++j) {
                const uint32_t h = vl.edges[d][j];
                for (uint32_t k = 0; k < N; ++k) {
                    if (k == d) continue;
                    const uint32_t w = host_inds[k][h];
                    if (visited[k][w]) continue;
                    visited[k][w] = 1;
                    for (uint64_t jj = vl.off[k][w]; jj < vl.off[k][w + 1]; ++jj) H.raise(mine[vl.edges[k][jj]]);
                }
            }
        }
    }
    return 0;
}

}  // namespace

// Lexi-order renumbering of a device COO tensor.  maps[m] (device, ndims[m])
// receives original index -> new index; with `apply` the tensor's own
// coordinates are renumbered, otherwise a working copy is.
int renumber_device(ptiB200Tensor *t, uint32_t iterations, uint32_t *const *maps, bool apply, cudaStream_t s)
{
    const char *mod = "B200 Renumber";
    PTI_CHECK(t && !t->hicoo, PTIERR_VALUE_ERROR, mod, "needs a device COO tensor");
    const uint32_t N = t->nmodes;
    DevBuf work[kMaxModes], org[kMaxModes];
    uint32_t *inds[kMaxModes];
    for (uint32_t m = 0; m < N; ++m) {
        if (apply) {
            inds[m] = t->inds[m].as<uint32_t>();
        } else {
            PTI_CUDA(work[m].alloc(padded(t->nnz * 4), s), mod);
            if (t->nnz)
                PTI_CUDA(cudaMemcpyAsync(work[m].ptr, t->inds[m].ptr, t->nnz * 4, cudaMemcpyDeviceToDevice, s), mod);
            inds[m] = work[m].as<uint32_t>();
        }
        PTI_CUDA(org[m].alloc(padded((uint64_t)t->ndims[m] * 4), s), mod);
        iota_k<<<grid_n(t->ndims[m]), 256, 0, s>>>(org[m].as<uint32_t>(), t->ndims[m]);
    }
    for (uint32_t it = 0; it < iterations; ++it)
        for (uint32_t m = 0; m < N; ++m) PTI_TRY(lexi_order_mode(N, t->ndims, t->nnz, inds, m, org[m], s));
    for (uint32_t m = 0; m < N; ++m)
        if (maps && maps[m]) final_map_k<<<grid_n(t->ndims[m]), 256, 0, s>>>(org[m].as<uint32_t>(), t->ndims[m], maps[m]);
    PTI_CUDA(cudaGetLastError(), mod);
    if (apply) {  // schedules built for the old numbering
        t->coo_plan = {};
        t->fiber_plan = {};
    }
    return 0;
}

}  // namespace pti

extern "C" {

int ptiB200Renumber(ptiB200Tensor *t, ptiIndex iterations, ptiIndex * const *new_indices, int apply, void *stream)
{
    using namespace pti;
    const char *mod = "B200 Renumber";
    PTI_CHECK(t, PTIERR_VALUE_ERROR, mod, "null tensor");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    DevBuf maps[kMaxModes];
    uint32_t *mp[kMaxModes] = {};
    for (uint32_t m = 0; m < t->nmodes; ++m) {
        if (!new_indices || !new_indices[m]) continue;
        PTI_CUDA(maps[m].alloc(padded((uint64_t)t->ndims[m] * 4), s), mod);
        mp[m] = maps[m].as<uint32_t>();
    }
    PTI_TRY(renumber_device(t, iterations, mp, apply != 0, s));
    for (uint32_t m = 0; m < t->nmodes; ++m)
        if (mp[m] && t->ndims[m])
            PTI_CUDA(cudaMemcpyAsync(new_indices[m], mp[m], (size_t)t->ndims[m] * 4, cudaMemcpyDeviceToHost, s), mod);
    PTI_CUDA(cudaStreamSynchronize(s), mod);
    return 0;
}

// include/includes/sptensors.h:100, src/sptensor/renumber.c:26-92; tsr is
// left as it was.  renumber == 1: Lexi-order on the GPU, `iterations` passes.
// impl_num 0, 1 and 2 all mean rows of exactly equal other-mode coordinates:
// impl_num 2 compares each mode by its block index and then its full index
// (sort.c:890-917), which orders the coordinates exactly as comparing the
// full indices does, and its quicksort (sort.c:1402-1431) sorts correctly, so
// the reference's own results for 2 are orderit's.  renumber == 2: BFS-like
// (bfs_like above; iterations and impl_num unused).  sb_bits and tk are not
// used.  Other choices (impl_num 3, which the reference marks as not
// working) record PTIERR_VALUE_ERROR (read it with ptiGetLastError) and
// return newIndices as the identity, as the call does on any other failure.
void ptiIndexRenumber(ptiSparseTensor *tsr, ptiIndex **newIndices, int renumber, ptiIndex iterations,
                      ptiElementIndex sb_bits, int tk, int impl_num)
{
    using namespace pti;
    (void)sb_bits;
    (void)tk;
    if (!tsr || !newIndices) return;
    for (ptiIndex m = 0; m < tsr->nmodes; ++m)
        for (ptiIndex i = 0; i < tsr->ndims[m]; ++i) newIndices[m][i] = i;
    const char *mod = "B200 Renumber";
    if (renumber == 2) {
        std::vector<const uint32_t *> hi(tsr->nmodes);
        for (ptiIndex m = 0; m < tsr->nmodes; ++m) hi[m] = tsr->inds[m].data;
        std::vector<std::vector<uint32_t>> out(tsr->nmodes);
        std::vector<uint32_t *> op(tsr->nmodes);
        for (ptiIndex m = 0; m < tsr->nmodes; ++m) {
            out[m].resize(tsr->ndims[m]);
            op[m] = out[m].data();
        }
        if (bfs_like(tsr->nmodes, tsr->ndims, tsr->nnz, hi.data(), op.data(), sync_stream()) != 0) return;
        for (ptiIndex m = 0; m < tsr->nmodes; ++m)
            if (tsr->ndims[m]) std::memcpy(newIndices[m], out[m].data(), (size_t)tsr->ndims[m] * 4);
        return;
    }
    if (renumber != 1 || impl_num < 0 || impl_num > 2) {
        complain(mod, PTIERR_VALUE_ERROR, __FILE__, __LINE__,
                 "renumber must be 1 (Lexi-order, impl_num 0..2) or 2 (BFS-like)");
        return;
    }
    cudaStream_t s = sync_stream();
    ptiB200Tensor t;
    if (upload_coo(&t, tsr, s) != 0) return;
    DevBuf maps[kMaxModes];
    uint32_t *mp[kMaxModes] = {};
    for (uint32_t m = 0; m < t.nmodes; ++m) {
        if (maps[m].alloc(padded((uint64_t)t.ndims[m] * 4), s) != cudaSuccess) {
            complain(mod, PTIERR_CUDA_ERROR, __FILE__, __LINE__, "allocation failed");
            return;
        }
        mp[m] = maps[m].as<uint32_t>();
    }
    if (renumber_device(&t, iterations, mp, true, s) != 0) return;
    std::vector<std::vector<uint32_t>> host(t.nmodes);
    for (uint32_t m = 0; m < t.nmodes; ++m) {
        host[m].resize(t.ndims[m]);
        if (t.ndims[m]) cudaMemcpyAsync(host[m].data(), mp[m], (size_t)t.ndims[m] * 4, cudaMemcpyDeviceToHost, s);
    }
    if (cudaStreamSynchronize(s) != cudaSuccess) {
        complain(mod, PTIERR_CUDA_ERROR, __FILE__, __LINE__, "renumbering failed on the device");
        return;
    }
    for (uint32_t m = 0; m < t.nmodes; ++m)
        if (t.ndims[m]) std::memcpy(newIndices[m], host[m].data(), (size_t)t.ndims[m] * 4);
}

// include/includes/sptensors.h:101, src/sptensor/orderit.c:121-208: the same
// Lexi-order (renumber == 1) or BFS-like (renumber == 2, orderit.c's copy of
// the same heap walk, :1030-1138).
void orderit(ptiSparseTensor *tsr, ptiIndex **newIndices, int const renumber, ptiIndex const iterations)
{
    ptiIndexRenumber(tsr, newIndices, renumber, iterations, 0, 1, 1);
}

// include/includes/sptensors.h:45: every coordinate replaced by its new index.
void ptiSparseTensorShuffleIndices(ptiSparseTensor *tsr, ptiIndex **map_inds)
{
    if (!tsr || !map_inds) return;
    for (ptiIndex m = 0; m < tsr->nmodes; ++m)
        for (ptiNnzIndex z = 0; z < tsr->nnz; ++z) tsr->inds[m].data[z] = map_inds[m][tsr->inds[m].data[z]];
}

// include/includes/matrices.h:30: row i of the result is row map[i] of the
// input (factor rows of a renumbered tensor back in the original numbering).
void ptiMatrixInverseShuffleIndices(ptiMatrix *mtx, ptiIndex *mode_map_inds)
{
    if (!mtx || !mode_map_inds) return;
    std::vector<ptiValue> tmp((size_t)mtx->nrows * mtx->stride);
    std::memcpy(tmp.data(), mtx->values, tmp.size() * sizeof(ptiValue));
    for (ptiIndex i = 0; i < mtx->nrows; ++i)
        std::memcpy(mtx->values + (size_t)i * mtx->stride, tmp.data() + (size_t)mode_map_inds[i] * mtx->stride,
                    mtx->stride * sizeof(ptiValue));
}

// include/includes/ktensors.h:24
void ptiKruskalTensorInverseShuffleIndices(ptiKruskalTensor *ktsr, ptiIndex **map_inds)
{
    if (!ktsr || !map_inds || !ktsr->factors) return;
    for (ptiIndex m = 0; m < ktsr->nmodes; ++m) ptiMatrixInverseShuffleIndices(ktsr->factors[m], map_inds[m]);
}

}  // extern "C"
