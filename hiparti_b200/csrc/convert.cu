// convert.cu -- COO -> HiCOO on the GPU, bit-identical to the reference's
// ptiSparseTensorToHiCOO (src/sptensor/hicoo/convert.c:646-860) for tensors
// with unique coordinates.
//
// Order.  The reference sorts nonzeros by their kernel coordinates
// (ind >> sk_bits, lexicographic over modes 0..N-1; src/sptensor/sort.c:929-953)
// and then, inside each kernel, by a Morton key (sort.c:1041-1098 for 3-D,
// :1109-1288 for 4-D).  Inside one kernel the coordinate bits >= sk_bits are
// equal, so the Morton order there is decided by the low sk_bits of each
// coordinate (3-D: only bits below 24 enter the reference's key).  Here every
// nonzero gets one integer key
//     [kernel coord of mode 0 | ... | kernel coord of mode N-1 | Morton(low bits)]
// (at most 128 bits) and a stable LSD radix sort orders the nonzeros by it.
//
// Structure.  After the sort, flags "starts a new block" / "starts a new
// kernel" and exclusive scans give bptr, binds, einds and kptr in parallel.
// cptr follows the reference's greedy chunk rule (convert.c:737-742,805-815),
// which only depends on the blocks of one kernel and the size of the last
// block of the previous kernel, so one thread walks each kernel.
#include "primitives.cuh"
#include "tensor.cuh"

namespace pti {

struct U128 {
    uint64_t lo, hi;
};

__device__ __forceinline__ void shl_or(U128 &k, uint32_t bits, uint64_t v)
{
    if (bits == 0) return;
    if (bits >= 64) {
        k.hi = k.lo;
        k.lo = 0;
        bits -= 64;
        if (bits) k.hi <<= bits;
        k.lo |= v;
        return;
    }
    k.hi = (k.hi << bits) | (k.lo >> (64 - bits));
    k.lo = (k.lo << bits) | v;
}

struct KeySpec {
    uint32_t nmodes;
    uint32_t sk;
    uint32_t kbits[kMaxModes];  // bits of each kernel coordinate
    uint32_t mbits_per_mode;    // low coordinate bits interleaved in the Morton part
    const uint32_t *inds[kMaxModes];
};

__device__ __forceinline__ U128 hicoo_key(const KeySpec &ks, uint64_t z)
{
    uint32_t c[kMaxModes];
#pragma unroll
    for (int m = 0; m < kMaxModes; ++m)
        if (m < (int)ks.nmodes) c[m] = ks.inds[m][z];
    U128 k{0, 0};
#pragma unroll
    for (int m = 0; m < kMaxModes; ++m)
        if (m < (int)ks.nmodes) shl_or(k, ks.kbits[m], ks.sk >= 32 ? 0u : (c[m] >> ks.sk));
    // Morton part: for bit b (most significant first), mode 0's bit is the
    // most significant of the group, mode N-1's the least.
    const uint32_t N = ks.nmodes;
    for (int b = (int)ks.mbits_per_mode - 1; b >= 0; --b) {
        uint64_t group = 0;
        for (uint32_t m = 0; m < N; ++m) group = (group << 1) | ((c[m] >> b) & 1u);
        shl_or(k, N, group);
    }
    return k;
}

__global__ void make_keys_kernel(KeySpec ks, uint64_t n, int word, const uint32_t *perm, uint64_t *keys,
                                 uint32_t *vals)
{
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t z = perm ? perm[i] : i;
        U128 k = hicoo_key(ks, z);
        keys[i] = word == 0 ? k.lo : k.hi;
        if (!perm) vals[i] = (uint32_t)i;
    }
}

struct GatherArgs {
    uint32_t nmodes;
    uint32_t sb;
    const uint32_t *perm;
    const uint32_t *inds[kMaxModes];
    const float *vals;
    uint32_t *sinds[kMaxModes];
    uint8_t *einds[kMaxModes];
    float *svals;
};

__global__ void gather_sorted_kernel(GatherArgs a, uint64_t n)
{
    const uint32_t emask = (1u << a.sb) - 1u;
    for (uint64_t z = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; z < n; z += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t p = a.perm[z];
#pragma unroll
        for (int m = 0; m < kMaxModes; ++m)
            if (m < (int)a.nmodes) {
                uint32_t c = a.inds[m][p];
                a.sinds[m][z] = c;
                a.einds[m][z] = (uint8_t)(c & emask);
            }
        a.svals[z] = a.vals[p];
    }
}

// 1 if nonzero z of the sorted tensor starts a new block (z == 0 or block
// coordinates differ from nonzero z-1).
struct NewBlockFlag {
    uint32_t nmodes, sb;
    const uint32_t *sinds[kMaxModes];
    __device__ uint32_t operator()(uint64_t z) const
    {
        if (z == 0) return 1u;
        uint32_t diff = 0;
#pragma unroll
        for (int m = 0; m < kMaxModes; ++m)
            if (m < (int)nmodes) diff |= (sinds[m][z] >> sb) ^ (sinds[m][z - 1] >> sb);
        return diff ? 1u : 0u;
    }
};

struct BlockOut {
    uint32_t nmodes, sb;
    const uint32_t *sinds[kMaxModes];
    uint64_t *bptr;
    uint32_t *binds[kMaxModes];
    __device__ void operator()(uint64_t z, uint32_t prefix, uint32_t flag) const
    {
        if (!flag) return;
        bptr[prefix] = z;
#pragma unroll
        for (int m = 0; m < kMaxModes; ++m)
            if (m < (int)nmodes) binds[m][prefix] = sinds[m][z] >> sb;
    }
};

// 1 if block b starts a new kernel.
struct NewKernelFlag {
    uint32_t nmodes, sk;
    const uint64_t *bptr;
    const uint32_t *sinds[kMaxModes];
    __device__ uint32_t operator()(uint64_t b) const
    {
        if (b == 0) return 1u;
        uint64_t z = bptr[b];
        uint32_t diff = 0;
#pragma unroll
        for (int m = 0; m < kMaxModes; ++m)
            if (m < (int)nmodes) {
                uint32_t a = sk >= 32 ? 0u : sinds[m][z] >> sk, c = sk >= 32 ? 0u : sinds[m][z - 1] >> sk;
                diff |= a ^ c;
            }
        return diff ? 1u : 0u;
    }
};

struct KernelOut {
    uint64_t *kptr;
    __device__ void operator()(uint64_t b, uint32_t prefix, uint32_t flag) const
    {
        if (flag) kptr[prefix] = b;
    }
};

// Greedy chunk pointers of one kernel (convert.c:737-742, 805-815); writes
// them if `out` is non-null, otherwise stores their count.  The reference
// walks the kernel's blocks keeping a running nonzero count that resets
// after each emitted chunk: at block step s (the count of block s-1 added)
// a chunk is emitted when the count reaches 2^sc.  A step's count is
// bptr[s] - bptr[s0 - 1], s0 the first step after the last reset, and bptr
// increases strictly, so the next emission is the first s >= s0 with
// bptr[s] >= bptr[s0 - 1] + 2^sc: a binary search per chunk instead of a
// step per block (one kernel can hold all blocks when sk is large).
__device__ uint64_t kernel_chunks(uint64_t k, const uint64_t *kptr, const uint64_t *bptr, uint64_t sc,
                                  uint64_t *out)
{
    const uint64_t first = kptr[k], last = kptr[k + 1];
    uint64_t n = 0;
    if (out) out[n] = first;
    ++n;
    // the first step of kernel k > 0 adds the previous kernel's last block
    uint64_t s0 = k > 0 ? first : first + 1;
    while (s0 < last) {
        const uint64_t target = bptr[s0 - 1] + sc;
        uint64_t lo = s0, hi = last;
        while (lo < hi) {
            const uint64_t mid = lo + (hi - lo) / 2;
            if (bptr[mid] >= target) hi = mid;
            else lo = mid + 1;
        }
        if (lo == last) break;
        if (out) out[n] = lo;
        ++n;
        s0 = lo + 1;
    }
    return n;
}

__global__ void chunk_count_kernel(uint64_t nk, const uint64_t *kptr, const uint64_t *bptr, uint64_t sc,
                                   uint32_t *counts)
{
    uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < nk) counts[k] = (uint32_t)kernel_chunks(k, kptr, bptr, sc, nullptr);
}

__global__ void chunk_fill_kernel(uint64_t nk, const uint64_t *kptr, const uint64_t *bptr, uint64_t sc,
                                  const uint32_t *offsets, uint64_t *cptr)
{
    uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < nk) kernel_chunks(k, kptr, bptr, sc, cptr + offsets[k]);
}

__global__ void block_max_kernel(const uint64_t *bptr, uint64_t nb, unsigned long long *mx)
{
    unsigned long long best = 0;
    for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += (uint64_t)gridDim.x * blockDim.x)
        best = max(best, (unsigned long long)(bptr[b + 1] - bptr[b]));
    for (int o = 16; o; o >>= 1) best = max(best, __shfl_xor_sync(0xffffffffu, best, o));
    if ((threadIdx.x & 31) == 0) atomicMax(mx, best);
}

__global__ void kernel_coords_kernel(uint64_t nk, uint32_t nmodes, uint32_t sk, const uint64_t *kptr,
                                     const uint64_t *bptr, KeySpec ks, uint32_t *kc)
{
    uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nk) return;
    uint64_t z = bptr[kptr[k]];
    for (uint32_t m = 0; m < nmodes; ++m) kc[m * nk + k] = sk >= 32 ? 0u : ks.inds[m][z] >> sk;
}

struct U32In {
    const uint32_t *p;
    __device__ uint32_t operator()(uint64_t i) const { return p[i]; }
};
struct U32OutPrefix {
    uint32_t *p;
    __device__ void operator()(uint64_t i, uint32_t prefix, uint32_t) const { p[i] = prefix; }
};

static uint32_t bits_for(uint64_t count)  // bits to hold values 0..count-1
{
    uint32_t b = 0;
    while (b < 64 && ((uint64_t)1 << b) < count) ++b;
    return b;
}

// Result of a device conversion, beyond the device HiCOO tensor itself.
struct ConvertExtras {
    uint64_t nk = 0, nc = 0, max_nnzb = 0;
    DevBuf kptr;      // uint64 [nk+1]
    DevBuf cptr;      // uint64 [nc]
    DevBuf kcoords;   // uint32 [nmodes][nk]
    std::array<DevBuf, kMaxModes> sinds;  // the COO indices in HiCOO order
    DevBuf svals;
};

int convert_device(const ptiB200Tensor *coo, ptiB200Tensor *h, uint8_t sb, uint8_t sk, uint8_t sc,
                   ConvertExtras &ex, cudaStream_t s)
{
    const char *mod = "B200 HiSpTns Convert";
    const uint32_t N = coo->nmodes;
    const uint64_t n = coo->nnz;
    PTI_CHECK(!coo->hicoo, PTIERR_VALUE_ERROR, mod, "input must be a COO tensor");
    PTI_CHECK(N == 3 || N == 4, PTIERR_VALUE_ERROR, mod, "only 3-D and 4-D tensors have a Morton order");
    PTI_CHECK(sk >= sb && sc >= sb, PTIERR_VALUE_ERROR, mod, "need sk_bits >= sb_bits and sc_bits >= sb_bits");
    PTI_CHECK(sb >= 1 && sb <= 8, PTIERR_VALUE_ERROR, mod, "sb_bits must be in [1, 8]");
    PTI_CHECK(sc < 64, PTIERR_VALUE_ERROR, mod, "sc_bits too large");
    PTI_CHECK(n > 0, PTIERR_VALUE_ERROR, mod, "empty tensor");
    PTI_CHECK(n < 0xFFFFFFFFull, PTIERR_VALUE_ERROR, mod, "too many nonzeros");

    KeySpec ks{};
    ks.nmodes = N;
    ks.sk = sk;
    uint32_t total = 0;
    for (uint32_t m = 0; m < N; ++m) {
        uint64_t kdim = sk >= 32 ? 1 : ((uint64_t)coo->ndims[m] + ((uint64_t)1 << sk) - 1) >> sk;
        ks.kbits[m] = bits_for(kdim);
        total += ks.kbits[m];
        ks.inds[m] = coo->inds[m].as<uint32_t>();
    }
    ks.mbits_per_mode = N == 3 ? (sk < 24 ? sk : 24) : (sk < 32 ? sk : 32);
    total += N * ks.mbits_per_mode;
    PTI_CHECK(total <= 128, PTIERR_VALUE_ERROR, mod, "sort key wider than 128 bits");

    DevBuf keys, perm;
    RadixScratch rs;
    PTI_CUDA(keys.alloc(padded(n * 8), s), mod);
    PTI_CUDA(perm.alloc(padded(n * 4), s), mod);
    PTI_TRY(rs.alloc(n, s));
    const unsigned grid = (unsigned)std::min<uint64_t>((n + 255) / 256, (uint64_t)sm_count() * 32);
    make_keys_kernel<<<grid, 256, 0, s>>>(ks, n, 0, nullptr, keys.as<uint64_t>(), perm.as<uint32_t>());
    PTI_CUDA(cudaGetLastError(), mod);
    PTI_TRY(radix_sort_pairs(keys, perm, n, total < 64 ? (int)total : 64, rs, s));
    if (total > 64) {
        make_keys_kernel<<<grid, 256, 0, s>>>(ks, n, 1, perm.as<uint32_t>(), keys.as<uint64_t>(), nullptr);
        PTI_CUDA(cudaGetLastError(), mod);
        PTI_TRY(radix_sort_pairs(keys, perm, n, (int)(total - 64), rs, s));
    }
    keys.reset();
    rs = RadixScratch();

    // Sorted COO, einds and values.
    h->hicoo = true;
    h->nmodes = N;
    h->ndims = coo->ndims;
    h->nnz = n;
    h->sb = sb;
    h->sk = sk;
    h->sc = sc;
    h->device = coo->device;
    GatherArgs ga{};
    ga.nmodes = N;
    ga.sb = sb;
    ga.perm = perm.as<uint32_t>();
    ga.vals = coo->vals.as<float>();
    for (uint32_t m = 0; m < N; ++m) {
        PTI_CUDA(ex.sinds[m].alloc(padded(n * 4), s), mod);
        PTI_CUDA(h->einds[m].alloc(padded(n), s), mod);
        ga.inds[m] = coo->inds[m].as<uint32_t>();
        ga.sinds[m] = ex.sinds[m].as<uint32_t>();
        ga.einds[m] = h->einds[m].as<uint8_t>();
    }
    PTI_CUDA(ex.svals.alloc(padded(n * 4), s), mod);
    PTI_CUDA(h->vals.alloc(padded(n * 4), s), mod);
    ga.svals = h->vals.as<float>();
    gather_sorted_kernel<<<grid, 256, 0, s>>>(ga, n);
    PTI_CUDA(cudaGetLastError(), mod);
    PTI_CUDA(cudaMemcpyAsync(ex.svals.ptr, h->vals.ptr, n * 4, cudaMemcpyDeviceToDevice, s), mod);
    perm.reset();

    // Blocks: bptr, binds.  Upper bound nb <= n until counted.
    DevBuf scan_tmp;
    PTI_CUDA(scan_tmp.alloc(padded(scan_tmp_elems<uint32_t>(n) * 4), s), mod);
    NewBlockFlag nbf{};
    nbf.nmodes = N;
    nbf.sb = sb;
    BlockOut bo{};
    bo.nmodes = N;
    bo.sb = sb;
    DevBuf bptr_full;
    std::array<DevBuf, kMaxModes> binds_full;
    PTI_CUDA(bptr_full.alloc(padded((n + 1) * 8), s), mod);
    for (uint32_t m = 0; m < N; ++m) {
        nbf.sinds[m] = ex.sinds[m].as<uint32_t>();
        bo.sinds[m] = ex.sinds[m].as<uint32_t>();
        PTI_CUDA(binds_full[m].alloc(padded(n * 4), s), mod);
        bo.binds[m] = binds_full[m].as<uint32_t>();
    }
    bo.bptr = bptr_full.as<uint64_t>();
    uint32_t nb32 = 0;
    PTI_TRY((exclusive_scan<uint32_t>(nbf, bo, n, scan_tmp.as<uint32_t>(), &nb32, s)));
    const uint64_t nb = nb32;
    h->nb = nb;
    PTI_CUDA(cudaMemcpyAsync(bptr_full.as<uint64_t>() + nb, &n, 8, cudaMemcpyHostToDevice, s), mod);
    // shrink to exact sizes
    PTI_CUDA(h->bptr.alloc(padded((nb + 1) * 8), s), mod);
    PTI_CUDA(cudaMemcpyAsync(h->bptr.ptr, bptr_full.ptr, (nb + 1) * 8, cudaMemcpyDeviceToDevice, s), mod);
    for (uint32_t m = 0; m < N; ++m) {
        PTI_CUDA(h->binds[m].alloc(padded(nb * 4), s), mod);
        PTI_CUDA(cudaMemcpyAsync(h->binds[m].ptr, binds_full[m].ptr, nb * 4, cudaMemcpyDeviceToDevice, s), mod);
        binds_full[m].reset();
    }
    bptr_full.reset();

    // Kernels: kptr over blocks.
    NewKernelFlag nkf{};
    nkf.nmodes = N;
    nkf.sk = sk;
    nkf.bptr = h->bptr.as<uint64_t>();
    for (uint32_t m = 0; m < N; ++m) nkf.sinds[m] = ex.sinds[m].as<uint32_t>();
    DevBuf kptr_full;
    PTI_CUDA(kptr_full.alloc(padded((nb + 1) * 8), s), mod);
    uint32_t nk32 = 0;
    PTI_TRY((exclusive_scan<uint32_t>(nkf, KernelOut{kptr_full.as<uint64_t>()}, nb, scan_tmp.as<uint32_t>(),
                                      &nk32, s)));
    const uint64_t nk = nk32;
    ex.nk = nk;
    PTI_CUDA(ex.kptr.alloc(padded((nk + 1) * 8), s), mod);
    PTI_CUDA(cudaMemcpyAsync(ex.kptr.ptr, kptr_full.ptr, nk * 8, cudaMemcpyDeviceToDevice, s), mod);
    PTI_CUDA(cudaMemcpyAsync(ex.kptr.as<uint64_t>() + nk, &nb, 8, cudaMemcpyHostToDevice, s), mod);
    kptr_full.reset();

    // Chunks.
    DevBuf ccount;
    PTI_CUDA(ccount.alloc(padded((nk + 1) * 4), s), mod);
    const uint64_t scv = (uint64_t)1 << sc;
    chunk_count_kernel<<<ceil_div(nk, 256), 256, 0, s>>>(nk, ex.kptr.as<uint64_t>(), h->bptr.as<uint64_t>(), scv,
                                                          ccount.as<uint32_t>());
    PTI_CUDA(cudaGetLastError(), mod);
    uint32_t nc_body = 0;
    PTI_TRY((exclusive_scan<uint32_t>(U32In{ccount.as<uint32_t>()}, U32OutPrefix{ccount.as<uint32_t>()}, nk,
                                      scan_tmp.as<uint32_t>(), &nc_body, s)));
    ex.nc = (uint64_t)nc_body + 1;
    PTI_CUDA(ex.cptr.alloc(padded(ex.nc * 8), s), mod);
    chunk_fill_kernel<<<ceil_div(nk, 256), 256, 0, s>>>(nk, ex.kptr.as<uint64_t>(), h->bptr.as<uint64_t>(), scv,
                                                         ccount.as<uint32_t>(), ex.cptr.as<uint64_t>());
    PTI_CUDA(cudaGetLastError(), mod);
    PTI_CUDA(cudaMemcpyAsync(ex.cptr.as<uint64_t>() + nc_body, &nb, 8, cudaMemcpyHostToDevice, s), mod);

    // max nonzeros per block, kernel coordinates
    DevBuf mx;
    PTI_CUDA(mx.alloc(64, s), mod);
    PTI_CUDA(cudaMemsetAsync(mx.ptr, 0, 8, s), mod);
    block_max_kernel<<<ceil_div(std::min<uint64_t>(nb, (uint64_t)sm_count() * 2048), 256), 256, 0, s>>>(
        h->bptr.as<uint64_t>(), nb, mx.as<unsigned long long>());
    KeySpec kcs = ks;
    for (uint32_t m = 0; m < N; ++m) kcs.inds[m] = ex.sinds[m].as<uint32_t>();
    PTI_CUDA(ex.kcoords.alloc(padded(nk * N * 4), s), mod);
    kernel_coords_kernel<<<ceil_div(nk, 256), 256, 0, s>>>(nk, N, sk, ex.kptr.as<uint64_t>(), h->bptr.as<uint64_t>(),
                                                            kcs, ex.kcoords.as<uint32_t>());
    PTI_CUDA(cudaGetLastError(), mod);
    unsigned long long mxh = 0;
    PTI_CUDA(cudaMemcpyAsync(&mxh, mx.ptr, 8, cudaMemcpyDeviceToHost, s), mod);
    PTI_CUDA(cudaStreamSynchronize(s), mod);
    ex.max_nnzb = mxh;
    return 0;
}

int finish_hicoo_layout(ptiB200Tensor *t, cudaStream_t s);
int upload_coo(ptiB200Tensor *t, const ptiSparseTensor *X, cudaStream_t s);
int assign_nnz_vector(ptiNnzIndexVector *v, const uint64_t *src, uint64_t len);
int assign_index_vector(ptiIndexVector *v, const uint32_t *src, uint64_t len);
int alloc_block_vector(ptiBlockIndexVector *v, uint64_t len);
int alloc_element_vector(ptiElementIndexVector *v, uint64_t len);
int alloc_value_vector(ptiValueVector *v, uint64_t len);
int alloc_nnz_vector(ptiNnzIndexVector *v, uint64_t len);
int balanced_schedule(ptiSparseTensorHiCOO *hitsr, uint64_t nnz);
int validate_coo(ptiB200Tensor *t, cudaStream_t s);

}  // namespace pti

extern "C" {

int ptiSparseTensorToHiCOO(ptiSparseTensorHiCOO *hitsr, ptiNnzIndex *max_nnzb, ptiSparseTensor *tsr,
                           const ptiElementIndex sb_bits, const ptiElementIndex sk_bits,
                           const ptiElementIndex sc_bits, int const tk)
{
    (void)tk;
    using namespace pti;
    const char *mod = "B200 HiSpTns Convert";
    PTI_CHECK(hitsr && tsr && max_nnzb, PTIERR_VALUE_ERROR, mod, "null argument");
    // src/sptensor/hicoo/convert.c:655-656 asserts these; src/sptensor/sort.c:414-430
    // has a Morton order for 3-D and 4-D tensors only.
    PTI_CHECK(tsr->nmodes == 3 || tsr->nmodes == 4, PTIERR_VALUE_ERROR, mod,
              "only 3-D and 4-D tensors have a Morton order");
    PTI_CHECK(sk_bits >= sb_bits && sc_bits >= sb_bits, PTIERR_VALUE_ERROR, mod,
              "need sk_bits >= sb_bits and sc_bits >= sb_bits");
    PTI_CHECK(sb_bits >= 1 && sb_bits <= 8, PTIERR_VALUE_ERROR, mod, "sb_bits must be in [1, 8]");
    cudaStream_t s = sync_stream();
    ptiB200Tensor coo, h;
    PTI_TRY(upload_coo(&coo, tsr, s));
    ConvertExtras ex;
    PTI_TRY(convert_device(&coo, &h, sb_bits, sk_bits, sc_bits, ex, s));
    const uint32_t N = tsr->nmodes;
    const uint64_t n = tsr->nnz, nb = h.nb, nk = ex.nk;

    PTI_TRY(ptiNewSparseTensorHiCOO(hitsr, N, tsr->ndims, n, sb_bits, sk_bits, sc_bits));
    // The caller's COO is left sorted in HiCOO order, as in the reference.
    for (uint32_t m = 0; m < N; ++m)
        PTI_CUDA(cudaMemcpyAsync(tsr->inds[m].data, ex.sinds[m].ptr, n * 4, cudaMemcpyDeviceToHost, s), mod);
    PTI_CUDA(cudaMemcpyAsync(tsr->values.data, ex.svals.ptr, n * 4, cudaMemcpyDeviceToHost, s), mod);
    for (uint32_t m = 0; m < N; ++m) tsr->sortorder[m] = m;

    PTI_TRY(alloc_nnz_vector(&hitsr->bptr, nb + 1));
    PTI_CUDA(cudaMemcpyAsync(hitsr->bptr.data, h.bptr.ptr, (nb + 1) * 8, cudaMemcpyDeviceToHost, s), mod);
    for (uint32_t m = 0; m < N; ++m) {
        PTI_TRY(alloc_block_vector(&hitsr->binds[m], nb));
        PTI_TRY(alloc_element_vector(&hitsr->einds[m], n));
        PTI_CUDA(cudaMemcpyAsync(hitsr->binds[m].data, h.binds[m].ptr, nb * 4, cudaMemcpyDeviceToHost, s), mod);
        PTI_CUDA(cudaMemcpyAsync(hitsr->einds[m].data, h.einds[m].ptr, n, cudaMemcpyDeviceToHost, s), mod);
    }
    PTI_TRY(alloc_value_vector(&hitsr->values, n));
    PTI_CUDA(cudaMemcpyAsync(hitsr->values.data, h.vals.ptr, n * 4, cudaMemcpyDeviceToHost, s), mod);
    PTI_TRY(alloc_nnz_vector(&hitsr->kptr, nk + 1));
    PTI_CUDA(cudaMemcpyAsync(hitsr->kptr.data, ex.kptr.ptr, (nk + 1) * 8, cudaMemcpyDeviceToHost, s), mod);
    PTI_TRY(alloc_nnz_vector(&hitsr->cptr, ex.nc));
    PTI_CUDA(cudaMemcpyAsync(hitsr->cptr.data, ex.cptr.ptr, ex.nc * 8, cudaMemcpyDeviceToHost, s), mod);
    std::vector<uint32_t> kc((size_t)nk * N);
    PTI_CUDA(cudaMemcpyAsync(kc.data(), ex.kcoords.ptr, kc.size() * 4, cudaMemcpyDeviceToHost, s), mod);
    PTI_CUDA(cudaStreamSynchronize(s), mod);

    // knnzs (convert.c:314-369): nonzeros of each kernel.
    PTI_TRY(alloc_nnz_vector(&hitsr->knnzs, nk));
    for (uint64_t k = 0; k < nk; ++k) {
        uint64_t zb = hitsr->bptr.data[hitsr->kptr.data[k]];
        uint64_t ze = hitsr->bptr.data[hitsr->kptr.data[k + 1]];
        hitsr->knnzs.data[k] = ze - zb;
    }
    // Kernel scheduler (convert.c:378-421): kschr[m][kernel row] lists the
    // kernels whose mode-m kernel coordinate is that row, in kernel order.
    const uint64_t skv = (uint64_t)1 << sk_bits;
    for (uint32_t m = 0; m < N; ++m) {
        uint64_t rows = ((uint64_t)tsr->ndims[m] + skv - 1) / skv;
        std::vector<uint32_t> cnt(rows + 1, 0);
        for (uint64_t k = 0; k < nk; ++k) cnt[kc[(size_t)m * nk + k]]++;
        std::vector<std::vector<uint32_t>> lists(rows);
        for (uint64_t r = 0; r < rows; ++r) lists[r].reserve(cnt[r]);
        for (uint64_t k = 0; k < nk; ++k) lists[kc[(size_t)m * nk + k]].push_back((uint32_t)k);
        uint32_t longest = 0;
        for (uint64_t r = 0; r < rows; ++r) {
            PTI_TRY(assign_index_vector(&hitsr->kschr[m][r], lists[r].data(), lists[r].size()));
            longest = std::max<uint32_t>(longest, (uint32_t)lists[r].size());
        }
        hitsr->nkiters[m] = longest;
    }
    PTI_TRY(balanced_schedule(hitsr, n));
    *max_nnzb = ex.max_nnzb;
    return 0;
}

int ptiB200TensorFromDeviceCOO(ptiB200Tensor **out, ptiIndex nmodes, const ptiIndex *ndims, ptiNnzIndex nnz,
                               const ptiIndex *const *dev_inds, const ptiValue *dev_vals, void *stream)
{
    using namespace pti;
    const char *mod = "B200 Upload";
    PTI_CHECK(out && ndims && dev_inds && dev_vals, PTIERR_VALUE_ERROR, mod, "null argument");
    PTI_CHECK(nmodes >= 2 && nmodes <= (uint32_t)kMaxModes, PTIERR_VALUE_ERROR, mod, "unsupported number of modes");
    configure_pool_once();
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    auto *t = new ptiB200Tensor();
    cudaGetDevice(&t->device);
    t->nmodes = nmodes;
    t->ndims.assign(ndims, ndims + nmodes);
    t->nnz = nnz;
    int r = 0;
    for (uint32_t m = 0; m < nmodes && r == 0; ++m) {
        if (t->inds[m].alloc(padded(nnz * 4), s) != cudaSuccess ||
            (nnz && cudaMemcpyAsync(t->inds[m].ptr, dev_inds[m], nnz * 4, cudaMemcpyDeviceToDevice, s) != cudaSuccess))
            r = PTIERR_CUDA_ERROR;
    }
    if (r == 0 && (t->vals.alloc(padded(nnz * 4), s) != cudaSuccess ||
                   (nnz && cudaMemcpyAsync(t->vals.ptr, dev_vals, nnz * 4, cudaMemcpyDeviceToDevice, s) != cudaSuccess)))
        r = PTIERR_CUDA_ERROR;
    if (r) {
        delete t;
        PTI_FAIL(r, mod, "device copy failed");
    }
    r = validate_coo(t, s);
    if (r) {
        delete t;
        return r;
    }
    *out = t;
    return 0;
}

int ptiB200ConvertToHiCOO(ptiB200Tensor **out, ptiB200Tensor *coo, ptiElementIndex sb_bits, ptiElementIndex sk_bits,
                          ptiElementIndex sc_bits, ptiNnzIndex *nb, ptiNnzIndex *max_nnzb, void *stream)
{
    using namespace pti;
    PTI_CHECK(out && coo, PTIERR_VALUE_ERROR, "B200 HiSpTns Convert", "null argument");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    auto *h = new ptiB200Tensor();
    ConvertExtras ex;
    int r = convert_device(coo, h, sb_bits, sk_bits, sc_bits, ex, s);
    if (r == 0) r = finish_hicoo_layout(h, s);
    if (r) {
        delete h;
        return r;
    }
    if (nb) *nb = h->nb;
    if (max_nnzb) *max_nnzb = ex.max_nnzb;
    *out = h;
    return 0;
}

}  // extern "C"
