// containers.cu -- host-side life cycle of the reference's structs and the
// reference's tensor loader (parsed on the GPU, ingest.cu).  Struct layouts are those of
// include/includes/structs.h in the reference; ownership follows its
// src/sptensor/sptensor.c, src/matrix/matrix.c, src/ktensor/ktensor.c and
// src/sptensor/hicoo/hicoo.c.
#include "common.cuh"
#include "tensor.cuh"

#include <cerrno>
#include <cmath>

namespace {

template <class V, class T>
int new_vector(V *v, uint64_t len, uint64_t cap)
{
    if (cap < len) cap = len;
    if (cap < 2) cap = 2;
    v->len = len;
    v->cap = cap;
    v->data = static_cast<T *>(std::malloc(cap * sizeof(T)));
    PTI_CHECK(v->data, PTIERR_OS_ERROR + ENOMEM, "Vec New", "out of memory");
    return 0;
}

template <class V>
void free_vector(V *v)
{
    std::free(v->data);
    v->data = nullptr;
    v->len = v->cap = 0;
}

}  // namespace

extern "C" {

int ptiNewSparseTensor(ptiSparseTensor *tsr, ptiIndex nmodes, const ptiIndex ndims[])
{
    tsr->nmodes = nmodes;
    tsr->sortorder = static_cast<ptiIndex *>(std::malloc(nmodes * sizeof(ptiIndex)));
    for (ptiIndex i = 0; i < nmodes; ++i) tsr->sortorder[i] = i;
    tsr->ndims = static_cast<ptiIndex *>(std::malloc(nmodes * sizeof(ptiIndex)));
    PTI_CHECK(tsr->ndims && tsr->sortorder, PTIERR_OS_ERROR + ENOMEM, "SpTns New", "out of memory");
    std::memcpy(tsr->ndims, ndims, nmodes * sizeof(ptiIndex));
    tsr->nnz = 0;
    tsr->inds = static_cast<ptiIndexVector *>(std::malloc(nmodes * sizeof(ptiIndexVector)));
    PTI_CHECK(tsr->inds, PTIERR_OS_ERROR + ENOMEM, "SpTns New", "out of memory");
    for (ptiIndex i = 0; i < nmodes; ++i)
        PTI_TRY((new_vector<ptiIndexVector, ptiIndex>(&tsr->inds[i], 0, 0)));
    PTI_TRY((new_vector<ptiValueVector, ptiValue>(&tsr->values, 0, 0)));
    return 0;
}

void ptiFreeSparseTensor(ptiSparseTensor *tsr)
{
    for (ptiIndex i = 0; i < tsr->nmodes; ++i) free_vector(&tsr->inds[i]);
    std::free(tsr->sortorder);
    std::free(tsr->ndims);
    std::free(tsr->inds);
    free_vector(&tsr->values);
    tsr->sortorder = nullptr;
    tsr->ndims = nullptr;
    tsr->inds = nullptr;
    tsr->nmodes = 0;
}

int ptiLoadSparseTensor(ptiSparseTensor *tsr, ptiIndex start_index, char const *const fname)
{
    const char *mod = "SpTns Load";
    PTI_CHECK(tsr && fname, PTIERR_VALUE_ERROR, mod, "null argument");
    cudaStream_t s = pti::sync_stream();
    ptiB200Tensor t;
    bool text = true;
    PTI_TRY(pti::ingest_file(&t, start_index, fname, &text, s));
    PTI_TRY(ptiNewSparseTensor(tsr, t.nmodes, t.ndims.data()));
    // The reference's text reader leaves sortorder zero-filled (load.c:68-71).
    if (text) std::memset(tsr->sortorder, 0, t.nmodes * sizeof(ptiIndex));
    const uint64_t nnz = t.nnz;
    tsr->nnz = nnz;
    for (ptiIndex m = 0; m < t.nmodes; ++m) {
        free_vector(&tsr->inds[m]);
        PTI_TRY((new_vector<ptiIndexVector, ptiIndex>(&tsr->inds[m], nnz, nnz)));
        if (nnz)
            PTI_CUDA(cudaMemcpyAsync(tsr->inds[m].data, t.inds[m].ptr, nnz * 4, cudaMemcpyDeviceToHost, s), mod);
    }
    free_vector(&tsr->values);
    PTI_TRY((new_vector<ptiValueVector, ptiValue>(&tsr->values, nnz, nnz)));
    if (nnz) PTI_CUDA(cudaMemcpyAsync(tsr->values.data, t.vals.ptr, nnz * 4, cudaMemcpyDeviceToHost, s), mod);
    PTI_CUDA(cudaStreamSynchronize(s), mod);
    return 0;
}

int ptiNewMatrix(ptiMatrix *mtx, ptiIndex const nrows, ptiIndex const ncols)
{
    mtx->nrows = nrows;
    mtx->ncols = ncols;
    mtx->cap = nrows != 0 ? nrows : 1;
    mtx->stride = ((ncols - 1) / 8 + 1) * 8;  // src/matrix/matrix.c:36-55
    size_t bytes = (size_t)mtx->cap * mtx->stride * sizeof(ptiValue);
    void *p = nullptr;
    if (posix_memalign(&p, 8 * sizeof(ptiValue), bytes ? bytes : 32) != 0) p = nullptr;
    mtx->values = static_cast<ptiValue *>(p);
    PTI_CHECK(mtx->values, PTIERR_OS_ERROR + ENOMEM, "Mtx New", "out of memory");
    return 0;
}

int ptiRandomizeMatrix(ptiMatrix *mtx)
{
    // src/matrix/matrix.c:67-74 fills A[i][j] = i + j + 1 (not random).
    for (ptiIndex i = 0; i < mtx->nrows; ++i)
        for (ptiIndex j = 0; j < mtx->ncols; ++j) mtx->values[(size_t)i * mtx->stride + j] = (ptiValue)(i + j + 1);
    return 0;
}

int ptiConstantMatrix(ptiMatrix *const mtx, ptiValue const val)
{
    for (ptiIndex i = 0; i < mtx->nrows; ++i)
        for (ptiIndex j = 0; j < mtx->ncols; ++j) mtx->values[(size_t)i * mtx->stride + j] = val;
    return 0;
}

void ptiFreeMatrix(ptiMatrix *mtx)
{
    std::free(mtx->values);
    mtx->values = nullptr;
    mtx->nrows = mtx->ncols = mtx->cap = mtx->stride = 0;
}

int ptiNewRankMatrix(ptiRankMatrix *mtx, ptiIndex const nrows, ptiElementIndex const ncols)
{
    mtx->nrows = nrows;
    mtx->ncols = ncols;
    mtx->cap = nrows != 0 ? nrows : 1;
    mtx->stride = (ptiElementIndex)(((ncols - 1) / 8 + 1) * 8);
    size_t bytes = (size_t)mtx->cap * mtx->stride * sizeof(ptiValue);
    void *p = nullptr;
    if (posix_memalign(&p, 8 * sizeof(ptiValue), bytes ? bytes : 32) != 0) p = nullptr;
    mtx->values = static_cast<ptiValue *>(p);
    PTI_CHECK(mtx->values, PTIERR_OS_ERROR + ENOMEM, "RankMtx New", "out of memory");
    return 0;
}

void ptiFreeRankMatrix(ptiRankMatrix *mtx)
{
    std::free(mtx->values);
    mtx->values = nullptr;
    mtx->nrows = mtx->cap = 0;
    mtx->ncols = mtx->stride = 0;
}

int ptiNewKruskalTensor(ptiKruskalTensor *ktsr, ptiIndex nmodes, const ptiIndex ndims[], ptiIndex rank)
{
    ktsr->nmodes = nmodes;
    ktsr->rank = rank;
    ktsr->ndims = static_cast<ptiIndex *>(std::malloc(nmodes * sizeof(ptiIndex)));
    std::memcpy(ktsr->ndims, ndims, nmodes * sizeof(ptiIndex));
    ktsr->lambda = static_cast<ptiValue *>(std::malloc((rank ? rank : 1) * sizeof(ptiValue)));
    ktsr->fit = 0.0;
    ktsr->factors = nullptr;
    return 0;
}

void ptiFreeKruskalTensor(ptiKruskalTensor *ktsr)
{
    ktsr->rank = 0;
    ktsr->fit = 0.0;
    std::free(ktsr->ndims);
    std::free(ktsr->lambda);
    if (ktsr->factors) {
        for (ptiIndex i = 0; i < ktsr->nmodes; ++i) {
            if (ktsr->factors[i]) {
                ptiFreeMatrix(ktsr->factors[i]);
                std::free(ktsr->factors[i]);
            }
        }
        if (ktsr->factors[ktsr->nmodes]) std::free(ktsr->factors[ktsr->nmodes]);
        std::free(ktsr->factors);
    }
    ktsr->ndims = nullptr;
    ktsr->lambda = nullptr;
    ktsr->factors = nullptr;
    ktsr->nmodes = 0;
}

int ptiNewRankKruskalTensor(ptiRankKruskalTensor *ktsr, ptiIndex nmodes, const ptiIndex ndims[],
                            ptiElementIndex rank)
{
    ktsr->nmodes = nmodes;
    ktsr->rank = rank;
    ktsr->ndims = static_cast<ptiIndex *>(std::malloc(nmodes * sizeof(ptiIndex)));
    std::memcpy(ktsr->ndims, ndims, nmodes * sizeof(ptiIndex));
    ktsr->lambda = static_cast<ptiValue *>(std::malloc((rank ? rank : 1) * sizeof(ptiValue)));
    ktsr->fit = 0.0;
    ktsr->factors = nullptr;
    return 0;
}

void ptiFreeRankKruskalTensor(ptiRankKruskalTensor *ktsr)
{
    ktsr->rank = 0;
    ktsr->fit = 0.0;
    std::free(ktsr->ndims);
    std::free(ktsr->lambda);
    if (ktsr->factors) {
        for (ptiIndex i = 0; i < ktsr->nmodes; ++i) {
            if (ktsr->factors[i]) {
                ptiFreeRankMatrix(ktsr->factors[i]);
                std::free(ktsr->factors[i]);
            }
        }
        if (ktsr->factors[ktsr->nmodes]) std::free(ktsr->factors[ktsr->nmodes]);
        std::free(ktsr->factors);
    }
    ktsr->ndims = nullptr;
    ktsr->lambda = nullptr;
    ktsr->factors = nullptr;
    ktsr->nmodes = 0;
}

int ptiNewSparseTensorHiCOO(ptiSparseTensorHiCOO *hitsr, const ptiIndex nmodes, const ptiIndex ndims[],
                            const ptiNnzIndex nnz, const ptiElementIndex sb_bits,
                            const ptiElementIndex sk_bits, const ptiElementIndex sc_bits)
{
    // src/sptensor/hicoo/hicoo.c:29-129: all vectors empty, kernel-row lists
    // allocated per mode (ceil(ndims[m] / 2^sk) rows each).
    std::memset(hitsr, 0, sizeof *hitsr);
    hitsr->nmodes = nmodes;
    hitsr->sortorder = static_cast<ptiIndex *>(std::malloc(nmodes * sizeof(ptiIndex)));
    for (ptiIndex i = 0; i < nmodes; ++i) hitsr->sortorder[i] = i;
    hitsr->ndims = static_cast<ptiIndex *>(std::malloc(nmodes * sizeof(ptiIndex)));
    std::memcpy(hitsr->ndims, ndims, nmodes * sizeof(ptiIndex));
    hitsr->nnz = nnz;
    hitsr->sb_bits = sb_bits;
    hitsr->sk_bits = sk_bits;
    hitsr->sc_bits = sc_bits;
    uint64_t sk = (uint64_t)1 << sk_bits;
    auto rows_lists = [&](ptiIndexVector **&lists) -> int {
        lists = static_cast<ptiIndexVector **>(std::malloc(nmodes * sizeof(ptiIndexVector *)));
        PTI_CHECK(lists, PTIERR_OS_ERROR + ENOMEM, "HiSpTns New", "out of memory");
        for (ptiIndex m = 0; m < nmodes; ++m) {
            uint64_t rows = (ndims[m] + sk - 1) / sk;
            lists[m] = static_cast<ptiIndexVector *>(std::malloc((rows ? rows : 1) * sizeof(ptiIndexVector)));
            for (uint64_t i = 0; i < rows; ++i)
                PTI_TRY((new_vector<ptiIndexVector, ptiIndex>(&lists[m][i], 0, 0)));
        }
        return 0;
    };
    PTI_TRY(rows_lists(hitsr->kschr));
    PTI_TRY(rows_lists(hitsr->kschr_balanced));
    PTI_TRY(rows_lists(hitsr->kschr_balanced_pos));
    hitsr->nkiters = static_cast<ptiIndex *>(std::calloc(nmodes, sizeof(ptiIndex)));
    hitsr->nkpars = static_cast<ptiIndex *>(std::calloc(nmodes, sizeof(ptiIndex)));
    hitsr->kschr_rest = static_cast<ptiIndexVector *>(std::malloc(nmodes * sizeof(ptiIndexVector)));
    for (ptiIndex m = 0; m < nmodes; ++m)
        PTI_TRY((new_vector<ptiIndexVector, ptiIndex>(&hitsr->kschr_rest[m], 0, 0)));
    PTI_TRY((new_vector<ptiNnzIndexVector, ptiNnzIndex>(&hitsr->kptr, 0, 0)));
    PTI_TRY((new_vector<ptiNnzIndexVector, ptiNnzIndex>(&hitsr->cptr, 0, 0)));
    PTI_TRY((new_vector<ptiNnzIndexVector, ptiNnzIndex>(&hitsr->knnzs, 0, 0)));
    PTI_TRY((new_vector<ptiNnzIndexVector, ptiNnzIndex>(&hitsr->bptr, 0, 0)));
    hitsr->binds = static_cast<ptiBlockIndexVector *>(std::malloc(nmodes * sizeof(ptiBlockIndexVector)));
    hitsr->einds = static_cast<ptiElementIndexVector *>(std::malloc(nmodes * sizeof(ptiElementIndexVector)));
    for (ptiIndex m = 0; m < nmodes; ++m) {
        PTI_TRY((new_vector<ptiBlockIndexVector, ptiBlockIndex>(&hitsr->binds[m], 0, 0)));
        PTI_TRY((new_vector<ptiElementIndexVector, ptiElementIndex>(&hitsr->einds[m], 0, 0)));
    }
    PTI_TRY((new_vector<ptiValueVector, ptiValue>(&hitsr->values, 0, 0)));
    return 0;
}

void ptiFreeSparseTensorHiCOO(ptiSparseTensorHiCOO *hitsr)
{
    ptiIndex nmodes = hitsr->nmodes;
    uint64_t sk = (uint64_t)1 << hitsr->sk_bits;
    auto free_lists = [&](ptiIndexVector **&lists) {
        if (!lists) return;
        for (ptiIndex m = 0; m < nmodes; ++m) {
            uint64_t rows = (hitsr->ndims[m] + sk - 1) / sk;
            for (uint64_t i = 0; i < rows; ++i) free_vector(&lists[m][i]);
            std::free(lists[m]);
        }
        std::free(lists);
        lists = nullptr;
    };
    free_lists(hitsr->kschr);
    free_lists(hitsr->kschr_balanced);
    free_lists(hitsr->kschr_balanced_pos);
    std::free(hitsr->nkiters);
    std::free(hitsr->nkpars);
    if (hitsr->kschr_rest)
        for (ptiIndex m = 0; m < nmodes; ++m) free_vector(&hitsr->kschr_rest[m]);
    std::free(hitsr->kschr_rest);
    free_vector(&hitsr->kptr);
    free_vector(&hitsr->cptr);
    free_vector(&hitsr->knnzs);
    free_vector(&hitsr->bptr);
    for (ptiIndex m = 0; m < nmodes; ++m) {
        if (hitsr->binds) free_vector(&hitsr->binds[m]);
        if (hitsr->einds) free_vector(&hitsr->einds[m]);
    }
    std::free(hitsr->binds);
    std::free(hitsr->einds);
    free_vector(&hitsr->values);
    std::free(hitsr->sortorder);
    std::free(hitsr->ndims);
    std::memset(hitsr, 0, sizeof *hitsr);
}

}  // extern "C"

namespace pti {

// Replaces the contents of a vector with `len` copied elements.
template <class V, class T>
int assign_vector(V *v, const T *src, uint64_t len)
{
    free_vector(v);
    PTI_TRY((new_vector<V, T>(v, len, len)));
    if (len) std::memcpy(v->data, src, len * sizeof(T));
    return 0;
}

int assign_nnz_vector(ptiNnzIndexVector *v, const uint64_t *src, uint64_t len)
{
    return assign_vector<ptiNnzIndexVector, ptiNnzIndex>(v, src, len);
}
int assign_index_vector(ptiIndexVector *v, const uint32_t *src, uint64_t len)
{
    return assign_vector<ptiIndexVector, ptiIndex>(v, src, len);
}
int alloc_block_vector(ptiBlockIndexVector *v, uint64_t len)
{
    free_vector(v);
    return new_vector<ptiBlockIndexVector, ptiBlockIndex>(v, len, len);
}
int alloc_element_vector(ptiElementIndexVector *v, uint64_t len)
{
    free_vector(v);
    return new_vector<ptiElementIndexVector, ptiElementIndex>(v, len, len);
}
int alloc_value_vector(ptiValueVector *v, uint64_t len)
{
    free_vector(v);
    return new_vector<ptiValueVector, ptiValue>(v, len, len);
}
int alloc_nnz_vector(ptiNnzIndexVector *v, uint64_t len)
{
    free_vector(v);
    return new_vector<ptiNnzIndexVector, ptiNnzIndex>(v, len, len);
}

}  // namespace pti
