// containers.cu -- host-side life cycle of the reference's structs and the
// .tns / .bin tensor reader.  Struct layouts are those of
// include/includes/structs.h in the reference; ownership follows its
// src/sptensor/sptensor.c, src/matrix/matrix.c, src/ktensor/ktensor.c and
// src/sptensor/hicoo/hicoo.c.
#include "common.cuh"

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

// Reads a whole file into memory.
int slurp(const char *fname, std::vector<char> &buf)
{
    FILE *fp = std::fopen(fname, "rb");
    PTI_CHECK(fp, PTIERR_OS_ERROR + errno, "SpTns Load", std::strerror(errno));
    std::fseek(fp, 0, SEEK_END);
    long n = std::ftell(fp);
    std::fseek(fp, 0, SEEK_SET);
    buf.resize(n > 0 ? (size_t)n + 1 : 1);
    size_t got = n > 0 ? std::fread(buf.data(), 1, (size_t)n, fp) : 0;
    std::fclose(fp);
    buf.resize(got + 1);
    buf[got] = 0;
    return 0;
}

// Text coordinate format, src/sptensor/load.c:63-115: "N", then N mode sizes,
// then one nonzero per line: N indices (start_index-based) and a value.
int read_text(ptiSparseTensor *tsr, ptiIndex start_index, const std::vector<char> &buf)
{
    const char *p = buf.data();
    char *end = nullptr;
    unsigned long nm = std::strtoul(p, &end, 10);
    PTI_CHECK(end != p && nm > 0 && nm < 64, PTIERR_VALUE_ERROR, "SpTns Load", "bad header");
    p = end;
    ptiIndex nmodes = (ptiIndex)nm;
    std::vector<ptiIndex> ndims(nmodes);
    for (ptiIndex m = 0; m < nmodes; ++m) {
        unsigned long d = std::strtoul(p, &end, 10);
        PTI_CHECK(end != p, PTIERR_VALUE_ERROR, "SpTns Load", "bad mode sizes");
        ndims[m] = (ptiIndex)d;
        p = end;
    }
    std::vector<std::vector<ptiIndex>> inds(nmodes);
    std::vector<ptiValue> vals;
    for (;;) {
        ptiIndex idx[64];
        bool ok = true;
        for (ptiIndex m = 0; m < nmodes; ++m) {
            unsigned long v = std::strtoul(p, &end, 10);
            if (end == p) { ok = false; break; }
            p = end;
            if (v < start_index) PTI_FAIL(PTIERR_VALUE_ERROR, "SpTns Load", "index < start_index");
            idx[m] = (ptiIndex)(v - start_index);
        }
        if (!ok) break;
        double val = std::strtod(p, &end);
        if (end == p) break;
        p = end;
        for (ptiIndex m = 0; m < nmodes; ++m) inds[m].push_back(idx[m]);
        vals.push_back((ptiValue)val);
    }
    uint64_t nnz = vals.size();
    tsr->nmodes = nmodes;
    // The reference's text reader leaves sortorder zero-filled (load.c:69-71).
    tsr->sortorder = static_cast<ptiIndex *>(std::calloc(nmodes, sizeof(ptiIndex)));
    tsr->ndims = static_cast<ptiIndex *>(std::malloc(nmodes * sizeof(ptiIndex)));
    std::memcpy(tsr->ndims, ndims.data(), nmodes * sizeof(ptiIndex));
    tsr->nnz = nnz;
    tsr->inds = static_cast<ptiIndexVector *>(std::malloc(nmodes * sizeof(ptiIndexVector)));
    for (ptiIndex m = 0; m < nmodes; ++m) {
        PTI_TRY((new_vector<ptiIndexVector, ptiIndex>(&tsr->inds[m], nnz, nnz)));
        if (nnz) std::memcpy(tsr->inds[m].data, inds[m].data(), nnz * sizeof(ptiIndex));
    }
    PTI_TRY((new_vector<ptiValueVector, ptiValue>(&tsr->values, nnz, nnz)));
    if (nnz) std::memcpy(tsr->values.data, vals.data(), nnz * sizeof(ptiValue));
    return 0;
}

// SPLATT binary format, src/sptensor/load.c:120-265: header {int32 magic,
// uint64 idx_width, uint64 val_width}, then nmodes, dims and nnz as idx_width
// integers, the indices mode by mode, then the values.
int read_binary(ptiSparseTensor *tsr, const std::vector<char> &buf)
{
    size_t pos = 0, n = buf.size() - 1;
    auto take = [&](void *dst, size_t bytes) -> bool {
        if (pos + bytes > n) return false;
        std::memcpy(dst, buf.data() + pos, bytes);
        pos += bytes;
        return true;
    };
    int32_t magic;
    uint64_t iw, vw;
    PTI_CHECK(take(&magic, 4) && take(&iw, 8) && take(&vw, 8), PTIERR_VALUE_ERROR, "SpTns Load",
              "truncated header");
    PTI_CHECK(iw == 4, PTIERR_VALUE_ERROR, "SpTns Load", "only 32-bit indices are supported");
    PTI_CHECK(vw == 4 || vw == 8, PTIERR_VALUE_ERROR, "SpTns Load", "bad value width");
    uint32_t nm;
    PTI_CHECK(take(&nm, 4) && nm > 0 && nm < 64, PTIERR_VALUE_ERROR, "SpTns Load", "bad nmodes");
    std::vector<ptiIndex> dims(nm);
    PTI_CHECK(take(dims.data(), 4 * nm), PTIERR_VALUE_ERROR, "SpTns Load", "truncated dims");
    uint32_t nnz32;
    PTI_CHECK(take(&nnz32, 4), PTIERR_VALUE_ERROR, "SpTns Load", "truncated nnz");
    uint64_t nnz = nnz32;
    PTI_TRY(ptiNewSparseTensor(tsr, nm, dims.data()));
    tsr->nnz = nnz;
    for (uint32_t m = 0; m < nm; ++m) {
        free_vector(&tsr->inds[m]);
        PTI_TRY((new_vector<ptiIndexVector, ptiIndex>(&tsr->inds[m], nnz, nnz)));
        PTI_CHECK(take(tsr->inds[m].data, 4 * nnz), PTIERR_VALUE_ERROR, "SpTns Load", "truncated indices");
    }
    free_vector(&tsr->values);
    PTI_TRY((new_vector<ptiValueVector, ptiValue>(&tsr->values, nnz, nnz)));
    if (vw == 4) {
        PTI_CHECK(take(tsr->values.data, 4 * nnz), PTIERR_VALUE_ERROR, "SpTns Load", "truncated values");
    } else {
        for (uint64_t z = 0; z < nnz; ++z) {
            double d;
            PTI_CHECK(take(&d, 8), PTIERR_VALUE_ERROR, "SpTns Load", "truncated values");
            tsr->values.data[z] = (ptiValue)d;
        }
    }
    return 0;
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
    PTI_CHECK(fname, PTIERR_VALUE_ERROR, "SpTns Load", "null file name");
    std::vector<char> buf;
    PTI_TRY(slurp(fname, buf));
    // File type by extension, src/sptensor/load.c:28-60.
    const char *suffix = std::strrchr(fname, '.');
    bool binary = suffix && std::strcmp(suffix, ".bin") == 0;
    return binary ? read_binary(tsr, buf) : read_text(tsr, start_index, buf);
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
