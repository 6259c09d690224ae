// checkpoint.cu -- Kruskal tensor text dumps (the reference's format) and
// CPD-ALS checkpoint files (the format is described in checkpoint.cuh).
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <fcntl.h>
#include <unistd.h>

#include "checkpoint.cuh"

namespace pti {
namespace {

constexpr uint64_t kFnvBasis = 0xcbf29ce484222325ull;
constexpr uint64_t kFnvPrime = 0x100000001b3ull;

uint64_t fnv_words(uint64_t h, const void *p, size_t bytes)
{
    const unsigned char *b = static_cast<const unsigned char *>(p);
    for (size_t i = 0; i + 8 <= bytes; i += 8) {
        uint64_t w;
        std::memcpy(&w, b + i, 8);
        h = (h ^ w) * kFnvPrime;
    }
    return h;
}

size_t round8(size_t n) { return (n + 7) & ~(size_t)7; }

struct Head {
    char magic[8];
    uint32_t version, nmodes, rank, iters, flags, reserved;
    uint64_t nnz;
    double normX2;
};
static_assert(sizeof(Head) == 48, "checkpoint header is 48 bytes");

// Writes `bytes` (a multiple of 8) and folds them into the checksum.
bool put(FILE *fp, uint64_t &h, const void *p, size_t bytes)
{
    h = fnv_words(h, p, bytes);
    return std::fwrite(p, 1, bytes, fp) == bytes;
}

}  // namespace

// ---------------------------------------------------------------------------
// Reading
// ---------------------------------------------------------------------------
int ckpt_read(const char *path, CkptState &st, bool *missing)
{
    const char *mod = "CPD checkpoint";
    PTI_CHECK(path, PTIERR_VALUE_ERROR, mod, "null path");
    if (missing) *missing = false;
    FILE *fp = std::fopen(path, "rb");
    if (!fp && errno == ENOENT && missing) {
        *missing = true;
        return 0;
    }
    PTI_CHECK(fp, PTIERR_OS_ERROR + errno, mod, std::strerror(errno));
    std::fseek(fp, 0, SEEK_END);
    const long len = std::ftell(fp);
    std::fseek(fp, 0, SEEK_SET);
    std::vector<unsigned char> buf(len > 0 ? (size_t)len : 0);
    const size_t got = buf.empty() ? 0 : std::fread(buf.data(), 1, buf.size(), fp);
    std::fclose(fp);
    PTI_CHECK(got == buf.size() && got >= sizeof(Head) + 8 && got % 8 == 0, PTIERR_VALUE_ERROR, mod,
              "truncated checkpoint file");
    Head h;
    std::memcpy(&h, buf.data(), sizeof h);
    PTI_CHECK(std::memcmp(h.magic, kCkptMagic, 8) == 0, PTIERR_VALUE_ERROR, mod, "not a CPD checkpoint file");
    PTI_CHECK(h.version == kCkptVersion, PTIERR_VALUE_ERROR, mod, "unsupported checkpoint version");
    PTI_CHECK(h.nmodes >= 1 && h.nmodes <= 64 && h.rank >= 1, PTIERR_VALUE_ERROR, mod, "bad checkpoint header");
    size_t off = sizeof(Head);
    const size_t dims_bytes = round8((size_t)h.nmodes * 4);
    PTI_CHECK(off + dims_bytes <= got, PTIERR_VALUE_ERROR, mod, "truncated checkpoint file");
    std::vector<uint32_t> ndims(h.nmodes);
    std::memcpy(ndims.data(), buf.data() + off, (size_t)h.nmodes * 4);
    off += dims_bytes;
    uint64_t rows = 0;
    for (uint32_t d : ndims) rows += d;
    const uint64_t body = (uint64_t)h.iters * 8 + round8(((uint64_t)h.rank + rows * h.rank) * 4);
    PTI_CHECK(off + body + 8 == got, PTIERR_VALUE_ERROR, mod, "checkpoint size does not match its header");
    uint64_t sum;
    std::memcpy(&sum, buf.data() + got - 8, 8);
    PTI_CHECK(fnv_words(kFnvBasis, buf.data(), got - 8) == sum, PTIERR_VALUE_ERROR, mod,
              "checkpoint checksum mismatch");

    st.nmodes = h.nmodes;
    st.rank = h.rank;
    st.iters = h.iters;
    st.flags = h.flags;
    st.nnz = h.nnz;
    st.normX2 = h.normX2;
    st.ndims = ndims;
    st.fits.resize(h.iters);
    if (h.iters) std::memcpy(st.fits.data(), buf.data() + off, (size_t)h.iters * 8);
    off += (size_t)h.iters * 8;
    st.lambda.resize(h.rank);
    std::memcpy(st.lambda.data(), buf.data() + off, (size_t)h.rank * 4);
    off += (size_t)h.rank * 4;
    st.factors.assign(h.nmodes, {});
    for (uint32_t m = 0; m < h.nmodes; ++m) {
        const size_t n = (size_t)ndims[m] * h.rank;
        st.factors[m].resize(n);
        if (n) std::memcpy(st.factors[m].data(), buf.data() + off, n * 4);
        off += n * 4;
    }
    return 0;
}

// ---------------------------------------------------------------------------
// Writing
// ---------------------------------------------------------------------------
CkptWriter::~CkptWriter()
{
    if (th_.joinable()) th_.join();
    if (ev_) cudaEventDestroy(ev_);
    if (host_) cudaFreeHost(host_);
}

int CkptWriter::init(const char *path, uint32_t nmodes, const uint32_t *ndims, uint64_t nnz, uint32_t rank,
                     uint32_t max_iters)
{
    const char *mod = "CPD checkpoint";
    PTI_CHECK(path && *path, PTIERR_VALUE_ERROR, mod, "empty checkpoint path");
    path_ = path;
    ndims_.assign(ndims, ndims + nmodes);
    nnz_ = nnz;
    rank_ = rank;
    max_iters_ = max_iters;
    factor_floats_ = 0;
    for (uint32_t d : ndims_) factor_floats_ += (size_t)d * rank;
    const size_t bytes = 8 + (size_t)max_iters * 8 + ((size_t)rank + factor_floats_) * 4;
    PTI_CUDA(cudaHostAlloc(reinterpret_cast<void **>(&host_), bytes, cudaHostAllocDefault), mod);
    PTI_CUDA(cudaEventCreateWithFlags(&ev_, cudaEventDisableTiming | cudaEventBlockingSync), mod);
    return 0;
}

int CkptWriter::save(float *const *A, uint32_t stride, const float *lambda, const double *fits,
                     const double *normX2, uint32_t iters, bool converged, cudaStream_t s)
{
    const char *mod = "CPD checkpoint";
    PTI_TRY(finish());  // the staging buffer is reused
    PTI_CHECK(iters <= max_iters_, PTIERR_VALUE_ERROR, mod, "more iterations than the writer was sized for");
    double *h_norm = reinterpret_cast<double *>(host_);
    double *h_fits = h_norm + 1;
    float *h_lam = reinterpret_cast<float *>(h_fits + max_iters_);
    float *h_fac = h_lam + rank_;
    PTI_CUDA(cudaMemcpyAsync(h_norm, normX2, 8, cudaMemcpyDeviceToHost, s), mod);
    if (iters) PTI_CUDA(cudaMemcpyAsync(h_fits, fits, (size_t)iters * 8, cudaMemcpyDeviceToHost, s), mod);
    PTI_CUDA(cudaMemcpyAsync(h_lam, lambda, (size_t)rank_ * 4, cudaMemcpyDeviceToHost, s), mod);
    for (size_t m = 0; m < ndims_.size(); ++m) {
        if (ndims_[m])
            PTI_CUDA(cudaMemcpy2DAsync(h_fac, (size_t)rank_ * 4, A[m], (size_t)stride * 4, (size_t)rank_ * 4,
                                       ndims_[m], cudaMemcpyDeviceToHost, s),
                     mod);
        h_fac += (size_t)ndims_[m] * rank_;
    }
    PTI_CUDA(cudaEventRecord(ev_, s), mod);
    iters_ = iters;
    flags_ = converged ? kCkptConverged : 0;
    th_ = std::thread([this] { write_file(); });
    return 0;
}

void CkptWriter::write_file()
{
    if (cudaEventSynchronize(ev_) != cudaSuccess) {
        err_ = PTIERR_CUDA_ERROR;
        why_ = "copy of the ALS state failed";
        return;
    }
    const double *h_norm = reinterpret_cast<const double *>(host_);
    const double *h_fits = h_norm + 1;
    const float *h_lam = reinterpret_cast<const float *>(h_fits + max_iters_);
    Head h{};
    std::memcpy(h.magic, kCkptMagic, 8);
    h.version = kCkptVersion;
    h.nmodes = (uint32_t)ndims_.size();
    h.rank = rank_;
    h.iters = iters_;
    h.flags = flags_;
    h.nnz = nnz_;
    h.normX2 = *h_norm;
    std::vector<uint32_t> dims(round8(ndims_.size() * 4) / 4, 0u);
    std::copy(ndims_.begin(), ndims_.end(), dims.begin());

    const std::string tmp = path_ + ".tmp";
    FILE *fp = std::fopen(tmp.c_str(), "wb");
    if (!fp) {
        err_ = PTIERR_OS_ERROR + errno;
        why_ = tmp + ": " + std::strerror(errno);
        return;
    }
    uint64_t sum = kFnvBasis;
    bool ok = put(fp, sum, &h, sizeof h) && put(fp, sum, dims.data(), dims.size() * 4) &&
              put(fp, sum, h_fits, (size_t)iters_ * 8);
    // lambda and the factors are contiguous in the staging buffer; the final
    // partial word (odd float count) is padded with zeros.
    const size_t vbytes = ((size_t)rank_ + factor_floats_) * 4;
    const size_t whole = vbytes & ~(size_t)7;
    ok = ok && put(fp, sum, h_lam, whole);
    if (ok && whole != vbytes) {
        unsigned char tail[8] = {0};
        std::memcpy(tail, reinterpret_cast<const unsigned char *>(h_lam) + whole, vbytes - whole);
        ok = put(fp, sum, tail, 8);
    }
    ok = ok && std::fwrite(&sum, 1, 8, fp) == 8;
    ok = ok && std::fflush(fp) == 0 && fsync(fileno(fp)) == 0;
    const int saved = errno;
    ok = (std::fclose(fp) == 0) && ok;
    if (!ok) {
        err_ = PTIERR_OS_ERROR + (saved ? saved : EIO);
        why_ = tmp + ": write failed";
        std::remove(tmp.c_str());
        return;
    }
    if (std::rename(tmp.c_str(), path_.c_str()) != 0) {
        err_ = PTIERR_OS_ERROR + errno;
        why_ = path_ + ": " + std::strerror(errno);
    }
}

int CkptWriter::finish()
{
    if (th_.joinable()) th_.join();
    if (err_) {
        const int e = err_;
        err_ = 0;
        return complain("CPD checkpoint", e, __FILE__, __LINE__, why_.c_str());
    }
    return 0;
}

}  // namespace pti

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

// Text dumps in the reference's format (src/matrix/dump.c:33-49,59-75 and
// src/ktensor/dump.c:23-88): a "<rows> x <cols> matrix" line, then every row
// as "%.2f\t" fields; a Kruskal tensor as its header, sizes, fit, weights and
// factor matrices.
int ptiDumpMatrix(ptiMatrix *mtx, FILE *fp)
{
    PTI_CHECK(mtx && fp, PTIERR_VALUE_ERROR, "Mtx Dump", "null argument");
    PTI_CHECK(std::fprintf(fp, "%u x %u matrix\n", mtx->nrows, mtx->ncols) >= 0, PTIERR_OS_ERROR + errno,
              "Mtx Dump", "write failed");
    for (ptiIndex i = 0; i < mtx->nrows; ++i) {
        const ptiValue *row = mtx->values + (size_t)i * mtx->stride;
        for (ptiIndex j = 0; j < mtx->ncols; ++j)
            PTI_CHECK(std::fprintf(fp, "%.2f\t", (double)row[j]) >= 0, PTIERR_OS_ERROR + errno, "Mtx Dump",
                      "write failed");
        std::fputc('\n', fp);
    }
    std::fputc('\n', fp);
    return 0;
}

int ptiDumpRankMatrix(ptiRankMatrix *mtx, FILE *fp)
{
    PTI_CHECK(mtx && fp, PTIERR_VALUE_ERROR, "RankMtx Dump", "null argument");
    PTI_CHECK(std::fprintf(fp, "%u x %u matrix\n", mtx->nrows, (unsigned)mtx->ncols) >= 0,
              PTIERR_OS_ERROR + errno, "RankMtx Dump", "write failed");
    for (ptiIndex i = 0; i < mtx->nrows; ++i) {
        const ptiValue *row = mtx->values + (size_t)i * mtx->stride;
        for (ptiElementIndex j = 0; j < mtx->ncols; ++j)
            PTI_CHECK(std::fprintf(fp, "%.2f\t", (double)row[j]) >= 0, PTIERR_OS_ERROR + errno, "RankMtx Dump",
                      "write failed");
        std::fputc('\n', fp);
    }
    std::fputc('\n', fp);
    return 0;
}

namespace {
// Header, sizes, fit and weights of a Kruskal tensor.
int dump_kruskal_head(const char *mod, ptiIndex nmodes, unsigned rank, const ptiIndex *ndims, double fit,
                      const ptiValue *lambda, FILE *fp)
{
    PTI_CHECK(std::fprintf(fp, "nmodes: %u, rank: %u\n", nmodes, rank) >= 0, PTIERR_OS_ERROR + errno, mod,
              "write failed");
    for (ptiIndex m = 0; m < nmodes; ++m) std::fprintf(fp, m ? " %u" : "%u", ndims[m]);
    std::fputc('\n', fp);
    std::fprintf(fp, "fit: %f\n", fit);
    std::fputs("lambda:\n", fp);
    for (unsigned r = 0; r < rank; ++r) std::fprintf(fp, "%f ", (double)lambda[r]);
    std::fputc('\n', fp);
    PTI_CHECK(std::fputs("Factor matrices:\n", fp) >= 0, PTIERR_OS_ERROR + errno, mod, "write failed");
    return 0;
}
}  // namespace

int ptiDumpKruskalTensor(ptiKruskalTensor *ktsr, FILE *fp)
{
    const char *mod = "KruskalTns Dump";
    PTI_CHECK(ktsr && fp && ktsr->factors, PTIERR_VALUE_ERROR, mod, "null argument");
    PTI_TRY(dump_kruskal_head(mod, ktsr->nmodes, ktsr->rank, ktsr->ndims, ktsr->fit, ktsr->lambda, fp));
    for (ptiIndex m = 0; m < ktsr->nmodes; ++m) PTI_TRY(ptiDumpMatrix(ktsr->factors[m], fp));
    return 0;
}

int ptiDumpRankKruskalTensor(ptiRankKruskalTensor *ktsr, FILE *fp)
{
    const char *mod = "RankKruskalTns Dump";
    PTI_CHECK(ktsr && fp && ktsr->factors, PTIERR_VALUE_ERROR, mod, "null argument");
    PTI_TRY(dump_kruskal_head(mod, ktsr->nmodes, ktsr->rank, ktsr->ndims, ktsr->fit, ktsr->lambda, fp));
    for (ptiIndex m = 0; m < ktsr->nmodes; ++m) PTI_TRY(ptiDumpRankMatrix(ktsr->factors[m], fp));
    return 0;
}

namespace {
int load_checkpoint(ptiKruskalTensor *ktsr, const pti::CkptState &st)
{
    using namespace pti;
    const char *mod = "CPD checkpoint";
    const uint32_t N = st.nmodes, R = st.rank;
    PTI_TRY(ptiNewKruskalTensor(ktsr, N, st.ndims.data(), R));
    ktsr->factors = static_cast<ptiMatrix **>(std::calloc(N + 1, sizeof(ptiMatrix *)));
    PTI_CHECK(ktsr->factors, PTIERR_OS_ERROR + ENOMEM, mod, "out of memory");
    std::memcpy(ktsr->lambda, st.lambda.data(), (size_t)R * 4);
    // The final weights, as the ALS loop computes them after its last
    // iteration (src/matrix/matrix.c:556-572): every factor column scaled to
    // unit 2-norm (FP64 sums), the weights multiplied by the norms.
    std::vector<double> colsq(R);
    for (uint32_t m = 0; m < N; ++m) {
        ktsr->factors[m] = static_cast<ptiMatrix *>(std::calloc(1, sizeof(ptiMatrix)));
        PTI_CHECK(ktsr->factors[m], PTIERR_OS_ERROR + ENOMEM, mod, "out of memory");
        PTI_TRY(ptiNewMatrix(ktsr->factors[m], st.ndims[m], R));
        ptiMatrix *F = ktsr->factors[m];
        const float *src = st.factors[m].data();
        std::fill(colsq.begin(), colsq.end(), 0.0);
        for (uint32_t i = 0; i < st.ndims[m]; ++i)
            for (uint32_t c = 0; c < R; ++c) colsq[c] += (double)src[(size_t)i * R + c] * src[(size_t)i * R + c];
        for (uint32_t i = 0; i < st.ndims[m]; ++i) {
            float *row = F->values + (size_t)i * F->stride;
            for (uint32_t c = 0; c < F->stride; ++c)
                row[c] = c < R ? src[(size_t)i * R + c] / (float)std::sqrt(colsq[c]) : 0.f;
        }
        for (uint32_t c = 0; c < R; ++c) ktsr->lambda[c] *= (float)std::sqrt(colsq[c]);
    }
    ktsr->factors[N] = static_cast<ptiMatrix *>(std::calloc(1, sizeof(ptiMatrix)));
    ktsr->fit = st.iters ? st.fits[st.iters - 1] : 0.0;
    return 0;
}
}  // namespace

int ptiB200LoadCpdCheckpoint(ptiKruskalTensor *ktsr, ptiIndex *iters_done, const char *path)
{
    using namespace pti;
    PTI_CHECK(ktsr && path, PTIERR_VALUE_ERROR, "CPD checkpoint", "null argument");
    CkptState st;
    PTI_TRY(ckpt_read(path, st, nullptr));
    const int r = load_checkpoint(ktsr, st);
    if (r) {
        ptiFreeKruskalTensor(ktsr);
        return r;
    }
    if (iters_done) *iters_done = st.iters;
    return 0;
}

}  // extern "C"
