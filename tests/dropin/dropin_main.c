/*
 * A caller of the reference's C API, compiled against the reference's own
 * header (HiParTI.h from the reference's include/ directory, not
 * include/hiparti_b200.h) and linked against libhiparti_b200.so: the drop-in
 * proof for the MTTKRP / CPD-ALS path.  It uses only names the reference
 * declares (plus CpdAlsStep, which the reference exports without declaring,
 * src/sptensor/cpd.c:32) and writes every result as raw little-endian
 * arrays into an output directory; tests/test_dropin_gpu.py compares them
 * with the reference library run on the same inputs.
 *
 *   dropin <tensor.tns> <outdir> <rank> <sb> <sk> <sc> <cpd_iters>
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "HiParTI.h"

double CpdAlsStep(ptiSparseTensor const * const ptien, ptiIndex const rank, ptiIndex const niters,
                  double const tol, ptiMatrix ** mats, ptiValue * const lambda);

static const char *g_out;

static int dump(const char *name, const void *data, size_t bytes)
{
    char path[4096];
    snprintf(path, sizeof path, "%s/%s.bin", g_out, name);
    FILE *f = fopen(path, "wb");
    if (!f) return 1;
    size_t w = bytes ? fwrite(data, 1, bytes, f) : 0;
    fclose(f);
    return w != bytes;
}

#define CHECK(x)                                                        \
    do {                                                                \
        int _r = (x);                                                   \
        if (_r) {                                                       \
            fprintf(stderr, "%s:%d: %s returned %d\n", __FILE__, __LINE__, #x, _r); \
            return 1;                                                   \
        }                                                               \
    } while (0)

/* deterministic factor entries in (0.1, 1.1) */
static void fill(ptiMatrix *m, ptiIndex mode)
{
    for (ptiIndex i = 0; i < m->nrows; ++i)
        for (ptiIndex j = 0; j < m->stride; ++j)
            m->values[(size_t)i * m->stride + j] =
                j < m->ncols ? 0.1f + (float)((i * 7u + j * 3u + mode * 5u) % 11u) / 10.0f : 0.0f;
}

/* row-major upper triangle of A^T A, as the reference's ssyrk_('L') calls leave it */
static void gram(const ptiMatrix *A, ptiMatrix *G)
{
    const ptiIndex R = A->ncols, st = A->stride;
    for (ptiIndex p = 0; p < R; ++p)
        for (ptiIndex q = 0; q < st; ++q) {
            double s = 0.0;
            if (q >= p && q < R)
                for (ptiIndex i = 0; i < A->nrows; ++i)
                    s += (double)A->values[(size_t)i * st + p] * A->values[(size_t)i * st + q];
            G->values[(size_t)p * st + q] = (float)s;
        }
}

int main(int argc, char **argv)
{
    if (argc != 8) {
        fprintf(stderr, "usage: %s tensor.tns outdir rank sb sk sc cpd_iters\n", argv[0]);
        return 2;
    }
    g_out = argv[2];
    const ptiIndex R = (ptiIndex)atoi(argv[3]);
    const ptiElementIndex sb = (ptiElementIndex)atoi(argv[4]), sk = (ptiElementIndex)atoi(argv[5]),
                          sc = (ptiElementIndex)atoi(argv[6]);
    const ptiIndex iters = (ptiIndex)atoi(argv[7]);

    ptiSparseTensor X;
    CHECK(ptiLoadSparseTensor(&X, 1, argv[1]));
    const ptiIndex N = X.nmodes;
    ptiIndex maxdim = 0;
    for (ptiIndex m = 0; m < N; ++m) maxdim = X.ndims[m] > maxdim ? X.ndims[m] : maxdim;
    CHECK(dump("ndims", X.ndims, N * sizeof(ptiIndex)));
    for (ptiIndex m = 0; m < N; ++m) {
        char nm[64];
        snprintf(nm, sizeof nm, "coo_ind%u", m);
        CHECK(dump(nm, X.inds[m].data, X.nnz * sizeof(ptiIndex)));
    }
    CHECK(dump("coo_vals", X.values.data, X.nnz * sizeof(ptiValue)));

    /* factors and MTTKRP output */
    ptiMatrix **mats = (ptiMatrix **)malloc((N + 1) * sizeof(ptiMatrix *));
    for (ptiIndex m = 0; m <= N; ++m) {
        mats[m] = (ptiMatrix *)malloc(sizeof(ptiMatrix));
        CHECK(ptiNewMatrix(mats[m], m < N ? X.ndims[m] : maxdim, R));
        if (m < N) fill(mats[m], m);
        else CHECK(ptiConstantMatrix(mats[m], 0));
    }
    ptiIndex *order = (ptiIndex *)malloc(N * sizeof(ptiIndex));
    for (ptiIndex mode = 0; mode < N; ++mode) {
        for (ptiIndex i = 0; i < N; ++i) order[i] = (mode + i) % N;
        char nm[64];
        CHECK(ptiMTTKRP(&X, mats, order, mode));
        snprintf(nm, sizeof nm, "mttkrp_coo%u", mode);
        CHECK(dump(nm, mats[N]->values, (size_t)X.ndims[mode] * mats[N]->stride * sizeof(ptiValue)));
    }

    /* COO -> HiCOO (sorts X in place, as the reference does) and HiCOO MTTKRP */
    ptiSparseTensorHiCOO H;
    ptiNnzIndex max_nnzb = 0;
    CHECK(ptiSparseTensorToHiCOO(&H, &max_nnzb, &X, sb, sk, sc, 1));
    const ptiNnzIndex nb = H.bptr.len - 1;
    CHECK(dump("h_bptr", H.bptr.data, (nb + 1) * sizeof(ptiNnzIndex)));
    CHECK(dump("h_kptr", H.kptr.data, H.kptr.len * sizeof(ptiNnzIndex)));
    CHECK(dump("h_cptr", H.cptr.data, H.cptr.len * sizeof(ptiNnzIndex)));
    CHECK(dump("h_vals", H.values.data, H.nnz * sizeof(ptiValue)));
    CHECK(dump("h_max_nnzb", &max_nnzb, sizeof max_nnzb));
    for (ptiIndex m = 0; m < N; ++m) {
        char nm[64];
        snprintf(nm, sizeof nm, "h_binds%u", m);
        CHECK(dump(nm, H.binds[m].data, nb * sizeof(ptiBlockIndex)));
        snprintf(nm, sizeof nm, "h_einds%u", m);
        CHECK(dump(nm, H.einds[m].data, H.nnz * sizeof(ptiElementIndex)));
    }
    for (ptiIndex mode = 0; mode < N; ++mode) {
        for (ptiIndex i = 0; i < N; ++i) order[i] = (mode + i) % N;
        char nm[64];
        CHECK(ptiMTTKRPHiCOO(&H, mats, order, mode));
        snprintf(nm, sizeof nm, "mttkrp_hicoo%u", mode);
        CHECK(dump(nm, mats[N]->values, (size_t)X.ndims[mode] * mats[N]->stride * sizeof(ptiValue)));
    }

    /* dense ALS helpers on Grams of the factors */
    ptiMatrix **ata = (ptiMatrix **)malloc((N + 1) * sizeof(ptiMatrix *));
    for (ptiIndex m = 0; m <= N; ++m) {
        ata[m] = (ptiMatrix *)malloc(sizeof(ptiMatrix));
        CHECK(ptiNewMatrix(ata[m], R, R));
        if (m < N) gram(mats[m], ata[m]);
        else CHECK(ptiConstantMatrix(ata[m], 0));
    }
    CHECK(ptiMatrixDotMulSeqTriangle(0, N, ata));
    CHECK(dump("dotmul_tri", ata[N]->values, (size_t)R * ata[N]->stride * sizeof(ptiValue)));
    ptiMatrix rhs;
    CHECK(ptiNewMatrix(&rhs, X.ndims[0], R));
    fill(&rhs, 7);
    CHECK(ptiMatrixSolveNormals(0, N, ata, &rhs));
    CHECK(dump("solve_normals", rhs.values, (size_t)rhs.nrows * rhs.stride * sizeof(ptiValue)));
    ptiValue *lam = (ptiValue *)malloc(R * sizeof(ptiValue));
    CHECK(ptiMatrix2Norm(&rhs, lam));
    CHECK(dump("norm2_lambda", lam, R * sizeof(ptiValue)));
    CHECK(dump("norm2_matrix", rhs.values, (size_t)rhs.nrows * rhs.stride * sizeof(ptiValue)));
    fill(&rhs, 9);
    CHECK(ptiMatrixMaxNorm(&rhs, lam));
    CHECK(dump("maxnorm_lambda", lam, R * sizeof(ptiValue)));
    CHECK(dump("maxnorm_matrix", rhs.values, (size_t)rhs.nrows * rhs.stride * sizeof(ptiValue)));
    for (ptiIndex r = 0; r < R; ++r) lam[r] = 1.0f + 0.25f * (float)r;
    double knorm = KruskalTensorFrobeniusNormSquared(N, lam, ata);
    CHECK(dump("kruskal_normsq", &knorm, sizeof knorm));
    double xnorm = SparseTensorFrobeniusNormSquared(&X);
    CHECK(dump("tensor_normsq", &xnorm, sizeof xnorm));

    /* CPD: the reference's driver entry and its ALS step from seeded factors */
    ptiKruskalTensor K;
    CHECK(ptiNewKruskalTensor(&K, N, X.ndims, R));
    CHECK(ptiCpdAls(&X, R, iters, 0.0, &K));
    CHECK(dump("cpd_lambda", K.lambda, R * sizeof(ptiValue)));
    CHECK(dump("cpd_fit", &K.fit, sizeof K.fit));
    for (ptiIndex m = 0; m < N; ++m) {
        char nm[64];
        snprintf(nm, sizeof nm, "cpd_factor%u", m);
        CHECK(dump(nm, K.factors[m]->values, (size_t)X.ndims[m] * K.factors[m]->stride * sizeof(ptiValue)));
    }
    for (ptiIndex m = 0; m < N; ++m) fill(mats[m], m);
    double step_fit = CpdAlsStep(&X, R, iters, 0.0, mats, lam);
    CHECK(dump("step_fit", &step_fit, sizeof step_fit));
    CHECK(dump("step_lambda", lam, R * sizeof(ptiValue)));
    for (ptiIndex m = 0; m < N; ++m) {
        char nm[64];
        snprintf(nm, sizeof nm, "step_factor%u", m);
        CHECK(dump(nm, mats[m]->values, (size_t)X.ndims[m] * mats[m]->stride * sizeof(ptiValue)));
    }
    /* the model's fit through KruskalTensorFit: Grams of the result, and the
       MTTKRP of the last mode with the result's factors */
    for (ptiIndex m = 0; m < N; ++m) gram(mats[m], ata[m]);
    for (ptiIndex i = 0; i < N; ++i) order[i] = (N - 1 + i) % N;
    CHECK(ptiMTTKRP(&X, mats, order, N - 1));
    double kfit = KruskalTensorFit(&X, lam, mats, ata);
    CHECK(dump("kruskal_fit", &kfit, sizeof kfit));

    ptiFreeKruskalTensor(&K);
    ptiFreeSparseTensorHiCOO(&H);
    ptiFreeSparseTensor(&X);
    printf("dropin ok\n");
    return 0;
}
