/*
 * orc.c -- TEST INFRASTRUCTURE ONLY (see orc.h).  CPU restatement of the
 * reference's MTTKRP, COO->HiCOO conversion and CPD-ALS, used to check the
 * GPU library.  Never linked into the product.
 */
#include "orc.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;

/* ------------------------------------------------------------------------ */
/* MTTKRP (COO) -- src/sptensor/mttkrp.c:39-163                              */
/* ------------------------------------------------------------------------ */
void orc_mttkrp_coo_f32(uint32_t nmodes, uint64_t nnz, const uint32_t *const *inds,
                        const float *vals, const float *const *mats, uint32_t R,
                        uint32_t stride, const uint32_t *mats_order, uint32_t mode,
                        uint32_t out_rows, float *out)
{
    memset(out, 0, (size_t)out_rows * stride * sizeof(float));
    float *scratch = (float *)malloc((R ? R : 1) * sizeof(float));
    const uint32_t *mode_ind = inds[mode];
    for (uint64_t x = 0; x < nnz; ++x) {
        /* first factor: scratch = entry * A[i] (mttkrp.c:83-90; the 3-D path
         * at :151-160 evaluates entry*A1*A2 left to right, the same order). */
        uint32_t k = mats_order[1];
        const float *row = mats[k] + (size_t)inds[k][x] * stride;
        float entry = vals[x];
        for (uint32_t r = 0; r < R; ++r) scratch[r] = entry * row[r];
        for (uint32_t i = 2; i < nmodes; ++i) {
            k = mats_order[i];
            row = mats[k] + (size_t)inds[k][x] * stride;
            for (uint32_t r = 0; r < R; ++r) scratch[r] *= row[r];
        }
        float *o = out + (size_t)mode_ind[x] * stride;
        for (uint32_t r = 0; r < R; ++r) o[r] += scratch[r];
    }
    free(scratch);
}

void orc_mttkrp_coo_f64(uint32_t nmodes, uint64_t nnz, const uint32_t *const *inds,
                        const float *vals, const double *const *mats, uint32_t R,
                        uint32_t stride, uint32_t mode, uint32_t out_rows, double *out)
{
    /* OpenMP over nonzeros with thread-private outputs summed at the end, so
     * the oracle finishes full-size CPD checks in seconds. */
    const size_t len = (size_t)out_rows * stride;
    memset(out, 0, len * sizeof(double));
#pragma omp parallel
    {
        double *priv = (double *)calloc(len ? len : 1, sizeof(double));
        double *scratch = (double *)malloc((R ? R : 1) * sizeof(double));
#pragma omp for schedule(static)
        for (uint64_t x = 0; x < nnz; ++x) {
            for (uint32_t r = 0; r < R; ++r) scratch[r] = (double)vals[x];
            for (uint32_t k = 0; k < nmodes; ++k) {
                if (k == mode) continue;
                const double *row = mats[k] + (size_t)inds[k][x] * stride;
                for (uint32_t r = 0; r < R; ++r) scratch[r] *= row[r];
            }
            double *o = priv + (size_t)inds[mode][x] * stride;
            for (uint32_t r = 0; r < R; ++r) o[r] += scratch[r];
        }
#pragma omp critical
        for (size_t i = 0; i < len; ++i) out[i] += priv[i];
        free(priv);
        free(scratch);
    }
}

/* ------------------------------------------------------------------------ */
/* MTTKRP (HiCOO) -- src/sptensor/hicoo/mttkrp.c:61-152, :232-310            */
/* Blocks are visited in storage order, which is the kernel -> block order   */
/* of the reference loops (kptr partitions the block range contiguously).    */
/* ------------------------------------------------------------------------ */
void orc_mttkrp_hicoo_f32(uint32_t nmodes, uint64_t nnz, uint64_t nb, uint8_t sb_bits,
                          const uint64_t *bptr, const uint32_t *const *binds,
                          const uint8_t *const *einds, const float *vals,
                          const float *const *mats, uint32_t R, uint32_t stride,
                          const uint32_t *mats_order, uint32_t mode, uint32_t out_rows,
                          float *out)
{
    (void)nnz;
    memset(out, 0, (size_t)out_rows * stride * sizeof(float));
    float *scratch = (float *)malloc((R ? R : 1) * sizeof(float));
    uint32_t coord[16];
    for (uint64_t b = 0; b < nb; ++b) {
        for (uint64_t z = bptr[b]; z < bptr[b + 1]; ++z) {
            for (uint32_t m = 0; m < nmodes; ++m)
                coord[m] = (binds[m][b] << sb_bits) + einds[m][z];
            uint32_t k = mats_order[1];
            const float *row = mats[k] + (size_t)coord[k] * stride;
            float entry = vals[z];
            for (uint32_t r = 0; r < R; ++r) scratch[r] = entry * row[r];
            for (uint32_t i = 2; i < nmodes; ++i) {
                k = mats_order[i];
                row = mats[k] + (size_t)coord[k] * stride;
                for (uint32_t r = 0; r < R; ++r) scratch[r] *= row[r];
            }
            float *o = out + (size_t)coord[mode] * stride;
            for (uint32_t r = 0; r < R; ++r) o[r] += scratch[r];
        }
    }
    free(scratch);
}

/* ------------------------------------------------------------------------ */
/* COO -> HiCOO                                                              */
/* ------------------------------------------------------------------------ */

/* 3-D Morton key of src/sptensor/sort.c:1041-1098.  Per byte j of the three
 * coordinates, bit i of z goes to 3i, of y to 3i+1, of x to 3i+2 (a 24-bit
 * group); the groups of bytes 0,1,2 sit at bit offsets 0, 24 and 72 of a
 * 128-bit key, and byte 3 is shifted out of the key entirely. */
static uint32_t spread3_byte(uint32_t b)
{
    uint32_t r = 0;
    for (int i = 0; i < 8; ++i) r |= ((b >> i) & 1u) << (3 * i);
    return r;
}
static u128 morton3(uint32_t x, uint32_t y, uint32_t z)
{
    static const int offs[3] = {0, 24, 72};
    u128 key = 0;
    for (int j = 0; j < 3; ++j) {
        uint32_t g = spread3_byte((z >> (8 * j)) & 0xFF) |
                     (spread3_byte((y >> (8 * j)) & 0xFF) << 1) |
                     (spread3_byte((x >> (8 * j)) & 0xFF) << 2);
        key |= (u128)g << offs[j];
    }
    return key;
}
/* 4-D Morton key of src/sptensor/sort.c:1109-1288: bit i of w, z, y, x goes
 * to 4i, 4i+1, 4i+2, 4i+3 over all 32 bits. */
static u128 morton4(uint32_t x, uint32_t y, uint32_t z, uint32_t w)
{
    u128 key = 0;
    for (int i = 0; i < 32; ++i) {
        key |= (u128)((w >> i) & 1u) << (4 * i);
        key |= (u128)((z >> i) & 1u) << (4 * i + 1);
        key |= (u128)((y >> i) & 1u) << (4 * i + 2);
        key |= (u128)((x >> i) & 1u) << (4 * i + 3);
    }
    return key;
}

typedef struct {
    uint32_t nmodes;
    uint8_t sk_bits;
    const uint32_t *const *inds;
    u128 *mkey;
} sort_ctx;
static sort_ctx g_ctx;

/* Order: kernel coordinates (ind >> sk_bits) lexicographically over modes
 * 0..N-1 (sort.c:929-953), then the Morton key (sort.c:1041-1288), then input
 * position (tie-break, see orc.h). */
static int cmp_hicoo(const void *pa, const void *pb)
{
    uint64_t a = *(const uint64_t *)pa, b = *(const uint64_t *)pb;
    for (uint32_t m = 0; m < g_ctx.nmodes; ++m) {
        uint32_t ka = g_ctx.inds[m][a] >> g_ctx.sk_bits, kb = g_ctx.inds[m][b] >> g_ctx.sk_bits;
        if (ka != kb) return ka < kb ? -1 : 1;
    }
    if (g_ctx.mkey[a] != g_ctx.mkey[b]) return g_ctx.mkey[a] < g_ctx.mkey[b] ? -1 : 1;
    return a < b ? -1 : (a > b);
}

struct orc_hicoo {
    uint32_t nmodes;
    uint64_t nnz, nb, nk, nc, max_nnzb;
    uint8_t sb_bits, sk_bits, sc_bits;
    uint64_t *perm;
    uint64_t *bptr;      /* nb+1 */
    uint32_t *binds;     /* nmodes*nb */
    uint8_t *einds;      /* nmodes*nnz */
    float *vals;
    uint64_t *kptr;      /* nk+1 (block indices) */
    uint64_t *cptr;      /* nc */
    uint64_t *knnzs;     /* nk */
    uint32_t *nkiters;   /* nmodes */
    uint32_t *kschr;     /* flattened lists */
    uint64_t *kschr_rowptr;
    uint64_t kschr_total, kschr_rows;
};

orc_hicoo *orc_hicoo_build(uint32_t nmodes, const uint32_t *ndims, uint64_t nnz,
                           const uint32_t *const *inds, const float *vals,
                           uint8_t sb_bits, uint8_t sk_bits, uint8_t sc_bits)
{
    if (nmodes < 3 || nmodes > 4 || nnz == 0) return NULL;
    orc_hicoo *h = (orc_hicoo *)calloc(1, sizeof(orc_hicoo));
    h->nmodes = nmodes; h->nnz = nnz;
    h->sb_bits = sb_bits; h->sk_bits = sk_bits; h->sc_bits = sc_bits;

    /* sort (convert.c:454 row-block sort + :585-596 Morton sort per kernel) */
    u128 *mkey = (u128 *)malloc(nnz * sizeof(u128));
    for (uint64_t z = 0; z < nnz; ++z)
        mkey[z] = nmodes == 3 ? morton3(inds[0][z], inds[1][z], inds[2][z])
                              : morton4(inds[0][z], inds[1][z], inds[2][z], inds[3][z]);
    h->perm = (uint64_t *)malloc(nnz * sizeof(uint64_t));
    for (uint64_t z = 0; z < nnz; ++z) h->perm[z] = z;
    g_ctx.nmodes = nmodes; g_ctx.sk_bits = sk_bits; g_ctx.inds = inds; g_ctx.mkey = mkey;
    qsort(h->perm, nnz, sizeof(uint64_t), cmp_hicoo);
    free(mkey);

    uint32_t *s[8];
    for (uint32_t m = 0; m < nmodes; ++m) {
        s[m] = (uint32_t *)malloc(nnz * sizeof(uint32_t));
        for (uint64_t z = 0; z < nnz; ++z) s[m][z] = inds[m][h->perm[z]];
    }

    /* kernel pointers over nonzeros (convert.c:314-369) */
    uint64_t *kz = (uint64_t *)malloc((nnz + 1) * sizeof(uint64_t));
    uint64_t nk = 0;
    kz[nk++] = 0;
    for (uint64_t z = 1; z < nnz; ++z) {
        int diff = 0;
        for (uint32_t m = 0; m < nmodes; ++m)
            if ((s[m][z] >> sk_bits) != (s[m][z - 1] >> sk_bits)) diff = 1;
        if (diff) kz[nk++] = z;
    }
    kz[nk] = nnz;
    h->nk = nk;
    h->knnzs = (uint64_t *)malloc(nk * sizeof(uint64_t));
    for (uint64_t k = 0; k < nk; ++k) h->knnzs[k] = kz[k + 1] - kz[k];

    /* kernel scheduler (convert.c:378-421): kschr[m][ind>>sk] lists kernels */
    uint32_t sk = 1u << sk_bits;
    h->kschr_rows = 0;
    uint64_t rowbase[8];
    for (uint32_t m = 0; m < nmodes; ++m) {
        rowbase[m] = h->kschr_rows;
        h->kschr_rows += (ndims[m] + sk - 1) / sk;
    }
    h->kschr_rowptr = (uint64_t *)calloc(h->kschr_rows + 1, sizeof(uint64_t));
    for (uint64_t k = 0; k < nk; ++k)
        for (uint32_t m = 0; m < nmodes; ++m)
            h->kschr_rowptr[rowbase[m] + (s[m][kz[k]] >> sk_bits) + 1]++;
    for (uint64_t r = 0; r < h->kschr_rows; ++r) h->kschr_rowptr[r + 1] += h->kschr_rowptr[r];
    h->kschr_total = h->kschr_rowptr[h->kschr_rows];
    h->kschr = (uint32_t *)malloc((h->kschr_total ? h->kschr_total : 1) * sizeof(uint32_t));
    uint64_t *fill = (uint64_t *)malloc((h->kschr_rows + 1) * sizeof(uint64_t));
    memcpy(fill, h->kschr_rowptr, (h->kschr_rows + 1) * sizeof(uint64_t));
    for (uint64_t k = 0; k < nk; ++k)
        for (uint32_t m = 0; m < nmodes; ++m)
            h->kschr[fill[rowbase[m] + (s[m][kz[k]] >> sk_bits)]++] = (uint32_t)k;
    free(fill);
    h->nkiters = (uint32_t *)calloc(nmodes, sizeof(uint32_t));
    for (uint32_t m = 0; m < nmodes; ++m) {
        uint64_t rows = (ndims[m] + sk - 1) / sk;
        for (uint64_t i = 0; i < rows; ++i) {
            uint64_t len = h->kschr_rowptr[rowbase[m] + i + 1] - h->kschr_rowptr[rowbase[m] + i];
            if (len > h->nkiters[m]) h->nkiters[m] = (uint32_t)len;
        }
    }

    /* single pass over sorted nonzeros (convert.c:718-846) */
    uint64_t sc = (uint64_t)1 << sc_bits;
    h->bptr = (uint64_t *)malloc((nnz + 1) * sizeof(uint64_t));
    uint32_t *bi = (uint32_t *)malloc((size_t)nmodes * nnz * sizeof(uint32_t));
    h->einds = (uint8_t *)malloc((size_t)nmodes * nnz);
    h->vals = (float *)malloc(nnz * sizeof(float));
    h->kptr = (uint64_t *)malloc((nk + 1) * sizeof(uint64_t));
    h->cptr = (uint64_t *)malloc((2 * nnz + 2) * sizeof(uint64_t));
    uint64_t nb = 1, ne = 0, nc = 0;
    uint32_t chunk_size = 0;
    uint32_t prior[8];
    for (uint32_t m = 0; m < nmodes; ++m) { prior[m] = s[m][0] >> sb_bits; bi[m * nnz + 0] = prior[m]; }
    uint64_t nbp = 0;
    h->bptr[nbp++] = 0;
    for (uint64_t k = 0; k < nk; ++k) {
        uint64_t nb_tmp = k == 0 ? 0 : nb;
        h->kptr[k] = nb_tmp;
        h->cptr[nc++] = nb_tmp;
        chunk_size = 0;
        for (uint64_t z = kz[k]; z < kz[k + 1]; ++z) {
            uint32_t blk[8];
            int same = 1;
            for (uint32_t m = 0; m < nmodes; ++m) {
                blk[m] = s[m][z] >> sb_bits;
                h->einds[m * nnz + z] = (uint8_t)(s[m][z] - (blk[m] << sb_bits));
                if (blk[m] != prior[m]) same = 0;
            }
            h->vals[z] = vals[h->perm[z]];
            if (same) {
                ++ne;
            } else {
                h->bptr[nbp++] = (uint32_t)z; /* the reference casts to ptiBlockIndex */
                for (uint32_t m = 0; m < nmodes; ++m) { bi[m * nnz + nb] = blk[m]; prior[m] = blk[m]; }
                if (chunk_size + ne >= sc) {
                    h->cptr[nc++] = nb;
                    chunk_size = 0;
                } else {
                    chunk_size += (uint32_t)ne;
                }
                ++nb;
                ne = 1;
            }
        }
    }
    h->kptr[nk] = nbp;
    h->cptr[nc++] = nbp;
    h->bptr[nbp++] = nnz;
    h->nb = nb; h->nc = nc;
    h->binds = (uint32_t *)malloc((size_t)nmodes * nb * sizeof(uint32_t));
    for (uint32_t m = 0; m < nmodes; ++m)
        memcpy(h->binds + (size_t)m * nb, bi + (size_t)m * nnz, nb * sizeof(uint32_t));
    free(bi);
    h->max_nnzb = h->bptr[1] - h->bptr[0];
    for (uint64_t b = 0; b < nb; ++b)
        if (h->bptr[b + 1] - h->bptr[b] > h->max_nnzb) h->max_nnzb = h->bptr[b + 1] - h->bptr[b];
    for (uint32_t m = 0; m < nmodes; ++m) free(s[m]);
    free(kz);
    return h;
}

void orc_hicoo_counts(const orc_hicoo *h, uint64_t counts[5])
{
    counts[0] = h->nb; counts[1] = h->nk; counts[2] = h->nc;
    counts[3] = h->max_nnzb; counts[4] = h->kschr_total;
}

void orc_hicoo_export(const orc_hicoo *h, uint64_t *bptr, uint32_t *const *binds,
                      uint8_t *const *einds, float *vals, uint64_t *kptr, uint64_t *cptr,
                      uint64_t *knnzs, uint64_t *perm, uint32_t *nkiters,
                      uint32_t *kschr_flat, uint64_t *kschr_rowptr)
{
    memcpy(bptr, h->bptr, (h->nb + 1) * sizeof(uint64_t));
    for (uint32_t m = 0; m < h->nmodes; ++m) {
        memcpy(binds[m], h->binds + (size_t)m * h->nb, h->nb * sizeof(uint32_t));
        memcpy(einds[m], h->einds + (size_t)m * h->nnz, h->nnz);
    }
    memcpy(vals, h->vals, h->nnz * sizeof(float));
    memcpy(kptr, h->kptr, (h->nk + 1) * sizeof(uint64_t));
    memcpy(cptr, h->cptr, h->nc * sizeof(uint64_t));
    memcpy(knnzs, h->knnzs, h->nk * sizeof(uint64_t));
    memcpy(perm, h->perm, h->nnz * sizeof(uint64_t));
    memcpy(nkiters, h->nkiters, h->nmodes * sizeof(uint32_t));
    memcpy(kschr_flat, h->kschr, h->kschr_total * sizeof(uint32_t));
    memcpy(kschr_rowptr, h->kschr_rowptr, (h->kschr_rows + 1) * sizeof(uint64_t));
}

void orc_hicoo_free(orc_hicoo *h)
{
    if (!h) return;
    free(h->perm); free(h->bptr); free(h->binds); free(h->einds); free(h->vals);
    free(h->kptr); free(h->cptr); free(h->knnzs); free(h->nkiters); free(h->kschr);
    free(h->kschr_rowptr); free(h);
}

/* ------------------------------------------------------------------------ */
/* CPD-ALS in FP64                                                           */
/* ------------------------------------------------------------------------ */
static void gram(const double *A, uint64_t I, uint32_t R, double *G)
{
    memset(G, 0, (size_t)R * R * sizeof(double));
    for (uint64_t i = 0; i < I; ++i) {
        const double *a = A + i * R;
        for (uint32_t p = 0; p < R; ++p)
            for (uint32_t q = p; q < R; ++q) G[p * R + q] += a[p] * a[q];
    }
    for (uint32_t p = 0; p < R; ++p)
        for (uint32_t q = 0; q < p; ++q) G[p * R + q] = G[q * R + p];
}

/* In-place Cholesky V = L L^T (lower in V).  Returns 0 if SPD. */
static int cholesky(double *V, uint32_t R)
{
    for (uint32_t j = 0; j < R; ++j) {
        double d = V[j * R + j];
        for (uint32_t k = 0; k < j; ++k) d -= V[j * R + k] * V[j * R + k];
        if (!(d > 0.0)) return 1;
        d = sqrt(d);
        V[j * R + j] = d;
        for (uint32_t i = j + 1; i < R; ++i) {
            double s = V[i * R + j];
            for (uint32_t k = 0; k < j; ++k) s -= V[i * R + k] * V[j * R + k];
            V[i * R + j] = s / d;
        }
    }
    return 0;
}

/* Solve x V = b for each row b of B (V symmetric), in place.
 * matrix_solver.c:49-61 (potrf/potrs), fallback :66-80 (gesv). */
static void solve_rows(double *Vin, uint32_t R, double *B, uint64_t I)
{
    double *V = (double *)malloc((size_t)R * R * sizeof(double));
    memcpy(V, Vin, (size_t)R * R * sizeof(double));
    if (cholesky(V, R) == 0) {
        for (uint64_t i = 0; i < I; ++i) {
            double *b = B + i * R;
            for (uint32_t p = 0; p < R; ++p) {          /* L y = b */
                double s = b[p];
                for (uint32_t k = 0; k < p; ++k) s -= V[p * R + k] * b[k];
                b[p] = s / V[p * R + p];
            }
            for (int p = (int)R - 1; p >= 0; --p) {     /* L^T x = y */
                double s = b[p];
                for (uint32_t k = p + 1; k < R; ++k) s -= V[k * R + p] * b[k];
                b[p] = s / V[p * R + p];
            }
        }
    } else {
        /* LU with partial pivoting on V (symmetric, so x V = b <=> V x^T = b^T) */
        memcpy(V, Vin, (size_t)R * R * sizeof(double));
        int *piv = (int *)malloc(R * sizeof(int));
        for (uint32_t j = 0; j < R; ++j) {
            uint32_t p = j;
            for (uint32_t i = j + 1; i < R; ++i)
                if (fabs(V[i * R + j]) > fabs(V[p * R + j])) p = i;
            piv[j] = (int)p;
            if (p != j)
                for (uint32_t k = 0; k < R; ++k) { double t = V[j * R + k]; V[j * R + k] = V[p * R + k]; V[p * R + k] = t; }
            double d = V[j * R + j];
            for (uint32_t i = j + 1; i < R; ++i) {
                double l = d != 0.0 ? V[i * R + j] / d : 0.0;
                V[i * R + j] = l;
                for (uint32_t k = j + 1; k < R; ++k) V[i * R + k] -= l * V[j * R + k];
            }
        }
        for (uint64_t i = 0; i < I; ++i) {
            double *b = B + i * R;
            for (uint32_t j = 0; j < R; ++j)
                if ((uint32_t)piv[j] != j) { double t = b[j]; b[j] = b[piv[j]]; b[piv[j]] = t; }
            for (uint32_t p = 0; p < R; ++p)
                for (uint32_t k = 0; k < p; ++k) b[p] -= V[p * R + k] * b[k];
            for (int p = (int)R - 1; p >= 0; --p) {
                double s = b[p];
                for (uint32_t k = p + 1; k < R; ++k) s -= V[p * R + k] * b[k];
                b[p] = s / V[p * R + p];
            }
        }
        free(piv);
    }
    free(V);
}

double orc_cpd_als_f64(uint32_t nmodes, const uint32_t *ndims, uint64_t nnz,
                       const uint32_t *const *inds, const float *vals, uint32_t R,
                       uint32_t niters, double *const *mats, double *lambda, double *fits)
{
    uint32_t maxI = 0;
    for (uint32_t m = 0; m < nmodes; ++m) if (ndims[m] > maxI) maxI = ndims[m];
    double **ata = (double **)malloc(nmodes * sizeof(double *));
    for (uint32_t m = 0; m < nmodes; ++m) {
        ata[m] = (double *)malloc((size_t)R * R * sizeof(double));
        gram(mats[m], ndims[m], R, ata[m]);                  /* cpd.c:65-72 */
    }
    double *M = (double *)malloc((size_t)maxI * R * sizeof(double));
    double *V = (double *)malloc((size_t)R * R * sizeof(double));
    double normX2 = 0;
    for (uint64_t z = 0; z < nnz; ++z) normX2 += (double)vals[z] * vals[z];
    double fit = 0;
    for (uint32_t it = 0; it < niters; ++it) {
        for (uint32_t m = 0; m < nmodes; ++m) {
            orc_mttkrp_coo_f64(nmodes, nnz, inds, vals, (const double *const *)mats, R, R, m,
                               ndims[m], M);                /* cpd.c:101 */
            memcpy(mats[m], M, (size_t)ndims[m] * R * sizeof(double));
            for (uint32_t x = 0; x < R * R; ++x) V[x] = 1.0;  /* matrix.c:340-385 */
            for (uint32_t k = 1; k < nmodes; ++k) {
                uint32_t pm = (m + k) % nmodes;
                for (uint32_t x = 0; x < R * R; ++x) V[x] *= ata[pm][x];
            }
            solve_rows(V, R, mats[m], ndims[m]);           /* cpd.c:109 */
            double *A = mats[m];
            if (it == 0) {                                  /* matrix.c:389-469 */
                for (uint32_t r = 0; r < R; ++r) lambda[r] = 0;
                for (uint64_t i = 0; i < ndims[m]; ++i)
                    for (uint32_t r = 0; r < R; ++r) lambda[r] += A[i * R + r] * A[i * R + r];
                for (uint32_t r = 0; r < R; ++r) lambda[r] = sqrt(lambda[r]);
            } else {                                        /* matrix.c:472-553 */
                for (uint32_t r = 0; r < R; ++r) lambda[r] = 0;
                for (uint64_t i = 0; i < ndims[m]; ++i)
                    for (uint32_t r = 0; r < R; ++r)
                        if (A[i * R + r] > lambda[r]) lambda[r] = A[i * R + r];
                for (uint32_t r = 0; r < R; ++r) if (lambda[r] < 1) lambda[r] = 1;
            }
            for (uint64_t i = 0; i < ndims[m]; ++i)
                for (uint32_t r = 0; r < R; ++r) A[i * R + r] /= lambda[r];
            gram(A, ndims[m], R, ata[m]);                   /* cpd.c:128 */
        }
        /* fit: ktensor.c:77-240 */
        for (uint32_t x = 0; x < R * R; ++x) V[x] = 1.0;
        for (uint32_t k = 0; k < nmodes; ++k)
            for (uint32_t x = 0; x < R * R; ++x) V[x] *= ata[k][x];
        double norm_mats = 0;
        for (uint32_t p = 0; p < R; ++p)
            for (uint32_t q = 0; q < R; ++q) norm_mats += V[p * R + q] * lambda[p] * lambda[q];
        norm_mats = fabs(norm_mats);
        uint32_t last = nmodes - 1;
        double inner = 0;
        for (uint32_t r = 0; r < R; ++r) {
            double acc = 0;
            for (uint64_t i = 0; i < ndims[last]; ++i) acc += mats[last][i * R + r] * M[i * R + r];
            inner += acc * lambda[r];
        }
        double residual = normX2 + norm_mats - 2 * inner;
        if (residual > 0.0) residual = sqrt(residual);
        fit = 1 - residual / sqrt(normX2);
        if (fits) fits[it] = fit;
    }
    /* GetFinalLambda: matrix.c:556-572 */
    for (uint32_t m = 0; m < nmodes; ++m) {
        double *A = mats[m];
        for (uint32_t r = 0; r < R; ++r) {
            double s = 0;
            for (uint64_t i = 0; i < ndims[m]; ++i) s += A[i * R + r] * A[i * R + r];
            s = sqrt(s);
            for (uint64_t i = 0; i < ndims[m]; ++i) A[i * R + r] /= s;
            lambda[r] *= s;
        }
    }
    for (uint32_t m = 0; m < nmodes; ++m) free(ata[m]);
    free(ata); free(M); free(V);
    return fit;
}

double orc_kruskal_fit_f64(uint32_t nmodes, const uint32_t *ndims, uint64_t nnz,
                           const uint32_t *const *inds, const float *vals, uint32_t R,
                           const double *const *mats, const double *lambda)
{
    double *V = (double *)malloc((size_t)R * R * sizeof(double));
    double *G = (double *)malloc((size_t)R * R * sizeof(double));
    for (uint32_t x = 0; x < R * R; ++x) V[x] = 1.0;
    for (uint32_t m = 0; m < nmodes; ++m) {
        gram(mats[m], ndims[m], R, G);
        for (uint32_t x = 0; x < R * R; ++x) V[x] *= G[x];
    }
    double norm_mats = 0;
    for (uint32_t p = 0; p < R; ++p)
        for (uint32_t q = 0; q < R; ++q) norm_mats += V[p * R + q] * lambda[p] * lambda[q];
    double normX2 = 0, inner = 0;
#pragma omp parallel for reduction(+ : normX2, inner) schedule(static)
    for (uint64_t z = 0; z < nnz; ++z) {
        double model = 0;
        for (uint32_t r = 0; r < R; ++r) {
            double p = lambda[r];
            for (uint32_t m = 0; m < nmodes; ++m) p *= mats[m][(size_t)inds[m][z] * R + r];
            model += p;
        }
        normX2 += (double)vals[z] * vals[z];
        inner += (double)vals[z] * model;
    }
    free(V); free(G);
    double residual = normX2 + fabs(norm_mats) - 2 * inner;
    if (residual > 0.0) residual = sqrt(residual);
    return 1 - residual / sqrt(normX2);
}
