/*
 * orc.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the reference algorithms on the MTTKRP / CPD-ALS path,
 * used as the checker for the GPU library.  Only tests/, the smoke check and
 * the bench's CPU-baseline leg may load it.  The product library never links,
 * calls or falls back to anything in this directory.
 *
 * Every function cites the reference file and lines it restates.  All arrays
 * are plain pointers so the functions can be driven from numpy via ctypes.
 */
#ifndef ORC_H
#define ORC_H
#include <stdint.h>

/* MTTKRP on a COO tensor in FP32, restating src/sptensor/mttkrp.c:39-163:
 * out[i_mode, r] = sum_z v_z * prod_{k=1..N-1} A_{order[k]}[i_order[k], r],
 * products taken left to right in mats_order[1..N-1] order, accumulation in
 * nonzero order.  inds is nmodes pointers of nnz uint32; mats is nmodes
 * pointers of row-major (ndims[k] x stride) floats; out is out_rows x stride
 * and is zeroed first (pad columns included). */
void orc_mttkrp_coo_f32(uint32_t nmodes, uint64_t nnz, const uint32_t *const *inds,
                        const float *vals, const float *const *mats, uint32_t R,
                        uint32_t stride, const uint32_t *mats_order, uint32_t mode,
                        uint32_t out_rows, float *out);

/* Same contraction with FP64 accumulation and FP64 factors (error bounds). */
void orc_mttkrp_coo_f64(uint32_t nmodes, uint64_t nnz, const uint32_t *const *inds,
                        const float *vals, const double *const *mats, uint32_t R,
                        uint32_t stride, uint32_t mode, uint32_t out_rows, double *out);

/* MTTKRP on a HiCOO tensor in FP32, restating src/sptensor/hicoo/mttkrp.c:61-152
 * (general order) and :232-310 (3-D blocked): iterate kernels -> blocks ->
 * nonzeros; coordinate = (binds << sb_bits) + einds. */
void orc_mttkrp_hicoo_f32(uint32_t nmodes, uint64_t nnz, uint64_t nb, uint8_t sb_bits,
                          const uint64_t *bptr, const uint32_t *const *binds,
                          const uint8_t *const *einds, const float *vals,
                          const float *const *mats, uint32_t R, uint32_t stride,
                          const uint32_t *mats_order, uint32_t mode, uint32_t out_rows,
                          float *out);

/* COO -> HiCOO, restating src/sptensor/hicoo/convert.c:314-421 (kernel
 * pointers, kernel scheduler), :430-604 (row-block sort, Morton sort inside
 * each kernel) and :646-860 (block, chunk and kernel pointers), with the sort
 * keys of src/sptensor/sort.c:929-953 (row-block), :1041-1098 (3-D Morton,
 * including its treatment of coordinate bits >= 24) and :1109-1288 (4-D Morton).
 * The reference quicksorts are unstable; for unique coordinates the keys are
 * unique and the order is fully determined.  Ties (duplicates, or 3-D
 * coordinates equal modulo 2^24) are broken by input position here.
 *
 * Phase 1 (orc_hicoo_build) sorts and counts; phase 2 copies the arrays out. */
typedef struct orc_hicoo orc_hicoo;
orc_hicoo *orc_hicoo_build(uint32_t nmodes, const uint32_t *ndims, uint64_t nnz,
                           const uint32_t *const *inds, const float *vals,
                           uint8_t sb_bits, uint8_t sk_bits, uint8_t sc_bits);
/* counts: [nb, nk, nc, max_nnzb, total kschr entries over all modes] */
void orc_hicoo_counts(const orc_hicoo *h, uint64_t counts[5]);
/* perm[z] = input position of the z-th nonzero in HiCOO order. */
void orc_hicoo_export(const orc_hicoo *h, uint64_t *bptr, uint32_t *const *binds,
                      uint8_t *const *einds, float *vals, uint64_t *kptr, uint64_t *cptr,
                      uint64_t *knnzs, uint64_t *perm, uint32_t *nkiters,
                      uint32_t *kschr_flat, uint64_t *kschr_rowptr);
void orc_hicoo_free(orc_hicoo *h);

/* FP64 CPD-ALS restating src/sptensor/cpd.c:32-160 with
 * src/matrix/matrix_solver.c:32-83 (normal equations against the Hadamard
 * product of the other modes' Grams; Cholesky, LU with partial pivoting if the
 * Gram is not SPD), src/matrix/matrix.c:389-572 (2-norm at iteration 0, then
 * max-norm clamped to >= 1; final lambda) and src/ktensor/ktensor.c:77-240
 * (fit from the Grams, the last MTTKRP and the last factor).  The Gram Hadamard
 * product in the fit uses the full symmetric Grams.
 * mats[k]: ndims[k] x R row-major doubles (stride R), in/out.  lambda: R out.
 * fits: niters out (fit after each iteration).  Returns the final fit. */
double orc_cpd_als_f64(uint32_t nmodes, const uint32_t *ndims, uint64_t nnz,
                       const uint32_t *const *inds, const float *vals, uint32_t R,
                       uint32_t niters, double *const *mats, double *lambda, double *fits);

/* Fit of a Kruskal model [[lambda; A_0..A_{N-1}]] to the sparse tensor,
 * computed directly: 1 - ||X - M|| / ||X|| with ||M||^2 from the Grams and
 * <X, M> by evaluating the model at every nonzero (FP64). */
double orc_kruskal_fit_f64(uint32_t nmodes, const uint32_t *ndims, uint64_t nnz,
                           const uint32_t *const *inds, const float *vals, uint32_t R,
                           const double *const *mats, const double *lambda);

#endif
