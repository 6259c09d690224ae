/*
 * hiparti_b200.h -- C ABI of the B200 (sm_100a) implementation of HiParTI's
 * sparse MTTKRP / CPD-ALS path.
 *
 * The types, struct layouts and function signatures below are byte- and
 * call-compatible with the reference headers, so a C program written against
 * HiParTI's MTTKRP/CPD entry points links against libhiparti_b200.so instead of
 * libHiParTI.so without source changes.  Every reference entry point declared
 * here runs its arithmetic on the GPU; there is no CPU fallback.  Functions
 * whose names start with ptiB200 are extensions with no reference counterpart:
 * they keep tensors and factor matrices resident in device memory.
 *
 * Citations are to files of the reference project (pnnl/HiParTI).
 */
#ifndef HIPARTI_B200_H
#define HIPARTI_B200_H

#include <stdint.h>
#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

/* ---------------------------------------------------------------------------
 * Scalar types: include/includes/types.h:27-98 (32-bit indices, FP32 values,
 * 8-bit element indices, 64-bit nonzero counters).
 * ------------------------------------------------------------------------ */
typedef uint32_t ptiIndex;
typedef uint32_t ptiBlockIndex;
typedef float    ptiValue;
typedef uint8_t  ptiElementIndex;
typedef uint16_t ptiBlockMatrixIndex;
typedef ptiBlockIndex ptiBlockNnzIndex;
typedef uint64_t ptiNnzIndex;

/* Error codes: include/includes/macros.h:47-56. */
typedef enum {
    PTIERR_NO_ERROR       = 0,
    PTIERR_UNKNOWN        = 1,
    PTIERR_SHAPE_MISMATCH = 2,
    PTIERR_VALUE_ERROR    = 3,
    PTIERR_ZERO_DIVISION  = 4,
    PTIERR_NO_MORE        = 99,
    PTIERR_OS_ERROR       = 0x10000,
    PTIERR_CUDA_ERROR     = 0x20000
} PtiError;

/* ---------------------------------------------------------------------------
 * Containers: include/includes/structs.h:27-56 (vectors), :64-82 (matrices),
 * :142-149 (COO tensor), :155-185 (HiCOO tensor), :254-271 (Kruskal tensors).
 * ------------------------------------------------------------------------ */
typedef struct { ptiNnzIndex len; ptiNnzIndex cap; ptiValue        *data; } ptiValueVector;
typedef struct { ptiNnzIndex len; ptiNnzIndex cap; ptiIndex        *data; } ptiIndexVector;
typedef struct { ptiNnzIndex len; ptiNnzIndex cap; ptiElementIndex *data; } ptiElementIndexVector;
typedef struct { ptiNnzIndex len; ptiNnzIndex cap; ptiBlockIndex   *data; } ptiBlockIndexVector;
typedef struct { ptiNnzIndex len; ptiNnzIndex cap; ptiNnzIndex     *data; } ptiNnzIndexVector;

/* Row-major dense matrix; stride = ncols rounded up to a multiple of 8. */
typedef struct {
    ptiIndex nrows;
    ptiIndex ncols;
    ptiIndex cap;
    ptiIndex stride;
    ptiValue *values;
} ptiMatrix;

/* Dense matrix with a small rank (ncols and stride are 8-bit). */
typedef struct {
    ptiIndex        nrows;
    ptiElementIndex ncols;
    ptiIndex        cap;
    ptiElementIndex stride;
    ptiValue        *values;
} ptiRankMatrix;

/* Coordinate (COO) sparse tensor, indices stored per mode. */
typedef struct {
    ptiIndex nmodes;
    ptiIndex *sortorder;
    ptiIndex *ndims;
    ptiNnzIndex nnz;
    ptiIndexVector *inds;
    ptiValueVector values;
} ptiSparseTensor;

/* Hierarchical COO (HiCOO) sparse tensor. */
typedef struct {
    ptiIndex    nmodes;
    ptiIndex    *sortorder;
    ptiIndex    *ndims;
    ptiNnzIndex nnz;
    ptiElementIndex sb_bits;      /* block edge = 2^sb_bits            */
    ptiElementIndex sk_bits;      /* kernel (super-block) edge = 2^sk  */
    ptiElementIndex sc_bits;      /* chunk size in nonzeros = 2^sc     */
    ptiNnzIndexVector kptr;       /* first block of each kernel, + nb  */
    ptiIndexVector  **kschr;      /* [mode][kernel row] -> kernel ids  */
    ptiIndex        *nkiters;     /* [mode] longest kschr list         */
    ptiNnzIndexVector cptr;       /* chunk pointers over blocks        */
    ptiIndexVector  **kschr_balanced;
    ptiIndexVector  **kschr_balanced_pos;
    ptiIndex        *nkpars;
    ptiIndexVector  *kschr_rest;
    ptiNnzIndexVector knnzs;      /* nonzeros of each kernel           */
    ptiNnzIndexVector bptr;       /* nb+1 nonzero offsets of blocks    */
    ptiBlockIndexVector   *binds; /* [mode] block coordinates, nb each */
    ptiElementIndexVector *einds; /* [mode] in-block offsets, nnz each */
    ptiValueVector values;
} ptiSparseTensorHiCOO;

typedef struct {
    ptiIndex nmodes;
    ptiIndex rank;
    ptiIndex *ndims;
    ptiValue *lambda;
    double fit;
    ptiMatrix **factors;
} ptiKruskalTensor;

typedef struct {
    ptiIndex nmodes;
    ptiElementIndex rank;
    ptiIndex *ndims;
    ptiValue *lambda;
    double fit;
    ptiRankMatrix **factors;
} ptiRankKruskalTensor;

/* Semi-sparse tensor (structs.h:219-233): dense along `mode`, sparse in the
 * other modes -- a sparse tensor of dense fibers.  inds[mode] is empty. */
typedef struct {
    ptiIndex nmodes;
    ptiIndex *ndims;
    ptiIndex mode;
    ptiNnzIndex nnz;           /* fibers */
    ptiIndexVector *inds;      /* [nmodes][nnz] fiber coordinates      */
    ptiIndex stride;           /* ndims[mode] rounded up to 8          */
    ptiMatrix values;          /* nnz x stride                         */
} ptiSemiSparseTensor;

/* ---------------------------------------------------------------------------
 * Error reporting: include/includes/helper_funcs.h:29-30,39-40.
 * A failing call records (module, file, line, reason) in a thread-local slot
 * and returns the code; ptiGetLastError returns that code and the strings.
 * ------------------------------------------------------------------------ */
int  ptiGetLastError(const char **module, const char **file, unsigned *line, const char **reason);
void ptiClearLastError(void);
int  ptiCudaSetDevice(int device);
int  ptiCudaGetLastError(void);

/* ---------------------------------------------------------------------------
 * Container life cycle.
 * ------------------------------------------------------------------------ */
/* include/includes/sptensors.h:23-25 */
int  ptiNewSparseTensor(ptiSparseTensor *tsr, ptiIndex nmodes, const ptiIndex ndims[]);
void ptiFreeSparseTensor(ptiSparseTensor *tsr);
/* include/includes/sptensors.h:26 (sum of squared values, FP64 accumulation; GPU) */
double SparseTensorFrobeniusNormSquared(ptiSparseTensor const * const ptien);
/* include/includes/sptensors.h:27 -- text .tns (header "N\nI_0 ... I_{N-1}")
 * or SPLATT .bin, selected by file extension as in src/sptensor/load.c:277-297.
 * The file is parsed on the GPU (see ptiB200LoadSparseTensor); the nonzeros,
 * their order and their values are those of the reference's fscanf reader. */
int  ptiLoadSparseTensor(ptiSparseTensor *tsr, ptiIndex start_index, char const * const fname);

/* include/includes/sptensors.h:100, src/sptensor/renumber.c:26-92;
 * newIndices[m][old] = new.  tsr is not modified.  renumber == 1: Lexi-order
 * on the GPU, `iterations` passes; impl_num 0, 1 or 2 (2 compares block
 * indices before indices, which orders coordinates the same way).
 * renumber == 2: BFS-like (renumber.c:534-839): the vertex lists are built on
 * the GPU and the heap walk runs on the host; every vertex starts unvisited
 * (the reference reads those marks uninitialised, renumber.c:768, so its own
 * output varies from call to call).  sb_bits and tk are unused.  Other
 * choices record PTIERR_VALUE_ERROR (see ptiGetLastError) and leave the
 * identity in newIndices. */
void ptiIndexRenumber(ptiSparseTensor * tsr, ptiIndex ** newIndices, int renumber, ptiIndex iterations,
                      ptiElementIndex sb_bits, int tk, int impl_num);
/* include/includes/sptensors.h:101, src/sptensor/orderit.c:121-208 -- the same
 * Lexi-order (renumber 1) or BFS-like (renumber 2).  (For impl_num 0 and 1 the
 * reference's ptiIndexRenumber sorts the nonzeros with a defective insertion
 * sort and so depends on their order; both entry points here give orderit's
 * result.) */
void orderit(ptiSparseTensor *tsr, ptiIndex **newIndices, int const renumber, ptiIndex const iterations);
/* include/includes/sptensors.h:45 -- coordinates replaced by map_inds[m][old] */
void ptiSparseTensorShuffleIndices(ptiSparseTensor *tsr, ptiIndex ** map_inds);

/* include/includes/matrices.h:26-34 */
int  ptiNewMatrix(ptiMatrix *mtx, ptiIndex const nrows, ptiIndex const ncols);
int  ptiRandomizeMatrix(ptiMatrix *mtx);           /* A[i,j] = i+j+1, src/matrix/matrix.c:67-74 */
int  ptiConstantMatrix(ptiMatrix * const mtx, ptiValue const val);
void ptiFreeMatrix(ptiMatrix *mtx);

/* include/includes/matrices.h:30, ktensors.h:24 -- row i becomes row map[i]
 * (factors of a renumbered tensor back in the original numbering) */
void ptiMatrixInverseShuffleIndices(ptiMatrix *mtx, ptiIndex * mode_map_inds);
void ptiKruskalTensorInverseShuffleIndices(ptiKruskalTensor * ktsr, ptiIndex ** map_inds);

/* include/includes/ktensors.h:23-25 */
int  ptiNewKruskalTensor(ptiKruskalTensor *ktsr, ptiIndex nmodes, const ptiIndex ndims[], ptiIndex rank);
void ptiFreeKruskalTensor(ptiKruskalTensor *ktsr);
int  ptiNewRankKruskalTensor(ptiRankKruskalTensor *ktsr, ptiIndex nmodes, const ptiIndex ndims[], ptiElementIndex rank);
void ptiFreeRankKruskalTensor(ptiRankKruskalTensor *ktsr);
/* include/includes/matrices.h:66,73 */
int  ptiNewRankMatrix(ptiRankMatrix *mtx, ptiIndex const nrows, ptiElementIndex const ncols);
void ptiFreeRankMatrix(ptiRankMatrix *mtx);

/* Text dumps in the reference's format: include/includes/matrices.h:35,74
 * (src/matrix/dump.c:33-75: "<rows> x <cols> matrix", then rows of "%.2f\t")
 * and include/includes/ktensors.h:26,46 (src/ktensor/dump.c:23-88: sizes,
 * "fit: ", "lambda:", "Factor matrices:").  Host only. */
int ptiDumpMatrix(ptiMatrix *mtx, FILE *fp);
int ptiDumpRankMatrix(ptiRankMatrix *mtx, FILE *fp);
int ptiDumpKruskalTensor(ptiKruskalTensor *ktsr, FILE *fp);
int ptiDumpRankKruskalTensor(ptiRankKruskalTensor *ktsr, FILE *fp);

/* include/includes/sptensors.h:104-119 */
int  ptiNewSparseTensorHiCOO(ptiSparseTensorHiCOO *hitsr, const ptiIndex nmodes, const ptiIndex ndims[],
                             const ptiNnzIndex nnz, const ptiElementIndex sb_bits,
                             const ptiElementIndex sk_bits, const ptiElementIndex sc_bits);
void ptiFreeSparseTensorHiCOO(ptiSparseTensorHiCOO *hitsr);

/* include/includes/sptensors.h:120-127, src/sptensor/hicoo/convert.c:646-860.
 * COO -> HiCOO on the GPU.  Output arrays are bit-identical to the reference
 * for tensors with unique coordinates (3-D: coordinates < 2^24; 4-D: any);
 * as in the reference, the caller's COO tensor is left sorted in HiCOO order
 * (kernels row-major, nonzeros in Morton order inside each kernel).  tk is
 * accepted and ignored.  Only 3-D and 4-D tensors are supported, as in
 * src/sptensor/sort.c:414-430. */
int  ptiSparseTensorToHiCOO(ptiSparseTensorHiCOO *hitsr, ptiNnzIndex *max_nnzb, ptiSparseTensor *tsr,
                            const ptiElementIndex sb_bits, const ptiElementIndex sk_bits,
                            const ptiElementIndex sc_bits, int const tk);

/* ---------------------------------------------------------------------------
 * TTM / TTV along one mode (include/includes/sptensors.h:156-161,
 * src/sptensor/mmul.c:36-86, vmul.c:26-70).  Y must be uninitialised; it is
 * created here (release it with ptiFreeSemiSparseTensor).  As in the
 * reference, X is sorted in place with `mode` last unless its sortorder
 * already says so, and each fiber's sum runs in that order with FP32
 * multiply-then-add, so Y is bit-identical to the reference's for distinct
 * coordinates.  All variants run the same GPU code (impl_num, smen_size
 * ignored); U has at most 256 columns.
 * ------------------------------------------------------------------------ */
int ptiNewSemiSparseTensor(ptiSemiSparseTensor *tsr, ptiIndex nmodes, ptiIndex mode, const ptiIndex ndims[]);
void ptiFreeSemiSparseTensor(ptiSemiSparseTensor *tsr);
int ptiSparseTensorMulMatrix(ptiSemiSparseTensor *Y, ptiSparseTensor * const X, ptiMatrix *const U, ptiIndex mode);
int ptiOmpSparseTensorMulMatrix(ptiSemiSparseTensor *Y, ptiSparseTensor * const X, ptiMatrix * const U,
                                ptiIndex mode);
int ptiCudaSparseTensorMulMatrix(ptiSemiSparseTensor *Y, ptiSparseTensor *X, const ptiMatrix *U, ptiIndex const mode);
int ptiCudaSparseTensorMulMatrixOneKernel(ptiSemiSparseTensor *Y, ptiSparseTensor *X, const ptiMatrix *U,
                                          ptiIndex const mode, ptiIndex const impl_num,
                                          ptiNnzIndex const smen_size);
int ptiSparseTensorMulVector(ptiSemiSparseTensor *Y, ptiSparseTensor * const X, ptiValueVector * const V,
                             ptiIndex mode);
/* include/includes/ssptensors.h:26, src/sptensor/fromssp.c:32-84: the entries
 * of src that are NaN, infinite or normal with |v| >= epsilon, as a sparse
 * tensor sorted lexicographically (dest uninitialised; epsilon >= 0). */
int ptiSemiSparseTensorToSparseTensor(ptiSparseTensor *dest, const ptiSemiSparseTensor *src, ptiValue epsilon);
/* include/includes/ssptensors.h:49-50, src/ssptensor/mmul.c:29-92: a semi-sparse
 * tensor's dense fibers times U (X->ndims[mode] x R): Y[i, k] = sum_r X[i, r] U[r, k]
 * in order, FP32 multiply-then-add (bit-identical); Y uninitialised. */
int ptiSemiSparseTensorMulMatrix(ptiSemiSparseTensor *Y, const ptiSemiSparseTensor *X, const ptiMatrix *U,
                                 ptiIndex mode);
int ptiCudaSemiSparseTensorMulMatrix(ptiSemiSparseTensor *Y, const ptiSemiSparseTensor *X, const ptiMatrix *U,
                                     ptiIndex mode);

/* ---------------------------------------------------------------------------
 * MTTKRP.  mats[0..N-1] are the factor matrices (row i of mats[k] is the rank-R
 * row of index i in mode k); mats[N] receives the result for `mode`
 * (mats[mode]->nrows rows of stride floats; rows are overwritten, pad columns
 * are zeroed).  mats_order[1..N-1] lists the modes multiplied together.
 * All entry points below run on the current CUDA device, copy the host
 * arguments in, and return once mats[N] has been written back.
 * ------------------------------------------------------------------------ */
/* include/includes/sptensors.h:179-183, src/sptensor/mttkrp.c:39-163 */
int ptiMTTKRP(ptiSparseTensor const * const X, ptiMatrix * mats[], ptiIndex const mats_order[],
              ptiIndex const mode);
/* include/includes/sptensors.h:184-189 (tk ignored) */
int ptiOmpMTTKRP(ptiSparseTensor const * const X, ptiMatrix * mats[], ptiIndex const mats_order[],
                 ptiIndex const mode, const int tk);
/* include/includes/sptensors.h:190-196 (copy_mats unused; tk ignored) */
int ptiOmpMTTKRP_Reduce(ptiSparseTensor const * const X, ptiMatrix * mats[], ptiMatrix * copy_mats[],
                        ptiIndex const mats_order[], ptiIndex const mode, const int tk);
/* include/includes/sptensors.h:197-203 (lock_pool accepted and unused: the GPU
 * path privatises rows instead of locking) and the OpenMP lock pool of
 * include/includes/helper_funcs.h:61-65 (opaque here). */
typedef struct ptiMutexPool ptiMutexPool;
ptiMutexPool * ptiMutexAlloc(void);
ptiMutexPool * SptMutexAllocCustom(ptiIndex const num_locks, ptiIndex const pad_size);
void ptiMutexFree(ptiMutexPool * pool);
int ptiOmpMTTKRP_Lock(ptiSparseTensor const * const X, ptiMatrix * mats[], ptiIndex const mats_order[],
                      ptiIndex const mode, const int tk, ptiMutexPool * lock_pool);
/* include/includes/sptensors.h:204-215, src/sptensor/mttkrp_cuda.cu:41-374 and
 * src/sptensor/mttkrp_cuda_onekernel.cu:41-426 (impl_num ignored; any order N). */
int ptiCudaMTTKRP(ptiSparseTensor const * const X, ptiMatrix * mats[], ptiIndex * const mats_order,
                  ptiIndex const mode, ptiIndex const impl_num);
int ptiCudaMTTKRPOneKernel(ptiSparseTensor const * const X, ptiMatrix ** const mats,
                           ptiIndex * const mats_order, ptiIndex const mode, ptiIndex const impl_num);
/* include/includes/sptensors.h:222-233, src/sptensor/mttkrp_cuda.cu:378-434:
 * COO MTTKRP on device arrays.  Xinds (nmodes pointers), dev_mats (nmodes+1
 * pointers) and dev_mats_order (nmodes entries) are device arrays, as are the
 * index, value and factor arrays they point to; Xndims is not read.  The
 * products are ADDED into dev_mats[nmodes] (rows of mode `mode`), which the
 * caller zeroes, as in the reference.  Factors and the output: `stride`
 * floats per row, 16-byte aligned, stride a multiple of 4.  dev_scratch (the
 * reference's nnz x rank staging) is not used and may be NULL.  Synchronous. */
int ptiCudaMTTKRPDevice(const ptiIndex mode, const ptiIndex nmodes, const ptiNnzIndex nnz, const ptiIndex rank,
                        const ptiIndex stride, const ptiIndex * Xndims, ptiIndex ** const Xinds,
                        const ptiValue * Xvals, const ptiIndex * dev_mats_order, ptiValue ** dev_mats,
                        ptiValue * dev_scratch);

/* include/includes/sptensors.h:253-257, src/sptensor/hicoo/mttkrp.c:61-310 */
int ptiMTTKRPHiCOO(ptiSparseTensorHiCOO const * const hitsr, ptiMatrix * mats[],
                   ptiIndex const mats_order[], ptiIndex const mode);
/* include/includes/sptensors.h:263-269 (tk, tb ignored) */
int ptiOmpMTTKRPHiCOO(ptiSparseTensorHiCOO const * const hitsr, ptiMatrix * mats[],
                      ptiIndex const mats_order[], ptiIndex const mode, const int tk, const int tb);
/* include/includes/sptensors.h:302-308, src/sptensor/hicoo/mttkrp_cuda.cu:41-265
 * (max_nnzb and impl_num ignored: no limit on nonzeros per block; any order N). */
/* include/includes/sptensors.h:258-300, src/sptensor/hicoo/mttkrp.c:313-404 and
 * hicoo/mttkrp_omp.c: the same MTTKRP with ptiRankMatrix factors (8-bit ncols and
 * stride).  tk, tb, balanced and copy_mats are accepted and unused. */
int ptiMTTKRPHiCOO_MatrixTiling(ptiSparseTensorHiCOO const * const hitsr, ptiRankMatrix * mats[],
                                ptiIndex const mats_order[], ptiIndex const mode);
int ptiOmpMTTKRPHiCOO_MatrixTiling(ptiSparseTensorHiCOO const * const hitsr, ptiRankMatrix * mats[],
                                   ptiIndex const mats_order[], ptiIndex const mode, const int tk, const int tb);
int ptiOmpMTTKRPHiCOO_MatrixTiling_Scheduled(ptiSparseTensorHiCOO const * const hitsr, ptiRankMatrix * mats[],
                                             ptiIndex const mats_order[], ptiIndex const mode, const int tk,
                                             const int tb, int balanced);
int ptiOmpMTTKRPHiCOO_MatrixTiling_Scheduled_Reduce(ptiSparseTensorHiCOO const * const hitsr,
                                                    ptiRankMatrix * mats[], ptiRankMatrix * copy_mats[],
                                                    ptiIndex const mats_order[], ptiIndex const mode,
                                                    const int tk, const int tb, int balanced);
int ptiOmpMTTKRPHiCOO_MatrixTiling_Scheduled_Reduce_Two(ptiSparseTensorHiCOO const * const hitsr,
                                                        ptiRankMatrix * mats[], ptiRankMatrix * copy_mats[],
                                                        ptiIndex const mats_order[], ptiIndex const mode,
                                                        const int tk, const int tb);
int ptiCudaMTTKRPHiCOO(ptiSparseTensorHiCOO const * const hitsr, ptiMatrix ** const mats,
                       ptiIndex * const mats_order, ptiIndex const mode, ptiNnzIndex const max_nnzb,
                       int const impl_num);

/* ---------------------------------------------------------------------------
 * CPD-ALS: include/includes/cpds.h:26-57, src/sptensor/cpd.c:32-208.
 * The ALS loop runs on the GPU in FP32 factors with FP64 Gram matrices,
 * Cholesky solve and fit.  Factors start from ptiRandomizeMatrix (i+j+1) as in
 * src/sptensor/cpd.c:181-187.  ktensor->lambda must come from
 * ptiNewKruskalTensor; ktensor->factors is allocated here (N+1 pointers,
 * factors[N] released) as in src/sptensor/cpd.c:200-205.
 * ------------------------------------------------------------------------ */
int ptiCpdAls(ptiSparseTensor const * const ptien, ptiIndex const rank, ptiIndex const niters,
              double const tol, ptiKruskalTensor * ktensor);
int ptiOmpCpdAls(ptiSparseTensor const * const ptien, ptiIndex const rank, ptiIndex const niters,
                 double const tol, const int tk, const int use_reduce, ptiKruskalTensor * ktensor);
int ptiCudaCpdAls(ptiSparseTensor const * const ptien, ptiIndex const rank, ptiIndex const niters,
                  double const tol, ptiKruskalTensor * ktensor);
int ptiCpdAlsHiCOO(ptiSparseTensorHiCOO const * const hitsr, ptiIndex const rank, ptiIndex const niters,
                   double const tol, ptiRankKruskalTensor * ktensor);
int ptiOmpCpdAlsHiCOO(ptiSparseTensorHiCOO const * const hitsr, ptiIndex const rank,
                      ptiIndex const niters, double const tol, const int tk, const int tb,
                      int balanced, ptiRankKruskalTensor * ktensor);

/* The ALS step on caller-initialised factors: src/sptensor/cpd.c:32-160
 * (CpdAlsStep), cpd_omp.c:32-178 (OmpCpdAlsStep), hicoo/cpd.c:31 and
 * hicoo/cpd_omp.c:32-202 (HiCOO twins).  The reference exports these without
 * declaring them in its headers.  mats[0..N-1] (ndims[m] x rank, one stride,
 * a multiple of 8) hold the initial factors and receive the result (columns
 * of unit 2-norm, GetFinalLambda applied); lambda (rank floats) receives the
 * weights; mats[N] (at least ndims[N-1] rows of that stride) receives the
 * last MTTKRP output (mode N-1 of the last iteration), as the reference
 * leaves it.  Runs the loop of ptiCpdAls on the GPU (tol as in cpd.c:144;
 * tk, tb, use_reduce, par_iters, balanced and copy_mats are unused).  Returns
 * the last iteration's fit, computed from the full symmetric Grams (see
 * KruskalTensorFit); NaN on bad arguments, with the last error set. */
double CpdAlsStep(ptiSparseTensor const * const ptien, ptiIndex const rank, ptiIndex const niters,
                  double const tol, ptiMatrix ** mats, ptiValue * const lambda);
double OmpCpdAlsStep(ptiSparseTensor const * const ptien, ptiIndex const rank, ptiIndex const niters,
                     double const tol, const int tk, const int use_reduce, ptiMatrix ** mats,
                     ptiMatrix ** copy_mats, ptiValue * const lambda);
double CpdAlsStepHiCOO(ptiSparseTensorHiCOO const * const hitsr, ptiIndex const rank, ptiIndex const niters,
                       double const tol, ptiRankMatrix ** mats, ptiValue * const lambda);
double OmpCpdAlsStepHiCOO(ptiSparseTensorHiCOO const * const hitsr, ptiIndex const rank,
                          ptiIndex const niters, double const tol, const int tk, const int tb,
                          const int * par_iters, ptiRankMatrix ** mats, ptiRankMatrix *** copy_mats,
                          ptiValue * const lambda, int balanced);

/* ---------------------------------------------------------------------------
 * Dense ALS helpers on host matrices, run on the GPU (each copies its
 * operands in and its results out).  Grams are rank x rank with the factors'
 * stride; as the reference's ssyrk_('L') calls leave them, only their
 * row-major upper triangle (i <= j) needs to be written.
 * ------------------------------------------------------------------------ */
/* include/includes/matrices.h:47,67, src/matrix/matrix.c:340-385:
 * mats[nmodes] = Hadamard product, in the order mode+1, ..., mode+nmodes-1
 * (mod nmodes), of the other Grams, FP32, written full symmetric. */
int ptiMatrixDotMulSeqTriangle(ptiIndex const mode, ptiIndex const nmodes, ptiMatrix ** mats);
int ptiRankMatrixDotMulSeqTriangle(ptiIndex const mode, ptiIndex const nmodes, ptiRankMatrix ** mats);
/* include/includes/matrices.h:61-65,81-85, src/matrix/matrix_solver.c:32-83:
 * rhs <- rhs V^{-1}, V = aTa[nmodes] = the Hadamard product above.  The solve
 * factors V formed in FP64 from the FP32 Grams and solves in FP64 (Cholesky;
 * Gauss-Jordan with pivoting where V is not positive definite, as the
 * reference falls back to sgesv; a singular V leaves rhs unchanged).  rhs pad
 * columns are written as zero.  aTa[nmodes] holds V (FP32) afterwards, where
 * the reference leaves its Cholesky factor. */
int ptiMatrixSolveNormals(ptiIndex const mode, ptiIndex const nmodes, ptiMatrix ** aTa, ptiMatrix * rhs);
int ptiRankMatrixSolveNormals(ptiIndex const mode, ptiIndex const nmodes, ptiRankMatrix ** aTa,
                              ptiRankMatrix * rhs);
/* include/includes/matrices.h:48,55,78-79, src/matrix/matrix.c:389-553:
 * lambda = column 2-norms (FP64 sums) / column maxima of the entries clamped
 * to >= 1; the columns are divided by lambda. */
int ptiMatrix2Norm(ptiMatrix * const A, ptiValue * const lambda);
int ptiMatrixMaxNorm(ptiMatrix * const A, ptiValue * const lambda);
int ptiRankMatrix2Norm(ptiRankMatrix * const A, ptiValue * const lambda);
int ptiRankMatrixMaxNorm(ptiRankMatrix * const A, ptiValue * const lambda);
/* include/includes/matrices.h:56-60,80, src/matrix/matrix.c:556-572: each
 * factor's columns to unit 2-norm, lambda multiplied by the norms. */
void GetFinalLambda(ptiIndex const rank, ptiIndex const nmodes, ptiMatrix ** mats, ptiValue * const lambda);
void GetRankFinalLambda(ptiElementIndex const rank, ptiIndex const nmodes, ptiRankMatrix ** mats,
                        ptiValue * const lambda);
/* include/includes/ktensors.h:27-60, src/ktensor/ktensor.c:77-240,
 * src/ktensor/rankktensor.c:76-242, src/sptensor/hicoo/hicoo.c:248-260.
 * KruskalTensorFrobeniusNormSquared = |lambda^T (Hadamard_m ata[m]) lambda|
 * in FP64, reading each Gram's row-major upper triangle (the reference's loop
 * reads the other triangle, which its ssyrk_ calls never write, so its value
 * depends on uninitialised memory); ata[nmodes] receives the FP32 product.
 * SparseKruskalTensorInnerProduct = sum_r lambda_r sum_i
 * mats[nmodes-1][i,r] mats[nmodes][i,r] (mats[nmodes]: the last MTTKRP
 * output).  KruskalTensorFit = 1 - sqrt(||X||^2 + norm - 2 inner) / ||X||
 * (the square root skipped when the residual is not positive).  NaN on bad
 * arguments (last error set). */
double KruskalTensorFit(ptiSparseTensor const * const ptien, ptiValue const * const lambda, ptiMatrix ** mats,
                        ptiMatrix ** ata);
double KruskalTensorFrobeniusNormSquared(ptiIndex const nmodes, ptiValue const * const lambda, ptiMatrix ** ata);
double SparseKruskalTensorInnerProduct(ptiIndex const nmodes, ptiValue const * const lambda, ptiMatrix ** mats);
double KruskalTensorFitHiCOO(ptiSparseTensorHiCOO const * const hitsr, ptiValue const * const lambda,
                             ptiRankMatrix ** mats, ptiRankMatrix ** ata);
double KruskalTensorFrobeniusNormSquaredRank(ptiIndex const nmodes, ptiValue const * const lambda,
                                             ptiRankMatrix ** ata);
double SparseKruskalTensorInnerProductRank(ptiIndex const nmodes, ptiValue const * const lambda,
                                           ptiRankMatrix ** mats);
/* include/includes/sptensors.h:131 (FP64 accumulation; GPU) */
double SparseTensorFrobeniusNormSquaredHiCOO(ptiSparseTensorHiCOO const * const hitsr);

/* ---------------------------------------------------------------------------
 * Extensions (no reference counterpart): device-resident tensors.
 * ------------------------------------------------------------------------ */
typedef struct ptiB200Tensor ptiB200Tensor;

/* Factor element types for the device entry points. */
enum { PTI_B200_F32 = 0, PTI_B200_BF16 = 1 };

/* Copy a COO or HiCOO tensor into device memory once.  The handle keeps the
 * tensor, plus the per-mode schedules built on first use, until freed. */
int ptiB200UploadSparseTensor(ptiB200Tensor **out, ptiSparseTensor const *X);
int ptiB200UploadSparseTensorHiCOO(ptiB200Tensor **out, ptiSparseTensorHiCOO const *H);
/* Build a device COO tensor from device arrays (inds[m] uint32 and vals f32,
 * nnz entries each); the arrays are copied.  `stream` is a cudaStream_t. */
int ptiB200TensorFromDeviceCOO(ptiB200Tensor **out, ptiIndex nmodes, const ptiIndex *ndims,
                               ptiNnzIndex nnz, const ptiIndex * const *dev_inds,
                               const ptiValue *dev_vals, void *stream);
/* Convert a device COO handle to a device HiCOO handle on the GPU (same
 * ordering rules as ptiSparseTensorToHiCOO); nb and max_nnzb may be NULL. */
int ptiB200ConvertToHiCOO(ptiB200Tensor **out, ptiB200Tensor *coo, ptiElementIndex sb_bits,
                          ptiElementIndex sk_bits, ptiElementIndex sc_bits,
                          ptiNnzIndex *nb, ptiNnzIndex *max_nnzb, void *stream);
/* Build the per-mode schedule for `mode` now (otherwise built on first use). */
int ptiB200Prepare(ptiB200Tensor *t, ptiIndex mode, void *stream);
/* Waits for `stream` and reports (then clears) an error that the tensor's
 * asynchronous kernels recorded on the device: PTIERR_VALUE_ERROR for a
 * coordinate outside its mode, PTIERR_CUDA_ERROR for a tile copy that did not
 * complete within its wait limit; 0 when there was none. */
int ptiB200CheckTensor(ptiB200Tensor *t, void *stream);
int ptiB200FreeTensor(ptiB200Tensor *t);
/* Copies a device HiCOO tensor's arrays to host buffers: bptr (nb+1),
 * binds[m] (nb each), einds[m] (nnz each), vals (nnz).  Synchronous. */
int ptiB200DownloadHiCOO(ptiB200Tensor const *t, ptiNnzIndex *bptr, void * const *binds,
                         void * const *einds, ptiValue *vals);
/* Shape and statistics of a device tensor.  info: [nmodes, nnz, nb, sb, sk, sc, is_hicoo]. */
int ptiB200TensorInfo(ptiB200Tensor const *t, ptiNnzIndex info[7], ptiIndex *ndims_out);

/* Loads a tensor file straight into device memory: the bytes are copied to
 * the GPU and parsed there (the reference parses on the host,
 * src/sptensor/load.c:63-265).  File types and results are those of
 * ptiLoadSparseTensor: .bin is SPLATT binary, other names are text
 * coordinates with 1-based (start_index 1) or 0-based indices; duplicates are
 * kept unless dedupe != 0, which sorts the nonzeros by coordinate (mode 0
 * first) and replaces each repeated coordinate by one nonzero holding the FP32
 * sum of its values in file order.  Indices must fit the mode sizes.  Hex
 * values, nan(...) payloads, values with more than 100 significant digits and
 * tokens longer than 4096 bytes are rejected.  The first load on a device
 * keeps 128 MB of pinned host staging (4 reader threads x 2 x 16 MB) for later
 * loads.  Synchronous on `stream`. */
int ptiB200LoadSparseTensor(ptiB200Tensor **out, ptiIndex start_index, const char *fname, int dedupe,
                            void *stream);
/* Copies a device COO tensor's arrays to host buffers: inds[m] and vals, nnz
 * entries each (NULL entries are skipped).  Synchronous. */
int ptiB200DownloadCOO(ptiB200Tensor const *t, ptiIndex * const *inds, ptiValue *vals);

/* TTM on a device COO tensor.  The fibers along `mode` (nonzeros sorted
 * with `mode` last, cut where another mode changes) are built on first use
 * and kept.  ptiB200TTMFibers returns their count and copies their
 * coordinates (dev_fiber_inds[m], nfibers uint32 each; NULL entries and the
 * mode itself skipped).  ptiB200TTM writes dev_Y (nfibers x ldy FP32, pad
 * columns zero) = fibers times dev_U (rows of ldu floats, rank <= 256 columns
 * used); rank == 0 is TTV with dev_U a vector.  Asynchronous on `stream`. */
int ptiB200TTMFibers(ptiB200Tensor *t, ptiIndex mode, ptiNnzIndex *nfibers, ptiIndex * const *dev_fiber_inds,
                     void *stream);
int ptiB200TTM(ptiB200Tensor *t, ptiIndex mode, const float *dev_U, ptiIndex rank, ptiIndex ldu, float *dev_Y,
               ptiIndex ldy, void *stream);

/* Lexi-order renumbering of a device COO tensor on the GPU (the reference runs
 * it on the host, src/sptensor/renumber.c:26-92).  Each mode in turn, for
 * `iterations` rounds, gets its indices ordered by the lexicographic order of
 * their row lists in the matricisation against the other modes (an index
 * present in the first differing row comes first; indices without nonzeros
 * come last; equal lists keep their current order).  new_indices (host, may be
 * NULL or hold NULL entries) receives original index -> new index per mode.
 * apply != 0 also renumbers the tensor's coordinates in place.  Synchronous. */
int ptiB200Renumber(ptiB200Tensor *t, ptiIndex iterations, ptiIndex * const *new_indices, int apply,
                    void *stream);

/* MTTKRP with everything in device memory.  dev_mats[k] points to ndims[k] x
 * stride row-major factors of element type `factor_type`; dev_out receives
 * ndims[mode] x stride FP32 rows (pad columns zeroed).  Runs asynchronously on
 * `stream` (a cudaStream_t; NULL = legacy default stream). */
int ptiB200MTTKRP(ptiB200Tensor *t, const void * const *dev_mats, int factor_type, ptiIndex rank,
                  ptiIndex stride, const ptiIndex *mats_order, ptiIndex mode, float *dev_out,
                  void *stream);

/* Gradient CP support (no reference counterpart), COO device tensors only.
 * ptiB200KruskalValues: dev_out[z] = sum_r prod_k A_k[i_k(z), r] for every
 * nonzero z in the tensor's input order (factors FP32, ndims[k] x stride).
 * ptiB200MTTKRPValues: ptiB200MTTKRP with the tensor's values replaced by
 * dev_vals (nnz floats in input order) -- the gradient of sum_z g_z model(z)
 * with respect to factor `mode`.  Both run asynchronously on `stream`. */
int ptiB200KruskalValues(ptiB200Tensor *t, const float * const *dev_factors, ptiIndex rank, ptiIndex stride,
                         float *dev_out, void *stream);
int ptiB200MTTKRPValues(ptiB200Tensor *t, const float *dev_vals, const void * const *dev_mats, int factor_type,
                        ptiIndex rank, ptiIndex stride, const ptiIndex *mats_order, ptiIndex mode,
                        float *dev_out, void *stream);

/* HiCOO MTTKRP that allocates no device memory (no counterpart in the
 * reference).  For callers that cannot call cudaMalloc while it runs: code
 * whose device memory is owned by a host framework's pool, services with a
 * fixed memory budget, real-time loops where an allocation could block.  The
 * caller passes the HiCOO arrays (bptr nb+1, binds[m] nb each, einds[m] and
 * vals nnz each; bptr strictly increasing), the FP32 factors (ndims[k] x
 * stride, 16-byte aligned) and the output (ndims[mode] x stride), all in
 * device memory; ndims, mats_order and the pointer arrays live in host memory.
 * The kernel's scratch (a tile table and an error word) sits in fixed arrays
 * in the library's device image -- about 1 MiB that every GPU which loads the
 * library keeps until exit -- which limits nnz to 268,435,456 (2^18 tiles of
 * 1024); larger tensors are rejected with PTIERR_VALUE_ERROR.  The first call
 * on a device looks up the arrays' device addresses, so make that first call
 * before any stream capture.  All calls share the scratch: calls that overlap
 * on the GPU (other streams, other host threads) race and must be ordered by
 * the caller.  Runs asynchronously on `stream`.  Nothing is reported back
 * from the device: nonzeros whose coordinates fall outside ndims are skipped,
 * and a bptr that is not strictly increasing (or that does not end at nnz)
 * is not detected and gives wrong results with return code 0, so validate
 * bptr before the call where it is not trusted.  The looked-up addresses are
 * kept for the life of the process: after cudaDeviceReset (or anything else
 * that destroys and recreates the device's primary context) they are stale,
 * and this entry point must not be called again in that process.  Uses the
 * direct-atomic kernel (no per-mode schedule, which would need memory). */
int ptiB200MTTKRPHiCOONoAlloc(ptiIndex nmodes, const ptiIndex *ndims, ptiNnzIndex nnz, ptiNnzIndex nb,
                              ptiElementIndex sb_bits, const ptiNnzIndex *dev_bptr,
                              const ptiBlockIndex * const *dev_binds,
                              const ptiElementIndex * const *dev_einds, const ptiValue *dev_vals,
                              const float * const *dev_mats, ptiIndex rank, ptiIndex stride,
                              const ptiIndex *mats_order, ptiIndex mode, float *dev_out, void *stream);

/* CPD-ALS with everything in device memory.  dev_factors[k] (ndims[k] x stride
 * FP32, stride a multiple of 8) hold the initial factors and receive the
 * result; dev_lambda (rank floats) receives the weights.  precision selects
 * the factor copy the MTTKRP gathers read: PTI_B200_F32, or PTI_B200_BF16 for
 * all but the last fp32_sweeps iterations.  Grams, solves and fits are FP64.
 * fits (host, niters doubles, may be NULL) receives the fit after every
 * iteration; iters_done the number of iterations run (tol > 0 stops early as
 * in src/sptensor/cpd.c:144).  rank <= 128.  Synchronous on `stream`. */
int ptiB200CpdAls(ptiB200Tensor *t, ptiIndex rank, ptiIndex niters, double tol, int precision,
                  ptiIndex fp32_sweeps, float * const *dev_factors, ptiIndex stride, float *dev_lambda,
                  double *fits, ptiIndex *iters_done, void *stream);

/* ptiB200CpdAls with checkpoints (the reference has none; its CPD writes its
 * result only as text, src/ktensor/dump.c:23-55).  ckpt_path (may be NULL:
 * none) receives the ALS loop state -- factors, weights and every fit so far
 * -- after every ckpt_every iterations (0: only the last) and after the last
 * iteration; the file is written from a background thread, as <path>.tmp
 * renamed over <path>.  With resume != 0 and an existing file, that state
 * replaces the initial factors and the loop continues after its last
 * iteration (a run that had converged under tol > 0 is not iterated further);
 * fits and iters_done then count the restored iterations too.  A checkpoint of
 * another shape, rank or tensor, or of more than niters iterations, is
 * rejected; a missing file starts from the initial factors. */
int ptiB200CpdAlsCheckpoint(ptiB200Tensor *t, ptiIndex rank, ptiIndex niters, double tol, int precision,
                            ptiIndex fp32_sweeps, float * const *dev_factors, ptiIndex stride,
                            float *dev_lambda, double *fits, ptiIndex *iters_done,
                            const char *ckpt_path, ptiIndex ckpt_every, int resume, void *stream);

/* Reads a checkpoint written by ptiB200CpdAlsCheckpoint into a host Kruskal
 * tensor, finished as the ALS loop finishes its result (columns scaled to unit
 * 2-norm, weights multiplied by the norms, src/matrix/matrix.c:556-572); fit is
 * the last fit.  ktsr is created here (release it with ptiFreeKruskalTensor);
 * iters_done (may be NULL) receives the stored iteration count.  Host only. */
int ptiB200LoadCpdCheckpoint(ptiKruskalTensor *ktsr, ptiIndex *iters_done, const char *path);

/* Batched CPD-ALS of many independent 3-D tensors of uneven size and rank (no
 * counterpart in the reference, whose CPD entry points factor one tensor per
 * call; each tensor follows src/sptensor/cpd.c:32-208).
 *
 * ptiB200BatchCreate copies the tensors (ndims: ntensors x 3; dev_inds:
 * ntensors x 3 device arrays of nnz[b] uint32; dev_vals: ntensors device
 * arrays), converts each to HiCOO on the GPU and builds its per-mode
 * schedules.  ranks[b] in [1, 32]; every tensor needs at least one nonzero.
 * tune != 0 times whole iterations for HiCOO block sizes sb_bits in {4..7} and
 * 4 or 8 factor columns per lane in BF16 iterations and keeps the fastest
 * (cached per batch shape); tune == 0 uses sb_bits 7 and 4 columns per lane.
 *
 * ptiB200BatchCpdAls runs niters ALS iterations on every tensor: each
 * iteration of the whole batch is one persistent kernel launch replayed from a
 * CUDA graph.  dev_factors: ntensors x 3 device arrays, ndims x stride FP32
 * with stride = rank rounded up to a multiple of 8, 16-byte aligned; they hold
 * the initial factors and receive the result.  dev_lambda: ntensors device
 * arrays of rank floats.  precision as for ptiB200CpdAls.  fits (host,
 * ntensors x niters, may be NULL) receives every tensor's fit after every
 * iteration; ms_per_iter (may be NULL) the device time of one iteration of the
 * batch.  Synchronous; ordered after the work already queued on `stream`. */
typedef struct ptiB200Batch ptiB200Batch;
int ptiB200BatchCreate(ptiB200Batch **out, ptiIndex ntensors, const ptiIndex *ndims,
                       const ptiNnzIndex *nnz, const ptiIndex * const *dev_inds,
                       const ptiValue * const *dev_vals, const ptiIndex *ranks, int tune,
                       void *stream);
int ptiB200BatchInfo(const ptiB200Batch *batch, int *sb_bits, int *cols_per_lane, float *tune_ms,
                     float *setup_ms, ptiNnzIndex *ntasks);
int ptiB200BatchCpdAls(ptiB200Batch *batch, ptiIndex niters, int precision, ptiIndex fp32_sweeps,
                       float * const *dev_factors, float * const *dev_lambda, double *fits,
                       float *ms_per_iter, void *stream);
void ptiB200BatchFree(ptiB200Batch *batch);

/* Self-checks of the bounded device waits (no reference counterpart; they
 * exercise the failure path without faulting or hanging the GPU).
 * ptiB200BatchWaitProbe runs the batched ALS kernel on a one-task queue whose
 * dependency nothing satisfies, with every wait bounded by wait_seconds (at
 * most 2): the wait gives up and the call returns PTIERR_CUDA_ERROR, as a run
 * whose queue stalled does; the batch stays usable (nothing it holds is
 * written).  ptiB200MbarrierWaitProbe arms a shared-memory barrier for bytes
 * that never arrive and waits `polls` polls: *gave_up = 1 when the bounded
 * wait gave up, *completed = 1 when a second barrier, completed by its
 * arrival alone, was seen complete. */
int ptiB200BatchWaitProbe(ptiB200Batch *bt, double wait_seconds);
int ptiB200MbarrierWaitProbe(unsigned polls, int *gave_up, int *completed);

/* The L2 read bandwidth of the current GPU (no reference counterpart): a
 * kernel of this library streams a buffer of `bytes` (1 MiB to 1 GiB; choose
 * one inside L2 and large enough for eight loads per thread, e.g. 64 MiB on
 * B200) with 16-byte L2-only loads `reps` times after one untimed pass;
 * *gbps receives bytes * reps / time.  The bench reads the MTTKRP's
 * factor-row gathers against it. */
int ptiB200ProbeL2ReadBandwidth(unsigned long long bytes, unsigned reps, double *gbps);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif /* HIPARTI_B200_H */
