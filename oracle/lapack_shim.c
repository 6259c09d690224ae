/* Test infrastructure only: forwards the four single-precision LAPACK/BLAS
 * symbols that the reference CPD path calls (ssyrk_, spotrf_, spotrs_, sgesv_)
 * to the OpenBLAS copy bundled with SciPy, whose symbols carry a "scipy_"
 * prefix.  Linked only into oracle/_ref/libHiParTI.so, never into the product. */
extern void scipy_ssyrk_(const char*, const char*, const int*, const int*, const float*,
                         const float*, const int*, const float*, float*, const int*);
extern void scipy_spotrf_(const char*, const int*, float*, const int*, int*);
extern void scipy_spotrs_(const char*, const int*, const int*, const float*, const int*,
                          float*, const int*, int*);
extern void scipy_sgesv_(const int*, const int*, float*, const int*, int*, float*, const int*, int*);

void ssyrk_(const char* u, const char* t, const int* n, const int* k, const float* al,
            const float* a, const int* lda, const float* be, float* c, const int* ldc)
{ scipy_ssyrk_(u, t, n, k, al, a, lda, be, c, ldc); }
void spotrf_(const char* u, const int* n, float* a, const int* lda, int* info)
{ scipy_spotrf_(u, n, a, lda, info); }
void spotrs_(const char* u, const int* n, const int* nrhs, const float* a, const int* lda,
             float* b, const int* ldb, int* info)
{ scipy_spotrs_(u, n, nrhs, a, lda, b, ldb, info); }
void sgesv_(const int* n, const int* nrhs, float* a, const int* lda, int* ipiv, float* b,
            const int* ldb, int* info)
{ scipy_sgesv_(n, nrhs, a, lda, ipiv, b, ldb, info); }
