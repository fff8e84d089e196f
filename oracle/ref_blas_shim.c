/* BLAS/LAPACK names the reference's CPU build links against (backend/Common/common.h:116-150),
 * forwarded to the OpenBLAS that scipy bundles, whose exported names carry a "scipy_" prefix.
 * Test infrastructure only: it lets oracle/build_ref_full.sh link the reference's own solver
 * (cput2cEXASIM) in a container with no system BLAS.  Character arguments get their hidden
 * Fortran length (1) passed explicitly. */
#include <stddef.h>

#define I int
typedef size_t flen;

double scipy_dnrm2_(I*, double*, I*);
double scipy_ddot_(I*, double*, I*, double*, I*);
void scipy_dcopy_(I*, double*, I*, double*, I*);
void scipy_dscal_(I*, double*, double*, I*);
void scipy_daxpy_(I*, double*, double*, I*, double*, I*);
void scipy_dgemv_(char*, I*, I*, double*, double*, I*, double*, I*, double*, double*, I*, flen);
void scipy_dgemm_(char*, char*, I*, I*, I*, double*, double*, I*, double*, I*, double*, double*, I*, flen, flen);
void scipy_dgetrf_(I*, I*, double*, I*, I*, I*);
void scipy_dgetri_(I*, double*, I*, I*, double*, I*, I*);
void scipy_dtrsm_(char*, char*, char*, char*, I*, I*, double*, double*, I*, double*, I*, flen, flen, flen, flen);
void scipy_dgeev_(char*, char*, I*, double*, I*, double*, double*, double*, I*, double*, I*, double*, I*, I*, flen,
                  flen);
void scipy_dgesv_(I*, I*, double*, I*, I*, double*, I*, I*);

double dnrm2_(I* n, double* x, I* incx) { return scipy_dnrm2_(n, x, incx); }
double ddot_(I* n, double* x, I* incx, double* y, I* incy) { return scipy_ddot_(n, x, incx, y, incy); }
void dcopy_(I* n, double* x, I* incx, double* y, I* incy) { scipy_dcopy_(n, x, incx, y, incy); }
void dscal_(I* n, double* a, double* x, I* incx) { scipy_dscal_(n, a, x, incx); }
void daxpy_(I* n, double* a, double* x, I* incx, double* y, I* incy) { scipy_daxpy_(n, a, x, incx, y, incy); }
void dgemv_(char* t, I* m, I* n, double* a, double* A, I* lda, double* x, I* incx, double* b, double* y, I* incy)
{
    scipy_dgemv_(t, m, n, a, A, lda, x, incx, b, y, incy, 1);
}
void dgemm_(char* ta, char* tb, I* m, I* n, I* k, double* a, double* A, I* lda, double* B, I* ldb, double* b,
            double* C, I* ldc)
{
    scipy_dgemm_(ta, tb, m, n, k, a, A, lda, B, ldb, b, C, ldc, 1, 1);
}
void dgetrf_(I* m, I* n, double* A, I* lda, I* ipiv, I* info) { scipy_dgetrf_(m, n, A, lda, ipiv, info); }
void dgetri_(I* n, double* A, I* lda, I* ipiv, double* w, I* lw, I* info) { scipy_dgetri_(n, A, lda, ipiv, w, lw, info); }
void dtrsm_(char* s, char* u, char* t, char* d, I* m, I* n, double* a, double* A, I* lda, double* B, I* ldb)
{
    scipy_dtrsm_(s, u, t, d, m, n, a, A, lda, B, ldb, 1, 1, 1, 1);
}
void dgeev_(char* jl, char* jr, I* n, double* A, I* lda, double* wr, double* wi, double* vl, I* ldvl, double* vr,
            I* ldvr, double* w, I* lw, I* info)
{
    scipy_dgeev_(jl, jr, n, A, lda, wr, wi, vl, ldvl, vr, ldvr, w, lw, info, 1, 1);
}
void dgesv_(I* n, I* nrhs, double* A, I* lda, I* ipiv, double* B, I* ldb, I* info)
{
    scipy_dgesv_(n, nrhs, A, lda, ipiv, B, ldb, info);
}
