/*
 * Minimal LAPACKE stand-in used ONLY to compile the reference into the test
 * oracle.  NOT product code.
 *
 * The block-Jacobi preconditioner calls dlange('1'), dgetrf, dgecon('1') and
 * dgetri on 3x3 row-major blocks (mappraiser/src/precond.c:530-566).  These
 * are implemented in shim_lapacke.c as restatements of reference LAPACK's
 * unblocked algorithms (DGETF2, DGECON with DLACN2 / Higham 1988, DTRTI2 +
 * DGETRI) and are checked against scipy.linalg.lapack in the CPU tests.
 * dsyev and dgelss (the two-level preconditioners, precond.c:770-1307) are
 * restated with Jacobi methods in shim_lapacke.c; dgesdd/dgesvd are only
 * reached by the out-of-scope templates and return an error.
 */
#ifndef ORACLE_SHIM_LAPACKE_H
#define ORACLE_SHIM_LAPACKE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef int lapack_int;

#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102

double     LAPACKE_dlange(int layout, char norm, lapack_int m, lapack_int n, const double *a, lapack_int lda);
lapack_int LAPACKE_dgetrf(int layout, lapack_int m, lapack_int n, double *a, lapack_int lda, lapack_int *ipiv);
lapack_int LAPACKE_dgecon(int layout, char norm, lapack_int n, const double *a, lapack_int lda, double anorm,
                          double *rcond);
lapack_int LAPACKE_dgetri(int layout, lapack_int n, double *a, lapack_int lda, const lapack_int *ipiv);

lapack_int LAPACKE_dsyev(int layout, char jobz, char uplo, lapack_int n, double *a, lapack_int lda, double *w);
lapack_int LAPACKE_dgelss(int layout, lapack_int m, lapack_int n, lapack_int nrhs, double *a, lapack_int lda,
                          double *b, lapack_int ldb, double *s, double rcond, lapack_int *rank);
lapack_int LAPACKE_dgesdd(int layout, char jobz, lapack_int m, lapack_int n, double *a, lapack_int lda, double *s,
                          double *u, lapack_int ldu, double *vt, lapack_int ldvt);
lapack_int LAPACKE_dgesdd_work(int layout, char jobz, lapack_int m, lapack_int n, double *a, lapack_int lda,
                               double *s, double *u, lapack_int ldu, double *vt, lapack_int ldvt, double *work,
                               lapack_int lwork, lapack_int *iwork);
lapack_int LAPACKE_dgesvd(int layout, char jobu, char jobvt, lapack_int m, lapack_int n, double *a, lapack_int lda,
                          double *s, double *u, lapack_int ldu, double *vt, lapack_int ldvt, double *superb);

/* cblas subset (two-level preconditioner only) */
enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
void cblas_dgemm(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE ta, enum CBLAS_TRANSPOSE tb, int m, int n, int k,
                 double alpha, const double *a, int lda, const double *b, int ldb, double beta, double *c, int ldc);

#ifdef __cplusplus
}
#endif

#endif /* ORACLE_SHIM_LAPACKE_H */
