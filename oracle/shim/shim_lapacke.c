/*
 * Test-oracle restatement of the LAPACK routines the block-Jacobi and the
 * two-level preconditioners use (see lapacke.h).  NOT product code.
 *
 * Row-major calls are handled the way LAPACKE does: the logical matrix is
 * copied to column-major, the column-major algorithm runs, and the result is
 * copied back.  The algorithms follow reference LAPACK 3.x:
 *   dgetrf  -> DGETF2 (partial pivoting, IDAMAX, reciprocal scaling when
 *              |pivot| >= sfmin, rank-1 update)
 *   dgecon  -> DGECON('1') with the DLACN2 estimator (Hager 1984, Higham 1988,
 *              ACM TOMS 14:381); DLATRS reduces to a plain triangular solve
 *              (scale 1) unless a diagonal of U is zero, where DGECON returns 0
 *   dgetri  -> DTRTI2 (inv(U)) then the unblocked DGETRI column sweep and the
 *              column interchanges in reverse order
 *   dlange  -> DLANGE('1') maximum absolute column sum
 */
#include "lapacke.h"

#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define CM(a, lda, i, j) (a)[(size_t) (j) * (lda) + (i)]

static void to_cm(int layout, int m, int n, const double *a, int lda, double *c) {
    for (int i = 0; i < m; i++)
        for (int j = 0; j < n; j++)
            c[(size_t) j * m + i] = (layout == LAPACK_ROW_MAJOR) ? a[(size_t) i * lda + j] : a[(size_t) j * lda + i];
}

static void from_cm(int layout, int m, int n, const double *c, double *a, int lda) {
    for (int i = 0; i < m; i++)
        for (int j = 0; j < n; j++) {
            if (layout == LAPACK_ROW_MAJOR) a[(size_t) i * lda + j] = c[(size_t) j * m + i];
            else a[(size_t) j * lda + i] = c[(size_t) j * m + i];
        }
}

static int idamax(int n, const double *x, int incx) {
    int    best = 0;
    double bv   = fabs(x[0]);
    for (int i = 1; i < n; i++) {
        double v = fabs(x[(size_t) i * incx]);
        if (v > bv) {
            bv   = v;
            best = i;
        }
    }
    return best;
}

double LAPACKE_dlange(int layout, char norm, lapack_int m, lapack_int n, const double *a, lapack_int lda) {
    if (norm != '1' && norm != 'O' && norm != 'o') {
        fprintf(stderr, "shim LAPACKE_dlange: only the 1-norm is implemented\n");
        return NAN;
    }
    double value = 0.0;
    for (int j = 0; j < n; j++) {
        double sum = 0.0;
        for (int i = 0; i < m; i++)
            sum += fabs(layout == LAPACK_ROW_MAJOR ? a[(size_t) i * lda + j] : a[(size_t) j * lda + i]);
        if (value < sum || isnan(sum)) value = sum;
    }
    return value;
}

/* DGETF2 on a column-major m x n matrix; ipiv is 1-based like LAPACK */
static int dgetf2_cm(int m, int n, double *a, int lda, int *ipiv) {
    const double sfmin = DBL_MIN;
    int          info  = 0;
    int          mn    = m < n ? m : n;
    for (int j = 0; j < mn; j++) {
        int jp      = j + idamax(m - j, &CM(a, lda, j, j), 1);
        ipiv[j]     = jp + 1;
        if (CM(a, lda, jp, j) != 0.0) {
            if (jp != j)
                for (int k = 0; k < n; k++) {
                    double t          = CM(a, lda, j, k);
                    CM(a, lda, j, k)  = CM(a, lda, jp, k);
                    CM(a, lda, jp, k) = t;
                }
            if (j < m - 1) {
                if (fabs(CM(a, lda, j, j)) >= sfmin) {
                    double r = 1.0 / CM(a, lda, j, j);
                    for (int i = j + 1; i < m; i++) CM(a, lda, i, j) *= r;
                } else {
                    for (int i = j + 1; i < m; i++) CM(a, lda, i, j) = CM(a, lda, i, j) / CM(a, lda, j, j);
                }
            }
        } else if (info == 0) {
            info = j + 1;
        }
        /* rank-1 update of the trailing block (DGER: column by column) */
        for (int k = j + 1; k < n; k++) {
            double t = CM(a, lda, j, k);
            if (t != 0.0)
                for (int i = j + 1; i < m; i++) CM(a, lda, i, k) += -t * CM(a, lda, i, j);
        }
    }
    return info;
}

lapack_int LAPACKE_dgetrf(int layout, lapack_int m, lapack_int n, double *a, lapack_int lda, lapack_int *ipiv) {
    double *c = malloc(sizeof(double) * (size_t) m * n);
    to_cm(layout, m, n, a, lda, c);
    int info = dgetf2_cm(m, n, c, m, ipiv);
    from_cm(layout, m, n, c, a, lda);
    free(c);
    return info;
}

/* x := inv(U) inv(L) x   (kase 1)   or   x := inv(L^T) inv(U^T) x   (kase 2) */
static void lu_solve(int n, const double *lu, int kase, double *x) {
    if (kase == 1) {
        for (int j = 0; j < n; j++) /* L unit lower, column oriented (DTRSV 'L','N','U') */
            if (x[j] != 0.0)
                for (int i = j + 1; i < n; i++) x[i] -= x[j] * CM(lu, n, i, j);
        for (int j = n - 1; j >= 0; j--) /* U upper non-unit (DTRSV 'U','N','N') */
            if (x[j] != 0.0) {
                x[j] = x[j] / CM(lu, n, j, j);
                double t = x[j];
                for (int i = j - 1; i >= 0; i--) x[i] -= t * CM(lu, n, i, j);
            }
    } else {
        for (int j = 0; j < n; j++) { /* U^T (DTRSV 'U','T','N') */
            double t = x[j];
            for (int i = 0; i < j; i++) t -= CM(lu, n, i, j) * x[i];
            x[j] = t / CM(lu, n, j, j);
        }
        for (int j = n - 1; j >= 0; j--) { /* L^T unit (DTRSV 'L','T','U') */
            double t = x[j];
            for (int i = n - 1; i > j; i--) t -= CM(lu, n, i, j) * x[i];
            x[j] = t;
        }
    }
}

static double dasum(int n, const double *x) {
    double s = 0.0;
    for (int i = 0; i < n; i++) s += fabs(x[i]);
    return s;
}

/* DGECON('1') driven by the DLACN2 estimator, written as a loop */
static double dgecon1_cm(int n, const double *lu, double anorm) {
    if (n == 0) return 1.0;
    if (anorm == 0.0) return 0.0;
    for (int j = 0; j < n; j++)
        if (CM(lu, n, j, j) == 0.0) return 0.0;
    double *x    = malloc(sizeof(double) * n);
    double *v    = malloc(sizeof(double) * n);
    int    *isgn = malloc(sizeof(int) * n);
    double  est = 0.0, estold;
    int     iter, j, jlast;
    int     ok = 1;

    for (int i = 0; i < n; i++) x[i] = 1.0 / (double) n;
    lu_solve(n, lu, 1, x); /* DLACN2 stage 20 */
    if (n == 1) {
        v[0] = x[0];
        est  = fabs(v[0]);
        goto done;
    }
    est = dasum(n, x);
    for (int i = 0; i < n; i++) {
        x[i]    = (x[i] >= 0.0) ? 1.0 : -1.0;
        isgn[i] = (int) lrint(x[i]);
    }
    lu_solve(n, lu, 2, x); /* stage 40 */
    j    = idamax(n, x, 1);
    iter = 2;
    for (;;) {
        /* stage 50 */
        for (int i = 0; i < n; i++) x[i] = 0.0;
        x[j] = 1.0;
        lu_solve(n, lu, 1, x);
        /* stage 70 */
        memcpy(v, x, sizeof(double) * n);
        estold = est;
        est    = dasum(n, v);
        int same = 1;
        for (int i = 0; i < n; i++) {
            double xs = (x[i] >= 0.0) ? 1.0 : -1.0;
            if ((int) lrint(xs) != isgn[i]) {
                same = 0;
                break;
            }
        }
        if (same) break;           /* repeated sign vector: converged */
        if (est <= estold) break;  /* stage 90: cycling test */
        for (int i = 0; i < n; i++) {
            x[i]    = (x[i] >= 0.0) ? 1.0 : -1.0;
            isgn[i] = (int) lrint(x[i]);
        }
        lu_solve(n, lu, 2, x);     /* stage 110 */
        jlast = j;
        j     = idamax(n, x, 1);
        if (x[jlast] != fabs(x[j]) && iter < 5) {
            iter++;
            continue;
        }
        break;
    }
    /* stage 120: alternating-sign extra vector */
    {
        double altsgn = 1.0;
        for (int i = 0; i < n; i++) {
            x[i]   = altsgn * (1.0 + (double) i / (double) (n - 1));
            altsgn = -altsgn;
        }
        lu_solve(n, lu, 1, x);
        double temp = 2.0 * (dasum(n, x) / (double) (3 * n)); /* stage 140 */
        if (temp > est) {
            memcpy(v, x, sizeof(double) * n);
            est = temp;
        }
    }
done:
    for (int i = 0; i < n; i++)
        if (!isfinite(x[i]) || !isfinite(v[i])) ok = 0;
    free(x);
    free(v);
    free(isgn);
    if (!ok || !isfinite(est)) return 0.0;
    if (est != 0.0) return (1.0 / est) / anorm;
    return 0.0;
}

lapack_int LAPACKE_dgecon(int layout, char norm, lapack_int n, const double *a, lapack_int lda, double anorm,
                          double *rcond) {
    if (norm != '1' && norm != 'O' && norm != 'o') {
        fprintf(stderr, "shim LAPACKE_dgecon: only the 1-norm is implemented\n");
        return -2;
    }
    double *c = malloc(sizeof(double) * (size_t) n * n);
    to_cm(layout, n, n, a, lda, c);
    *rcond = dgecon1_cm(n, c, anorm);
    free(c);
    return 0;
}

/* DTRTI2 ('U','N') followed by the unblocked DGETRI sweep */
static int dgetri_cm(int n, double *a, const int *ipiv) {
    for (int j = 0; j < n; j++)
        if (CM(a, n, j, j) == 0.0) return j + 1;
    for (int j = 0; j < n; j++) {
        CM(a, n, j, j) = 1.0 / CM(a, n, j, j);
        double ajj     = -CM(a, n, j, j);
        /* DTRMV('U','N','N', j, A, x = A(0:j-1, j)) */
        double *x = &CM(a, n, 0, j);
        for (int jj = 0; jj < j; jj++) {
            if (x[jj] != 0.0) {
                double temp = x[jj];
                for (int i = 0; i < jj; i++) x[i] += temp * CM(a, n, i, jj);
                x[jj] *= CM(a, n, jj, jj);
            }
        }
        for (int i = 0; i < j; i++) x[i] *= ajj;
    }
    double *work = malloc(sizeof(double) * n);
    for (int j = n - 1; j >= 0; j--) {
        for (int i = j + 1; i < n; i++) {
            work[i]        = CM(a, n, i, j);
            CM(a, n, i, j) = 0.0;
        }
        if (j < n - 1) /* DGEMV('N', n, n-j-1, -1, A(:, j+1:), work(j+1:), 1, A(:, j)) */
            for (int jj = j + 1; jj < n; jj++) {
                double temp = -work[jj];
                if (temp != 0.0)
                    for (int i = 0; i < n; i++) CM(a, n, i, j) += temp * CM(a, n, i, jj);
            }
    }
    free(work);
    for (int j = n - 2; j >= 0; j--) {
        int jp = ipiv[j] - 1;
        if (jp != j)
            for (int i = 0; i < n; i++) {
                double t        = CM(a, n, i, j);
                CM(a, n, i, j)  = CM(a, n, i, jp);
                CM(a, n, i, jp) = t;
            }
    }
    return 0;
}

lapack_int LAPACKE_dgetri(int layout, lapack_int n, double *a, lapack_int lda, const lapack_int *ipiv) {
    double *c = malloc(sizeof(double) * (size_t) n * n);
    to_cm(layout, n, n, a, lda, c);
    int info = dgetri_cm(n, c, ipiv);
    from_cm(layout, n, n, c, a, lda);
    free(c);
    return info;
}

static lapack_int unavailable(const char *name) {
    fprintf(stderr, "shim %s: not available in the test oracle (templates only)\n",
            name);
    return -1;
}

/*
 * The two-level preconditioners (precond.c:791-1307) call dsyev('V','U') on
 * the Lanczos tridiagonal matrix and dgelss on E = Z^T A Z (pseudo-inverse).
 * Both are restated with Jacobi methods, which give the same eigen/singular
 * decompositions as LAPACK's QR-based drivers up to rounding and the signs of
 * the vectors (the preconditioners only depend on the spanned subspace):
 *   dsyev  -> cyclic two-sided Jacobi (Golub & Van Loan, Matrix Computations,
 *             4th ed., section 8.5), eigenvalues sorted ascending
 *   dgelss -> one-sided Jacobi SVD (Hestenes 1958; Demmel & Veselic 1992),
 *             minimum-norm solution with singular values <= rcond * s_max
 *             treated as zero (rcond < 0: machine epsilon), as DGELSS
 */
static void jacobi_eig_cm(int n, double *a, double *v) {
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) CM(v, n, i, j) = (i == j) ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0.0, tot = 0.0;
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                tot += CM(a, n, i, j) * CM(a, n, i, j);
                if (i != j) off += CM(a, n, i, j) * CM(a, n, i, j);
            }
        if (off <= DBL_EPSILON * DBL_EPSILON * tot || off == 0.0) break;
        for (int p = 0; p < n - 1; p++)
            for (int q = p + 1; q < n; q++) {
                double apq = CM(a, n, p, q);
                if (apq == 0.0) continue;
                double theta = (CM(a, n, q, q) - CM(a, n, p, p)) / (2.0 * apq);
                double t     = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < n; k++) { /* A <- A J (columns p, q) */
                    double akp = CM(a, n, k, p), akq = CM(a, n, k, q);
                    CM(a, n, k, p) = c * akp - s * akq;
                    CM(a, n, k, q) = s * akp + c * akq;
                }
                for (int k = 0; k < n; k++) { /* A <- J^T A (rows p, q) */
                    double apk = CM(a, n, p, k), aqk = CM(a, n, q, k);
                    CM(a, n, p, k) = c * apk - s * aqk;
                    CM(a, n, q, k) = s * apk + c * aqk;
                }
                for (int k = 0; k < n; k++) {
                    double vkp = CM(v, n, k, p), vkq = CM(v, n, k, q);
                    CM(v, n, k, p) = c * vkp - s * vkq;
                    CM(v, n, k, q) = s * vkp + c * vkq;
                }
            }
    }
}

lapack_int LAPACKE_dsyev(int layout, char jobz, char uplo, lapack_int n, double *a, lapack_int lda, double *w) {
    if (n <= 0) return 0;
    double *c = malloc(sizeof(double) * (size_t) n * n), *v = malloc(sizeof(double) * (size_t) n * n);
    int    *ord = malloc(sizeof(int) * (size_t) n);
    to_cm(layout, n, n, a, lda, c);
    const int up = (uplo == 'U' || uplo == 'u');
    for (int j = 0; j < n; j++) /* symmetric from the referenced triangle */
        for (int i = 0; i < n; i++)
            if ((up && i > j) || (!up && i < j)) CM(c, n, i, j) = CM(c, n, j, i);
    jacobi_eig_cm(n, c, v);
    for (int i = 0; i < n; i++) ord[i] = i;
    for (int i = 1; i < n; i++) /* insertion sort, ascending eigenvalues */
        for (int k = i; k > 0 && CM(c, n, ord[k], ord[k]) < CM(c, n, ord[k - 1], ord[k - 1]); k--) {
            int t = ord[k]; ord[k] = ord[k - 1]; ord[k - 1] = t;
        }
    double *out = malloc(sizeof(double) * (size_t) n * n);
    for (int j = 0; j < n; j++) {
        w[j] = CM(c, n, ord[j], ord[j]);
        for (int i = 0; i < n; i++) CM(out, n, i, j) = (jobz == 'V' || jobz == 'v') ? CM(v, n, i, ord[j]) : 0.0;
    }
    if (jobz == 'V' || jobz == 'v') from_cm(layout, n, n, out, a, lda);
    free(c), free(v), free(ord), free(out);
    return 0;
}

lapack_int LAPACKE_dgelss(int layout, lapack_int m, lapack_int n, lapack_int nrhs, double *a, lapack_int lda,
                          double *b, lapack_int ldb, double *s, double rcond, lapack_int *rank) {
    const int mb = m > n ? m : n;                       /* rows of b */
    double   *u = malloc(sizeof(double) * (size_t) m * n), *v = malloc(sizeof(double) * (size_t) n * n);
    double   *bc = calloc((size_t) mb * nrhs, sizeof(double)), *sv = malloc(sizeof(double) * (size_t) n);
    double   *x = calloc((size_t) n * nrhs, sizeof(double));
    int      *ord = malloc(sizeof(int) * (size_t) n);
    to_cm(layout, m, n, a, lda, u);
    for (int i = 0; i < m; i++)
        for (int r = 0; r < nrhs; r++)
            CM(bc, mb, i, r) = (layout == LAPACK_ROW_MAJOR) ? b[(size_t) i * ldb + r] : b[(size_t) r * ldb + i];
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) CM(v, n, i, j) = (i == j) ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 100; sweep++) {
        int rotated = 0;
        for (int p = 0; p < n - 1; p++)
            for (int q = p + 1; q < n; q++) {
                double al = 0.0, be = 0.0, ga = 0.0;
                for (int k = 0; k < m; k++) {
                    al += CM(u, m, k, p) * CM(u, m, k, p);
                    be += CM(u, m, k, q) * CM(u, m, k, q);
                    ga += CM(u, m, k, p) * CM(u, m, k, q);
                }
                if (ga == 0.0 || fabs(ga) <= DBL_EPSILON * sqrt(al * be)) continue;
                rotated = 1;
                double zeta = (be - al) / (2.0 * ga);
                double t    = (zeta >= 0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
                double c = 1.0 / sqrt(1.0 + t * t), sn = c * t;
                for (int k = 0; k < m; k++) {
                    double up = CM(u, m, k, p), uq = CM(u, m, k, q);
                    CM(u, m, k, p) = c * up - sn * uq;
                    CM(u, m, k, q) = sn * up + c * uq;
                }
                for (int k = 0; k < n; k++) {
                    double vp = CM(v, n, k, p), vq = CM(v, n, k, q);
                    CM(v, n, k, p) = c * vp - sn * vq;
                    CM(v, n, k, q) = sn * vp + c * vq;
                }
            }
        if (!rotated) break;
    }
    double smax = 0.0;
    for (int j = 0; j < n; j++) {
        double nn = 0.0;
        for (int k = 0; k < m; k++) nn += CM(u, m, k, j) * CM(u, m, k, j);
        sv[j] = sqrt(nn);
        if (sv[j] > smax) smax = sv[j];
    }
    const double thr = (rcond < 0 ? DBL_EPSILON : rcond) * smax;
    int          kept = 0;
    for (int j = 0; j < n; j++) {
        if (!(sv[j] > thr)) continue;
        kept++;
        for (int r = 0; r < nrhs; r++) { /* x += v_j (u_j^T b_r) / s_j^2 (u_j unnormalised) */
            double d = 0.0;
            for (int k = 0; k < m; k++) d += CM(u, m, k, j) * CM(bc, mb, k, r);
            d /= sv[j] * sv[j];
            for (int i = 0; i < n; i++) CM(x, n, i, r) += CM(v, n, i, j) * d;
        }
    }
    for (int i = 0; i < n; i++) ord[i] = i;
    for (int i = 1; i < n; i++) /* singular values in decreasing order */
        for (int k = i; k > 0 && sv[ord[k]] > sv[ord[k - 1]]; k--) {
            int t = ord[k]; ord[k] = ord[k - 1]; ord[k - 1] = t;
        }
    for (int j = 0; j < (m < n ? m : n); j++) s[j] = sv[ord[j]];
    for (int i = 0; i < n; i++)
        for (int r = 0; r < nrhs; r++) {
            if (layout == LAPACK_ROW_MAJOR) b[(size_t) i * ldb + r] = CM(x, n, i, r);
            else b[(size_t) r * ldb + i] = CM(x, n, i, r);
        }
    if (rank) *rank = kept;
    free(u), free(v), free(bc), free(sv), free(x), free(ord);
    return 0;
}

lapack_int LAPACKE_dgesdd(int layout, char jobz, lapack_int m, lapack_int n, double *a, lapack_int lda, double *s,
                          double *u, lapack_int ldu, double *vt, lapack_int ldvt) {
    (void) layout, (void) jobz, (void) m, (void) n, (void) a, (void) lda, (void) s, (void) u, (void) ldu,
            (void) vt, (void) ldvt;
    return unavailable("LAPACKE_dgesdd");
}
lapack_int LAPACKE_dgesdd_work(int layout, char jobz, lapack_int m, lapack_int n, double *a, lapack_int lda,
                               double *s, double *u, lapack_int ldu, double *vt, lapack_int ldvt, double *work,
                               lapack_int lwork, lapack_int *iwork) {
    (void) layout, (void) jobz, (void) m, (void) n, (void) a, (void) lda, (void) s, (void) u, (void) ldu,
            (void) vt, (void) ldvt, (void) work, (void) lwork, (void) iwork;
    return unavailable("LAPACKE_dgesdd_work");
}
lapack_int LAPACKE_dgesvd(int layout, char jobu, char jobvt, lapack_int m, lapack_int n, double *a, lapack_int lda,
                          double *s, double *u, lapack_int ldu, double *vt, lapack_int ldvt, double *superb) {
    (void) layout, (void) jobu, (void) jobvt, (void) m, (void) n, (void) a, (void) lda, (void) s, (void) u,
            (void) ldu, (void) vt, (void) ldvt, (void) superb;
    return unavailable("LAPACKE_dgesvd");
}

void cblas_dgemm(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE ta, enum CBLAS_TRANSPOSE tb, int m, int n, int k,
                 double alpha, const double *a, int lda, const double *b, int ldb, double beta, double *c, int ldc) {
    for (int i = 0; i < m; i++)
        for (int j = 0; j < n; j++) {
            double s = 0.0;
            for (int p = 0; p < k; p++) {
                double av, bv;
                if (order == CblasRowMajor) {
                    av = (ta == CblasNoTrans) ? a[(size_t) i * lda + p] : a[(size_t) p * lda + i];
                    bv = (tb == CblasNoTrans) ? b[(size_t) p * ldb + j] : b[(size_t) j * ldb + p];
                } else {
                    av = (ta == CblasNoTrans) ? a[(size_t) p * lda + i] : a[(size_t) i * lda + p];
                    bv = (tb == CblasNoTrans) ? b[(size_t) j * ldb + p] : b[(size_t) p * ldb + j];
                }
                s += av * bv;
            }
            double *cij = (order == CblasRowMajor) ? &c[(size_t) i * ldc + j] : &c[(size_t) j * ldc + i];
            *cij        = alpha * s + (beta == 0.0 ? 0.0 : beta * *cij);
        }
}
