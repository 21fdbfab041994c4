/*
 * Test-oracle FFT behind the FFTW3 API subset the reference uses (see
 * fftw3.h).  NOT product code.
 *
 * Power-of-two sizes use a real FFT packed into a half-size complex FFT
 * (iterative radix-2 Cooley-Tukey, twiddles computed once per plan in long
 * double); any other size falls back to a direct O(n^2) DFT accumulated in
 * long double.  Conventions follow FFTW: r2c writes n/2+1 bins, c2r is the
 * unnormalised inverse (c2r(r2c(x)) == n*x).
 */
#include "fftw3.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

struct shim_fftw_plan_s {
    int     kind; /* 0 = r2c, 1 = c2r */
    int     n, howmany, idist, odist;
    double *rin;
    double *rout;
    fftw_complex *cin;
    fftw_complex *cout;
    int     pow2;
    double *tw;   /* exp(-2 pi i k / n), k < n/2, interleaved re/im */
    int    *rev;  /* bit reversal for the n/2-point complex FFT */
    double *work; /* n doubles (n/2 complex) */
};

void *fftw_malloc(size_t n) {
    void *p = NULL;
    if (posix_memalign(&p, 64, n ? n : 1) != 0) return NULL;
    return p;
}
void fftw_free(void *p) { free(p); }
void fftw_cleanup(void) {}
int  fftw_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int nthreads) { (void) nthreads; }
void fftw_cleanup_threads(void) {}

static int is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

static void plan_tables(struct shim_fftw_plan_s *p) {
    int n = p->n;
    p->pow2 = is_pow2(n) && n >= 4;
    if (!p->pow2) return;
    int m  = n / 2;
    p->tw  = (double *) malloc(sizeof(double) * (size_t) n);
    p->rev = (int *) malloc(sizeof(int) * (size_t) m);
    p->work = (double *) fftw_malloc(sizeof(double) * (size_t) n);
    for (int k = 0; k < m; k++) {
        long double a = -2.0L * 3.14159265358979323846264338327950288L * (long double) k / (long double) n;
        p->tw[2 * k]     = (double) cosl(a);
        p->tw[2 * k + 1] = (double) sinl(a);
    }
    int bits = 0;
    while ((1 << bits) < m) bits++;
    for (int i = 0; i < m; i++) {
        int r = 0;
        for (int b = 0; b < bits; b++)
            if (i & (1 << b)) r |= 1 << (bits - 1 - b);
        p->rev[i] = r;
    }
}

/* in-place complex FFT of size m = n/2 over interleaved z; twiddle stride 2 in tw (size-n table) */
static void cfft(const struct shim_fftw_plan_s *p, double *z, int inverse) {
    int m = p->n / 2;
    for (int i = 0; i < m; i++) {
        int r = p->rev[i];
        if (r > i) {
            double t0 = z[2 * i], t1 = z[2 * i + 1];
            z[2 * i]     = z[2 * r];
            z[2 * i + 1] = z[2 * r + 1];
            z[2 * r]     = t0;
            z[2 * r + 1] = t1;
        }
    }
    double sgn = inverse ? -1.0 : 1.0;
    for (int len = 2; len <= m; len <<= 1) {
        int half = len >> 1;
        int step = (p->n / len); /* twiddle index stride in the size-n table: exp(-2pi i j / len) */
        for (int base = 0; base < m; base += len) {
            for (int j = 0; j < half; j++) {
                double wr = p->tw[2 * (j * step)];
                double wi = sgn * p->tw[2 * (j * step) + 1];
                double *a = z + 2 * (base + j);
                double *b = z + 2 * (base + j + half);
                double br = b[0] * wr - b[1] * wi;
                double bi = b[0] * wi + b[1] * wr;
                b[0] = a[0] - br;
                b[1] = a[1] - bi;
                a[0] += br;
                a[1] += bi;
            }
        }
    }
}

static void r2c_one(const struct shim_fftw_plan_s *p, const double *x, fftw_complex *X) {
    int n = p->n;
    if (!p->pow2) {
        double *tmp = (double *) malloc(sizeof(double) * (size_t) n);
        memcpy(tmp, x, sizeof(double) * (size_t) n);
        for (int k = 0; k <= n / 2; k++) {
            long double sr = 0, si = 0;
            for (int j = 0; j < n; j++) {
                long double a = -2.0L * 3.14159265358979323846264338327950288L
                              * (long double) (((long long) j * k) % n) / (long double) n;
                sr += tmp[j] * cosl(a);
                si += tmp[j] * sinl(a);
            }
            X[k][0] = (double) sr;
            X[k][1] = (double) si;
        }
        free(tmp);
        return;
    }
    int     m = n / 2;
    double *z = p->work;
    memcpy(z, x, sizeof(double) * (size_t) n);
    cfft(p, z, 0);
    for (int k = 0; k <= m / 2; k++) {
        int    k2  = (m - k) % m;
        double zr  = z[2 * k], zi = z[2 * k + 1];
        double cr  = z[2 * k2], ci = -z[2 * k2 + 1]; /* conj(Z[m-k]) */
        double er  = 0.5 * (zr + cr), ei = 0.5 * (zi + ci);
        double dr  = 0.5 * (zr - cr), di = 0.5 * (zi - ci); /* (Z - conj)/2 = i * O */
        double or_ = di, oi = -dr;                         /* O = (Z - conj)/(2i) */
        double wr  = p->tw[2 * k], wi = p->tw[2 * k + 1];
        double tr  = wr * or_ - wi * oi, ti = wr * oi + wi * or_;
        double Xr = er + tr, Xi = ei + ti;
        /* mirror bin m-k: X[m-k] = conj(E[k]) - conj(w^k O[k]) * ... use symmetry of E/O */
        double er2 = er, ei2 = -ei;   /* E[m-k] = conj(E[k]) */
        double or2 = or_, oi2 = -oi;  /* O[m-k] = conj(O[k]) */
        int    km  = m - k;
        double w2r = (km < m) ? p->tw[2 * km] : -1.0, w2i = (km < m) ? p->tw[2 * km + 1] : 0.0;
        double t2r = w2r * or2 - w2i * oi2, t2i = w2r * oi2 + w2i * or2;
        X[k][0] = Xr;
        X[k][1] = Xi;
        X[km][0] = er2 + t2r;
        X[km][1] = ei2 + t2i;
    }
}

static void c2r_one(const struct shim_fftw_plan_s *p, const fftw_complex *Xin, double *x) {
    int n = p->n;
    if (!p->pow2) {
        int           h   = n / 2;
        fftw_complex *tmp = (fftw_complex *) malloc(sizeof(fftw_complex) * (size_t) (h + 1));
        memcpy(tmp, Xin, sizeof(fftw_complex) * (size_t) (h + 1));
        for (int j = 0; j < n; j++) {
            long double s = 0;
            for (int k = 0; k < n; k++) {
                double xr, xi;
                if (k <= h) {
                    xr = tmp[k][0];
                    xi = tmp[k][1];
                } else {
                    xr = tmp[n - k][0];
                    xi = -tmp[n - k][1];
                }
                if (k == 0 || (n % 2 == 0 && k == h)) xi = 0.0;
                long double a = 2.0L * 3.14159265358979323846264338327950288L
                              * (long double) (((long long) j * k) % n) / (long double) n;
                s += xr * cosl(a) - xi * sinl(a);
            }
            x[j] = (double) s;
        }
        free(tmp);
        return;
    }
    int     m = n / 2;
    double *z = p->work;
    for (int k = 0; k < m; k++) {
        double Xr = Xin[k][0], Xi = (k == 0) ? 0.0 : Xin[k][1];
        int    km = m - k;
        double Yr = Xin[km][0], Yi = (km == m || km == 0) ? 0.0 : Xin[km][1];
        if (k == 0) {
            Yr = Xin[m][0];
            Yi = 0.0;
        }
        double cr = Yr, ci = -Yi; /* conj(X[m-k]) */
        double Er = Xr + cr, Ei = Xi + ci;       /* 2 E[k] */
        double Dr = Xr - cr, Di = Xi - ci;       /* 2 w^k O[k] */
        double wr = p->tw[2 * k], wi = -p->tw[2 * k + 1]; /* conj(w^k) = 1/w^k */
        double Or = Dr * wr - Di * wi, Oi = Dr * wi + Di * wr; /* 2 O[k] */
        z[2 * k]     = Er - Oi; /* 2(E + i O) */
        z[2 * k + 1] = Ei + Or;
    }
    cfft(p, z, 1);
    memcpy(x, z, sizeof(double) * (size_t) n);
}

fftw_plan fftw_plan_many_dft_r2c(int rank, const int *n, int howmany, double *in, const int *inembed,
                                 int istride, int idist, fftw_complex *out, const int *onembed,
                                 int ostride, int odist, unsigned flags) {
    (void) rank;
    (void) inembed;
    (void) istride;
    (void) onembed;
    (void) ostride;
    (void) flags;
    struct shim_fftw_plan_s *p = calloc(1, sizeof(*p));
    p->kind    = 0;
    p->n       = n[0];
    p->howmany = howmany;
    p->idist   = idist;
    p->odist   = odist;
    p->rin     = in;
    p->cout    = out;
    plan_tables(p);
    return p;
}

fftw_plan fftw_plan_many_dft_c2r(int rank, const int *n, int howmany, fftw_complex *in,
                                 const int *inembed, int istride, int idist, double *out,
                                 const int *onembed, int ostride, int odist, unsigned flags) {
    (void) rank;
    (void) inembed;
    (void) istride;
    (void) onembed;
    (void) ostride;
    (void) flags;
    struct shim_fftw_plan_s *p = calloc(1, sizeof(*p));
    p->kind    = 1;
    p->n       = n[0];
    p->howmany = howmany;
    p->idist   = idist;
    p->odist   = odist;
    p->cin     = in;
    p->rout    = out;
    plan_tables(p);
    return p;
}

fftw_plan fftw_plan_dft_r2c_1d(int n, double *in, fftw_complex *out, unsigned flags) {
    return fftw_plan_many_dft_r2c(1, &n, 1, in, NULL, 1, n, out, NULL, 1, n / 2 + 1, flags);
}

void fftw_execute(const fftw_plan p) {
    for (int b = 0; b < p->howmany; b++) {
        if (p->kind == 0) {
            /* copy first: the reference runs in-place r2c (toeplitz.c:455-466) */
            double *tmp = (double *) malloc(sizeof(double) * (size_t) p->n);
            memcpy(tmp, p->rin + (size_t) b * p->idist, sizeof(double) * (size_t) p->n);
            r2c_one(p, tmp, p->cout + (size_t) b * p->odist);
            free(tmp);
        } else {
            c2r_one(p, p->cin + (size_t) b * p->idist, p->rout + (size_t) b * p->odist);
        }
    }
}

void fftw_destroy_plan(fftw_plan p) {
    if (!p) return;
    free(p->tw);
    free(p->rev);
    fftw_free(p->work);
    free(p);
}
