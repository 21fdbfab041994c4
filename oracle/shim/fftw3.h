/*
 * Minimal FFTW3 stand-in used ONLY to compile the reference's Toeplitz code
 * (algebra/src/toeplitz/toeplitz.c) into the test oracle.  NOT product code.
 *
 * The reference calls 8 FFTW entry points (toeplitz.c:408-470, 569-616):
 * fftw_malloc/free, fftw_plan_many_dft_r2c/c2r, fftw_plan_dft_r2c_1d,
 * fftw_execute, fftw_destroy_plan, fftw_cleanup.  They are implemented in
 * shim_fftw.c with FFTW's conventions: unnormalised transforms, r2c writes
 * n/2+1 complex outputs, c2r reads them and ignores the imaginary parts of the
 * DC and Nyquist bins.
 */
#ifndef ORACLE_SHIM_FFTW3_H
#define ORACLE_SHIM_FFTW3_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct shim_fftw_plan_s *fftw_plan;

#define FFTW_MEASURE    (0U)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_UNALIGNED  (1U << 1)
#define FFTW_EXHAUSTIVE (1U << 3)
#define FFTW_PRESERVE_INPUT (1U << 4)
#define FFTW_PATIENT    (1U << 5)
#define FFTW_ESTIMATE   (1U << 6)

void     *fftw_malloc(size_t n);
void      fftw_free(void *p);
fftw_plan fftw_plan_many_dft_r2c(int rank, const int *n, int howmany, double *in, const int *inembed,
                                 int istride, int idist, fftw_complex *out, const int *onembed,
                                 int ostride, int odist, unsigned flags);
fftw_plan fftw_plan_many_dft_c2r(int rank, const int *n, int howmany, fftw_complex *in,
                                 const int *inembed, int istride, int idist, double *out,
                                 const int *onembed, int ostride, int odist, unsigned flags);
fftw_plan fftw_plan_dft_r2c_1d(int n, double *in, fftw_complex *out, unsigned flags);
void      fftw_execute(const fftw_plan p);
void      fftw_destroy_plan(fftw_plan p);
void      fftw_cleanup(void);
int       fftw_init_threads(void);
void      fftw_plan_with_nthreads(int nthreads);
void      fftw_cleanup_threads(void);

#ifdef __cplusplus
}
#endif

#endif /* ORACLE_SHIM_FFTW3_H */
