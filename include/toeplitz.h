/*
 * Drop-in Toeplitz API of midapack, B200 implementation.
 * Same names, signatures and struct layouts as the reference
 * (algebra/include/toeplitz/toeplitz.h:152-203, 257-367).  FFTW types appear
 * in tpltz_init's signature; they are declared here ABI-compatibly
 * (fftw_complex = double[2], fftw_plan = opaque pointer) so callers need no
 * FFTW.  The spectra live on the GPU and are built once per Tpltz.
 */
#ifndef MDP_DROPIN_TOEPLITZ_H
#define MDP_DROPIN_TOEPLITZ_H

#include <stdint.h>

#include "mdp_mpi_compat.h"

#ifdef __cplusplus
extern "C" {
#endif

#ifndef FFTW3_H
typedef double fftw_complex[2];
typedef struct mdp_fftw_plan_s *fftw_plan;
#endif

/* toeplitz.h:152-167 */
typedef struct {
    int64_t idv;
    double *T_block;
    int     lambda;
    int     n;
} Block;

/* toeplitz.h:169-182 */
typedef struct {
    int flag_bs;
    int flag_nfft;
    int flag_fftw;
    int flag_no_rshp;
    int flag_nofft;
    int flag_blockingcomm;
    int fixed_nfft;
    int fixed_bs;
    int flag_verbose;
    int flag_skip_build_gappy_blocks;
    int flag_param_distmin_fixed;
    int flag_precompute_lvl;
} Flag;

/* toeplitz.h:184-188 */
typedef struct {
    int64_t *id0gap;
    int     *lgap;
    int      ngap;
} Gap;

/* toeplitz.h:190-203 */
typedef struct {
    int64_t  nrow;
    int      m_cw;
    int      m_rw;
    Block   *tpltzblocks;
    int      nb_blocks_loc;
    int      nb_blocks_tot;
    int64_t  idp;
    int      local_V_size;
    Flag     flag_stgy;
    MPI_Comm comm;
} Tpltz;

/* toeplitz.h:257-260 -> toeplitz.c:298-367.  Computes blocksize (define_blocksize,
 * toeplitz.c:168-253), nfft = 1 and the circulant spectrum T_fft (bs/2+1 complex,
 * host memory from malloc); V_fft/V_rfft are allocated, plans are opaque handles. */
int tpltz_init(int n, int lambda, int *nfft, int *blocksize, fftw_complex **T_fft, double *T,
               fftw_complex **V_fft, double **V_rfft, fftw_plan *plan_f, fftw_plan *plan_b, Flag flag_stgy);
/* toeplitz.h:262-263 -> toeplitz.c:485-498 */
int tpltz_cleanup(fftw_complex **T_fft, fftw_complex **V_fft, double **V_rfft, fftw_plan *plan_f,
                  fftw_plan *plan_b);
/* toeplitz.h:315 -> toeplitz_params.c (flag_stgy_init_auto) */
int flag_stgy_init_auto(Flag *flag_stgy);
int flag_stgy_init_zeros(Flag *flag_stgy);
/* toeplitz.h:321 -> toeplitz.c:168-253 */
int define_blocksize(int n, int lambda, int bs_flag, int fixed_bs);
/* toeplitz.h:365 -> toeplitz_wizard.c:80-111: V <- N^-1 V in place (block mean removal + banded Toeplitz) */
int stbmmProd(Tpltz *Nm1, double *V);

#ifdef __cplusplus
}
#endif
#endif
