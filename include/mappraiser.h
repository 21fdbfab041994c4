/*
 * Drop-in MAPPRAISER API (GLS map-making), B200 implementation.
 * Same names and signatures as the reference:
 *   mappraiser/include/mappraiser/map.h:10-18          MLmap, MTmap
 *   mappraiser/include/mappraiser/pcg_true.h:8-12      get_pixshare_pond, PCG_GLS_true
 *   mappraiser/include/mappraiser/precond.h:6-35       Precond, build_precond, apply_precond, free_precond,
 *                                                      precondblockjacobilike
 *   mappraiser/include/mappraiser/create_toeplitz.h    defineTpltz_avg, defineBlocks_avg
 *   mappraiser/include/mappraiser/ecg.h:6-7            ECG_GLS
 *   mappraiser/include/mappraiser/iofiles.h:24         write_map
 * Scope: solver 0 (PCG) with precond 0 (block Jacobi), 1 and 2 (two-level),
 * solver 1 (ECG, block Jacobi), on one GPU; MTmap with solver 0, precond 0.
 * Other solver/precond values return an error (MLmap/MTmap print it and return).
 */
#ifndef MDP_DROPIN_MAPPRAISER_H
#define MDP_DROPIN_MAPPRAISER_H

#include "mapmat.h"
#include "toeplitz.h"

#ifdef __cplusplus
extern "C" {
#endif

/* precond.h:6-22 */
typedef struct {
    int      precond;
    int      n;
    int      Zn;
    Mat      BJ_inv;
    Mat      BJ;
    double  *pixpond;
    double **Z;
    double **AZ;
    double  *Em1;
    double  *Qg;
    double  *AQg;
    double  *Qtx;
    double  *w;
} Precond;

/* create_toeplitz.c:10-25 */
int defineTpltz_avg(Tpltz *Nm1, int64_t nrow, int m_cw, int m_rw, Block *tpltzblocks, int nb_blocks_loc,
                    int nb_blocks_tot, int64_t idp, int local_V_size, Flag flag_stgy, MPI_Comm comm);
/* create_toeplitz.c:27-47 */
int defineBlocks_avg(Block *tpltzblocks, double *T, int nb_blocks_loc, void *local_blocks_sizes, int lambda_block_avg,
                     int64_t id0);

/* precond.c:456-702 */
int  precondblockjacobilike(Mat *A, Tpltz *Nm1, Mat *BJ_inv, Mat *BJ, double *b, double *cond, int *lhits);
/* precond.c:1310-1400 (precond 0 only) */
void build_precond(Precond **out_p, double **out_pixpond, int *out_n, Mat *A, Tpltz *Nm1, double **in_out_x,
                   double *b, double *noise, double *cond, int *lhits, double tol, int Zn, int precond);
/* precond.c:1403-1423 */
void apply_precond(Precond *p, const Mat *A, Tpltz *Nm1, double *g, double *Cg);
/* precond.c:1426-1455 */
void free_precond(Precond **in_out_p);
/* precond.c:432-444; one GPU: every pixel has weight 1 */
void get_pixshare_pond(Mat *A, double *pixpond);
/* pcg_true.c:578-600 */
int  apply_weights(Tpltz *Nm1, double *tod);

/* pcg_true.h:11-12 -> pcg_true.c:20-241 (precond 0, 1, 2) */
int PCG_GLS_true(char *outpath, char *ref, Mat *A, Tpltz *Nm1, double *x, double *b, double *noise, double *cond,
                 int *lhits, double tol, int K, int precond, int Z_2lvl);

/* ecg.h:6-7 -> ecg.c:44-175 (enlarged CG; the preAlps iteration restated) */
int ECG_GLS(char *outpath, char *ref, Mat *A, Tpltz *Nm1, double *x, double *b, double *noise, double *cond,
            int *lhits, double tol, int maxIter, int enlFac, int ortho_alg, int bs_red);

/* map.h:10-13 -> mappraiser.c:34-385 (solver 0 with precond 0, 1, 2; solver 1).  Writes the
 * I, Q, U, Cond and Hits maps (12*nside^2 entries each) to
 * outpath/{mapI,mapQ,mapU,Cond,Hits}_<ref>.fits as HEALPix binary tables. */
void MLmap(MPI_Comm comm, char *outpath, char *ref, int solver, int precond, int Z_2lvl, int pointing_commflag,
           double tol, int maxiter, int enlFac, int ortho_alg, int bs_red, int nside, void *data_size_proc,
           int nb_blocks_loc, void *local_blocks_sizes, int Nnz, void *pix, void *pixweights, void *signal,
           double *noise, int lambda, double *invtt);

/* map.h:15-18: MLmap with per-block template amplitudes marginalised
 * (PCG_GLS_templates, pcg_true.c:243-560): Legendre polynomials per sweep,
 * azimuth-binned ground signal, HWP harmonics; white noise per block (invtt: one
 * weight per block).  Here: solver 0 with precond 0, one rank, every block as long
 * as its CES (sweeptstamps[i][nsweeps[i]] samples), detector-minor within a CES. */
void MTmap(MPI_Comm comm, char *outpath, char *ref, int solver, int precond, int Z_2lvl, int pointing_commflag,
           int npoly, int nhwp, double delta_t, int ground, int n_sss_bins, double tol, int maxiter, int enlFac,
           int ortho_alg, int bs_red, int nside, int **sweeptstamps, int *nsweeps, double **az, double *az_min,
           double *az_max, double **hwp_angle, int nces, void *data_size_proc, int nb_blocks_loc,
           void *local_blocks_sizes, int Nnz, void *pix, void *pixweights, void *signal, double *noise,
           double sampling_freq, double *invtt);

/* iofiles.h:24 -> iofiles.c:19-52: one HEALPix map (12*nside^2 values of type
 * 82 = TDOUBLE or 31 = TINT, CFITSIO's codes) as a FITS binary table with one
 * column SIGNAL of 8-byte doubles (integers converted, as CFITSIO converts them),
 * ORDERING NESTED (nest != 0) or RING, COORDSYS from coordsys[0].  Written by
 * the library itself (CFITSIO is not needed). */
void write_map(void *signal, int type, long nside, const char *filename, char nest, const char *coordsys);

/* Extension (no reference counterpart): MLmap's solve with the maps returned in
 * caller buffers (12*nside^2 each, any may be NULL) instead of files, and the
 * iteration count / final relative residual.  Inputs are not modified.
 * Returns 0 on success or an MDP_E* code. */
int MLmap_b200(int solver, int precond, double tol, int maxiter, int nside, int m, int nb_blocks_loc,
               const int *local_blocks_sizes, int Nnz, const int *pix, const double *pixweights, const double *signal,
               const double *noise, int lambda, const double *invtt, double *mapI, double *mapQ, double *mapU,
               double *Cond, int *Hits, int *iterations, double *res_rel);

#ifdef __cplusplus
}
#endif
#endif
