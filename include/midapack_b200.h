/*
 * midapack_b200 device-level C API.
 *
 * The GLS map-making hot path (P^T N^-1 P) m = P^T N^-1 d on one B200, on
 * device-resident data: every pointer named d_* is device memory owned by the
 * caller, every h_* pointer is host memory.  The reference-compatible API
 * (MatInit, MatVecProd, TrMatVecProd, stbmmProd, PCG_GLS_true, MLmap; host
 * pointers) is declared in mapmat.h, toeplitz.h and mappraiser.h and is built
 * on top of this one.
 *
 * All functions return 0 (MDP_OK) or an MDP_E* code; mdp_last_error() gives a
 * one-line description of the last failure on the calling thread.  Work is
 * queued on the context's stream; functions that return host-visible results
 * synchronise that stream.
 */
#ifndef MIDAPACK_B200_H
#define MIDAPACK_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MDP_OK           0
#define MDP_EINVAL       1 /* bad argument (size, pointer, index out of range) */
#define MDP_ENOMEM       2 /* device or host allocation failed */
#define MDP_ECUDA        3 /* CUDA runtime error */
#define MDP_EUNSUPPORTED 4 /* valid input this build does not handle */
#define MDP_ENAN         5 /* NaN/Inf met in a reduction */
#define MDP_ETIMEOUT     6 /* a bounded device-side wait gave up */
#define MDP_ENOCONV      7 /* an iterative fit did not converge within its evaluation limit */

typedef struct mdp_context  mdp_context;
typedef struct mdp_pointing mdp_pointing;
typedef struct mdp_noise    mdp_noise;

const char *mdp_strerror(int code);
const char *mdp_last_error(void);

/* ---- context: one device, one stream ---------------------------------- */
int      mdp_context_create(int device, mdp_context **out);
void     mdp_context_destroy(mdp_context *ctx);
/* The solves keep their work buffers (TOD- and map-sized) in the context for
 * its next solve, so that repeated solves do not cudaMalloc/cudaFree (which
 * synchronise the device); mdp_context_trim frees them (after synchronising
 * the context's stream). */
int      mdp_context_trim(mdp_context *ctx);
/* queue work on an existing cudaStream_t (e.g. the caller's; pass cudaStreamLegacy,
 * i.e. (void *) 1, for the legacy default stream); NULL = a stream of its own */
int      mdp_context_set_stream(mdp_context *ctx, void *cuda_stream);
void    *mdp_context_stream(mdp_context *ctx);
int      mdp_synchronize(mdp_context *ctx);
/* number of kernels this library launched on ctx since creation */
uint64_t mdp_launch_count(const mdp_context *ctx);
/* per-operator timing of PCG iterations (CUDA events on the context stream):
 * enable = 1 starts (and zeroes) the counters; ms[4]/count[4] receive the
 * accumulated milliseconds and launches of P, N^-1, P^T and the fused
 * vector/dot kernels. */
int      mdp_profile_enable(mdp_context *ctx, int enable);
int      mdp_profile_read(const mdp_context *ctx, double *ms, int64_t *count);

/* ---- pointing matrix P (reference: Mat, algebra/include/mapmat/mapmat.h:46-69) ----
 * m rows (time samples), nnz entries per row, global column indices d_gindices
 * [m*nnz] (int32, e.g. 3*pixel+stokes, negative = flagged) and weights
 * d_values [m*nnz].  Creation compresses the indices exactly as MatInit /
 * MatLocalShape do (sorted unique set, position = local index, trash pixel
 * when the smallest index is negative).  d_values is borrowed, not copied: it
 * must stay valid while the pointing exists. */
int  mdp_pointing_create(mdp_context *ctx, int64_t m, int nnz, const int32_t *d_gindices,
                         const double *d_values, mdp_pointing **out);
void mdp_pointing_destroy(mdp_pointing *A);
/* lcount = #unique indices, n_map = lcount - nnz*trash_pix (map-domain size) */
int  mdp_pointing_shape(const mdp_pointing *A, int64_t *lcount, int *trash_pix, int64_t *n_map,
                        int *triplet_layout);
int  mdp_pointing_lindices(mdp_context *ctx, const mdp_pointing *A, int32_t *d_lindices);
int  mdp_pointing_local_indices(mdp_context *ctx, const mdp_pointing *A, int32_t *d_local);
/* y[m] = P x[n_map]          (reference MatVecProd, mapmat.c:704-729) */
int  mdp_matvec(mdp_context *ctx, const mdp_pointing *A, const double *d_x, double *d_y);
/* x[n_map] = P^T y[m]        (reference TrMatVecProd, mapmat.c:819-859) */
int  mdp_trmatvec(mdp_context *ctx, const mdp_pointing *A, const double *d_y, double *d_x);

/* ---- inverse noise N^-1: block-diagonal banded symmetric Toeplitz --------
 * (reference: Tpltz/Block, algebra/include/toeplitz/toeplitz.h:152-203)
 * Block b covers rows [h_idv[b], h_idv[b] + h_n[b]) and its first row is
 * h_T[b*lambda .. b*lambda+lambda).  Spectra are computed once here. */
int  mdp_noise_create(mdp_context *ctx, int nb_blocks, const int64_t *h_idv, const int32_t *h_n,
                      int lambda, const double *h_T, mdp_noise **out);
void mdp_noise_destroy(mdp_noise *N);
/* out = N^-1 in: per block, subtract the block mean then apply the banded
 * Toeplitz block (reference stbmmProd, toeplitz_wizard.c:80-111; with
 * lambda == 1 the diagonal scaling of apply_weights, pcg_true.c:578-600).
 * in == out is allowed. */
int  mdp_stbmm(mdp_context *ctx, const mdp_noise *N, const double *d_in, double *d_out);
int  mdp_noise_tile(const mdp_noise *N, int *fft_size, int *cluster_ctas, int64_t *n_tiles);
/* FP32 variant of mdp_stbmm (the operator of the mixed-precision solver):
 * FP32 input/output, FP32 spectra and FFTs, block means accumulated in FP64.
 * d_in != d_out required. */
int  mdp_stbmm_fp32(mdp_context *ctx, mdp_noise *N, const float *d_in, float *d_out);
/* FP32 tile plan (builds it on first use) */
int  mdp_noise_tile_fp32(mdp_context *ctx, mdp_noise *N, int *fft_size, int *cluster_ctas, int64_t *n_tiles);
/* No counterpart in the reference.  Builds the FP32 operator state of the
 * mixed-precision solves ahead of them (FP32 weights of A, FP32 tile plan and
 * spectra of N), which they otherwise build on first use. */
int  mdp_prepare_fp32(mdp_context *ctx, mdp_pointing *A, mdp_noise *N);
/* Launch shape of a tile plan (fp32 = 0: FP64 tiles, 1: FP32 tiles, built on
 * first use): 2^log2_cta_points complex points per CTA, CTAs per cluster,
 * threads per CTA, and whether the autotuner picked it (1) by timing the
 * candidate plans on this device, or the cost model did (0).  A split plan
 * (three kernels, four-step FFT of 2^split_log_m1 x 2^split_log_m2 points)
 * reports split_log_m1 > 0 and cluster 0; a cluster four-step plan (one
 * cluster of C CTAs per tile, 2C x 4096 points, the tile on chip) reports
 * split_log_m1 = log2(2C), split_log_m2 = 12 and cluster C.  The autotuner runs
 * once per precision, band (ceil log2 lambda) and block length class. */
int  mdp_noise_plan(mdp_context *ctx, mdp_noise *N, int fp32, int *log2_cta_points, int *cluster_ctas,
                    int *threads, int *tuned, int *split_log_m1, int *split_log_m2);
/* No counterpart in the reference.  Replaces the tile plan of one precision
 * (fp32 = 0: the FP64 operator, 1: the FP32 operator of the mixed solves):
 * "auto" (the autotuner's choice), "model" (the cost model's choice, nothing
 * timed), "fft:N" (the cost model's choice among one-kernel tiles of N real
 * samples), "log2_cta_points,cluster,threads" (one-kernel tiles),
 * "s,log_m1,log_m2" (three-kernel split tiles) or "c,C" (cluster four-step
 * tiles of C CTAs).  For tests and tuning; MDP_EINVAL when the plan does not
 * hold the band. */
int  mdp_noise_set_plan(mdp_context *ctx, mdp_noise *N, int fp32, const char *plan);
/* No counterpart in the reference.  out = N^-1 in like mdp_stbmm, but the call
 * allocates no device memory: for callers that cannot call cudaMalloc while
 * they apply the operator (a memory arena or pool that owns the device memory,
 * a solve loop that must not synchronise the device through cudaMalloc/cudaFree,
 * a plugin that may only touch buffers its host gives it).  The block-mean
 * scratch lives in a fixed 1 MiB device array (131072 doubles) that the library
 * keeps on every device it is loaded on until the process exits; a noise
 * operator needing more (one double per block plus one per 65536-row chunk of
 * every block) is rejected with MDP_EINVAL, as is d_in == d_out.  The first
 * call on a device looks up that array's device address (once per device), so
 * make the first call before any stream capture.  The cached address belongs
 * to the device's primary context (the runtime's): calls from another context
 * on that device, or after cudaDeviceReset, are not supported.  All calls
 * share the array: calls that overlap on the GPU (other streams, other
 * threads) race on it and must be serialised by the caller. */
int  mdp_stbmm_noalloc(mdp_context *ctx, const mdp_noise *N, const double *d_in, double *d_out);

/* ---- GLS solve (reference PCG_GLS_true, pcg_true.c:20-241) ---- */
typedef struct {
    double tol;      /* relative residual: stop when sum(g^2) <= tol^2 sum(g0^2) */
    int    maxiter;  /* K: at most K-1 iterations, as the reference */
    int    verbose;  /* 1: print the reference's per-iteration line on stdout */
    int    precond;  /* 0: block Jacobi; 1: two-level a priori (build_Z); 2: two-level
                        a posteriori (Lanczos Ritz vectors); precond.c:1310-1423.
                        mdp_gls_solve and mdp_gls_solve_mixed (there the deflation
                        columns are built with the FP64 operator and precondition
                        the inner FP32-operator PCGs) */
    int    z_2lvl;   /* deflation columns of the two-level preconditioners, 1..128
                        (0: one, the reference's default of one per rank) */
} mdp_solve_params;

typedef struct {
    int     iterations;    /* k at exit (the reference's loop index) */
    int     converged;
    double  res0, res;     /* sum(g0^2) and final sum(g^2) */
    int64_t n_map;         /* unknowns after the rcond cut */
    int64_t n_cut;         /* pixels removed by the rcond cut */
    double  precond_seconds, solve_seconds;
    int     outer_iterations;   /* mixed precision: refinement steps (FP64 residuals) */
    int     fp64_applications;  /* operator applications in FP64 */
} mdp_solve_info;

/* Builds the block-Jacobi preconditioner (rcond > 0.1 cut, exactly as
 * precondblockjacobilike, precond.c:456-702; A is updated in place to the
 * post-cut pointing) and solves with x0 = 0.  Outputs (device, capacity
 * n_map of A before the cut, i.e. mdp_pointing_shape's n_map):
 *   d_x      solution, n_map entries after the cut
 *   d_lstid  global index of each solution entry (lindices minus trash)
 *   d_cond   rcond of each kept pixel (n_map/3)
 *   d_hits   hit count of each kept pixel (n_map/3)
 * h_res_rel (optional, maxiter+1 entries) receives sqrt(res/res0) per iteration. */
int mdp_gls_solve(mdp_context *ctx, mdp_pointing *A, const mdp_noise *N, const double *d_signal,
                  const double *d_noise, const mdp_solve_params *params, double *d_x, int32_t *d_lstid,
                  double *d_cond, int32_t *d_hits, double *h_res_rel, mdp_solve_info *info);

/* ---- ECG solve (reference ECG_GLS, mappraiser/src/ecg.c:44-175, solver 1) ----
 * Enlarged conjugate gradient with enl_fac search directions per iteration
 * (the residual split over enl_fac contiguous ranges of the map's pixels),
 * block-Jacobi preconditioner and rcond cut as mdp_gls_solve, Orthomin
 * (ortho_alg 1) or Orthodir (ortho_alg 0) block recurrences, A-orthonormal
 * blocks by Cholesky or, with bs_red = 1, by eigenvectors with the block
 * shrinking when it loses rank; stops when ||r|| < tol ||r0||.  FP64.
 * Outputs as mdp_gls_solve; h_res_rel (maxiter+1 entries) receives ||r||/||r0||. */
#define MDP_ECG_MAX_ENL 64
typedef struct {
    double tol;
    int    maxiter;
    int    enl_fac;    /* 1..MDP_ECG_MAX_ENL */
    int    ortho_alg;  /* 0: Orthodir, 1: Orthomin */
    int    bs_red;     /* 1: adaptive block size */
    int    verbose;
} mdp_ecg_params;
int mdp_ecg_solve(mdp_context *ctx, mdp_pointing *A, const mdp_noise *N, const double *d_signal,
                  const double *d_noise, const mdp_ecg_params *params, double *d_x, int32_t *d_lstid,
                  double *d_cond, int32_t *d_hits, double *h_res_rel, mdp_solve_info *info);

/* Mixed precision: the same solve as mdp_gls_solve (same preconditioner, cut
 * and stop test on the FP64 residual sum(g^2) <= tol^2 sum(g0^2)), computed as
 * FP64 iterative refinement.  Each step recomputes g = P^T N^-1 (d - P x) in
 * FP64, then solves A delta = g approximately with block-Jacobi PCG whose
 * operator P^T N^-1 P runs with FP32 weights, FP32 TOD and FP32 Toeplitz FFTs
 * (dot products, PCG scalars, the 3x3 blocks and the map stay FP64), until the
 * inner residual drops by inner_tol (or by the reduction still needed, with a
 * factor 2 margin, when that is smaller) or inner_maxiter iterations, and adds
 * delta to x.  info->iterations counts inner iterations; h_res_rel (optional,
 * maxiter+1 entries) receives sqrt(res/res0) after each refinement step. */
int mdp_gls_solve_mixed(mdp_context *ctx, mdp_pointing *A, const mdp_noise *N, const double *d_signal,
                        const double *d_noise, const mdp_solve_params *params, double inner_tol, int inner_maxiter,
                        double *d_x, int32_t *d_lstid, double *d_cond, int32_t *d_hits, double *h_res_rel,
                        mdp_solve_info *info);

/* No counterpart in the reference (MLmap solves one right-hand side per call).
 * Multi-RHS mixed-precision solve: nrhs right-hand sides that share A and N,
 * column r's TOD being d_r = noise_r (+ signal on column signal_col, zeroed on
 * cut samples as in MLmap).  Each column is the mdp_gls_solve_mixed solve
 * (same block-Jacobi preconditioner and cut, built once, FP64 refinement, stop
 * on sum(g^2) <= tol^2 sum(g0^2)); the inner FP32 PCGs of up to `slots`
 * columns advance together in batched iterations (one pass over the pointing
 * for all of them, their Toeplitz tiles in one launch), a column that
 * converges leaves its slot to the next column, and the batched iteration is
 * replayed as a CUDA graph (use_graph = 1).  slots = 0 times one batched
 * operator application for 1, 2, 4 and 8 slots and keeps the cheapest per
 * column.  Needs the (I,Q,U) triplet layout, lambda > 1 and noise blocks
 * covering every row.
 *   d_noise   column r at d_noise + r*noise_stride elements (float when
 *             noise_fp32 = 1, else double); FP32 values are used exactly
 *   d_signal  FP64 signal of column signal_col (signal_col < 0: none)
 *   d_x       [nrhs][n_map] solutions (n_map after the cut, as mdp_gls_solve)
 *   col_info  [nrhs] per-column iterations, refinements, convergence, res0/res */
typedef struct {
    double tol;            /* relative residual of the FP64 stop test */
    int    maxiter;        /* inner iterations per column, all refinements together */
    double inner_tol;      /* relative residual of each inner FP32 solve */
    int    inner_maxiter;  /* iterations of each inner solve */
    int    slots;          /* columns iterated together: 1, 2, 4, 8, or 0 = timed choice */
    int    use_graph;      /* 1: replay the batched iteration as a CUDA graph */
    int    verbose;
} mdp_multi_params;

typedef struct {
    int    iterations;        /* inner iterations of this column */
    int    outer_iterations;  /* FP64 refinement steps */
    int    converged;
    double res0, res;         /* sum(g^2) at x = 0 and at the end */
} mdp_multi_col_info;

typedef struct {
    int     slots;                /* columns per batched iteration */
    int     graph;                /* 1 when the iteration ran as a CUDA graph */
    int     total_iterations;     /* sum of the columns' inner iterations */
    int     batched_iterations;   /* batched iterations launched */
    int     fp64_applications;    /* FP64 operator applications (refinement residuals) */
    int64_t n_map, n_cut;
    double  precond_seconds, solve_seconds;
} mdp_multi_info;

int mdp_gls_solve_multi(mdp_context *ctx, mdp_pointing *A, const mdp_noise *N, int nrhs, const void *d_noise,
                        int noise_fp32, int64_t noise_stride, const double *d_signal, int signal_col,
                        const mdp_multi_params *params, double *d_x, int32_t *d_lstid, double *d_cond,
                        int32_t *d_hits, mdp_multi_col_info *col_info, mdp_multi_info *info);

/* ---- Pieces of a solve sharded over ranks (no counterpart in the reference,
 * whose ranks exchange through MPI inside precondblockjacobilike and
 * PCG_GLS_true).  Each rank holds the samples of some detectors/intervals;
 * the caller sums the blocks and the maps over ranks.  npix below is the
 * pointing's current pixel count, n_map/3 of mdp_pointing_shape. */
/* getlocalW (precond.c:42-161) on this rank's samples: d_W [npix][9]
 * (upper triangle and diagonal filled) and d_hits [npix], zeroed first. */
int  mdp_local_blocks(mdp_context *ctx, mdp_pointing *A, const mdp_noise *N, double *d_W, int32_t *d_hits);
/* Per 3x3 block (summed over ranks): rcond (LAPACK dgecon 1-norm estimate), the
 * inverse when rcond > 0.1, otherwise a zero block and d_cut[q] = 1
 * (precond.c:456-702).  d_W is symmetrised in place. */
int  mdp_block_inverse(mdp_context *ctx, int64_t npix, double *d_W, double *d_inv, double *d_rcond, int32_t *d_cut,
                       int64_t *n_cut);
/* The samples of every pixel q with d_target[q] != 0 become cut rows (weights
 * ignored, signal zeroed in residuals); the other pixels keep their order and
 * are renumbered; *kept_pixels gets their count. */
int  mdp_pointing_cut(mdp_context *ctx, mdp_pointing *A, const int32_t *d_target, int64_t *kept_pixels);
/* d_r = P^T N^-1 (d - P x), d = signal (zero on cut rows) + noise; d_x may be
 * NULL for x = 0.  FP64. */
int  mdp_gls_residual(mdp_context *ctx, mdp_pointing *A, const mdp_noise *N, const double *d_signal,
                      const double *d_noise, const double *d_x, double *d_r);
/* d_q = P^T N^-1 P d_h (maps FP64); fp32 = 1 runs the FP32 operator of the
 * mixed-precision solver. */
int  mdp_apply_op(mdp_context *ctx, mdp_pointing *A, const mdp_noise *N, const double *d_h, double *d_q, int fp32);

/* ---- inverse-noise first rows from noise timestreams -------------------
 * compute_invtt / noise2invtt (mappraiser/python/TOAST_interface/utils.py:439-481,
 * 500-602), which the reference runs in Python (scipy) before MLmap.  Blocks are
 * consecutive in d_noise: block b has h_n[b] samples.  FP64 throughout. */
#define MDP_APOD_CHEBWIN  0   /* scipy get_window(("chebwin", 150), 2*lambda) */
#define MDP_APOD_GAUSSIAN 1   /* scipy get_window(("general_gaussian", 1, lambda/3), 2*lambda) */
/* The apodisation window after ifftshift, first lambda points (utils.py:567-582). */
int  mdp_apod_window(mdp_context *ctx, int lambda, int apod, double *d_window);
/* scipy.signal.welch(x_b, fsamp, window='hann', nperseg=h_n[b], detrend='linear')
 * of every block (utils.py:531): d_psd gets h_n[b]/2 + 1 values per block, blocks
 * one after the other.  h_n[b] >= 4. */
int  mdp_periodogram(mdp_context *ctx, int nb, const int32_t *h_n, const double *d_noise, double fsamp,
                     double *d_psd);
/* noise2invtt of every block: periodogram, fit of the log PSD model
 * a + log10(1 + ((f + fmin)/fknee)^alpha) under the reference's bounds and
 * starting point (bounded Levenberg-Marquardt run to the least-squares minimum),
 * inverse PSD, irfft, times the window.  d_invtt gets nb*lambda doubles (block
 * b at b*lambda); h_params (nb*4: a, alpha, fknee, fmin) and h_evals (model
 * evaluations per block, -1 when not converged) may be NULL.  Errors: MDP_EINVAL
 * when lambda > h_n[b]/2 ("Bandwidth cannot be larger than timestream") or a
 * block has fewer than 8 samples; MDP_EUNSUPPORTED when a block needs a
 * transform longer than 2^24 points (a power of two above 2^24 samples, any
 * other length above 2^23); MDP_ENAN when a periodogram value is zero or not
 * finite; MDP_ENOCONV (outputs written) when a fit used 1000 evaluations,
 * curve_fit's maxfev. */
int  mdp_noise2invtt(mdp_context *ctx, int nb, const int32_t *h_n, const double *d_noise, int lambda, double fsamp,
                     int apod, double *d_invtt, double *h_params, int32_t *h_evals);

/* ---- templates of MTmap's filtered solve: set-up (host) ------------------
 * MTmap (mappraiser/src/mappraiser.c:387-391) takes the scan as per-CES rows:
 * sweep time stamps (nsweeps[i] + 1, the last one the CES length), boresight
 * azimuth and its range, HWP angle.  Here the rows are flattened one CES after
 * the other.  Block b = i*ndet + j is detector j in CES i (ces_length(i) samples). */
typedef struct {
    int            nces, ndet;
    int            npoly;        /* Legendre orders 0..npoly-1 per sweep */
    int            ground;       /* 1: scan-synchronous signal in n_sss_bins azimuth bins */
    int            n_sss_bins;
    int            nhwp;         /* HWP harmonics (cos and sin amplitudes per delta_t) */
    double         delta_t;      /* seconds */
    double         fs;           /* sampling frequency, Hz */
    const int32_t *nsweeps;      /* [nces] */
    const int32_t *sweeps;       /* rows of nsweeps[i] + 1 stamps, sweeps[row 0] = 0 */
    const double  *az;           /* rows of ces_length(i) samples (ground = 1) */
    const double  *az_min, *az_max;   /* [nces] (ground = 1) */
    const double  *hwp;          /* rows of ces_length(i) samples (nhwp > 0) */
} mdp_template_scan;
/* The template classes of every CES in ELL form (Tlist_init + expandpolydata /
 * expandSSSdata / expandHWPSSdata, algebra/src/templates/templates.c:634-800):
 * h_bins/h_wghts [sum ces_length][n_class], n_class = npoly + ground + 2*nhwp, bins
 * numbered from 0 within a block in the reference's amplitude order (Legendre order
 * k on sweep q: k*nsweeps + q; azimuth bins; per harmonic h its cos chunks then its
 * sin chunks); h_nt [nces] (may be NULL) receives the amplitudes per block.  A
 * first stamp other than 0, a sweep of fewer than 2 samples or an azimuth below
 * az_min is MDP_EINVAL (the reference leaves such samples on a foreign bin or
 * divides by zero). */
int  mdp_template_layout(const mdp_template_scan *scan, int32_t *h_bins, double *h_wghts, int32_t *h_nt);
/* The kernels B_b = pinv(w_b T_b^T T_b) of every block (BuildKernel + InvKernel,
 * templates.c:192-418: singular values <= 1e-12 s_max dropped), block after
 * block in h_kinv (nt_i^2 doubles each, row-major); h_w_block [nces*ndet] = the
 * white-noise weight of each block (MTmap: invtt[b], lambda = 1). */
int  mdp_template_kernels(const mdp_template_scan *scan, const double *h_w_block, double *h_kinv);
/* The weighting of MTmap's PCG on the device (PCG_GLS_templates,
 * mappraiser/src/pcg_true.c:301-365, 433-462): d_out = W d_in - W T B T^T W d_in
 * with W = diag(h_w_block[b]) per block (MTmap's white N^-1, lambda = 1) and B the
 * kernels above.  TOD blocks are consecutive, block b = i*ndet + j of
 * ces_length(i) samples; d_out may be d_in.  At most 6144 amplitudes per block
 * (MDP_EUNSUPPORTED beyond).  The template amplitude sums use atomic adds, so
 * results vary in the last bits from call to call. */
typedef struct mdp_templates mdp_templates;
int  mdp_templates_create(mdp_context *ctx, const mdp_template_scan *scan, const double *h_w_block,
                          mdp_templates **out);
void mdp_templates_destroy(mdp_templates *T);
/* samples of the TOD the filter covers and its template amplitudes in total */
int  mdp_templates_samples(const mdp_templates *T, int64_t *m, int64_t *n_amplitudes);
int  mdp_templates_filter(mdp_context *ctx, const mdp_templates *T, const double *d_in, double *d_out);
/* MTmap's solve (PCG_GLS_templates, pcg_true.c:243-560): block Jacobi from the
 * white noise operator N (lambda = 1, first row = the block's weight; one block
 * per template block) with the rcond cut applied to A, then the PCG_GLS_true
 * recurrences and stop test with the weighting of mdp_templates_filter in place of
 * N^-1.  Outputs as mdp_gls_solve.  params->precond must be 0. */
int  mdp_gls_solve_templates(mdp_context *ctx, mdp_pointing *A, const mdp_noise *N, const mdp_templates *T,
                             const double *d_signal, const double *d_noise, const mdp_solve_params *params,
                             double *d_x, int32_t *d_lstid, double *d_cond, int32_t *d_hits, double *h_res_rel,
                             mdp_solve_info *info);

#ifdef __cplusplus
}
#endif

#endif /* MIDAPACK_B200_H */
