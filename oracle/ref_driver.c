/*
 * Test-oracle driver: thin C entry points around the reference's own
 * operators, compiled together with the unmodified reference sources into
 * oracle/_ref/libmidapack_ref.so by oracle/build_ref.sh.  NOT product code;
 * only tests/, the smoke check and bench.py's CPU-baseline leg load it.
 *
 * Each entry point reproduces the call sequence of the reference caller it
 * names, so a test compares against exactly what MAPPRAISER would compute:
 *   ref_local_shape   MatInit -> MatLocalShape   (algebra/src/mapmat/mapmat.c:54-73,496-521)
 *   ref_matvec        MatVecProd                 (mapmat.c:704-729)
 *   ref_trmatvec      TrMatVecProd               (mapmat.c:819-859)
 *   ref_stbmm         defineBlocks_avg/defineTpltz_avg + stbmmProd
 *                     (mappraiser/src/create_toeplitz.c:10-47, toeplitz_wizard.c:80-111)
 *   ref_pcg           MLmap's set-up (mappraiser.c:64-200) + PCG_GLS_true (pcg_true.c:20-241)
 *   ref_mlmap         MLmap on n forked ranks (mappraiser.c:34-385)
 *   ref_operator_time one A = P^T N^-1 P application, timed (CPU baseline)
 *   ref_templates_ops MTmap's template classes (Tlist_init) + TrTVecProd, TVecProd,
 *                     BuildKernel, InvKernel (algebra/src/templates/templates.c)
 *   ref_mtmap         MTmap on one rank (mappraiser.c:387-800, PCG_GLS_templates)
 */
#include <math.h>
#include <mpi.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mappraiser/create_toeplitz.h"
#include "mappraiser/map.h"
#include "mappraiser/pcg_true.h"
#include "mappraiser/precond.h"
#include "midapack.h"

int apply_weights(Tpltz *Nm1, double *tod);

/* indices: in = global, out = local (in place, as MatInit does). Returns lcount. */
int ref_local_shape(int m, int nnz, int *indices, double *values, int *lindices_out, int cap, int *trash_pix) {
    Mat A;
    memset(&A, 0, sizeof(A));
    A.trash_pix = 0;
    MatInit(&A, m, nnz, indices, values, ALLREDUCE, MPI_COMM_WORLD);
    int lc = A.lcount;
    if (lindices_out) memcpy(lindices_out, A.lindices, sizeof(int) * (size_t) (lc < cap ? lc : cap));
    *trash_pix = A.trash_pix;
    MatFree(&A);
    return lc;
}

static void build_mat(Mat *A, int m, int nnz, int *gindices, double *values) {
    memset(A, 0, sizeof(*A));
    A->trash_pix = 0;
    MatInit(A, m, nnz, gindices, values, ALLREDUCE, MPI_COMM_WORLD);
}

/* y = P x; gindices are global and are rewritten in place to local indices */
int ref_matvec(int m, int nnz, int *gindices, double *values, double *x, double *y) {
    Mat A;
    build_mat(&A, m, nnz, gindices, values);
    MatVecProd(&A, x, y, 0);
    MatFree(&A);
    return 0;
}

/* x = P^T y */
int ref_trmatvec(int m, int nnz, int *gindices, double *values, double *y, double *x) {
    Mat A;
    build_mat(&A, m, nnz, gindices, values);
    TrMatVecProd(&A, y, x, 0);
    MatFree(&A);
    return 0;
}

static void build_tpltz(Tpltz *Nm1, Block **blocks, int nb_blocks, int *block_sizes, int lambda, double *invtt,
                        int64_t nrow) {
    Flag flag_stgy;
    flag_stgy_init_auto(&flag_stgy);
    flag_stgy.flag_verbose = 0;
    *blocks = (Block *) malloc(sizeof(Block) * (size_t) nb_blocks);
    defineBlocks_avg(*blocks, invtt, nb_blocks, block_sizes, lambda, 0);
    defineTpltz_avg(Nm1, nrow, 1, 1, *blocks, nb_blocks, nb_blocks, 0, (int) nrow, flag_stgy, MPI_COMM_WORLD);
}

/* V <- N^-1 V in place (mean removal + banded Toeplitz per block), as apply_weights does */
int ref_stbmm(int nb_blocks, int *block_sizes, int lambda, double *invtt, double *V) {
    int64_t nrow = 0;
    for (int i = 0; i < nb_blocks; i++) nrow += block_sizes[i];
    Tpltz  Nm1;
    Block *blocks;
    build_tpltz(&Nm1, &blocks, nb_blocks, block_sizes, lambda, invtt, nrow);
    apply_weights(&Nm1, V);
    free(blocks);
    return 0;
}

/* Replicates MLmap's pixel-to-time linked list (mappraiser.c:110-145). */
static void build_ll(Mat *A, int m) {
    int nvalid = A->lcount - (A->trash_pix ? A->nnz : 0);
    A->id_last_pix = (int *) malloc(sizeof(int) * (size_t) (nvalid / A->nnz > 0 ? nvalid / A->nnz : 1));
    A->ll = (int *) malloc(sizeof(int) * (size_t) (m > 0 ? m : 1));
    for (int i = 0; i < m; i++) A->ll[i] = -1;
    for (int j = 0; j < nvalid / A->nnz; j++) A->id_last_pix[j] = -1;
    for (int i = 0; i < m; i++) {
        if (!A->trash_pix || (A->trash_pix && (A->indices[i * A->nnz] != 0))) {
            int vpix_i = A->indices[i * A->nnz] / A->nnz - A->trash_pix;
            if (A->id_last_pix[vpix_i] == -1) A->id_last_pix[vpix_i] = i;
            else {
                A->ll[i]               = A->id_last_pix[vpix_i];
                A->id_last_pix[vpix_i] = i;
            }
        }
    }
}

/*
 * Single-rank GLS solve exactly as MLmap drives it (solver 0); precond 0 is
 * block Jacobi, 1 and 2 the two-level preconditioners with z_2lvl columns
 * (0: one per rank).
 * gindices/values/signal are modified in place like the reference does.
 * Outputs: x_out (capacity 3*npix_cap unknowns), lstid_out (global ids of x),
 * cond_out, hits_out; returns the number of unknowns n.
 */
int ref_pcg_precond(int m, int nnz, int *gindices, double *values, double *signal, double *noise, int nb_blocks,
                    int *block_sizes, int lambda, double *invtt, double tol, int maxiter, int precond, int z_2lvl,
                    const char *outpath, const char *ref, double *x_out, int *lstid_out, double *cond_out,
                    int *hits_out, int cap) {
    Mat A;
    build_mat(&A, m, nnz, gindices, values);
    build_ll(&A, m);
    int     nvalid = A.lcount - (A.trash_pix ? A.nnz : 0);
    double *x      = (double *) calloc((size_t) nvalid, sizeof(double));
    double *cond   = (double *) calloc((size_t) (nvalid / 3 + 1), sizeof(double));
    int    *lhits  = (int *) calloc((size_t) (nvalid / 3 + 1), sizeof(int));
    Tpltz   Nm1;
    Block  *blocks;
    build_tpltz(&Nm1, &blocks, nb_blocks, block_sizes, lambda, invtt, (int64_t) m);
    PCG_GLS_true((char *) outpath, (char *) ref, &A, &Nm1, x, signal, noise, cond, lhits, tol, maxiter, precond,
                 z_2lvl);
    int n = A.lcount - A.nnz * A.trash_pix;
    if (n > cap) n = cap;
    memcpy(x_out, x, sizeof(double) * (size_t) n);
    for (int i = 0; i < n; i++) lstid_out[i] = A.lindices[i + A.nnz * A.trash_pix];
    memcpy(cond_out, cond, sizeof(double) * (size_t) (n / 3));
    memcpy(hits_out, lhits, sizeof(int) * (size_t) (n / 3));
    MatFree(&A);
    free(x);
    free(cond);
    free(lhits);
    free(blocks);
    return n;
}

int ref_pcg(int m, int nnz, int *gindices, double *values, double *signal, double *noise, int nb_blocks,
            int *block_sizes, int lambda, double *invtt, double tol, int maxiter, const char *outpath,
            const char *ref, double *x_out, int *lstid_out, double *cond_out, int *hits_out, int cap) {
    return ref_pcg_precond(m, nnz, gindices, values, signal, noise, nb_blocks, block_sizes, lambda, invtt, tol,
                           maxiter, 0, 0, outpath, ref, x_out, lstid_out, cond_out, hits_out, cap);
}

/* ---- MLmap over forked ranks ---- */
typedef struct {
    char   *outpath, *ref;
    double  tol;
    int     maxiter, nside, nnz, lambda, nranks;
    int    *data_size_proc; /* [nranks] */
    int    *nb_blocks_proc; /* [nranks] */
    int    *block_sizes;    /* all blocks, rank-major */
    int    *pix;            /* global arrays (rank-major) */
    double *weights, *signal, *noise, *invtt;
} mlmap_args;

static void mlmap_rank(int rank, void *vp) {
    mlmap_args *a = (mlmap_args *) vp;
    int64_t     s0 = 0;
    int         b0 = 0;
    for (int r = 0; r < rank; r++) {
        s0 += a->data_size_proc[r];
        b0 += a->nb_blocks_proc[r];
    }
    int m = a->data_size_proc[rank];
    /* MLmap rewrites its inputs in place; work on private copies */
    int    *pix = (int *) malloc(sizeof(int) * (size_t) m * a->nnz);
    double *w   = (double *) malloc(sizeof(double) * (size_t) m * a->nnz);
    double *sig = (double *) malloc(sizeof(double) * (size_t) m);
    double *noi = (double *) malloc(sizeof(double) * (size_t) m);
    memcpy(pix, a->pix + s0 * a->nnz, sizeof(int) * (size_t) m * a->nnz);
    memcpy(w, a->weights + s0 * a->nnz, sizeof(double) * (size_t) m * a->nnz);
    memcpy(sig, a->signal + s0, sizeof(double) * (size_t) m);
    memcpy(noi, a->noise + s0, sizeof(double) * (size_t) m);
    MLmap(MPI_COMM_WORLD, a->outpath, a->ref, 0, 0, 0, ALLREDUCE, a->tol, a->maxiter, 0, 0, 0, a->nside,
          a->data_size_proc, a->nb_blocks_proc[rank], a->block_sizes + b0, a->nnz, pix, w, sig, noi, a->lambda,
          a->invtt + (size_t) b0 * a->lambda);
    free(pix);
    free(w);
    free(sig);
    free(noi);
}

int ref_mlmap(int nranks, const char *outpath, const char *ref, double tol, int maxiter, int nside, int nnz,
              int lambda, int *data_size_proc, int *nb_blocks_proc, int *block_sizes, int *pix, double *weights,
              double *signal, double *noise, double *invtt) {
    mlmap_args a = {(char *) outpath, (char *) ref, tol,   maxiter, nside,  nnz,   lambda, nranks,
                    data_size_proc,   nb_blocks_proc, block_sizes, pix,   weights, signal, noise, invtt};
    return shim_mpi_run(nranks, mlmap_rank, &a);
}

/* ---- CPU baseline: time one operator application P^T N^-1 P on n ranks ---- */
typedef struct {
    int     nranks, nnz, lambda, reps;
    int    *data_size_proc, *nb_blocks_proc, *block_sizes, *pix;
    double *weights, *invtt;
    double *seconds; /* shared result: max over ranks, written by rank 0 via Allreduce */
    double *shared_out;
} optime_args;

static void optime_rank(int rank, void *vp) {
    optime_args *a  = (optime_args *) vp;
    int64_t      s0 = 0;
    int          b0 = 0;
    for (int r = 0; r < rank; r++) {
        s0 += a->data_size_proc[r];
        b0 += a->nb_blocks_proc[r];
    }
    int     m   = a->data_size_proc[rank];
    int    *pix = (int *) malloc(sizeof(int) * (size_t) m * a->nnz);
    memcpy(pix, a->pix + s0 * a->nnz, sizeof(int) * (size_t) m * a->nnz);
    Mat A;
    memset(&A, 0, sizeof(A));
    MatInit(&A, m, a->nnz, pix, a->weights + s0 * a->nnz, ALLREDUCE, MPI_COMM_WORLD);
    int64_t M = 0;
    for (int r = 0; r < a->nranks; r++) M += a->data_size_proc[r];
    int nb_tot = 0;
    for (int r = 0; r < a->nranks; r++) nb_tot += a->nb_blocks_proc[r];
    Flag flag_stgy;
    flag_stgy_init_auto(&flag_stgy);
    flag_stgy.flag_verbose = 0;
    Block *blocks = (Block *) malloc(sizeof(Block) * (size_t) a->nb_blocks_proc[rank]);
    defineBlocks_avg(blocks, a->invtt + (size_t) b0 * a->lambda, a->nb_blocks_proc[rank], a->block_sizes + b0,
                     a->lambda, s0);
    Tpltz Nm1;
    defineTpltz_avg(&Nm1, M, 1, 1, blocks, a->nb_blocks_proc[rank], nb_tot, s0, m, flag_stgy, MPI_COMM_WORLD);
    int     n   = A.lcount - A.nnz * A.trash_pix;
    double *h   = (double *) malloc(sizeof(double) * (size_t) (n > 0 ? n : 1));
    double *out = (double *) malloc(sizeof(double) * (size_t) (n > 0 ? n : 1));
    double *tod = (double *) malloc(sizeof(double) * (size_t) m);
    for (int i = 0; i < n; i++) h[i] = 1.0 + 1e-3 * (double) (i % 97);
    /* each application timed on its own (max over ranks after a barrier): the
       file gets one double per application, in order */
    double *times = (double *) malloc(sizeof(double) * (size_t) a->reps);
    for (int r = 0; r < a->reps; r++) {
        MPI_Barrier(MPI_COMM_WORLD);
        double t0 = MPI_Wtime();
        MatVecProd(&A, h, tod, 0);
        apply_weights(&Nm1, tod);
        TrMatVecProd(&A, tod, out, 0);
        double dt = MPI_Wtime() - t0, dmax;
        MPI_Allreduce(&dt, &dmax, 1, MPI_DOUBLE, MPI_MAX, MPI_COMM_WORLD);
        times[r] = dmax;
    }
    if (rank == 0) {
        FILE *f = fopen((char *) a->shared_out, "wb");
        if (f) {
            fwrite(times, sizeof(double), (size_t) a->reps, f);
            fclose(f);
        }
    }
    free(times);
    MatFree(&A);
    free(pix);
    free(blocks);
    free(h);
    free(out);
    free(tod);
}

/* writes max-over-ranks seconds of each of the reps applications to the file named by result_path */
int ref_operator_time(int nranks, int nnz, int lambda, int reps, int *data_size_proc, int *nb_blocks_proc,
                      int *block_sizes, int *pix, double *weights, double *invtt, const char *result_path) {
    optime_args a = {nranks, nnz, lambda, reps, data_size_proc, nb_blocks_proc, block_sizes, pix, weights,
                     invtt,  NULL, (double *) result_path};
    return shim_mpi_run(nranks, optime_rank, &a);
}

/* ---- templates: the operators of MTmap's filtered solve ------------------
 * (algebra/src/templates/templates.c; MTmap's set-up, mappraiser/src/mappraiser.c:586-660).
 * nces CESs x ndet detectors, block (i, j) = i*ndet + j of ces_length[i] =
 * sweeps[i][nsweeps[i]] samples.  sweeps_flat: the nces rows of nsweeps[i] + 1 stamps one
 * after the other; az_flat, hwp_flat: the nces rows of ces_length[i] samples.  As MTmap:
 * az bins by bin_az, hwp_mod = (cos, sin) of the HWP angle, classes by Tlist_init with
 * weights on the fly.  Outputs: amp = T^T d (TrTVecProd), tod = T tau (TVecProd), and per
 * block the kernel w_b T_b^T T_b (BuildKernel) in kern and its pseudo-inverse (InvKernel)
 * in kinv, blocks one after the other.  Returns the number of template amplitudes. */
#include "templates.h"

static int **rows_i(int nces, const int *len, int *flat) {
    int **r = (int **) malloc(sizeof(int *) * (size_t) nces);
    for (int i = 0, at = 0; i < nces; at += len[i], i++) r[i] = flat + at;
    return r;
}
static double **rows_d(int nces, const int *len, double *flat) {
    double **r = (double **) malloc(sizeof(double *) * (size_t) nces);
    for (int i = 0, at = 0; i < nces; at += len[i], i++) r[i] = flat + at;
    return r;
}

int ref_templates_ops(int nces, int ndet, int *nsweeps, int *sweeps_flat, double *az_flat, double *az_min,
                      double *az_max, double *hwp_flat, int npoly, int ground, int n_sss_bins, int nhwp,
                      double delta_t, double fs, double *w_block, double *d, double *tau, double *amp, double *tod,
                      double *kern, double *kinv) {
    int *slen = (int *) malloc(sizeof(int) * (size_t) nces);
    for (int i = 0; i < nces; i++) slen[i] = nsweeps[i] + 1;
    int **sweeptstamps = rows_i(nces, slen, sweeps_flat);
    int *ces_length = (int *) malloc(sizeof(int) * (size_t) nces);
    int *hwp_bins = (int *) malloc(sizeof(int) * (size_t) nces);
    int **detnsweeps = (int **) malloc(sizeof(int *) * (size_t) nces);
    for (int i = 0; i < nces; i++) {
        ces_length[i] = sweeptstamps[i][nsweeps[i]];
        hwp_bins[i] = (int) ceil(ces_length[i] / (delta_t * fs));
        detnsweeps[i] = (int *) malloc(sizeof(int) * (size_t) ndet);
        for (int j = 0; j < ndet; j++) detnsweeps[i][j] = nsweeps[i];
    }
    double **az = rows_d(nces, ces_length, az_flat);
    double **hwp_angle = rows_d(nces, ces_length, hwp_flat);
    int **az_binned = bin_az(az, az_min, az_max, ces_length, ground, n_sss_bins, nces);
    double ***hwp_mod = (double ***) malloc(sizeof(double **) * (size_t) nces);
    for (int i = 0; i < nces && nhwp; i++) {
        hwp_mod[i] = (double **) malloc(2 * sizeof(double *));
        hwp_mod[i][0] = (double *) malloc(sizeof(double) * (size_t) ces_length[i]);
        hwp_mod[i][1] = (double *) malloc(sizeof(double) * (size_t) ces_length[i]);
        for (int t = 0; t < ces_length[i]; t++) {
            hwp_mod[i][0][t] = cos(hwp_angle[i][t]);
            hwp_mod[i][1][t] = sin(hwp_angle[i][t]);
        }
    }
    int nb = nces * ndet;
    int *block_sizes = (int *) malloc(sizeof(int) * (size_t) nb);
    for (int i = 0; i < nces; i++)
        for (int j = 0; j < ndet; j++) block_sizes[i * ndet + j] = ces_length[i];
    int n_class = npoly + ground + 2 * nhwp;
    TemplateClass *X = (TemplateClass *) malloc(sizeof(TemplateClass) * (size_t) n_class * nb);
    Tlist_init(X, ndet, nces, block_sizes, detnsweeps, ces_length, sweeptstamps, n_sss_bins, az_binned, fs, npoly,
               ground, nhwp, delta_t, 0, hwp_mod);
    TrTVecProd(X, nces, n_class * ndet, fs, ces_length, sweeptstamps, az_binned, hwp_mod, nhwp, delta_t, 0, d, amp);
    TVecProd(X, nces, n_class * ndet, fs, ces_length, sweeptstamps, az_binned, hwp_mod, nhwp, delta_t, 0, tau, tod);
    int ntot = 0;
    size_t at = 0;
    for (int i = 0; i < nces; i++) {
        hwpss_w hw;
        memset(&hw, 0, sizeof(hw));
        if (nhwp) build_hwpss_w(&hw, hwp_mod[i], ces_length[i], nhwp, i);
        int nt = npoly * nsweeps[i] + ground * n_sss_bins + 2 * nhwp * hwp_bins[i];
        for (int j = 0; j < ndet; j++) {
            double *Bk = kern + at;
            memset(Bk, 0, sizeof(double) * (size_t) nt * nt);
            BuildKernel(X + (i * ndet + j) * n_class, n_class, Bk, w_block[i * ndet + j], sweeptstamps[i],
                        ground ? az_binned[i] : NULL, hw, delta_t, fs);
            double *tmp = (double *) malloc(sizeof(double) * (size_t) nt * nt);
            double *binv = (double *) calloc((size_t) nt * nt, sizeof(double));
            memcpy(tmp, Bk, sizeof(double) * (size_t) nt * nt);
            InvKernel(tmp, nt, binv);
            memcpy(kinv + at, binv, sizeof(double) * (size_t) nt * nt);
            free(tmp);
            free(binv);
            at += (size_t) nt * nt;
            ntot += nt;
        }
        if (nhwp) free_hwpss_w(&hw, nhwp);
    }
    return ntot;
}

/* ---- MTmap on one rank (mappraiser/src/mappraiser.c:387-800): the template-filtered
 * solve (PCG_GLS_templates, pcg_true.c:243-560) with white noise per block (invtt: one
 * weight per block); maps written like MLmap's. */
typedef struct {
    const char *outpath, *ref;
    int nces, ndet, npoly, ground, n_sss_bins, nhwp, maxiter, nside, nnz;
    double delta_t, fs, tol;
    int *nsweeps, *sweeps_flat, *pix;
    double *az_flat, *az_min, *az_max, *hwp_flat, *weights, *signal, *noise, *invtt;
} mtmap_args;

static void mtmap_rank(int rank, void *vp) {
    (void) rank;
    mtmap_args *a = (mtmap_args *) vp;
    int nces = a->nces;
    int *slen = (int *) malloc(sizeof(int) * (size_t) nces);
    for (int i = 0; i < nces; i++) slen[i] = a->nsweeps[i] + 1;
    int **sweeptstamps = rows_i(nces, slen, a->sweeps_flat);
    int *ces_length = (int *) malloc(sizeof(int) * (size_t) nces);
    int m = 0;
    for (int i = 0; i < nces; i++) {
        ces_length[i] = sweeptstamps[i][a->nsweeps[i]];
        m += ces_length[i] * a->ndet;
    }
    double **az = rows_d(nces, ces_length, a->az_flat);
    double **hwp_angle = rows_d(nces, ces_length, a->hwp_flat);
    int nb = nces * a->ndet;
    int *block_sizes = (int *) malloc(sizeof(int) * (size_t) nb);
    for (int i = 0; i < nces; i++)
        for (int j = 0; j < a->ndet; j++) block_sizes[i * a->ndet + j] = ces_length[i];
    int *pix = (int *) malloc(sizeof(int) * (size_t) m * a->nnz);
    double *w = (double *) malloc(sizeof(double) * (size_t) m * a->nnz);
    double *sig = (double *) malloc(sizeof(double) * (size_t) m);
    double *noi = (double *) malloc(sizeof(double) * (size_t) m);
    memcpy(pix, a->pix, sizeof(int) * (size_t) m * a->nnz);
    memcpy(w, a->weights, sizeof(double) * (size_t) m * a->nnz);
    memcpy(sig, a->signal, sizeof(double) * (size_t) m);
    memcpy(noi, a->noise, sizeof(double) * (size_t) m);
    int dsp[1] = {m};
    MTmap(MPI_COMM_WORLD, (char *) a->outpath, (char *) a->ref, 0, 0, 0, ALLREDUCE, a->npoly, a->nhwp, a->delta_t,
          a->ground, a->n_sss_bins, a->tol, a->maxiter, 0, 0, 0, a->nside, sweeptstamps, a->nsweeps, az, a->az_min,
          a->az_max, hwp_angle, nces, dsp, nb, block_sizes, a->nnz, pix, w, sig, noi, a->fs, a->invtt);
    free(pix);
    free(w);
    free(sig);
    free(noi);
}

int ref_mtmap(const char *outpath, const char *ref, int nces, int ndet, int *nsweeps, int *sweeps_flat,
              double *az_flat, double *az_min, double *az_max, double *hwp_flat, int npoly, int ground,
              int n_sss_bins, int nhwp, double delta_t, double fs, double tol, int maxiter, int nside, int nnz,
              int *pix, double *weights, double *signal, double *noise, double *invtt) {
    mtmap_args a = {outpath, ref, nces, ndet, npoly, ground, n_sss_bins, nhwp, maxiter, nside, nnz, delta_t, fs, tol,
                    nsweeps, sweeps_flat, pix, az_flat, az_min, az_max, hwp_flat, weights, signal, noise, invtt};
    return shim_mpi_run(1, mtmap_rank, &a);
}
