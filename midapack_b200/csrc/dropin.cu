// Reference-compatible C API (host pointers) on top of the device API.
//
// Each entry point keeps the reference's name, signature, argument meaning
// and side effects (in-place index rewrite by MatInit, in-place V by
// stbmmProd, cut rewrite of A and b by the preconditioner); see the
// declarations in include/{mapmat,toeplitz,mappraiser}.h for the reference
// lines each one replaces.  Device mirrors of Mat and Tpltz objects are kept
// in registries keyed by the struct's address.
#include <sys/stat.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <mutex>
#include <unordered_map>

#include "mdp_internal.cuh"

extern "C" {
#include "mappraiser.h"
}

// ------------------------------------------------------------------ shared state
static std::mutex   g_mu;
static mdp_context *g_ctx = nullptr;

static mdp_context *default_ctx() {
    if (g_ctx) return g_ctx;
    int dev = 0;
    cudaGetDevice(&dev);
    if (mdp_context_create(dev, &g_ctx) != MDP_OK) {
        fprintf(stderr, "midapack_b200: no usable CUDA device: %s\n", mdp_last_error());
        return nullptr;
    }
    return g_ctx;
}

struct MatDev {
    mdp_pointing *P = nullptr;
    DevBuf        values;
    int           m = 0, nnz = 0;
    ~MatDev() { mdp_pointing_destroy(P); }
};
static std::unordered_map<const void *, MatDev *> g_mats;

struct NoiseDev {
    mdp_noise           *N = nullptr;
    std::vector<int64_t> key;  // block layout it was built for
    std::vector<const double *> tptr;
    ~NoiseDev() { mdp_noise_destroy(N); }
};
static std::unordered_map<const void *, NoiseDev *> g_noises;

static void drop_mat(const void *A) {
    auto it = g_mats.find(A);
    if (it != g_mats.end()) {
        delete it->second;
        g_mats.erase(it);
    }
}

static int fail(const char *where, int rc) {
    fprintf(stderr, "midapack_b200 %s: %s (%s)\n", where, mdp_strerror(rc), mdp_last_error());
    return rc ? rc : 1;
}

// ------------------------------------------------------------------ Mat
extern "C" void MatSetIndices(Mat *A, int m, int nnz, int *indices) {
    A->m = m;
    A->nnz = nnz;
    A->indices = indices;
}

extern "C" void MatSetValues(Mat *A, int m, int nnz, double *values) {
    A->m = m;
    A->nnz = nnz;
    A->values = values;
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_mats.find(A);
    if (it != g_mats.end() && it->second->values.p && (int64_t) m * nnz > 0) {
        mdp_context *ctx = default_ctx();
        cudaMemcpyAsync(it->second->values.p, values, sizeof(double) * (size_t) m * nnz, cudaMemcpyHostToDevice,
                        ctx->stream);
        cudaStreamSynchronize(ctx->stream);
    }
}

// compress A->indices (global) on the device; rewrite them to local indices in place
static int local_shape(Mat *A) {
    mdp_context *ctx = default_ctx();
    if (!ctx) return MDP_ECUDA;
    const int64_t n = (int64_t) A->m * A->nnz;
    if (A->m <= 0 || A->nnz <= 0 || !A->indices || !A->values) {
        mdp_set_error("MatLocalShape: empty or unset matrix");
        return MDP_EINVAL;
    }
    drop_mat(A);
    MatDev *D = new MatDev();
    D->m = A->m;
    D->nnz = A->nnz;
    DevBuf gidx, loc;
    int    rc;
    if ((rc = gidx.alloc(4 * n)) || (rc = loc.alloc(4 * n)) || (rc = D->values.alloc(8 * n))) {
        delete D;
        return rc;
    }
    cudaMemcpyAsync(gidx.p, A->indices, 4 * n, cudaMemcpyHostToDevice, ctx->stream);
    cudaMemcpyAsync(D->values.p, A->values, 8 * n, cudaMemcpyHostToDevice, ctx->stream);
    rc = mdp_pointing_create_ex(ctx, A->m, A->nnz, gidx.as<int32_t>(), D->values.as<double>(), loc.as<int32_t>(), &D->P);
    if (rc) {
        delete D;
        return rc;
    }
    cudaMemcpyAsync(A->indices, loc.p, 4 * n, cudaMemcpyDeviceToHost, ctx->stream);
    A->lcount = (int) D->P->lcount;
    A->lindices = (int *) malloc(sizeof(int) * std::max<int64_t>(D->P->lcount, 1));
    cudaMemcpyAsync(A->lindices, D->P->lindices.p, 4 * D->P->lcount, cudaMemcpyDeviceToHost, ctx->stream);
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
        delete D;
        mdp_set_error("MatLocalShape: %s", cudaGetErrorString(cudaGetLastError()));
        return MDP_ECUDA;
    }
    if (A->lindices[0] < 0) A->trash_pix = 1;  // mapmat.c:518 (never reset, as the reference)
    if (A->trash_pix != D->P->trash_pix) {
        delete D;
        mdp_set_error("MatLocalShape: trash_pix was set on input but the indices have no negative entry");
        return MDP_EUNSUPPORTED;
    }
    g_mats[A] = D;
    return MDP_OK;
}

extern "C" int MatLocalShape(Mat *A, int sflag) {
    (void) sflag;  // every sort method yields the same sorted unique set
    std::lock_guard<std::mutex> lk(g_mu);
    int                         rc = local_shape(A);
    return rc ? fail("MatLocalShape", rc) : 0;
}

extern "C" int MatComShape(Mat *A, int flag, MPI_Comm comm) {
    A->flag = flag;
    A->comm = comm;
    A->com_indices = nullptr;
    A->com_count = 0;
    A->steps = 0;
    A->nS = A->nR = nullptr;
    A->R = A->S = nullptr;
    return 0;
}

extern "C" int MatInit(Mat *A, int m, int nnz, int *indices, double *values, int flag, MPI_Comm comm) {
    MatSetIndices(A, m, nnz, indices);
    A->values = values;
    int err = MatLocalShape(A, 3);
    MatComShape(A, flag, comm);
    return err;
}

extern "C" void MatFree(Mat *A) {
    std::lock_guard<std::mutex> lk(g_mu);
    free(A->lindices);
    A->lindices = nullptr;
    drop_mat(A);
}

static MatDev *mat_dev(const Mat *A) {
    auto it = g_mats.find(A);
    if (it == g_mats.end() || it->second->m != A->m || it->second->nnz != A->nnz) return nullptr;
    return it->second;
}

extern "C" int MatVecProd(Mat *A, double *x, double *y, int pflag) {
    (void) pflag;
    std::lock_guard<std::mutex> lk(g_mu);
    MatDev                     *D = mat_dev(A);
    mdp_context                *ctx = default_ctx();
    if (!D || !ctx) {
        mdp_set_error("MatVecProd: matrix not initialised with MatInit/MatLocalShape");
        return fail("MatVecProd", MDP_EINVAL);
    }
    const int64_t n = D->P->n_map();
    DevBuf        dx, dy;
    int           rc;
    if ((rc = dx.alloc(8 * std::max<int64_t>(n, 1))) || (rc = dy.alloc(8 * (int64_t) A->m))) return fail("MatVecProd", rc);
    cudaMemcpyAsync(dx.p, x, 8 * n, cudaMemcpyHostToDevice, ctx->stream);
    if ((rc = mdp_matvec_launch(ctx, D->P, dx.as<double>(), dy.as<double>()))) return fail("MatVecProd", rc);
    cudaMemcpyAsync(y, dy.p, 8 * (int64_t) A->m, cudaMemcpyDeviceToHost, ctx->stream);
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) return fail("MatVecProd", MDP_ECUDA);
    return 0;
}

extern "C" int TrMatVecProd(Mat *A, double *y, double *x, int pflag) {
    (void) pflag;
    std::lock_guard<std::mutex> lk(g_mu);
    MatDev                     *D = mat_dev(A);
    mdp_context                *ctx = default_ctx();
    if (!D || !ctx) {
        mdp_set_error("TrMatVecProd: matrix not initialised with MatInit/MatLocalShape");
        return fail("TrMatVecProd", MDP_EINVAL);
    }
    const int64_t n = D->P->n_map();
    DevBuf        dx, dy;
    int           rc;
    if ((rc = dx.alloc(8 * std::max<int64_t>(n, 1))) || (rc = dy.alloc(8 * (int64_t) A->m)))
        return fail("TrMatVecProd", rc);
    cudaMemcpyAsync(dy.p, y, 8 * (int64_t) A->m, cudaMemcpyHostToDevice, ctx->stream);
    if ((rc = mdp_trmatvec_launch(ctx, D->P, dy.as<double>(), dx.as<double>()))) return fail("TrMatVecProd", rc);
    cudaMemcpyAsync(x, dx.p, 8 * n, cudaMemcpyDeviceToHost, ctx->stream);
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) return fail("TrMatVecProd", MDP_ECUDA);
    return 0;
}

extern "C" int greedyreduce(Mat *A, double *x) {
    (void) A;
    (void) x;
    return 0;
}

// ------------------------------------------------------------------ Toeplitz
extern "C" int flag_stgy_init_zeros(Flag *f) {
    memset(f, 0, sizeof(*f));
    return 0;
}

extern "C" int flag_stgy_init_auto(Flag *f) {
    memset(f, 0, sizeof(*f));
    f->flag_fftw = 1 << 6;  // FFTW_ESTIMATE, as the reference's FLAG_FFTW default
    return 0;
}

// toeplitz.c:168-253 (flags 0-4 and 6; 5 is the MADmap formula)
extern "C" int define_blocksize(int n, int lambda, int bs_flag, int fixed_bs) {
    auto pow2ceil = [](double v) { return (int) std::pow(2.0, std::ceil(std::log(v) / std::log(2.0))); };
    int  bs;
    if (bs_flag == 1) return fixed_bs;
    if (bs_flag == 5) {
        bs = 1;
        while (bs < 2 * (lambda - 1) * std::log(bs + 1) && bs < n) bs *= 2;
        return bs;
    }
    int mult = (bs_flag == 2) ? 2 : (bs_flag == 3) ? 3 : 4;
    int min_bs = mult * lambda;
    bs = pow2ceil(min_bs);
    if (bs_flag == 6) bs = std::max(bs, 1 << 14);
    if (bs > n) bs = min_bs;
    return bs;
}

struct HostPlan {
    int n;
};

extern "C" int tpltz_init(int n, int lambda, int *nfft, int *blocksize, fftw_complex **T_fft, double *T,
                          fftw_complex **V_fft, double **V_rfft, fftw_plan *plan_f, fftw_plan *plan_b,
                          Flag flag_stgy) {
    *blocksize = define_blocksize(n, lambda, flag_stgy.flag_bs, flag_stgy.fixed_bs);
    *nfft = (flag_stgy.flag_nfft == 1) ? flag_stgy.fixed_nfft : 1;
    const int bs = *blocksize, h = bs / 2 + 1;
    *T_fft = (fftw_complex *) malloc(sizeof(fftw_complex) * h);
    *V_fft = (fftw_complex *) malloc(sizeof(fftw_complex) * (size_t) (*nfft) * h);
    *V_rfft = (double *) malloc(sizeof(double) * (size_t) (*nfft) * bs);
    if (!*T_fft || !*V_fft || !*V_rfft) return 2;  // toeplitz.c error 2: bad allocation
    // spectrum of the circulant embedding, computed on the device (circ_init_fftw's
    // r2c transform of c[0] = T[0], c[i] = c[bs-i] = T[i])
    mdp_context *ctx = default_ctx();
    if (!ctx || mdp_circulant_spectrum(ctx, T, lambda, bs, &(*T_fft)[0][0]) != MDP_OK) {
        fprintf(stderr, "tpltz_init: %s\n", mdp_last_error());
        return 3;
    }
    HostPlan *pf = new HostPlan{bs}, *pb = new HostPlan{bs};
    *plan_f = (fftw_plan) pf;
    *plan_b = (fftw_plan) pb;
    return 0;
}

extern "C" int tpltz_cleanup(fftw_complex **T_fft, fftw_complex **V_fft, double **V_rfft, fftw_plan *plan_f,
                             fftw_plan *plan_b) {
    free(*T_fft);
    free(*V_fft);
    free(*V_rfft);
    delete (HostPlan *) *plan_f;
    delete (HostPlan *) *plan_b;
    *T_fft = nullptr;
    *V_fft = nullptr;
    *V_rfft = nullptr;
    *plan_f = nullptr;
    *plan_b = nullptr;
    return 0;
}

extern "C" int defineTpltz_avg(Tpltz *Nm1, int64_t nrow, int m_cw, int m_rw, Block *tpltzblocks, int nb_blocks_loc,
                               int nb_blocks_tot, int64_t idp, int local_V_size, Flag flag_stgy, MPI_Comm comm) {
    Nm1->nrow = nrow;
    Nm1->m_cw = m_cw;
    Nm1->m_rw = m_rw;
    Nm1->tpltzblocks = tpltzblocks;
    Nm1->nb_blocks_loc = nb_blocks_loc;
    Nm1->nb_blocks_tot = nb_blocks_tot;
    Nm1->idp = idp;
    Nm1->local_V_size = local_V_size;
    Nm1->flag_stgy = flag_stgy;
    Nm1->comm = comm;
    return 0;
}

extern "C" int defineBlocks_avg(Block *tpltzblocks, double *T, int nb_blocks_loc, void *local_blocks_sizes,
                                int lambda_block_avg, int64_t id0) {
    const int *sizes = (const int *) local_blocks_sizes;
    int64_t    idv = id0;
    for (int i = 0; i < nb_blocks_loc; i++) {
        tpltzblocks[i].n = sizes[i];
        tpltzblocks[i].lambda = lambda_block_avg;
        tpltzblocks[i].idv = idv;
        idv += sizes[i];
        tpltzblocks[i].T_block = T + (size_t) i * lambda_block_avg;
    }
    return 0;
}

// device noise operator for a Tpltz, rebuilt when its block layout changes
static int noise_for(Tpltz *Nm1, mdp_noise **out) {
    mdp_context *ctx = default_ctx();
    if (!ctx) return MDP_ECUDA;
    const int nb = Nm1->nb_blocks_loc;
    if (nb <= 0 || !Nm1->tpltzblocks) {
        mdp_set_error("stbmmProd: no Toeplitz blocks");
        return MDP_EINVAL;
    }
    if (Nm1->m_cw != 1 || Nm1->m_rw != 1) {
        mdp_set_error("stbmmProd: only one column (m_cw = m_rw = 1) is supported, as MAPPRAISER uses");
        return MDP_EUNSUPPORTED;
    }
    std::vector<int64_t>         key = {(int64_t) nb, Nm1->idp, (int64_t) Nm1->local_V_size};
    std::vector<const double *> tp;
    const int                    lam = Nm1->tpltzblocks[0].lambda;
    for (int b = 0; b < nb; b++) {
        const Block &B = Nm1->tpltzblocks[b];
        if (B.lambda != lam) {
            mdp_set_error("stbmmProd: blocks with different lambda are not supported");
            return MDP_EUNSUPPORTED;
        }
        key.push_back(B.idv);
        key.push_back(B.n);
        key.push_back(B.lambda);
        tp.push_back(B.T_block);
    }
    auto it = g_noises.find(Nm1);
    if (it != g_noises.end() && it->second->key == key && it->second->tptr == tp) {
        *out = it->second->N;
        return MDP_OK;
    }
    if (it != g_noises.end()) {
        delete it->second;
        g_noises.erase(it);
    }
    std::vector<int64_t> idv(nb);
    std::vector<int32_t> n(nb);
    std::vector<double>  T((size_t) nb * lam);
    for (int b = 0; b < nb; b++) {
        idv[b] = Nm1->tpltzblocks[b].idv - Nm1->idp;
        n[b] = Nm1->tpltzblocks[b].n;
        memcpy(T.data() + (size_t) b * lam, Nm1->tpltzblocks[b].T_block, sizeof(double) * lam);
    }
    NoiseDev *D = new NoiseDev();
    int       rc = mdp_noise_create(ctx, nb, idv.data(), n.data(), lam, T.data(), &D->N);
    if (rc) {
        delete D;
        return rc;
    }
    D->key = key;
    D->tptr = tp;
    g_noises[Nm1] = D;
    *out = D->N;
    return MDP_OK;
}

extern "C" int stbmmProd(Tpltz *Nm1, double *V) {
    std::lock_guard<std::mutex> lk(g_mu);
    mdp_noise                  *N;
    int                         rc = noise_for(Nm1, &N);
    if (rc) return fail("stbmmProd", rc);
    mdp_context  *ctx = default_ctx();
    const int64_t rows = std::max<int64_t>(Nm1->local_V_size, N->nrow_end);
    DevBuf        dv, dout;
    if ((rc = dv.alloc(8 * rows)) || (rc = dout.alloc(8 * rows))) return fail("stbmmProd", rc);
    cudaMemcpyAsync(dv.p, V, 8 * Nm1->local_V_size, cudaMemcpyHostToDevice, ctx->stream);
    cudaMemcpyAsync(dout.p, dv.p, 8 * Nm1->local_V_size, cudaMemcpyDeviceToDevice, ctx->stream);
    if ((rc = mdp_stbmm_impl(ctx, N, dv.as<double>(), dout.as<double>(), nullptr))) return fail("stbmmProd", rc);
    cudaMemcpyAsync(V, dout.p, 8 * Nm1->local_V_size, cudaMemcpyDeviceToHost, ctx->stream);
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) return fail("stbmmProd", MDP_ECUDA);
    return 0;
}

extern "C" int apply_weights(Tpltz *Nm1, double *tod) { return stbmmProd(Nm1, tod); }

// ------------------------------------------------------------------ preconditioner and PCG
extern "C" void get_pixshare_pond(Mat *A, double *pixpond) {
    const int n = A->lcount - A->nnz * A->trash_pix;
    for (int i = 0; i < n; i++) pixpond[i] = 1.0;
}

// After the device cut, mirror the reference's side effects on the host Mat:
// new local indices, zero weights on cut rows, b = 0 on cut rows, new lindices.
static int mirror_cut_to_host(mdp_context *ctx, Mat *A, MatDev *D, double *b) {
    mdp_pointing *P = D->P;
    const int64_t m = A->m;
    std::vector<int32_t> off(m);
    cudaMemcpyAsync(off.data(), P->off.p, 4 * m, cudaMemcpyDeviceToHost, ctx->stream);
    DevBuf loc;
    int    rc;
    if ((rc = loc.alloc(12 * m))) return rc;
    if ((rc = mdp_pointing_local_indices(ctx, P, loc.as<int32_t>()))) return rc;
    cudaMemcpyAsync(A->indices, loc.p, 12 * m, cudaMemcpyDeviceToHost, ctx->stream);
    free(A->lindices);
    A->lcount = (int) P->lcount;
    A->lindices = (int *) malloc(sizeof(int) * std::max<int64_t>(P->lcount, 1));
    cudaMemcpyAsync(A->lindices, P->lindices.p, 4 * P->lcount, cudaMemcpyDeviceToHost, ctx->stream);
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) return MDP_ECUDA;
    A->trash_pix = P->trash_pix;
    bool any = false;
    for (int64_t t = 0; t < m; t++)
        if (off[t] == -2) {
            any = true;
            for (int j = 0; j < 3; j++) A->values[3 * t + j] = 0.0;
            if (b) b[t] = 0.0;
        }
    if (any) cudaMemcpy(D->values.p, A->values, 24 * m, cudaMemcpyHostToDevice);
    return MDP_OK;
}

static void set_bj_mat(Mat *M, int n, int *indices, double *values) {
    memset(M, 0, sizeof(*M));
    M->m = n;
    M->nnz = 3;
    M->indices = indices;
    M->values = values;
    M->lcount = n;
    M->lindices = (int *) malloc(sizeof(int) * std::max(n, 1));
}

extern "C" int precondblockjacobilike(Mat *A, Tpltz *Nm1, Mat *BJ_inv, Mat *BJ, double *b, double *cond, int *lhits) {
    std::lock_guard<std::mutex> lk(g_mu);
    mdp_context                *ctx = default_ctx();
    MatDev                     *D = mat_dev(A);
    mdp_noise                  *N;
    int                         rc;
    if (!D) return fail("precondblockjacobilike", MDP_EINVAL);
    if ((rc = noise_for(Nm1, &N))) return fail("precondblockjacobilike", rc);
    BJState bj;
    if ((rc = mdp_bj_build(ctx, D->P, N, &bj))) return fail("precondblockjacobilike", rc);
    if (bj.ncut > 0 && (rc = mirror_cut_to_host(ctx, A, D, b))) return fail("precondblockjacobilike", rc);
    const int n = (int) (3 * bj.npix);
    cudaMemcpy(cond, bj.rcond.p, 8 * bj.npix, cudaMemcpyDeviceToHost);
    cudaMemcpy(lhits, bj.hits.p, 4 * bj.npix, cudaMemcpyDeviceToHost);
    // BJ_inv and BJ as n x 3 matrices whose row i reads pixel i/3 (precond.c:672-699)
    int    *idx = (int *) malloc(sizeof(int) * std::max(3 * n, 1));
    double *vinv = (double *) malloc(sizeof(double) * std::max(3 * n, 1));
    double *vw = (double *) malloc(sizeof(double) * std::max(3 * n, 1));
    cudaMemcpy(vinv, bj.inv.p, 8 * 3 * (size_t) n, cudaMemcpyDeviceToHost);
    cudaMemcpy(vw, bj.W.p, 8 * 3 * (size_t) n, cudaMemcpyDeviceToHost);
    for (int i = 0; i < n; i++)
        for (int j = 0; j < 3; j++) idx[3 * i + j] = 3 * (i / 3) + j;  // local numbering of the map
    set_bj_mat(BJ_inv, n, idx, vinv);
    set_bj_mat(BJ, n, idx, vw);
    for (int i = 0; i < n; i++) BJ_inv->lindices[i] = BJ->lindices[i] = A->lindices[3 * A->trash_pix + i];
    if (A->id_last_pix) free(A->id_last_pix);
    if (A->ll) free(A->ll);
    A->id_last_pix = nullptr;
    A->ll = nullptr;
    return 0;
}

// Two-level state of the device pointing/noise after the block-Jacobi cut;
// precond 2 starts its Lanczos run from the first residual P^T N^-1 (b + noise)
// with b the (cut) host signal.
static int twolevel_for(mdp_context *ctx, MatDev *D, mdp_noise *N, int precond, int zn, const double *b,
                        const double *noise, mdp_twolevel *tl) {
    DevBuf g0;
    if (precond == 2) {
        const int64_t m = D->P->m;
        DevBuf        db, dn;
        MDP_TRY(db.alloc(8 * m));
        MDP_TRY(dn.alloc(8 * m));
        MDP_TRY(g0.alloc(8 * std::max<int64_t>(D->P->n_map(), 1)));
        MDP_CUDA(cudaMemcpyAsync(db.p, b, 8 * m, cudaMemcpyHostToDevice, ctx->stream));
        MDP_CUDA(cudaMemcpyAsync(dn.p, noise, 8 * m, cudaMemcpyHostToDevice, ctx->stream));
        MDP_TRY(mdp_gls_rhs(ctx, D->P, N, db.as<double>(), dn.as<double>(), g0.as<double>()));
        MDP_CUDA(cudaStreamSynchronize(ctx->stream));  // db, dn are released on return
    }
    return mdp_twolevel_build(ctx, D->P, N, precond, zn, g0.as<double>(), tl);
}

extern "C" void build_precond(Precond **out_p, double **out_pixpond, int *out_n, Mat *A, Tpltz *Nm1, double **in_out_x,
                              double *b, double *noise, double *cond, int *lhits, double tol, int Zn, int precond) {
    (void) tol;
    *out_p = nullptr;
    if (precond < 0 || precond > 2) {
        fprintf(stderr, "midapack_b200 build_precond: precond must be 0 (block Jacobi), 1 or 2 (two-level), got %d\n",
                precond);
        return;
    }
    Precond *p = (Precond *) calloc(1, sizeof(Precond));
    p->precond = precond;
    p->Zn = Zn;
    if (precondblockjacobilike(A, Nm1, &p->BJ_inv, &p->BJ, b, cond, lhits) != 0) {
        free(p);
        return;
    }
    p->n = A->lcount - A->nnz * A->trash_pix;
    p->pixpond = (double *) malloc(sizeof(double) * std::max(p->n, 1));
    get_pixshare_pond(A, p->pixpond);
    if (precond != 0) {
        // Z, AZ (Zn columns of n) and Em1 (Zn x Zn) built on the device and
        // kept in the reference's host fields (precond.c:1341-1394)
        std::lock_guard<std::mutex> lk(g_mu);
        mdp_context                *ctx = default_ctx();
        MatDev                     *D = mat_dev(A);
        mdp_noise                  *N = nullptr;
        mdp_twolevel                tl;
        int                         rc = D ? noise_for(Nm1, &N) : MDP_EINVAL;
        if (!rc) rc = twolevel_for(ctx, D, N, precond, Zn, b, noise, &tl);
        if (rc) {
            fail("build_precond", rc);
            free(p->pixpond);
            free(p);
            return;
        }
        const int zn = tl.zn, n = p->n;
        p->Zn = zn;
        p->Z = (double **) calloc(zn, sizeof(double *));
        p->AZ = (double **) calloc(zn, sizeof(double *));
        for (int j = 0; j < zn; j++) {
            p->Z[j] = (double *) malloc(sizeof(double) * std::max(n, 1));
            p->AZ[j] = (double *) malloc(sizeof(double) * std::max(n, 1));
            cudaMemcpy(p->Z[j], tl.Z.as<double>() + (int64_t) j * n, 8 * (size_t) n, cudaMemcpyDeviceToHost);
            cudaMemcpy(p->AZ[j], tl.AZ.as<double>() + (int64_t) j * n, 8 * (size_t) n, cudaMemcpyDeviceToHost);
        }
        p->Em1 = (double *) malloc(sizeof(double) * (size_t) zn * zn);
        memcpy(p->Em1, tl.h_Em1.data(), sizeof(double) * (size_t) zn * zn);
        p->Qg = (double *) calloc(std::max(n, 1), sizeof(double));
        p->AQg = (double *) calloc(std::max(n, 1), sizeof(double));
        p->w = (double *) calloc(zn, sizeof(double));
        p->Qtx = (double *) calloc(zn, sizeof(double));
    }
    *out_p = p;
    *out_pixpond = p->pixpond;
    *out_n = p->n;
    (void) in_out_x;  // x keeps its allocation (it is at least n long)
}

// Host arrays in and out, as the reference's apply_precond: block Jacobi, or
// the two-level product Cg = BJ_inv (g - AZ Qtx) + Z Qtx with Qtx = Em1 Z^T g
// (precond.c:1403-1423)
extern "C" void apply_precond(Precond *p, const Mat *A, Tpltz *Nm1, double *g, double *Cg) {
    (void) A;
    (void) Nm1;
    const int n = p->BJ_inv.m;
    const double *src = g;
    if (p->precond != 0) {
        const int zn = p->Zn;
        for (int j = 0; j < zn; j++) {
            double s = 0.0;
            for (int k = 0; k < n; k++) s += p->Z[j][k] * g[k] * p->pixpond[k];
            p->w[j] = s;
        }
        for (int i = 0; i < zn; i++) {
            double s = 0.0;
            for (int j = 0; j < zn; j++) s += p->Em1[i * zn + j] * p->w[j];
            p->Qtx[i] = s;
        }
        for (int k = 0; k < n; k++) p->Qg[k] = p->AQg[k] = 0.0;
        for (int j = 0; j < zn; j++)
            for (int k = 0; k < n; k++) {
                p->Qg[k] += p->Z[j][k] * p->Qtx[j];
                p->AQg[k] += p->AZ[j][k] * p->Qtx[j];
            }
        for (int k = 0; k < n; k++) p->AQg[k] = g[k] - p->AQg[k];
        src = p->AQg;
    }
    for (int i = 0; i < n; i++) {
        const double *r = p->BJ_inv.values + 3 * i;
        const int     q = 3 * (i / 3);
        Cg[i] = r[0] * src[q] + r[1] * src[q + 1] + r[2] * src[q + 2];
    }
    if (p->precond != 0)
        for (int i = 0; i < n; i++) Cg[i] += p->Qg[i];
}

extern "C" void free_precond(Precond **in_out_p) {
    Precond *p = *in_out_p;
    if (!p) return;
    free(p->pixpond);
    free(p->BJ_inv.indices);
    free(p->BJ_inv.values);
    free(p->BJ_inv.lindices);
    free(p->BJ.values);
    free(p->BJ.lindices);
    if (p->precond != 0) {
        for (int j = 0; j < p->Zn; j++) {
            if (p->Z) free(p->Z[j]);
            if (p->AZ) free(p->AZ[j]);
        }
        free(p->Z);
        free(p->AZ);
        free(p->Em1);
        free(p->Qg);
        free(p->AQg);
        free(p->w);
        free(p->Qtx);
    }
    free(p);
    *in_out_p = nullptr;
}

static void write_residuals(const char *outpath, const char *ref, const std::vector<double> &res, int k) {
    if (!outpath || !ref) return;
    char fn[4096];
    snprintf(fn, sizeof(fn), "%s/pcg_residuals_%s.dat", outpath, ref);
    FILE *f = fopen(fn, "wb");
    if (!f) return;
    fwrite(res.data(), sizeof(double), (size_t) std::min<int>(k + 1, (int) res.size()), f);
    fclose(f);
}

// ECG_GLS's relative residuals (ecg.c:156-161): <outpath>/rel_res_<ref>_enlfac_<t>_o=<ortho_alg>.txt
static void write_ecg_residuals(const char *outpath, const char *ref, const std::vector<double> &res, int iters,
                                int enl_fac, int ortho_alg) {
    if (!outpath || !ref) return;
    char fn[4096];
    snprintf(fn, sizeof(fn), "%s/rel_res_%s_enlfac_%d_o=%d.txt", outpath, ref, enl_fac, ortho_alg);
    FILE *f = fopen(fn, "w");
    if (!f) return;
    for (int i = 0; i <= iters && i < (int) res.size(); i++) fprintf(f, "%.15e\n", res[i]);
    fclose(f);
}

extern "C" int PCG_GLS_true(char *outpath, char *ref, Mat *A, Tpltz *Nm1, double *x, double *b, double *noise,
                            double *cond, int *lhits, double tol, int K, int precond, int Z_2lvl) {
    if (precond < 0 || precond > 2) {
        fprintf(stderr, "midapack_b200 PCG_GLS_true: precond must be 0 (block Jacobi), 1 or 2 (two-level)\n");
        return 1;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    mdp_context                *ctx = default_ctx();
    MatDev                     *D = mat_dev(A);
    mdp_noise                  *N;
    int                         rc;
    if (!D || !ctx) return fail("PCG_GLS_true", MDP_EINVAL);
    if ((rc = noise_for(Nm1, &N))) return fail("PCG_GLS_true", rc);
    const int64_t m = A->m;
    BJState       bj;
    if ((rc = mdp_bj_build(ctx, D->P, N, &bj))) return fail("PCG_GLS_true", rc);
    if (bj.ncut > 0 && (rc = mirror_cut_to_host(ctx, A, D, b))) return fail("PCG_GLS_true", rc);
    if (A->id_last_pix) free(A->id_last_pix);  // precond.c:673-675
    if (A->ll) free(A->ll);
    A->id_last_pix = nullptr;
    A->ll = nullptr;
    DevBuf db, dn, dx;
    const int64_t nmap = D->P->n_map();
    if ((rc = db.alloc(8 * m)) || (rc = dn.alloc(8 * m)) || (rc = dx.alloc(8 * std::max<int64_t>(nmap, 1))))
        return fail("PCG_GLS_true", rc);
    cudaMemcpyAsync(db.p, b, 8 * m, cudaMemcpyHostToDevice, ctx->stream);
    cudaMemcpyAsync(dn.p, noise, 8 * m, cudaMemcpyHostToDevice, ctx->stream);
    mdp_twolevel tl;
    if (precond != 0 && (rc = twolevel_for(ctx, D, N, precond, Z_2lvl, b, noise, &tl))) return fail("PCG_GLS_true", rc);
    mdp_solve_params prm = {tol, K, 1, precond, Z_2lvl};
    mdp_solve_info   info = {};
    std::vector<double> res(std::max(K, 1) + 1, 0.0);
    rc = mdp_pcg_run(ctx, D->P, N, bj.inv.as<double>(), bj.npix, db.as<double>(), dn.as<double>(), &prm, dx.as<double>(),
                     res.data(), &info, precond != 0 ? &tl : nullptr);
    if (rc) return fail("PCG_GLS_true", rc);
    cudaMemcpy(x, dx.p, 8 * 3 * bj.npix, cudaMemcpyDeviceToHost);
    cudaMemcpy(cond, bj.rcond.p, 8 * bj.npix, cudaMemcpyDeviceToHost);
    cudaMemcpy(lhits, bj.hits.p, 4 * bj.npix, cudaMemcpyDeviceToHost);
    if (info.converged && info.iterations < K) {
        printf("--> converged (%e < %e)\n", info.res, tol * tol * info.res0);
    } else {
        printf("--> unconverged, max iterate reached (%le > %le)\n", info.res, tol * tol * info.res0);
    }
    write_residuals(outpath, ref, res, info.iterations < K ? info.iterations : K - 1);
    return 0;
}

// ECG_GLS (ecg.c:44-175): block-Jacobi preconditioner with the cut mirrored on
// the host Mat and b, then the enlarged CG on the device; x receives the
// solution, cond/lhits the kept pixels' rcond and hits, and
// <outpath>/rel_res_<ref>_enlfac_<t>_o=<ortho_alg>.txt the relative residuals.
extern "C" int ECG_GLS(char *outpath, char *ref, Mat *A, Tpltz *Nm1, double *x, double *b, double *noise,
                       double *cond, int *lhits, double tol, int maxIter, int enlFac, int ortho_alg, int bs_red) {
    std::lock_guard<std::mutex> lk(g_mu);
    mdp_context                *ctx = default_ctx();
    MatDev                     *D = mat_dev(A);
    mdp_noise                  *N;
    int                         rc;
    if (!D || !ctx) return fail("ECG_GLS", MDP_EINVAL);
    if (enlFac < 1 || enlFac > MDP_ECG_MAX_ENL) {
        mdp_set_error("ECG_GLS: enlFac must be in 1..%d", MDP_ECG_MAX_ENL);
        return fail("ECG_GLS", MDP_EINVAL);
    }
    if ((rc = noise_for(Nm1, &N))) return fail("ECG_GLS", rc);
    const int64_t m = A->m;
    BJState       bj;
    if ((rc = mdp_bj_build(ctx, D->P, N, &bj))) return fail("ECG_GLS", rc);
    if (bj.ncut > 0 && (rc = mirror_cut_to_host(ctx, A, D, b))) return fail("ECG_GLS", rc);
    if (A->id_last_pix) free(A->id_last_pix);
    if (A->ll) free(A->ll);
    A->id_last_pix = nullptr;
    A->ll = nullptr;
    DevBuf        db, dn, dx;
    const int64_t nmap = D->P->n_map();
    if ((rc = db.alloc(8 * m)) || (rc = dn.alloc(8 * m)) || (rc = dx.alloc(8 * std::max<int64_t>(nmap, 1))))
        return fail("ECG_GLS", rc);
    cudaMemcpyAsync(db.p, b, 8 * m, cudaMemcpyHostToDevice, ctx->stream);
    cudaMemcpyAsync(dn.p, noise, 8 * m, cudaMemcpyHostToDevice, ctx->stream);
    mdp_ecg_params      prm = {tol, maxIter, enlFac, ortho_alg, bs_red, 0};
    mdp_solve_info      info = {};
    std::vector<double> res(std::max(maxIter, 1) + 1, 0.0);
    rc = mdp_ecg_run(ctx, D->P, N, bj.inv.as<double>(), bj.npix, db.as<double>(), dn.as<double>(), &prm,
                     dx.as<double>(), res.data(), &info);
    if (rc) return fail("ECG_GLS", rc);
    cudaMemcpy(x, dx.p, 8 * 3 * bj.npix, cudaMemcpyDeviceToHost);
    cudaMemcpy(cond, bj.rcond.p, 8 * bj.npix, cudaMemcpyDeviceToHost);
    cudaMemcpy(lhits, bj.hits.p, 4 * bj.npix, cudaMemcpyDeviceToHost);
    printf("*** ECG: %d iterations, relative residual %e (%s)\n", info.iterations, std::sqrt(info.res / info.res0),
           info.converged ? "converged" : "not converged");
    write_ecg_residuals(outpath, ref, res, info.iterations, enlFac, ortho_alg);
    return 0;
}

// ------------------------------------------------------------------ MLmap
// x2map_pol (mappraiser.c:836-853)
static void x2map(double *mapI, double *mapQ, double *mapU, double *Cond, int *Hits, const double *x, const int *lstid,
                  const double *cond, const int *lhits, int64_t xsize, int64_t npix) {
    for (int64_t i = 0; i < xsize; i++) {
        int64_t p = lstid[i] / 3;
        if (p < 0 || p >= npix) continue;
        if (i % 3 == 0) {
            if (mapI) mapI[p] = x[i];
            if (Hits) Hits[p] = lhits[i / 3];
            if (Cond) Cond[p] = cond[i / 3];
        } else if (i % 3 == 1) {
            if (mapQ) mapQ[p] = x[i];
        } else if (mapU) {
            mapU[p] = x[i];
        }
    }
}

// scan != nullptr: MTmap's template-filtered solve (lambda 1, one weight per block in invtt)
static int mlmap_device(int m, int nb, const int *blocks, const int *pix, const double *w, const double *sig,
                        const double *noi, int lambda, const double *invtt, double tol, int maxiter, int verbose,
                        int precond, int z_2lvl, int solver, int enl_fac, int ortho_alg, int bs_red,
                        std::vector<double> &x, std::vector<int> &lstid, std::vector<double> &cond,
                        std::vector<int> &hits, int *iters, double *res_rel,
                        const mdp_template_scan *scan = nullptr, std::vector<double> *res_hist = nullptr) {
    mdp_context *ctx = default_ctx();
    if (!ctx) return MDP_ECUDA;
    const int64_t n3 = 3LL * m;
    DevBuf        dpix, dw, ds, dn;
    int           rc;
    if ((rc = dpix.alloc(4 * n3)) || (rc = dw.alloc(8 * n3)) || (rc = ds.alloc(8LL * m)) || (rc = dn.alloc(8LL * m))) return rc;
    cudaStream_t st = ctx->stream;
    cudaMemcpyAsync(dpix.p, pix, 4 * n3, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(dw.p, w, 8 * n3, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(ds.p, sig, 8LL * m, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(dn.p, noi, 8LL * m, cudaMemcpyHostToDevice, st);
    mdp_pointing *P = nullptr;
    if ((rc = mdp_pointing_create(ctx, m, 3, dpix.as<int32_t>(), dw.as<double>(), &P))) return rc;
    std::vector<int64_t> idv(nb);
    std::vector<int32_t> nn(nb);
    int64_t              acc = 0;
    for (int b = 0; b < nb; b++) {
        idv[b] = acc;
        nn[b] = blocks[b];
        acc += blocks[b];
    }
    mdp_noise *N = nullptr;
    if ((rc = mdp_noise_create(ctx, nb, idv.data(), nn.data(), lambda, invtt, &N))) {
        mdp_pointing_destroy(P);
        return rc;
    }
    const int64_t nmap = P->n_map();
    DevBuf        dx, dl, dc, dh;
    if ((rc = dx.alloc(8 * nmap)) || (rc = dl.alloc(4 * nmap)) || (rc = dc.alloc(8 * (nmap / 3 + 1))) ||
        (rc = dh.alloc(4 * (nmap / 3 + 1)))) {
        mdp_pointing_destroy(P);
        mdp_noise_destroy(N);
        return rc;
    }
    mdp_solve_params    prm = {tol, maxiter, verbose, precond, z_2lvl};
    mdp_solve_info      info = {};
    std::vector<double> res(std::max(maxiter, 1) + 1, 0.0);
    mdp_templates *T = nullptr;
    if (scan && (rc = mdp_templates_create(ctx, scan, invtt, &T))) {
        mdp_pointing_destroy(P);
        mdp_noise_destroy(N);
        return rc;
    }
    if (T) {
        rc = mdp_gls_solve_templates(ctx, P, N, T, ds.as<double>(), dn.as<double>(), &prm, dx.as<double>(),
                                     dl.as<int32_t>(), dc.as<double>(), dh.as<int32_t>(), res.data(), &info);
        mdp_templates_destroy(T);
    } else if (solver == 1) {
        mdp_ecg_params eprm = {tol, maxiter, enl_fac, ortho_alg, bs_red, verbose};
        rc = mdp_ecg_solve(ctx, P, N, ds.as<double>(), dn.as<double>(), &eprm, dx.as<double>(), dl.as<int32_t>(),
                           dc.as<double>(), dh.as<int32_t>(), res.data(), &info);
    } else {
        rc = mdp_gls_solve(ctx, P, N, ds.as<double>(), dn.as<double>(), &prm, dx.as<double>(), dl.as<int32_t>(),
                           dc.as<double>(), dh.as<int32_t>(), res.data(), &info);
    }
    if (!rc) {
        const int64_t n = info.n_map;
        x.resize(n);
        lstid.resize(n);
        cond.resize(n / 3);
        hits.resize(n / 3);
        cudaMemcpyAsync(x.data(), dx.p, 8 * n, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(lstid.data(), dl.p, 4 * n, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(cond.data(), dc.p, 8 * (n / 3), cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(hits.data(), dh.p, 4 * (n / 3), cudaMemcpyDeviceToHost, st);
        if (cudaStreamSynchronize(st) != cudaSuccess) rc = MDP_ECUDA;
        if (iters) *iters = info.iterations;
        if (res_rel) *res_rel = std::sqrt(info.res / info.res0);
        if (res_hist) *res_hist = res;
    }
    mdp_pointing_destroy(P);
    mdp_noise_destroy(N);
    return rc;
}

// HEALPix FITS map writer with the layout the reference's write_map
// (iofiles.c:19-52) gets from CFITSIO: an empty primary array (BITPIX 16,
// NAXIS 0, EXTEND) with its creation DATE, then one binary table of 12 nside^2
// rows and one column SIGNAL of format 1D (8-byte doubles, big endian; integer
// maps are converted, as fits_write_col converts them into that column) with
// PIXTYPE, ORDERING, NSIDE, COORDSYS and the coordinate-system comment.
static void fits_card(std::string &h, const char *key, const char *val, const char *comment) {
    char c[81];
    if (val)
        snprintf(c, sizeof(c), "%-8.8s= %20s / %-47.47s", key, val, comment ? comment : "");
    else
        snprintf(c, sizeof(c), "%-80.80s", key);
    std::string s(c);
    s.resize(80, ' ');
    h += s;
}
static void fits_string_card(std::string &h, const char *key, const char *val, const char *comment) {
    char q[72];
    snprintf(q, sizeof(q), "'%-8s'", val);  // strings padded to at least 8 characters
    char c[81];
    snprintf(c, sizeof(c), "%-8.8s= %-20s / %-47.47s", key, q, comment);
    std::string s(c);
    s.resize(80, ' ');
    h += s;
}
static void fits_pad(std::string &h, char fill) {
    while (h.size() % 2880) h.push_back(fill);
}
// CFITSIO's data type codes of the two maps MLmap writes
#define MDP_FITS_TINT 31
#define MDP_FITS_TDOUBLE 82
static int write_fits_map(const char *path, const void *data, int type, long nside, bool nest, char coordsys) {
    const int64_t npix = 12LL * nside * nside;
    std::string   hdr;
    fits_card(hdr, "SIMPLE", "T", "file does conform to FITS standard");
    fits_card(hdr, "BITPIX", "16", "number of bits per data pixel");
    fits_card(hdr, "NAXIS", "0", "number of data axes");
    fits_card(hdr, "EXTEND", "T", "FITS dataset may contain extensions");
    {
        char           date[32];
        const time_t   now = time(nullptr);
        struct tm      ut;
        gmtime_r(&now, &ut);
        strftime(date, sizeof(date), "%Y-%m-%dT%H:%M:%S", &ut);
        fits_string_card(hdr, "DATE", date, "file creation date (YYYY-MM-DDThh:mm:ss UT)");
    }
    fits_card(hdr, "END", nullptr, nullptr);
    fits_pad(hdr, ' ');
    std::string ext;
    char        v[32];
    fits_string_card(ext, "XTENSION", "BINTABLE", "binary table extension");
    fits_card(ext, "BITPIX", "8", "8-bit bytes");
    fits_card(ext, "NAXIS", "2", "2-dimensional binary table");
    fits_card(ext, "NAXIS1", "8", "width of table in bytes");
    snprintf(v, sizeof(v), "%lld", (long long) npix);
    fits_card(ext, "NAXIS2", v, "number of rows in table");
    fits_card(ext, "PCOUNT", "0", "size of special data area");
    fits_card(ext, "GCOUNT", "1", "one data group (required keyword)");
    fits_card(ext, "TFIELDS", "1", "number of fields in each row");
    fits_string_card(ext, "TTYPE1", "SIGNAL", "label for field   1");
    fits_string_card(ext, "TFORM1", "1D", "data format of field: 8-byte DOUBLE");
    fits_string_card(ext, "TUNIT1", " ", "physical unit of field");
    fits_string_card(ext, "EXTNAME", "BINTABLE", "name of this binary table extension");
    fits_string_card(ext, "PIXTYPE", "HEALPIX", "HEALPIX Pixelisation");
    fits_string_card(ext, "ORDERING", nest ? "NESTED" : "RING", "Pixel ordering scheme, either RING or NESTED");
    snprintf(v, sizeof(v), "%ld", nside);
    fits_card(ext, "NSIDE", v, "Resolution parameter for HEALPIX");
    const char cs[2] = {coordsys, 0};
    fits_string_card(ext, "COORDSYS", cs, "Pixelisation coordinate system");
    fits_card(ext, "COMMENT G = Galactic, E = ecliptic, C = celestial = equatorial", nullptr, nullptr);
    fits_card(ext, "END", nullptr, nullptr);
    fits_pad(ext, ' ');
    FILE *f = fopen(path, "wb");
    if (!f) return 1;
    fwrite(hdr.data(), 1, hdr.size(), f);
    fwrite(ext.data(), 1, ext.size(), f);
    std::vector<char> buf(8 * (size_t) npix);
    for (int64_t i = 0; i < npix; i++) {
        const double d = (type == MDP_FITS_TINT) ? (double) ((const int *) data)[i] : ((const double *) data)[i];
        const unsigned char *src = (const unsigned char *) &d;
        for (int b = 0; b < 8; b++) buf[8 * i + b] = (char) src[7 - b];  // big endian
    }
    fwrite(buf.data(), 1, buf.size(), f);
    size_t            tail = (2880 - buf.size() % 2880) % 2880;
    std::vector<char> z(tail, 0);
    fwrite(z.data(), 1, tail, f);
    return fclose(f) == 0 ? 0 : 1;
}

// iofiles.h:24 -> iofiles.c:19-52
extern "C" void write_map(void *signal, int type, long nside, const char *filename, char nest, const char *coordsys) {
    if (!signal || !filename || nside < 1 || (type != MDP_FITS_TINT && type != MDP_FITS_TDOUBLE)) {
        fprintf(stderr, "write_map: a TDOUBLE (82) or TINT (31) map of nside >= 1 is needed\n");
        return;
    }
    const char c = (coordsys && coordsys[0]) ? coordsys[0] : 'C';
    if (write_fits_map(filename, signal, type, nside, nest != 0, c)) fprintf(stderr, "write_map: cannot write %s\n", filename);
}

// the five maps as FITS files <outpath>/{mapI,mapQ,mapU,Cond,Hits}_<ref>.fits
static void write_maps(const char *outpath, const char *ref, int nside, const std::vector<double> &x,
                       const std::vector<int> &lstid, const std::vector<double> &cond, const std::vector<int> &hits,
                       const char *who);

extern "C" void MLmap(MPI_Comm comm, char *outpath, char *ref, int solver, int precond, int Z_2lvl,
                      int pointing_commflag, double tol, int maxiter, int enlFac, int ortho_alg, int bs_red, int nside,
                      void *data_size_proc, int nb_blocks_loc, void *local_blocks_sizes, int Nnz, void *pix,
                      void *pixweights, void *signal, double *noise, int lambda, double *invtt) {
    (void) comm, (void) pointing_commflag;
    if (solver < 0 || solver > 1 || precond < 0 || precond > 2 || Nnz != 3 || (solver == 1 && precond != 0)) {
        fprintf(stderr, "midapack_b200 MLmap: solver 0 (PCG, precond 0, 1, 2) or 1 (ECG, block Jacobi) with Nnz 3\n");
        return;
    }
    const int m = ((int *) data_size_proc)[0];
    printf("\n############# MAPPRAISER (midapack_b200, one GPU) ################\n");
    std::vector<double> x, cond, hist;
    std::vector<int>    lstid, hits;
    int                 it = 0;
    double              rr = 0;
    int rc;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        rc = mlmap_device(m, nb_blocks_loc, (const int *) local_blocks_sizes, (const int *) pix,
                          (const double *) pixweights, (const double *) signal, noise, lambda, invtt, tol, maxiter, 1,
                          precond, Z_2lvl, solver, enlFac, ortho_alg, bs_red, x, lstid, cond, hits, &it, &rr, nullptr,
                          &hist);
    }
    if (rc) {
        fail("MLmap", rc);
        return;
    }
    // the residual history the reference's solver writes (PCG_GLS_true,
    // pcg_true.c:119-123,195: one double per iteration from k = 0; ECG_GLS,
    // ecg.c:156-161: one line per iteration)
    if (solver == 0) write_residuals(outpath, ref, hist, it < maxiter ? it : maxiter - 1);
    else write_ecg_residuals(outpath, ref, hist, it, enlFac, ortho_alg);
    write_maps(outpath, ref, nside, x, lstid, cond, hits, "MLmap");
    printf("[midapack_b200] %d iterations, final res_rel %e\n", it, rr);
}

static void write_maps(const char *outpath, const char *ref, int nside, const std::vector<double> &x,
                       const std::vector<int> &lstid, const std::vector<double> &cond, const std::vector<int> &hits,
                       const char *who) {
    const int64_t       npix = 12LL * nside * nside;
    std::vector<double> mI(npix, 0.0), mQ(npix, 0.0), mU(npix, 0.0), mC(npix, 0.0);
    std::vector<int>    mH(npix, 0);
    x2map(mI.data(), mQ.data(), mU.data(), mC.data(), mH.data(), x.data(), lstid.data(), cond.data(), hits.data(),
          (int64_t) x.size(), npix);
    const char *names[5] = {"mapI", "mapQ", "mapU", "Cond", "Hits"};
    const void *data[5] = {mI.data(), mQ.data(), mU.data(), mC.data(), mH.data()};
    for (int i = 0; i < 5; i++) {
        char fn[4096];
        snprintf(fn, sizeof(fn), "%s/%s_%s.fits", outpath, names[i], ref);
        if (write_fits_map(fn, data[i], i == 4 ? MDP_FITS_TINT : MDP_FITS_TDOUBLE, nside, true, 'C'))
            fprintf(stderr, "%s: cannot write %s\n", who, fn);
    }
}

// MTmap (mappraiser/src/mappraiser.c:387-800; map.h:15-18): MLmap with per-block template
// amplitudes marginalised (PCG_GLS_templates), white noise per block (invtt: one weight
// per block, lambda 1).  One rank, solver 0 with precond 0; every block as long as its
// CES (sweeptstamps[i][nsweeps[i]] samples), detector-minor within each CES.
extern "C" void MTmap(MPI_Comm comm, char *outpath, char *ref, int solver, int precond, int Z_2lvl,
                      int pointing_commflag, int npoly, int nhwp, double delta_t, int ground, int n_sss_bins,
                      double tol, int maxiter, int enlFac, int ortho_alg, int bs_red, int nside, int **sweeptstamps,
                      int *nsweeps, double **az, double *az_min, double *az_max, double **hwp_angle, int nces,
                      void *data_size_proc, int nb_blocks_loc, void *local_blocks_sizes, int Nnz, void *pix,
                      void *pixweights, void *signal, double *noise, double sampling_freq, double *invtt) {
    (void) comm, (void) pointing_commflag, (void) Z_2lvl, (void) enlFac, (void) ortho_alg, (void) bs_red;
    if (solver != 0 || precond != 0 || Nnz != 3 || nces < 1 || nb_blocks_loc % nces != 0) {
        fprintf(stderr, "midapack_b200 MTmap: solver 0 with precond 0, Nnz 3, nb_blocks_loc a multiple of nces\n");
        return;
    }
    const int m = ((int *) data_size_proc)[0];
    const int ndet = nb_blocks_loc / nces;
    const int *blocks = (const int *) local_blocks_sizes;
    std::vector<int32_t> nsw(nces), sw;
    std::vector<double>  azf, hwpf;
    for (int i = 0; i < nces; ++i) {
        nsw[i] = nsweeps[i];
        const int L = sweeptstamps[i][nsweeps[i]];
        for (int k = 0; k <= nsweeps[i]; ++k) sw.push_back(sweeptstamps[i][k]);
        for (int j = 0; j < ndet; ++j)
            if (blocks[i * ndet + j] != L) {
                fprintf(stderr, "midapack_b200 MTmap: block %d has %d samples, its CES %d has %d\n", i * ndet + j,
                        blocks[i * ndet + j], i, L);
                return;
            }
        if (ground) azf.insert(azf.end(), az[i], az[i] + L);
        if (nhwp) hwpf.insert(hwpf.end(), hwp_angle[i], hwp_angle[i] + L);
    }
    mdp_template_scan scan = {nces, ndet, npoly, ground, n_sss_bins, nhwp, delta_t, sampling_freq, nsw.data(),
                              sw.data(), ground ? azf.data() : nullptr, ground ? az_min : nullptr,
                              ground ? az_max : nullptr, nhwp ? hwpf.data() : nullptr};
    printf("\n############# MAPPRAISER MTmap (midapack_b200, one GPU) ################\n");
    std::vector<double> x, cond, hist;
    std::vector<int>    lstid, hits;
    int                 it = 0;
    double              rr = 0;
    int                 rc;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        rc = mlmap_device(m, nb_blocks_loc, blocks, (const int *) pix, (const double *) pixweights,
                          (const double *) signal, noise, 1, invtt, tol, maxiter, 1, 0, 0, 0, 1, 1, 0, x, lstid, cond,
                          hits, &it, &rr, &scan, &hist);
    }
    if (rc) {
        fail("MTmap", rc);
        return;
    }
    // PCG_GLS_templates' residual history (pcg_true.c:415-420,520-523)
    write_residuals(outpath, ref, hist, it < maxiter ? it : maxiter - 1);
    write_maps(outpath, ref, nside, x, lstid, cond, hits, "MTmap");
    printf("[midapack_b200] %d iterations, final res_rel %e\n", it, rr);
}

extern "C" int MLmap_b200(int solver, int precond, double tol, int maxiter, int nside, int m, int nb_blocks_loc,
                          const int *local_blocks_sizes, int Nnz, const int *pix, const double *pixweights,
                          const double *signal, const double *noise, int lambda, const double *invtt, double *mapI,
                          double *mapQ, double *mapU, double *Cond, int *Hits, int *iterations, double *res_rel) {
    if (solver < 0 || solver > 1 || precond < 0 || precond > 2 || Nnz != 3 || (solver == 1 && precond != 0)) {
        mdp_set_error("MLmap_b200: solver 0 (PCG, precond 0, 1, 2) or 1 (ECG with enlFac 1, block Jacobi), Nnz 3");
        return MDP_EUNSUPPORTED;
    }
    std::vector<double> x, cond;
    std::vector<int>    lstid, hits;
    int                 rc;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        rc = mlmap_device(m, nb_blocks_loc, local_blocks_sizes, pix, pixweights, signal, noise, lambda, invtt, tol,
                          maxiter, 0, precond, 0, solver, 1, 1, 0, x, lstid, cond, hits, iterations, res_rel);
    }
    if (rc) return rc;
    const int64_t npix = 12LL * nside * nside;
    x2map(mapI, mapQ, mapU, Cond, Hits, x.data(), lstid.data(), cond.data(), hits.data(), (int64_t) x.size(), npix);
    return MDP_OK;
}
