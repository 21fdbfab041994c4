// Enlarged conjugate gradient (ECG) solve of (P^T N^-1 P) x = P^T N^-1 d:
// MAPPRAISER's solver 1 (mappraiser/src/ecg.c:44-175, ECG_GLS, and its block
// operators Opmmmatrix / Opmmpreconditioner at :196-245).  The reference takes
// the ECG iteration from preAlps (overlap_ecg.h, not part of the reference
// and not in this image); the iteration here restates the published method
// (Grigori, Moufawad & Nataf, SIAM J. Matrix Anal. Appl. 37:744, 2016;
// Grigori & Tissot, Numer. Algorithms 80:1333, 2019):
//
//   R_0 = T(r_0) (t = enlFac columns: the residual split over t contiguous
//   ranges of the map's pixels), P = M^-1 R_0, AP = A P, A-orthonormalised;
//   per iteration: alpha = P^T R, X += P alpha, R -= AP alpha, stop when
//   ||sum_j R_j|| < tol ||r_0||; Orthomin (ortho_alg 1): Z = M^-1 R,
//   P <- Z - P (AP^T Z); Orthodir (ortho_alg 0): Z = M^-1 AP,
//   P <- Z - P (AP^T Z) - P_prev (AP_prev^T Z); AP = A P; A-orthonormalise
//   by the Cholesky factor of P^T A P, or (bs_red) by its eigenvectors,
//   dropping the directions whose eigenvalue is below 1e-12 of the largest
//   (the block shrinks); x = sum_j X_j.  Without bs_red a block that loses
//   rank (no Cholesky factor) ends the solve with an error.
//
// M is the block-Jacobi preconditioner with the rcond cut (the cut rewrites
// the pointing, ecg.c:67).  Device layout: each block of vectors is [cols][n]
// FP64 (one contiguous map per column).  The small matrices (t x t Gram
// products, alpha, beta) are formed on the device by deterministic
// reductions; only P^T A P goes to the host for its t x t factorisation.
#include <chrono>
#include <cmath>
#include <vector>

#include "mdp_internal.cuh"
#include "smalldense.h"

namespace {

constexpr int ET = 256;    // threads of the block kernels
constexpr int EBLK = 296;  // blocks of the reductions (2 per SM)
constexpr int GK = 16;     // rows staged per Gram step

// Gram partials: part[e][bx], e = a * nb + b, the sum over bx's rows k of
// X[a][k] * Y[b][k]; one entry per thread, the rows staged 16 at a time.
__global__ void __launch_bounds__(ET) gram_kernel(const double *__restrict__ X, int na, const double *__restrict__ Y,
                                                 int nb, int64_t n, double *__restrict__ part) {
    extern __shared__ double gs[];  // Xs[na][GK], Ys[nb][GK]
    double   *Xs = gs, *Ys = gs + na * GK;
    const int e = blockIdx.y * ET + threadIdx.x;
    const int a = e / nb, b = e % nb;
    double    s = 0.0;
    for (int64_t k0 = (int64_t) blockIdx.x * GK; k0 < n; k0 += (int64_t) gridDim.x * GK) {
        __syncthreads();
        for (int l = threadIdx.x; l < (na + nb) * GK; l += ET) {
            const int     c = l / GK, kk = l % GK;
            const int64_t k = k0 + kk;
            const double *src = c < na ? X + (int64_t) c * n : Y + (int64_t) (c - na) * n;
            gs[l] = k < n ? src[k] : 0.0;
        }
        __syncthreads();
        if (e < na * nb)
#pragma unroll
            for (int kk = 0; kk < GK; kk++) s += Xs[a * GK + kk] * Ys[b * GK + kk];
    }
    if (e < na * nb) part[(int64_t) e * gridDim.x + blockIdx.x] = s;
}

// out[e] = sum of part[e][0..nblk) in block order
__global__ void sum_kernel(const double *__restrict__ part, int nblk, int ne, double *__restrict__ out) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int b = 0; b < nblk; b++) s += part[(int64_t) e * nblk + b];
        out[e] = s;
    }
}

// out[j][i] = base[j][i] + sgn * sum_l C[l * ldc + j] V[l][i] (j < nout; base
// null: 0).  out may be base (element-wise in place).
constexpr int CJ = 8;
__global__ void __launch_bounds__(ET) combine_kernel(const double *base, double sgn, const double *__restrict__ V,
                                                    int nl, const double *__restrict__ C, int ldc, int nout, int64_t n,
                                                    double *out) {
    extern __shared__ double cs[];  // C [nl][nout]
    for (int l = threadIdx.x; l < nl * nout; l += ET) cs[l] = C[(l / nout) * ldc + l % nout];
    __syncthreads();
    for (int64_t i = (int64_t) blockIdx.x * ET + threadIdx.x; i < n; i += (int64_t) gridDim.x * ET) {
        for (int j0 = 0; j0 < nout; j0 += CJ) {
            double acc[CJ];
#pragma unroll
            for (int r = 0; r < CJ; r++) acc[r] = 0.0;
            for (int l = 0; l < nl; l++) {
                const double v = V[(int64_t) l * n + i];
#pragma unroll
                for (int r = 0; r < CJ; r++)
                    if (j0 + r < nout) acc[r] += cs[l * nout + j0 + r] * v;
            }
#pragma unroll
            for (int r = 0; r < CJ; r++)
                if (j0 + r < nout) {
                    const int64_t o = (int64_t) (j0 + r) * n + i;
                    out[o] = (base ? base[o] : 0.0) + sgn * acc[r];
                }
        }
    }
}

// Z[j] = BJ_inv R[j] for j < ncol (apply_precond, precond 0, per column)
__global__ void bj_cols_kernel(const double *__restrict__ inv, const double *__restrict__ R, int ncol, int64_t npix,
                               double *__restrict__ Z) {
    const int64_t n = 3 * npix;
    for (int64_t q = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; q < npix; q += (int64_t) gridDim.x * blockDim.x) {
        const double *I = inv + 9 * q;
        for (int j = 0; j < ncol; j++) {
            const double *r = R + (int64_t) j * n + 3 * q;
            double       *z = Z + (int64_t) j * n + 3 * q;
            const double  g0 = r[0], g1 = r[1], g2 = r[2];
            z[0] = I[0] * g0 + I[1] * g1 + I[2] * g2;
            z[1] = I[3] * g0 + I[4] * g1 + I[5] * g2;
            z[2] = I[6] * g0 + I[7] * g1 + I[8] * g2;
        }
    }
}

// part[bx] = partial sum over i of (sum_j R[j][i])^2
__global__ void __launch_bounds__(ET) colsum_sq_kernel(const double *__restrict__ R, int t, int64_t n,
                                                      double *__restrict__ part) {
    double s = 0.0;
    for (int64_t i = (int64_t) blockIdx.x * ET + threadIdx.x; i < n; i += (int64_t) gridDim.x * ET) {
        double r = 0.0;
        for (int j = 0; j < t; j++) r += R[(int64_t) j * n + i];
        s += r * r;
    }
    __shared__ double sh[ET / 32];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double u = 0.0;
        for (int w = 0; w < ET / 32; w++) u += sh[w];
        part[blockIdx.x] = u;
    }
}

// x = sum_j X[j]
__global__ void colsum_kernel(const double *__restrict__ X, int t, int64_t n, double *__restrict__ x) {
    for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int j = 0; j < t; j++) s += X[(int64_t) j * n + i];
        x[i] = s;
    }
}

// T(r): R[j][i] = r[i] on the j-th of t contiguous pixel ranges, 0 elsewhere
__global__ void split_kernel(const double *__restrict__ r, int t, int64_t npix, double *__restrict__ R) {
    const int64_t n = 3 * npix;
    for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x) {
        const int c = (int) ((i / 3) * t / npix);
        for (int j = 0; j < t; j++) R[(int64_t) j * n + i] = (j == c) ? r[i] : 0.0;
    }
}

struct Ecg {
    mdp_context *ctx;
    int64_t      n;
    DevBuf       part, small;  // reduction partials; small matrices on the device

    // G = X Y^T ([na][nb]) into small + off (device)
    int gram(const double *X, int na, const double *Y, int nb, int64_t off) {
        const int ne = na * nb, gy = (ne + ET - 1) / ET;
        MDP_TRY(part.alloc(8 * (size_t) ne * EBLK));
        const size_t sm = 8 * (size_t) (na + nb) * GK;
        gram_kernel<<<dim3(EBLK, gy), ET, sm, ctx->stream>>>(X, na, Y, nb, n, part.as<double>());
        MDP_CHECK_LAUNCH(ctx);
        sum_kernel<<<(ne + 255) / 256, 256, 0, ctx->stream>>>(part.as<double>(), EBLK, ne, small.as<double>() + off);
        MDP_CHECK_LAUNCH(ctx);
        return MDP_OK;
    }
    int combine(const double *base, double sgn, const double *V, int nl, const double *C, int ldc, int nout,
                double *out) {
        const size_t sm = 8 * (size_t) nl * nout;
        combine_kernel<<<grid_for(n, ET, ctx->sm_count * 4), ET, sm, ctx->stream>>>(base, sgn, V, nl, C, ldc, nout,
                                                                                     n, out);
        MDP_CHECK_LAUNCH(ctx);
        return MDP_OK;
    }
    int norm_colsum(const double *R, int t, double *out) {
        MDP_TRY(part.alloc(8 * (size_t) (EBLK + 1)));
        colsum_sq_kernel<<<EBLK, ET, 0, ctx->stream>>>(R, t, n, part.as<double>());
        MDP_CHECK_LAUNCH(ctx);
        sum_kernel<<<1, 32, 0, ctx->stream>>>(part.as<double>(), EBLK, 1, part.as<double>() + EBLK);
        MDP_CHECK_LAUNCH(ctx);
        MDP_CUDA(cudaMemcpyAsync(ctx->h_pinned, part.as<double>() + EBLK, 8, cudaMemcpyDeviceToHost, ctx->stream));
        MDP_CUDA(cudaStreamSynchronize(ctx->stream));
        *out = std::sqrt(ctx->h_pinned[0]);
        return MDP_OK;
    }
};

}  // namespace

// The ECG iteration on the post-cut pointing with the block-Jacobi inverse
// blocks inv [npix][9]; d_x receives the n_map unknowns.
int mdp_ecg_run(mdp_context *ctx, mdp_pointing *A, const mdp_noise *N, const double *inv, int64_t npix,
                const double *d_signal, const double *d_noise, const mdp_ecg_params *prm, double *d_x,
                double *h_res_rel, mdp_solve_info *info) {
    const int     t = prm->enl_fac;
    const bool    omin = prm->ortho_alg != 0;
    const int64_t n = 3 * npix;
    cudaStream_t  st = ctx->stream;
    Ecg           E{ctx, n, {}, {}};
    // block vectors (t columns of n each) and the small matrices
    DevBuf bX, bR, bZ, bP, bAP, bPn, bAPn, bPp, bAPp, r0;
    const size_t blk = 8 * (size_t) t * std::max<int64_t>(n, 1);
    MDP_TRY(bX.alloc(blk));
    MDP_TRY(bR.alloc(blk));
    MDP_TRY(bZ.alloc(blk));
    MDP_TRY(bP.alloc(blk));
    MDP_TRY(bAP.alloc(blk));
    MDP_TRY(bPn.alloc(blk));
    MDP_TRY(bAPn.alloc(blk));
    if (!omin) {
        MDP_TRY(bPp.alloc(blk));
        MDP_TRY(bAPp.alloc(blk));
    }
    MDP_TRY(r0.alloc(8 * (size_t) std::max<int64_t>(n, 1)));
    MDP_TRY(E.small.alloc(8 * (size_t) 3 * t * t));
    double *X = bX.as<double>(), *R = bR.as<double>(), *Z = bZ.as<double>(), *P = bP.as<double>(),
           *AP = bAP.as<double>(), *Pn = bPn.as<double>(), *APn = bAPn.as<double>(), *Pp = bPp.as<double>(),
           *APp = bAPp.as<double>();
    double   *S = E.small.as<double>();  // [0, t*t): alpha / beta; [t*t, 2t*t): gamma; [2t*t, 3t*t): factor
    const int gn = grid_for(npix, 256, ctx->sm_count * 8);
    MDP_CUDA(cudaMemsetAsync(X, 0, blk, st));
    MDP_TRY(mdp_gls_rhs(ctx, A, N, d_signal, d_noise, r0.as<double>()));
    split_kernel<<<grid_for(n, 256, ctx->sm_count * 8), 256, 0, st>>>(r0.as<double>(), t, npix, R);
    MDP_CHECK_LAUNCH(ctx);
    double normb = 0.0;
    MDP_TRY(E.norm_colsum(R, t, &normb));
    if (!std::isfinite(normb)) {
        mdp_set_error("ECG: initial residual norm is %f", normb);
        return MDP_ENAN;
    }
    // A-orthonormalise the c columns of (Pn, APn) into (P, AP); returns the block size
    auto orthonormalize = [&](int c, int *bs) -> int {
        MDP_TRY(E.gram(Pn, c, APn, c, 2 * (int64_t) t * t));
        std::vector<double> G((size_t) c * c), F;
        MDP_CUDA(cudaMemcpyAsync(G.data(), S + 2 * (int64_t) t * t, 8 * (size_t) c * c, cudaMemcpyDeviceToHost, st));
        MDP_CUDA(cudaStreamSynchronize(st));
        for (int i = 0; i < c; i++)
            for (int j = 0; j < i; j++) G[(size_t) i * c + j] = G[(size_t) j * c + i] = 0.5 * (G[(size_t) i * c + j] + G[(size_t) j * c + i]);
        int                 k = c;
        std::vector<double> L;
        if (!prm->bs_red && mdp_dense::cholesky(c, G, L)) {
            const std::vector<double> Li = mdp_dense::lower_inverse(c, L);
            F.assign((size_t) c * c, 0.0);  // F[l][j] = Li[j][l]: P_j = sum_l Li[j][l] Pn_l
            for (int l = 0; l < c; l++)
                for (int j = 0; j < c; j++) F[(size_t) l * c + j] = Li[(size_t) j * c + l];
        } else if (prm->bs_red) {
            std::vector<double> w, V, Gc(G);
            mdp_dense::jacobi_eigh(c, Gc, w, V);
            const double top = w.empty() ? 0.0 : w.back();
            std::vector<int> keep;
            for (int j = 0; j < c; j++)
                if (w[j] > 1e-12 * top && w[j] > 0.0) keep.push_back(j);
            k = (int) keep.size();
            F.assign((size_t) c * std::max(k, 1), 0.0);
            for (int l = 0; l < c; l++)
                for (int j = 0; j < k; j++) F[(size_t) l * k + j] = V[(size_t) l * c + keep[j]] / std::sqrt(w[keep[j]]);
        } else {
            mdp_set_error("ECG: the block of search directions lost rank (P^T A P is not positive definite); "
                          "bs_red = 1 shrinks the block instead");
            return MDP_ENAN;
        }
        *bs = k;
        if (k == 0) return MDP_OK;
        MDP_CUDA(cudaMemcpyAsync(S + 2 * (int64_t) t * t, F.data(), 8 * (size_t) c * k, cudaMemcpyHostToDevice, st));
        MDP_TRY(E.combine(nullptr, 1.0, Pn, c, S + 2 * (int64_t) t * t, k, k, P));
        MDP_TRY(E.combine(nullptr, 1.0, APn, c, S + 2 * (int64_t) t * t, k, k, AP));
        MDP_CUDA(cudaStreamSynchronize(st));  // F is a host temporary
        return MDP_OK;
    };
    auto apply_block = [&](const double *V, int c, double *out) -> int {
        for (int j = 0; j < c; j++) MDP_TRY(mdp_apply_op_impl(ctx, A, N, V + (int64_t) j * n, out + (int64_t) j * n));
        return MDP_OK;
    };
    bj_cols_kernel<<<gn, 256, 0, st>>>(inv, R, t, npix, Pn);
    MDP_CHECK_LAUNCH(ctx);
    MDP_TRY(apply_block(Pn, t, APn));
    int bs = 0, bsp = 0;
    MDP_TRY(orthonormalize(t, &bs));
    if (h_res_rel) h_res_rel[0] = 1.0;
    if (prm->verbose) printf("ECG k = 0, ||r0|| = %e, bs = %d\n", normb, bs);
    int    it = 0, converged = 0;
    double res = normb;
    while (it < prm->maxiter && bs > 0) {
        MDP_TRY(E.gram(P, bs, R, t, 0));                     // alpha = P^T R [bs][t]
        MDP_TRY(E.combine(X, 1.0, P, bs, S, t, t, X));      // X += P alpha
        MDP_TRY(E.combine(R, -1.0, AP, bs, S, t, t, R));    // R -= AP alpha
        it++;
        MDP_TRY(E.norm_colsum(R, t, &res));
        if (!std::isfinite(res)) {
            mdp_set_error("ECG: residual became %f at iteration %d", res, it);
            return MDP_ENAN;
        }
        if (h_res_rel) h_res_rel[it] = res / normb;
        if (prm->verbose) printf("ECG k = %d, res_rel = %e, bs = %d\n", it, res / normb, bs);
        if (res < prm->tol * normb) {
            converged = 1;
            break;
        }
        if (it >= prm->maxiter) break;
        int c;
        if (omin) {
            bj_cols_kernel<<<gn, 256, 0, st>>>(inv, R, t, npix, Z);  // Z = M^-1 R
            MDP_CHECK_LAUNCH(ctx);
            MDP_TRY(E.gram(AP, bs, Z, t, 0));                       // beta = AP^T Z [bs][t]
            MDP_TRY(E.combine(Z, -1.0, P, bs, S, t, t, Pn));        // Pn = Z - P beta
            c = t;
        } else {
            bj_cols_kernel<<<gn, 256, 0, st>>>(inv, AP, bs, npix, Z);  // Z = M^-1 AP
            MDP_CHECK_LAUNCH(ctx);
            MDP_TRY(E.gram(AP, bs, Z, bs, 0));                         // beta = AP^T Z [bs][bs]
            MDP_TRY(E.combine(Z, -1.0, P, bs, S, bs, bs, Pn));         // Pn = Z - P beta
            if (bsp > 0) {
                MDP_TRY(E.gram(APp, bsp, Z, bs, (int64_t) t * t));     // gamma = AP_prev^T Z [bsp][bs]
                MDP_TRY(E.combine(Pn, -1.0, Pp, bsp, S + (int64_t) t * t, bs, bs, Pn));
            }
            std::swap(P, Pp);
            std::swap(AP, APp);
            bsp = bs;
            c = bs;
        }
        MDP_TRY(apply_block(Pn, c, APn));
        MDP_TRY(orthonormalize(c, &bs));
    }
    colsum_kernel<<<grid_for(n, 256, ctx->sm_count * 8), 256, 0, st>>>(X, t, n, d_x);
    MDP_CHECK_LAUNCH(ctx);
    MDP_CUDA(cudaStreamSynchronize(st));
    if (info) {
        info->iterations = it;
        info->converged = converged;
        info->res0 = normb * normb;
        info->res = res * res;
        info->n_map = n;
        info->outer_iterations = 0;
        info->fp64_applications = 0;
    }
    return MDP_OK;
}

extern "C" int mdp_ecg_solve(mdp_context *ctx, mdp_pointing *A, const mdp_noise *N, const double *d_signal,
                             const double *d_noise, const mdp_ecg_params *params, double *d_x, int32_t *d_lstid,
                             double *d_cond, int32_t *d_hits, double *h_res_rel, mdp_solve_info *info) {
    if (!ctx || !A || !N || !d_signal || !d_noise || !params || !d_x) {
        mdp_set_error("mdp_ecg_solve: invalid arguments");
        return MDP_EINVAL;
    }
    if (params->enl_fac < 1 || params->enl_fac > MDP_ECG_MAX_ENL) {
        mdp_set_error("mdp_ecg_solve: enlFac must be in 1..%d (got %d)", MDP_ECG_MAX_ENL, params->enl_fac);
        return MDP_EINVAL;
    }
    if (N->nrow_end > A->m) {
        mdp_set_error("mdp_ecg_solve: noise blocks extend past the pointing rows");
        return MDP_EINVAL;
    }
    MDP_CUDA(cudaSetDevice(ctx->device));
    auto           tp0 = std::chrono::steady_clock::now();
    const BJState *bjp = nullptr;
    MDP_TRY(mdp_bj_cached(ctx, A, N, &bjp));
    const BJState &bj = *bjp;
    cudaStream_t   st = ctx->stream;
    if (d_lstid)
        MDP_CUDA(cudaMemcpyAsync(d_lstid, A->lindices.as<int32_t>() + 3 * A->trash_pix, 4 * A->n_map(),
                                 cudaMemcpyDeviceToDevice, st));
    if (d_cond) MDP_CUDA(cudaMemcpyAsync(d_cond, bj.rcond.p, 8 * bj.npix, cudaMemcpyDeviceToDevice, st));
    if (d_hits) MDP_CUDA(cudaMemcpyAsync(d_hits, bj.hits.p, 4 * bj.npix, cudaMemcpyDeviceToDevice, st));
    MDP_CUDA(cudaStreamSynchronize(st));
    auto tp1 = std::chrono::steady_clock::now();
    MDP_TRY(mdp_ecg_run(ctx, A, N, bj.inv.as<double>(), bj.npix, d_signal, d_noise, params, d_x, h_res_rel, info));
    auto tp2 = std::chrono::steady_clock::now();
    if (info) {
        info->n_cut = bj.ncut;
        info->precond_seconds = std::chrono::duration<double>(tp1 - tp0).count();
        info->solve_seconds = std::chrono::duration<double>(tp2 - tp1).count();
    }
    return MDP_OK;
}
