// Two-level preconditioners of the PCG: precond 1 ("a priori": deflation
// columns from the sample counts of row groups) and precond 2 ("a
// posteriori": Ritz vectors of a Lanczos run from the first residual).
//
// Reference: mappraiser/src/precond.c:770-788 (inverse_svd_bis: dgelss
// pseudo-inverse, rcond 1e-15), 791-938 (build_Z), 951-1000 (build_Em1),
// 1003-1024 (build_AZ), 1026-1069 (build_Qtx, mul_ZQtx), 1028-1252
// (Lanczos_eig), 1310-1423 (build_precond, apply_precond); pcg_true.c:52
// (z_2lvl = 0 means one column per rank).
//
// The preconditioner is M g = BJ_inv (g - AZ qtx) + Z qtx with
// qtx = E^+ Z^T g, E = Z^T AZ and AZ = P^T N^-1 P Z.
//
// Device layout: Z and AZ are [zn][n] FP64, one contiguous column per
// deflation vector, so Z^T g is zn coalesced dot products and M g reads each
// column once per pixel triple.  The dense zn x zn and K x K problems (the
// pseudo-inverse of E, the eigenvectors of the Lanczos tridiagonal matrix) are
// solved on the host with Jacobi methods, as the reference calls LAPACK on the
// host; they are at most 128 x 128.  Everything of size n runs on the device:
// the counts, the operator applications, the Lanczos vectors, the Ritz
// combinations and the Gram matrix.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <vector>

#include "mdp_internal.cuh"
#include "smalldense.h"

namespace {

constexpr double EPS_2LVL = 1.0e-15;  // precond.c:25
constexpr int    TLT = 256;           // threads of the reduction kernels

// ------------------------------------------------------------ a priori columns
// cnt[g][L] += 1 for the rows t of group g (t < group * rows_per), L the local
// pixel of the row counting the trash pixel first: the reference's count of
// local index 3L (and 3L+1, 3L+2) in build_Z.  Trash and cut rows point to
// the trash pixel L = 0.
__global__ void z_count_kernel(const int32_t *__restrict__ off, int64_t rows_per, int group, int trash,
                               int64_t npix_l, int32_t *__restrict__ cnt) {
    const int64_t total = rows_per * group;
    for (int64_t t = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t) gridDim.x * blockDim.x) {
        const int32_t o = off[t];
        const int64_t L = o >= 0 ? (int64_t) (o / 3) + trash : 0;
        atomicAdd(&cnt[(int64_t) (t / rows_per) * npix_l + L], 1);
    }
}

// Z[g][3q] = count_flat[g * group + i] / tcount[i] with i = 3 (q + trash) and
// count_flat the [group][lcount] entry counts flattened (precond.c:873-879,
// its index kept as it is); Z[g][3q+1] = Z[g][3q+2] = 0.
__global__ void z_fill_kernel(const int32_t *__restrict__ cnt, int group, int trash, int64_t npix_l, int64_t npix,
                              double *__restrict__ Z) {
    const int64_t lcount = 3 * npix_l, n = 3 * npix;
    for (int64_t q = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; q < npix; q += (int64_t) gridDim.x * blockDim.x) {
        const int64_t i = 3 * (q + trash);
        int64_t       tc = 0;
        for (int g = 0; g < group; g++) tc += cnt[(int64_t) g * npix_l + i / 3];
        for (int g = 0; g < group; g++) {
            const int64_t idx = (int64_t) g * group + i;  // < group * lcount (checked on the host)
            const int64_t c = cnt[(idx / lcount) * npix_l + (idx % lcount) / 3];
            double       *z = Z + (int64_t) g * n + 3 * q;
            z[0] = (double) c / (double) tc;
            z[1] = 0.0;
            z[2] = 0.0;
        }
    }
}

// ------------------------------------------------------------ reductions
// part[blockIdx.y][blockIdx.x] = partial sum of a[y][k] * b[k] (b shared by
// every y when b_stride = 0)
__global__ void __launch_bounds__(TLT) dot_partial_kernel(const double *__restrict__ a, int64_t a_stride,
                                                         const double *__restrict__ b, int64_t b_stride, int64_t n,
                                                         double *__restrict__ part) {
    const double *x = a + (int64_t) blockIdx.y * a_stride;
    const double *y = b + (int64_t) blockIdx.y * b_stride;
    double        s = 0.0;
    for (int64_t k = (int64_t) blockIdx.x * TLT + threadIdx.x; k < n; k += (int64_t) gridDim.x * TLT) s += x[k] * y[k];
    __shared__ double sh[TLT / 32];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < TLT / 32; w++) t += sh[w];
        part[(int64_t) blockIdx.y * gridDim.x + blockIdx.x] = t;
    }
}

// out[y] = sum of part[y][0..nb) in block order
__global__ void sum_partials_kernel(const double *__restrict__ part, int nb, int ny, double *__restrict__ out) {
    for (int y = threadIdx.x; y < ny; y += blockDim.x) {
        double s = 0.0;
        for (int b = 0; b < nb; b++) s += part[(int64_t) y * nb + b];
        out[y] = s;
    }
}

// qtx = Em1 (Z^T g): w[j] from the partials in block order, then the small product (precond.c:1036-1051)
__global__ void qtx_kernel(const double *__restrict__ part, int nb, const double *__restrict__ Em1, int zn,
                           double *__restrict__ qtx) {
    __shared__ double w[MDP_TL_MAX_ZN];
    for (int j = threadIdx.x; j < zn; j += blockDim.x) {
        double s = 0.0;
        for (int b = 0; b < nb; b++) s += part[(int64_t) j * nb + b];
        w[j] = s;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < zn; i += blockDim.x) {
        double s = 0.0;
        for (int j = 0; j < zn; j++) s += Em1[i * zn + j] * w[j];
        qtx[i] = s;
    }
}

// E partials: part[e][bx] with e = i * zn + j, the sum over bx's rows k of
// Z[j][k] * AZ[i][k] (build_Em1's E[i][j]); one entry per thread, the block's
// rows staged in shared memory 16 at a time.
constexpr int GK = 16;
__global__ void __launch_bounds__(TLT) gram_partial_kernel(const double *__restrict__ Z, const double *__restrict__ AZ,
                                                          int zn, int64_t n, double *__restrict__ part) {
    extern __shared__ double gsm[];  // Zs[zn][GK], AZs[zn][GK]
    double   *Zs = gsm, *AZs = gsm + zn * GK;
    const int e = blockIdx.y * TLT + threadIdx.x;
    const int i = e / zn, j = e % zn;
    double    s = 0.0;
    for (int64_t k0 = (int64_t) blockIdx.x * GK; k0 < n; k0 += (int64_t) gridDim.x * GK) {
        __syncthreads();
        for (int l = threadIdx.x; l < zn * GK; l += TLT) {
            const int     c = l / GK, kk = l % GK;
            const int64_t k = k0 + kk;
            Zs[l] = k < n ? Z[(int64_t) c * n + k] : 0.0;
            AZs[l] = k < n ? AZ[(int64_t) c * n + k] : 0.0;
        }
        __syncthreads();
        if (e < zn * zn)
#pragma unroll
            for (int kk = 0; kk < GK; kk++) s += Zs[j * GK + kk] * AZs[i * GK + kk];
    }
    if (e < zn * zn) part[(int64_t) e * gridDim.x + blockIdx.x] = s;
}

// ------------------------------------------------------------ Lanczos vectors
// v = w / beta
__global__ void scale_copy_kernel(const double *__restrict__ w, double beta, double *__restrict__ v, int64_t n) {
    for (int64_t k = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t) gridDim.x * blockDim.x)
        v[k] = w[k] / beta;
}

// w = Av - alpha v - beta vold
__global__ void lanczos_w_kernel(const double *__restrict__ Av, const double *__restrict__ v,
                                 const double *__restrict__ vold, double alpha, double beta, double *__restrict__ w,
                                 int64_t n) {
    for (int64_t k = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t) gridDim.x * blockDim.x)
        w[k] = Av[k] - (alpha * v[k]) - (beta * vold[k]);
}

// out[j][k] = sum over l of V[l][k] * Y[l][j] in l order (the Ritz vectors,
// precond.c:1217-1236); 8 outputs per pass over the rows of V
constexpr int RJ = 8;
__global__ void ritz_kernel(const double *__restrict__ V, const double *__restrict__ Y, int K, int64_t n,
                            double *__restrict__ out) {
    extern __shared__ double ysm[];  // Y [K][K]
    for (int l = threadIdx.x; l < K * K; l += blockDim.x) ysm[l] = Y[l];
    __syncthreads();
    for (int64_t k = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t) gridDim.x * blockDim.x) {
        for (int j0 = 0; j0 < K; j0 += RJ) {
            double acc[RJ];
#pragma unroll
            for (int r = 0; r < RJ; r++) acc[r] = 0.0;
            for (int l = 0; l < K; l++) {
                const double v = V[(int64_t) l * n + k];
#pragma unroll
                for (int r = 0; r < RJ; r++)
                    if (j0 + r < K) acc[r] += v * ysm[l * K + j0 + r];
            }
#pragma unroll
            for (int r = 0; r < RJ; r++)
                if (j0 + r < K) out[(int64_t) (j0 + r) * n + k] = acc[r];
        }
    }
}

// deterministic dot product on the device, read back to the host
int dot_host(mdp_context *ctx, const double *a, const double *b, int64_t n, DevBuf &part, double *out) {
    MDP_TRY(part.alloc(8 * (MDP_TL_BLOCKS + 1)));
    dot_partial_kernel<<<dim3(MDP_TL_BLOCKS, 1), TLT, 0, ctx->stream>>>(a, 0, b, 0, n, part.as<double>());
    MDP_CHECK_LAUNCH(ctx);
    sum_partials_kernel<<<1, 32, 0, ctx->stream>>>(part.as<double>(), MDP_TL_BLOCKS, 1,
                                                   part.as<double>() + MDP_TL_BLOCKS);
    MDP_CHECK_LAUNCH(ctx);
    MDP_CUDA(cudaMemcpyAsync(ctx->h_pinned, part.as<double>() + MDP_TL_BLOCKS, 8, cudaMemcpyDeviceToHost,
                             ctx->stream));
    MDP_CUDA(cudaStreamSynchronize(ctx->stream));
    *out = ctx->h_pinned[0];
    return MDP_OK;
}

int ritz(mdp_context *ctx, const double *V, const std::vector<double> &Y, int K, int64_t n, double *out) {
    DevBuf dY;
    MDP_TRY(dY.alloc(8 * (size_t) K * K));
    MDP_CUDA(cudaMemcpyAsync(dY.p, Y.data(), 8 * (size_t) K * K, cudaMemcpyHostToDevice, ctx->stream));
    const size_t smem = 8 * (size_t) K * K;
    MDP_CUDA(cudaFuncSetAttribute((const void *) ritz_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int) (8 * MDP_TL_MAX_ZN * MDP_TL_MAX_ZN)));
    ritz_kernel<<<grid_for(n, 256, ctx->sm_count * 4), 256, smem, ctx->stream>>>(V, dY.as<double>(), K, n, out);
    MDP_CHECK_LAUNCH(ctx);
    MDP_CUDA(cudaStreamSynchronize(ctx->stream));  // dY is released on return
    return MDP_OK;
}

}  // namespace

// qtx = Em1 Z^T g on the device
int mdp_twolevel_qtx(mdp_context *ctx, const mdp_twolevel *tl, const double *d_g) {
    dot_partial_kernel<<<dim3(MDP_TL_BLOCKS, tl->zn), TLT, 0, ctx->stream>>>(tl->Z.as<double>(), tl->n, d_g, 0, tl->n,
                                                                             tl->part.as<double>());
    MDP_CHECK_LAUNCH(ctx);
    qtx_kernel<<<1, 128, 0, ctx->stream>>>(tl->part.as<double>(), MDP_TL_BLOCKS, tl->Em1.as<double>(), tl->zn,
                                           tl->qtx.as<double>());
    MDP_CHECK_LAUNCH(ctx);
    return MDP_OK;
}

// Builds Z, AZ and Em1 for the post-cut pointing A.  d_g0 (precond 2): the
// first residual P^T N^-1 (b + noise), the Lanczos start (precond.c:1100-1110).
int mdp_twolevel_build(mdp_context *ctx, mdp_pointing *A, const mdp_noise *N, int precond, int zn,
                       const double *d_g0, mdp_twolevel *tl) {
    if (zn == 0) zn = 1;  // one column per rank (pcg_true.c:52), one rank here
    if (precond != 1 && precond != 2) {
        mdp_set_error("two-level preconditioner: precond must be 1 or 2 (got %d)", precond);
        return MDP_EINVAL;
    }
    if (zn < 1 || zn > MDP_TL_MAX_ZN) {
        mdp_set_error("two-level preconditioner: z_2lvl must be in 1..%d (got %d)", MDP_TL_MAX_ZN, zn);
        return MDP_EINVAL;
    }
    cudaStream_t  st = ctx->stream;
    const int64_t n = A->n_map(), npix = n / 3, m = A->m;
    tl->precond = precond;
    tl->zn = zn;
    tl->n = n;
    MDP_TRY(tl->Z.alloc(8 * (size_t) zn * n));
    MDP_TRY(tl->AZ.alloc(8 * (size_t) zn * n));
    MDP_TRY(tl->Em1.alloc(8 * (size_t) zn * zn));
    MDP_TRY(tl->qtx.alloc(8 * (size_t) zn));
    MDP_TRY(tl->part.alloc(8 * (size_t) std::max(zn, 1) * MDP_TL_BLOCKS));
    double *Z = tl->Z.as<double>(), *AZ = tl->AZ.as<double>();
    if (precond == 1) {
        const int     group = zn > 1 ? zn : 1;
        const int64_t npix_l = A->lcount / 3, lcount = A->lcount;
        // the reference's column index g * group + i stays inside its count array
        if ((int64_t) (group - 1) * group + lcount - 3 >= (int64_t) group * lcount) {
            mdp_set_error("two-level a priori: %d columns for a map of %lld local indices", zn, (long long) lcount);
            return MDP_EINVAL;
        }
        DevBuf cnt;
        MDP_TRY(cnt.alloc(4 * (size_t) group * npix_l));
        MDP_CUDA(cudaMemsetAsync(cnt.p, 0, 4 * (size_t) group * npix_l, st));
        const int64_t rows_per = m / group;
        z_count_kernel<<<grid_for(rows_per * group, 256, ctx->sm_count * 16), 256, 0, st>>>(
                A->off.as<int32_t>(), rows_per, group, A->trash_pix, npix_l, cnt.as<int32_t>());
        MDP_CHECK_LAUNCH(ctx);
        z_fill_kernel<<<grid_for(npix, 256, ctx->sm_count * 8), 256, 0, st>>>(cnt.as<int32_t>(), group, A->trash_pix,
                                                                              npix_l, npix, Z);
        MDP_CHECK_LAUNCH(ctx);
        for (int j = 0; j < zn; j++) MDP_TRY(mdp_apply_op_impl(ctx, A, N, Z + (int64_t) j * n, AZ + (int64_t) j * n));
        MDP_CUDA(cudaStreamSynchronize(st));  // cnt is released on return
    } else {
        if (!d_g0) return MDP_EINVAL;
        const int K = zn;
        DevBuf    Vb, AVb, wb, zero;
        MDP_TRY(Vb.alloc(8 * (size_t) K * n));
        MDP_TRY(AVb.alloc(8 * (size_t) K * n));
        MDP_TRY(wb.alloc(8 * (size_t) n));
        MDP_TRY(zero.alloc(8 * (size_t) n));
        double   *V = Vb.as<double>(), *AV = AVb.as<double>(), *w = wb.as<double>();
        const int gn = grid_for(n, 256, ctx->sm_count * 8);
        MDP_CUDA(cudaMemsetAsync(V, 0, 8 * (size_t) K * n, st));
        MDP_CUDA(cudaMemsetAsync(zero.p, 0, 8 * (size_t) n, st));
        std::vector<double> T((size_t) K * K, 0.0);
        double              dot = 0.0, alpha = 0.0, beta;
        // v0 = w0 / ||w0||, Av0, alpha0, w = Av0 - alpha0 v0 (precond.c:1112-1143)
        MDP_TRY(dot_host(ctx, d_g0, d_g0, n, tl->part, &dot));
        beta = std::sqrt(dot);
        if (beta > EPS_2LVL) {
            scale_copy_kernel<<<gn, 256, 0, st>>>(d_g0, beta, V, n);
            MDP_CHECK_LAUNCH(ctx);
        }
        const double *v = V, *vold = zero.as<double>();
        MDP_TRY(mdp_apply_op_impl(ctx, A, N, v, AV));
        MDP_TRY(dot_host(ctx, v, AV, n, tl->part, &alpha));
        lanczos_w_kernel<<<gn, 256, 0, st>>>(AV, v, vold, alpha, 0.0, w, n);
        MDP_CHECK_LAUNCH(ctx);
        // steps 1..K-1; the reference's step K only feeds T and V entries its
        // K x K truncation drops (precond.c:1203-1215), so it is not made
        for (int i = 0; i + 1 < K; i++) {
            MDP_TRY(dot_host(ctx, w, w, n, tl->part, &dot));
            beta = std::sqrt(dot);
            double *vn = V + (int64_t) (i + 1) * n;
            if (beta > EPS_2LVL) {  // else the column stays zero and v is kept (precond.c:1163-1170)
                scale_copy_kernel<<<gn, 256, 0, st>>>(w, beta, vn, n);
                MDP_CHECK_LAUNCH(ctx);
                v = vn;
            }
            T[(size_t) i * K + i] = alpha;
            T[(size_t) i * K + i + 1] = beta;
            T[(size_t) (i + 1) * K + i] = beta;
            double *Av = AV + (int64_t) (i + 1) * n;
            MDP_TRY(mdp_apply_op_impl(ctx, A, N, v, Av));
            MDP_TRY(dot_host(ctx, v, Av, n, tl->part, &alpha));
            // vold is still zero at the first step (precond.c:1196-1200)
            lanczos_w_kernel<<<gn, 256, 0, st>>>(Av, v, vold, alpha, beta, w, n);
            MDP_CHECK_LAUNCH(ctx);
            vold = v;
        }
        T[(size_t) (K - 1) * K + K - 1] = alpha;
        std::vector<double> ev, Y;
        mdp_dense::jacobi_eigh(K, T, ev, Y);
        MDP_TRY(ritz(ctx, V, Y, K, n, Z));
        MDP_TRY(ritz(ctx, AV, Y, K, n, AZ));
    }
    // E[i][j] = Z[j] . AZ[i] and its pseudo-inverse (precond.c:951-1000)
    const int ey = (zn * zn + TLT - 1) / TLT;
    DevBuf    gpart, dE;
    MDP_TRY(gpart.alloc(8 * (size_t) zn * zn * MDP_TL_BLOCKS));
    MDP_TRY(dE.alloc(8 * (size_t) zn * zn));
    const size_t gsm = 2 * 8 * (size_t) zn * GK;
    gram_partial_kernel<<<dim3(MDP_TL_BLOCKS, ey), TLT, gsm, st>>>(Z, AZ, zn, n, gpart.as<double>());
    MDP_CHECK_LAUNCH(ctx);
    sum_partials_kernel<<<1, 256, 0, st>>>(gpart.as<double>(), MDP_TL_BLOCKS, zn * zn, dE.as<double>());
    MDP_CHECK_LAUNCH(ctx);
    std::vector<double> E((size_t) zn * zn);
    MDP_CUDA(cudaMemcpyAsync(E.data(), dE.p, 8 * (size_t) zn * zn, cudaMemcpyDeviceToHost, st));
    MDP_CUDA(cudaStreamSynchronize(st));
    for (double e : E)
        if (!std::isfinite(e)) {
            mdp_set_error("two-level preconditioner: E = Z^T A Z is not finite");
            return MDP_ENAN;
        }
    tl->h_Em1 = mdp_dense::pinv_gelss(zn, E, EPS_2LVL);
    MDP_CUDA(cudaMemcpyAsync(tl->Em1.p, tl->h_Em1.data(), 8 * (size_t) zn * zn, cudaMemcpyHostToDevice, st));
    MDP_CUDA(cudaStreamSynchronize(st));
    return MDP_OK;
}
