// Block-Jacobi preconditioner and the PCG solve of (P^T N^-1 P) x = P^T N^-1 d.
//
// Reference: mappraiser/src/precond.c:42-161 (getlocalW), 456-702
// (precondblockjacobilike: per-pixel dlange/dgetrf/dgecon/dgetri, rcond > 0.1
// cut, trash rewrite, MatInit again), 1310-1423 (build_precond, apply_precond);
// mappraiser/src/pcg_true.c:20-241 (PCG_GLS_true, Polak-Ribiere, stop test on
// the unpreconditioned residual), 578-600 (apply_weights).
//
// Device layout: map-domain vectors are contiguous FP64 arrays of n = 3*npix
// unknowns; the 3x3 blocks are row-major [npix][9].  Dot products are
// deterministic two-level reductions (fixed grid, partials summed in block
// order by the last block to finish); P^T and the block-Jacobi blocks add
// their terms in a fixed order too (map bins, below and in pointing.cu), so a
// solve on pointings of 2^20 rows or more is bitwise reproducible.
#include <cfloat>
#include <chrono>
#include <cmath>

#include "mdp_internal.cuh"


// ================================================================= getlocalW
__device__ __forceinline__ int find_block(const int64_t *__restrict__ bstart, const int32_t *__restrict__ blen, int nb,
                                          int64_t t) {
    int lo = 0, hi = nb - 1, ans = -1;
    while (lo <= hi) {
        int mid = (lo + hi) >> 1;
        if (bstart[mid] <= t) {
            ans = mid;
            lo = mid + 1;
        } else {
            hi = mid - 1;
        }
    }
    if (ans >= 0 && t < bstart[ans] + blen[ans]) return ans;
    return -1;
}

// W[q] += w w^T * T0(block of t)  (weight 1 outside every block), hits[q] += 1
__global__ void localW_kernel(const int32_t *__restrict__ off, const double *__restrict__ w, int64_t m,
                              const int64_t *__restrict__ bstart, const int32_t *__restrict__ blen,
                              const double *__restrict__ t0, int nb, double *__restrict__ W, int *__restrict__ hits) {
    for (int64_t t = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; t < m; t += (int64_t) gridDim.x * blockDim.x) {
        const int32_t o = off[t];
        if (o < 0) continue;
        const int    b = find_block(bstart, blen, nb, t);
        const double d = (b >= 0) ? t0[b] : 1.0;
        const double w0 = w[3 * t], w1 = w[3 * t + 1], w2 = w[3 * t + 2];
        double      *Wq = W + 3 * (int64_t) o;  // o = 3q -> 9q = 3*o
        const double a00 = __dmul_rn(__dmul_rn(w0, w0), d), a01 = __dmul_rn(__dmul_rn(w0, w1), d);
        const double a02 = __dmul_rn(__dmul_rn(w0, w2), d), a11 = __dmul_rn(__dmul_rn(w1, w1), d);
        const double a12 = __dmul_rn(__dmul_rn(w1, w2), d), a22 = __dmul_rn(__dmul_rn(w2, w2), d);
        atomicAdd(Wq + 0, a00);
        atomicAdd(Wq + 1, a01);
        atomicAdd(Wq + 2, a02);
        atomicAdd(Wq + 4, a11);
        atomicAdd(Wq + 5, a12);
        atomicAdd(Wq + 8, a22);
        atomicAdd(hits + o / 3, 1);
    }
}

// The same sums over the P^T map bins (pointing.cu): warp k of a CTA owns bin
// LW_WARPS*blockIdx.x + k and adds, in the bin's time-ordered row list, each
// row's six products and its hit into shared-memory accumulators; rows of one
// step on one pixel are added in lane order.  Every pixel's sums run in time
// order, as getlocalW's loop over the rows does (precond.c:42-161), and are
// reproducible bit for bit.
#define LW_WARPS 3
__global__ void __launch_bounds__(32 * LW_WARPS) localW_bins_kernel(
        const int32_t *__restrict__ off, const double *__restrict__ w, const int64_t *__restrict__ bin_start,
        const uint32_t *__restrict__ perm, int64_t nbins, int64_t npix, const int64_t *__restrict__ bstart,
        const int32_t *__restrict__ blen, const double *__restrict__ t0, int nb, double *__restrict__ W,
        int *__restrict__ hits) {
    constexpr int BP = MDP_PT_BIN_PIX;
    __shared__ double acc_s[LW_WARPS][BP * 7];  // per pixel: W00 W01 W02 W11 W12 W22 hits
    const int     wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t bin = (int64_t) blockIdx.x * LW_WARPS + wid;
    if (bin >= nbins) return;  // whole warps only; no CTA-wide barrier follows
    double *acc = acc_s[wid];
    for (int i = lane; i < BP * 7; i += 32) acc[i] = 0.0;
    __syncwarp();
    const int64_t s0 = bin_start[bin], s1 = bin_start[bin + 1];
    const int64_t base = bin * 3 * BP;
    for (int64_t i0 = s0; i0 < s1; i0 += 32) {
        const int64_t i = i0 + lane;
        int           q = -1;
        double        a[6] = {0, 0, 0, 0, 0, 0};
        if (i < s1) {
            const int64_t t = perm[i];
            q = (int) ((off[t] - base) / 3);
            const int    b = find_block(bstart, blen, nb, t);
            const double d = (b >= 0) ? t0[b] : 1.0;
            const double w0 = w[3 * t], w1 = w[3 * t + 1], w2 = w[3 * t + 2];
            a[0] = __dmul_rn(__dmul_rn(w0, w0), d);
            a[1] = __dmul_rn(__dmul_rn(w0, w1), d);
            a[2] = __dmul_rn(__dmul_rn(w0, w2), d);
            a[3] = __dmul_rn(__dmul_rn(w1, w1), d);
            a[4] = __dmul_rn(__dmul_rn(w1, w2), d);
            a[5] = __dmul_rn(__dmul_rn(w2, w2), d);
        }
        const unsigned peers = __match_any_sync(0xffffffffu, q);
        const bool     alone = q < 0 || peers == (1u << lane);
        if (__all_sync(0xffffffffu, alone)) {
            if (q >= 0) {
#pragma unroll
                for (int k = 0; k < 6; k++) acc[7 * q + k] = __dadd_rn(acc[7 * q + k], a[k]);
                acc[7 * q + 6] += 1.0;
            }
        } else {
            for (int src = 0; src < 32; src++) {  // rows in lane order
                const int qq = __shfl_sync(0xffffffffu, q, src);
                double    d[6];
#pragma unroll
                for (int k = 0; k < 6; k++) d[k] = __shfl_sync(0xffffffffu, a[k], src);
                if (lane == 0 && qq >= 0) {
#pragma unroll
                    for (int k = 0; k < 6; k++) acc[7 * qq + k] = __dadd_rn(acc[7 * qq + k], d[k]);
                    acc[7 * qq + 6] += 1.0;
                }
            }
        }
        __syncwarp();
    }
    const int64_t p0 = bin * BP;
    const int     np = (int) min((int64_t) BP, npix - p0);
    for (int j = lane; j < np; j += 32) {
        double *Wq = W + 9 * (p0 + j);
        const double *s = acc + 7 * j;
        Wq[0] = s[0];
        Wq[1] = s[1];
        Wq[2] = s[2];
        Wq[3] = 0.0;
        Wq[4] = s[3];
        Wq[5] = s[4];
        Wq[6] = 0.0;
        Wq[7] = 0.0;
        Wq[8] = s[5];
        hits[p0 + j] = (int) s[6];
    }
}

// W and hits of every pixel: by map bins (time order) when the pointing has
// them, else with atomics
static int localW_launch(mdp_context *ctx, mdp_pointing *A, const mdp_noise *N, double *d_W, int *d_hits) {
    cudaStream_t  st = ctx->stream;
    const int64_t npix = A->n_map() / 3;
    if (mdp_pointing_binned(A)) {
        MDP_TRY(mdp_pointing_bins(ctx, A));
        if (A->bins.nbins > 0)
            localW_bins_kernel<<<(unsigned) ((A->bins.nbins + LW_WARPS - 1) / LW_WARPS), 32 * LW_WARPS, 0, st>>>(
                    A->off.as<int32_t>(), A->values, A->bins.start.as<int64_t>(), A->bins.perm.as<uint32_t>(),
                    A->bins.nbins, npix, N->blk_start.as<int64_t>(), N->blk_len.as<int32_t>(), N->blk_t0.as<double>(),
                    N->nb, d_W, d_hits);
        MDP_CHECK_LAUNCH(ctx);
        return MDP_OK;
    }
    MDP_CUDA(cudaMemsetAsync(d_W, 0, 72 * npix, st));
    MDP_CUDA(cudaMemsetAsync(d_hits, 0, 4 * npix, st));
    localW_kernel<<<grid_for(A->m, 256, ctx->sm_count * 16), 256, 0, st>>>(
            A->off.as<int32_t>(), A->values, A->m, N->blk_start.as<int64_t>(), N->blk_len.as<int32_t>(),
            N->blk_t0.as<double>(), N->nb, d_W, d_hits);
    MDP_CHECK_LAUNCH(ctx);
    return MDP_OK;
}

// ================================================================= 3x3 LAPACK restatement
// Column-major 3x3 (a[i + 3j] = A(i,j)) on the logical block, as LAPACKE does
// for row-major calls.  Products and sums are rounded separately (no FMA
// contraction) like reference LAPACK built without FMA.
#define MUL __dmul_rn
#define ADD __dadd_rn
#define SUB __dsub_rn

__device__ int idamax3(const double *x, int n, int inc) {
    int    best = 0;
    double bv = fabs(x[0]);
    for (int i = 1; i < n; i++) {
        double v = fabs(x[i * inc]);
        if (v > bv) {
            bv = v;
            best = i;
        }
    }
    return best;
}

// DGETF2; ipiv 0-based
__device__ void getf2_3(double *a, int *ipiv) {
    for (int j = 0; j < 3; j++) {
        int jp = j + idamax3(a + j + 3 * j, 3 - j, 1);
        ipiv[j] = jp;
        if (a[jp + 3 * j] != 0.0) {
            if (jp != j)
                for (int k = 0; k < 3; k++) {
                    double t = a[j + 3 * k];
                    a[j + 3 * k] = a[jp + 3 * k];
                    a[jp + 3 * k] = t;
                }
            if (j < 2) {
                if (fabs(a[j + 3 * j]) >= DBL_MIN) {
                    double r = __drcp_rn(a[j + 3 * j]);
                    for (int i = j + 1; i < 3; i++) a[i + 3 * j] = MUL(a[i + 3 * j], r);
                } else {
                    for (int i = j + 1; i < 3; i++) a[i + 3 * j] = __ddiv_rn(a[i + 3 * j], a[j + 3 * j]);
                }
            }
        }
        for (int k = j + 1; k < 3; k++) {
            double t = a[j + 3 * k];
            if (t != 0.0)
                for (int i = j + 1; i < 3; i++) a[i + 3 * k] = ADD(a[i + 3 * k], MUL(-t, a[i + 3 * j]));
        }
    }
}

__device__ void lu_solve3(const double *lu, int kase, double *x) {
    if (kase == 1) {
        for (int j = 0; j < 3; j++)
            if (x[j] != 0.0)
                for (int i = j + 1; i < 3; i++) x[i] = SUB(x[i], MUL(x[j], lu[i + 3 * j]));
        for (int j = 2; j >= 0; j--)
            if (x[j] != 0.0) {
                x[j] = __ddiv_rn(x[j], lu[j + 3 * j]);
                double t = x[j];
                for (int i = j - 1; i >= 0; i--) x[i] = SUB(x[i], MUL(t, lu[i + 3 * j]));
            }
    } else {
        for (int j = 0; j < 3; j++) {
            double t = x[j];
            for (int i = 0; i < j; i++) t = SUB(t, MUL(lu[i + 3 * j], x[i]));
            x[j] = __ddiv_rn(t, lu[j + 3 * j]);
        }
        for (int j = 2; j >= 0; j--) {
            double t = x[j];
            for (int i = 2; i > j; i--) t = SUB(t, MUL(lu[i + 3 * j], x[i]));
            x[j] = t;
        }
    }
}

__device__ double dasum3(const double *x) { return ADD(ADD(fabs(x[0]), fabs(x[1])), fabs(x[2])); }

// DGECON('1') with the DLACN2 estimator (Higham 1988); 0 for a zero pivot
__device__ double gecon1_3(const double *lu, double anorm) {
    if (anorm == 0.0) return 0.0;
    for (int j = 0; j < 3; j++)
        if (lu[j + 3 * j] == 0.0) return 0.0;
    double x[3], v[3];
    int    isgn[3];
    double est, estold;
    for (int i = 0; i < 3; i++) x[i] = 1.0 / 3.0;
    lu_solve3(lu, 1, x);
    est = dasum3(x);
    for (int i = 0; i < 3; i++) {
        x[i] = (x[i] >= 0.0) ? 1.0 : -1.0;
        isgn[i] = (int) x[i];
    }
    lu_solve3(lu, 2, x);
    int j = idamax3(x, 3, 1), iter = 2;
    for (;;) {
        x[0] = x[1] = x[2] = 0.0;
        x[j] = 1.0;
        lu_solve3(lu, 1, x);
        v[0] = x[0];
        v[1] = x[1];
        v[2] = x[2];
        estold = est;
        est = dasum3(v);
        bool same = true;
        for (int i = 0; i < 3; i++)
            if (((x[i] >= 0.0) ? 1 : -1) != isgn[i]) same = false;
        if (same) break;
        if (est <= estold) break;
        for (int i = 0; i < 3; i++) {
            x[i] = (x[i] >= 0.0) ? 1.0 : -1.0;
            isgn[i] = (int) x[i];
        }
        lu_solve3(lu, 2, x);
        int jlast = j;
        j = idamax3(x, 3, 1);
        if (x[jlast] != fabs(x[j]) && iter < 5) {
            iter++;
            continue;
        }
        break;
    }
    double alt = 1.0;
    for (int i = 0; i < 3; i++) {
        x[i] = alt * (1.0 + (double) i / 2.0);
        alt = -alt;
    }
    lu_solve3(lu, 1, x);
    double temp = 2.0 * (dasum3(x) / 9.0);
    if (temp > est) {
        v[0] = x[0];
        v[1] = x[1];
        v[2] = x[2];
        est = temp;
    }
    if (!isfinite(est) || !isfinite(v[0]) || !isfinite(v[1]) || !isfinite(v[2])) return 0.0;
    if (est != 0.0) return __ddiv_rn(__drcp_rn(est), anorm);
    return 0.0;
}

// DTRTI2('U','N') + unblocked DGETRI + column interchanges
__device__ void getri_3(double *a, const int *ipiv) {
    for (int j = 0; j < 3; j++) {
        a[j + 3 * j] = __drcp_rn(a[j + 3 * j]);
        double ajj = -a[j + 3 * j];
        double *x = a + 3 * j;
        for (int jj = 0; jj < j; jj++) {
            if (x[jj] != 0.0) {
                double temp = x[jj];
                for (int i = 0; i < jj; i++) x[i] = ADD(x[i], MUL(temp, a[i + 3 * jj]));
                x[jj] = MUL(x[jj], a[jj + 3 * jj]);
            }
        }
        for (int i = 0; i < j; i++) x[i] = MUL(x[i], ajj);
    }
    double work[3];
    for (int j = 2; j >= 0; j--) {
        for (int i = j + 1; i < 3; i++) {
            work[i] = a[i + 3 * j];
            a[i + 3 * j] = 0.0;
        }
        for (int jj = j + 1; jj < 3; jj++) {
            double temp = -work[jj];
            if (temp != 0.0)
                for (int i = 0; i < 3; i++) a[i + 3 * j] = ADD(a[i + 3 * j], MUL(temp, a[i + 3 * jj]));
        }
    }
    for (int j = 1; j >= 0; j--) {
        int jp = ipiv[j];
        if (jp != j)
            for (int i = 0; i < 3; i++) {
                double t = a[i + 3 * j];
                a[i + 3 * j] = a[i + 3 * jp];
                a[i + 3 * jp] = t;
            }
    }
}

// per pixel: symmetrise the accumulated upper triangle, rcond, inverse when kept
__global__ void bj_pixel_kernel(double *__restrict__ W, int64_t npix, double *__restrict__ inv,
                                double *__restrict__ rcond, int *__restrict__ cut, int *__restrict__ ncut) {
    int local_cut = 0;
    for (int64_t q = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; q < npix; q += (int64_t) gridDim.x * blockDim.x) {
        double *Wq = W + 9 * q;
        Wq[3] = Wq[1];
        Wq[6] = Wq[2];
        Wq[7] = Wq[5];
        double a[9];
        for (int r = 0; r < 3; r++)
            for (int c = 0; c < 3; c++) a[r + 3 * c] = Wq[3 * r + c];
        double anorm = 0.0;
        for (int c = 0; c < 3; c++) {
            double s = ADD(ADD(fabs(a[0 + 3 * c]), fabs(a[1 + 3 * c])), fabs(a[2 + 3 * c]));
            if (anorm < s || isnan(s)) anorm = s;
        }
        int ipiv[3];
        getf2_3(a, ipiv);
        double rc = gecon1_3(a, anorm);
        rcond[q] = rc;
        int is_cut = !(rc > 1e-1);
        cut[q] = is_cut;
        double *Iq = inv + 9 * q;
        if (!is_cut) {
            getri_3(a, ipiv);
            for (int r = 0; r < 3; r++)
                for (int c = 0; c < 3; c++) Iq[3 * r + c] = a[r + 3 * c];
        } else {
            for (int i = 0; i < 9; i++) Iq[i] = 0.0;
            local_cut++;
        }
    }
    if (local_cut) atomicAdd(ncut, local_cut);
}

// ----------------------------------------------------------------- the rcond cut
// target[q] = 1 for the pixel whose samples the reference rewrites when block
// u is cut: q = u + trash_pix (precond.c:521,585-600 with MLmap's id_last_pix
// numbering, mappraiser.c:130-142).
__global__ void cut_target_kernel(const int *__restrict__ cut, int64_t npix, int trash, uint32_t *__restrict__ target) {
    for (int64_t u = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; u < npix; u += (int64_t) gridDim.x * blockDim.x)
        if (cut[u] && u + trash < npix) target[u + trash] = 1u;
}

__global__ void invert_flags_kernel(const uint32_t *__restrict__ in, uint32_t *__restrict__ out, int64_t n) {
    for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x)
        out[i] = 1u - in[i];
}

__global__ void keep_from_cut_kernel(const int *__restrict__ cut, uint32_t *__restrict__ keep, int64_t n) {
    for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x)
        keep[i] = cut[i] ? 0u : 1u;
}

// rows of removed pixels become cut rows (-2); kept pixels are renumbered
__global__ void rewrite_off_kernel(int32_t *__restrict__ off, int64_t m, const uint32_t *__restrict__ target,
                                   const uint32_t *__restrict__ remap) {
    for (int64_t t = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; t < m; t += (int64_t) gridDim.x * blockDim.x) {
        int32_t o = off[t];
        if (o < 0) continue;
        int32_t q = o / 3;
        off[t] = target[q] ? -2 : 3 * (int32_t) remap[q];
    }
}

// compact kept blocks (original order) and kept pixel ids
__global__ void compact_blocks_kernel(const uint32_t *__restrict__ keepb, const uint32_t *__restrict__ rankb,
                                      int64_t npix, const double *__restrict__ inv, const double *__restrict__ rcond,
                                      const int *__restrict__ hits, double *__restrict__ inv_out,
                                      double *__restrict__ cond_out, int32_t *__restrict__ hits_out) {
    for (int64_t u = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; u < npix; u += (int64_t) gridDim.x * blockDim.x) {
        if (!keepb[u]) continue;
        int64_t k = rankb[u];
        for (int i = 0; i < 9; i++) inv_out[9 * k + i] = inv[9 * u + i];
        cond_out[k] = rcond[u];
        hits_out[k] = hits[u];
    }
}

__global__ void new_lindices_kernel(const int32_t *__restrict__ old_lind, int old_trash, int64_t npix,
                                    const uint32_t *__restrict__ target, const uint32_t *__restrict__ remap,
                                    int32_t *__restrict__ lind) {
    for (int64_t q = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; q < npix; q += (int64_t) gridDim.x * blockDim.x) {
        if (q == 0) {
            lind[0] = -3;
            lind[1] = -2;
            lind[2] = -1;
        }
        if (target[q]) continue;
        int64_t k = remap[q];
        for (int j = 0; j < 3; j++) lind[3 + 3 * k + j] = old_lind[3 * old_trash + 3 * q + j];
    }
}

// ================================================================= vector kernels
#define RED_THREADS 256
#define RED_BLOCKS 296

struct Scal {       // device scalars of the solve
    double g2pix, g2pixp, g2pix_polak, coeff, res, ro, gamma;
    double pad;
    double partial[4][RED_BLOCKS];
    unsigned int count[4];
};

template <int K>
__device__ __forceinline__ void block_reduce_store(double (&v)[K], Scal *S, int slot0) {
    __shared__ double sh[K][RED_THREADS / 32];
#pragma unroll
    for (int k = 0; k < K; k++)
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    if ((threadIdx.x & 31) == 0)
#pragma unroll
        for (int k = 0; k < K; k++) sh[k][threadIdx.x >> 5] = v[k];
    __syncthreads();
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < K; k++) {
            double s = 0.0;
            for (int w = 0; w < RED_THREADS / 32; w++) s += sh[k][w];
            S->partial[slot0 + k][blockIdx.x] = s;
        }
}

// last block to finish sums the partials in block order (deterministic)
__device__ __forceinline__ bool last_block(Scal *S, int slot) {
    __shared__ bool is_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned int prev = atomicAdd(&S->count[slot], 1u);
        is_last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (is_last) __threadfence();
    return is_last;
}

__device__ __forceinline__ double sum_partials(const Scal *S, int slot) {
    double s = 0.0;
    for (int b = 0; b < (int) gridDim.x; b++) s += ((volatile const Scal *) S)->partial[slot][b];
    return s;
}

// RHS: _g = b + noise - P x0 with x0 = 0; cut rows have b zeroed (precond.c:605-615)
__global__ void rhs_kernel(const int32_t *__restrict__ off, const double *__restrict__ b,
                           const double *__restrict__ noise, double *__restrict__ out, int64_t m) {
    for (int64_t t = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; t < m; t += (int64_t) gridDim.x * blockDim.x)
        out[t] = ((off[t] == -2) ? 0.0 : b[t]) + noise[t];
}

__device__ __forceinline__ void bj3(const double *__restrict__ inv, const double *__restrict__ g, int64_t q,
                                    double &c0, double &c1, double &c2) {
    const double *I = inv + 9 * q;
    const double  g0 = g[3 * q], g1 = g[3 * q + 1], g2 = g[3 * q + 2];
    c0 = I[0] * g0 + I[1] * g1 + I[2] * g2;
    c1 = I[3] * g0 + I[4] * g1 + I[5] * g2;
    c2 = I[6] * g0 + I[7] * g1 + I[8] * g2;
}

// init: Cg = M^-1 g, h = Cg, g2pix = (Cg, g), res = (g, g)
__global__ void __launch_bounds__(RED_THREADS) pcg_init_kernel(const double *__restrict__ inv, const double *__restrict__ g,
                                                               double *__restrict__ Cg, double *__restrict__ h,
                                                               int64_t npix, Scal *S) {
    double v[2] = {0.0, 0.0};
    for (int64_t q = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; q < npix; q += (int64_t) gridDim.x * blockDim.x) {
        double c0, c1, c2;
        bj3(inv, g, q, c0, c1, c2);
        Cg[3 * q] = c0;
        Cg[3 * q + 1] = c1;
        Cg[3 * q + 2] = c2;
        h[3 * q] = c0;
        h[3 * q + 1] = c1;
        h[3 * q + 2] = c2;
        const double g0 = g[3 * q], g1 = g[3 * q + 1], g2 = g[3 * q + 2];
        v[0] += c0 * g0 + c1 * g1 + c2 * g2;
        v[1] += g0 * g0 + g1 * g1 + g2 * g2;
    }
    block_reduce_store<2>(v, S, 0);
    if (last_block(S, 0) && threadIdx.x == 0) {
        S->g2pix = sum_partials(S, 0);
        S->res = sum_partials(S, 1);
        S->count[0] = 0;
    }
}

// coeff = (h, AtNm1Ah)
__global__ void __launch_bounds__(RED_THREADS) pcg_coeff_kernel(const double *__restrict__ h,
                                                                const double *__restrict__ q_, int64_t n, Scal *S) {
    double v[1] = {0.0};
    for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x)
        v[0] += h[i] * q_[i];
    block_reduce_store<1>(v, S, 0);
    if (last_block(S, 1) && threadIdx.x == 0) {
        S->coeff = sum_partials(S, 0);
        S->ro = S->g2pix / S->coeff;
        S->count[1] = 0;
    }
}

// x += ro h; g = gp - ro AtNm1Ah; Cg = M^-1 g; dots (Cg,g), (Cg,g-gp), (g,g)
__global__ void __launch_bounds__(RED_THREADS) pcg_update_kernel(const double *__restrict__ inv, double *__restrict__ x,
                                                                 const double *__restrict__ h,
                                                                 const double *__restrict__ q_,
                                                                 const double *__restrict__ gp, double *__restrict__ g,
                                                                 double *__restrict__ Cg, int64_t npix, Scal *S) {
    const double ro = S->ro;
    double       v[3] = {0.0, 0.0, 0.0};
    for (int64_t q = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; q < npix; q += (int64_t) gridDim.x * blockDim.x) {
        double gn[3], go[3];
#pragma unroll
        for (int j = 0; j < 3; j++) {
            const int64_t i = 3 * q + j;
            x[i] = x[i] + ro * h[i];
            go[j] = gp[i];
            gn[j] = go[j] - ro * q_[i];
            g[i] = gn[j];
        }
        const double *I = inv + 9 * q;
        double        c[3];
        c[0] = I[0] * gn[0] + I[1] * gn[1] + I[2] * gn[2];
        c[1] = I[3] * gn[0] + I[4] * gn[1] + I[5] * gn[2];
        c[2] = I[6] * gn[0] + I[7] * gn[1] + I[8] * gn[2];
#pragma unroll
        for (int j = 0; j < 3; j++) {
            Cg[3 * q + j] = c[j];
            v[0] += c[j] * gn[j];
            v[1] += c[j] * (gn[j] - go[j]);
            v[2] += gn[j] * gn[j];
        }
    }
    block_reduce_store<3>(v, S, 0);
    if (last_block(S, 2) && threadIdx.x == 0) {
        S->g2pixp = S->g2pix;
        S->g2pix = sum_partials(S, 0);
        S->g2pix_polak = sum_partials(S, 1);
        S->res = sum_partials(S, 2);
        S->gamma = S->g2pix_polak / S->g2pixp;
        S->count[2] = 0;
    }
}

// ---------------------------------------------------------------- two-level preconditioner
// c = M g for pixel q: BJ_inv (g - AZ qtx) + Z qtx, sums over the columns in
// column order (apply_precond, precond.c:1412-1423; mul_ZQtx :1053-1069)
__device__ __forceinline__ void tl_apply3(const double *__restrict__ inv, const double *__restrict__ Z,
                                          const double *__restrict__ AZ, const double *qtx, int zn, int64_t n,
                                          int64_t q, const double (&gq)[3], double (&c)[3]) {
    double qg[3] = {0.0, 0.0, 0.0}, aq[3] = {0.0, 0.0, 0.0};
    for (int j = 0; j < zn; j++) {
        const double  t = qtx[j];
        const double *z = Z + (int64_t) j * n + 3 * q, *az = AZ + (int64_t) j * n + 3 * q;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            qg[k] += z[k] * t;
            aq[k] += az[k] * t;
        }
    }
    double r[3];
#pragma unroll
    for (int k = 0; k < 3; k++) r[k] = gq[k] - aq[k];
    const double *I = inv + 9 * q;
    c[0] = I[0] * r[0] + I[1] * r[1] + I[2] * r[2];
    c[1] = I[3] * r[0] + I[4] * r[1] + I[5] * r[2];
    c[2] = I[6] * r[0] + I[7] * r[1] + I[8] * r[2];
#pragma unroll
    for (int k = 0; k < 3; k++) c[k] += qg[k];
}

// init with the two-level preconditioner: Cg = M g, h = Cg, g2pix = (Cg, g), res = (g, g)
__global__ void __launch_bounds__(RED_THREADS) pcg_init_tl_kernel(const double *__restrict__ inv,
                                                                  const double *__restrict__ g, double *__restrict__ Cg,
                                                                  double *__restrict__ h, int64_t npix,
                                                                  const double *__restrict__ Z,
                                                                  const double *__restrict__ AZ,
                                                                  const double *__restrict__ qtx_g, int zn, Scal *S) {
    __shared__ double qtx[MDP_TL_MAX_ZN];
    for (int j = threadIdx.x; j < zn; j += blockDim.x) qtx[j] = qtx_g[j];
    __syncthreads();
    const int64_t n = 3 * npix;
    double        v[2] = {0.0, 0.0};
    for (int64_t q = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; q < npix; q += (int64_t) gridDim.x * blockDim.x) {
        const double gq[3] = {g[3 * q], g[3 * q + 1], g[3 * q + 2]};
        double       c[3];
        tl_apply3(inv, Z, AZ, qtx, zn, n, q, gq, c);
#pragma unroll
        for (int k = 0; k < 3; k++) {
            Cg[3 * q + k] = c[k];
            h[3 * q + k] = c[k];
            v[0] += c[k] * gq[k];
            v[1] += gq[k] * gq[k];
        }
    }
    block_reduce_store<2>(v, S, 0);
    if (last_block(S, 0) && threadIdx.x == 0) {
        S->g2pix = sum_partials(S, 0);
        S->res = sum_partials(S, 1);
        S->count[0] = 0;
    }
}

// x += ro h; g = gp - ro AtNm1Ah (the preconditioner follows once Z^T g is known)
__global__ void pcg_step_kernel(double *__restrict__ x, const double *__restrict__ h, const double *__restrict__ q_,
                                const double *__restrict__ gp, double *__restrict__ g, int64_t n, const Scal *S) {
    const double ro = S->ro;
    for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x) {
        x[i] = x[i] + ro * h[i];
        g[i] = gp[i] - ro * q_[i];
    }
}

// Cg = M g with the two-level preconditioner; dots (Cg,g), (Cg,g-gp), (g,g)
__global__ void __launch_bounds__(RED_THREADS) pcg_precond_tl_kernel(const double *__restrict__ inv,
                                                                     const double *__restrict__ g,
                                                                     const double *__restrict__ gp,
                                                                     double *__restrict__ Cg, int64_t npix,
                                                                     const double *__restrict__ Z,
                                                                     const double *__restrict__ AZ,
                                                                     const double *__restrict__ qtx_g, int zn, Scal *S) {
    __shared__ double qtx[MDP_TL_MAX_ZN];
    for (int j = threadIdx.x; j < zn; j += blockDim.x) qtx[j] = qtx_g[j];
    __syncthreads();
    const int64_t n = 3 * npix;
    double        v[3] = {0.0, 0.0, 0.0};
    for (int64_t q = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; q < npix; q += (int64_t) gridDim.x * blockDim.x) {
        const double gq[3] = {g[3 * q], g[3 * q + 1], g[3 * q + 2]};
        double       c[3];
        tl_apply3(inv, Z, AZ, qtx, zn, n, q, gq, c);
#pragma unroll
        for (int k = 0; k < 3; k++) {
            Cg[3 * q + k] = c[k];
            v[0] += c[k] * gq[k];
            v[1] += c[k] * (gq[k] - gp[3 * q + k]);
            v[2] += gq[k] * gq[k];
        }
    }
    block_reduce_store<3>(v, S, 0);
    if (last_block(S, 2) && threadIdx.x == 0) {
        S->g2pixp = S->g2pix;
        S->g2pix = sum_partials(S, 0);
        S->g2pix_polak = sum_partials(S, 1);
        S->res = sum_partials(S, 2);
        S->gamma = S->g2pix_polak / S->g2pixp;
        S->count[2] = 0;
    }
}

// out = d' - out where d' = b (0 on cut rows) + noise: the TOD residual d' - P x
__global__ void tod_residual_kernel(const int32_t *__restrict__ off, const double *__restrict__ b,
                                    const double *__restrict__ noise, double *__restrict__ out, int64_t m) {
    for (int64_t t = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; t < m; t += (int64_t) gridDim.x * blockDim.x)
        out[t] = ((off[t] == -2) ? 0.0 : b[t]) + noise[t] - out[t];
}

// x += d
__global__ void axpy1_kernel(double *__restrict__ x, const double *__restrict__ d, int64_t n) {
    for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x)
        x[i] += d[i];
}

// res = (g, g)
__global__ void __launch_bounds__(RED_THREADS) dot_self_kernel(const double *__restrict__ g, int64_t n, Scal *S) {
    double v[1] = {0.0};
    for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x)
        v[0] += g[i] * g[i];
    block_reduce_store<1>(v, S, 0);
    if (last_block(S, 3) && threadIdx.x == 0) {
        S->res = sum_partials(S, 0);
        S->count[3] = 0;
    }
}

// h = gamma h + Cg
__global__ void pcg_direction_kernel(double *__restrict__ h, const double *__restrict__ Cg, int64_t n, const Scal *S) {
    const double gamma = S->gamma;
    for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x)
        h[i] = h[i] * gamma + Cg[i];
}

// ================================================================= the solve
int mdp_bj_build(mdp_context *ctx, mdp_pointing *A, const mdp_noise *N, BJState *bj) {
    if (!A->triplet) {
        mdp_set_error("block Jacobi needs the (I,Q,U) triplet pointing layout");
        return MDP_EUNSUPPORTED;
    }
    cudaStream_t  st = ctx->stream;
    const int64_t m = A->m;
    const int64_t npix0 = A->n_map() / 3;
    DevBuf        W, inv, rcond, cut, hits, ncut;
    int           rc;
    if ((rc = W.alloc(72 * npix0)) || (rc = inv.alloc(72 * npix0)) || (rc = rcond.alloc(8 * npix0)) ||
        (rc = cut.alloc(4 * npix0)) || (rc = hits.alloc(4 * npix0)) || (rc = ncut.alloc(4)))
        return rc;
    MDP_CUDA(cudaMemsetAsync(ncut.p, 0, 4, st));
    MDP_TRY(localW_launch(ctx, A, N, W.as<double>(), hits.as<int>()));
    bj_pixel_kernel<<<grid_for(npix0, 128, ctx->sm_count * 8), 128, 0, st>>>(W.as<double>(), npix0, inv.as<double>(),
                                                                            rcond.as<double>(), cut.as<int>(),
                                                                            ncut.as<int>());
    MDP_CHECK_LAUNCH(ctx);
    int h_ncut = 0;
    MDP_CUDA(cudaMemcpyAsync(&h_ncut, ncut.p, 4, cudaMemcpyDeviceToHost, st));
    MDP_CUDA(cudaStreamSynchronize(st));
    bj->ncut = h_ncut;
    if (h_ncut == 0) {
        std::swap(bj->inv.p, inv.p), std::swap(bj->inv.bytes, inv.bytes);
        std::swap(bj->W.p, W.p), std::swap(bj->W.bytes, W.bytes);
        std::swap(bj->rcond.p, rcond.p), std::swap(bj->rcond.bytes, rcond.bytes);
        std::swap(bj->hits.p, hits.p), std::swap(bj->hits.bytes, hits.bytes);
        bj->npix = npix0;
        return MDP_OK;
    }
    // pixels whose samples become trash, and the renumbering of the others
    DevBuf target, remap, keep, lind2, rankb;
    if ((rc = target.alloc(4 * npix0)) || (rc = remap.alloc(4 * npix0)) || (rc = keep.alloc(4 * npix0)) ||
        (rc = lind2.alloc(4 * (3 * npix0 + 3))) || (rc = rankb.alloc(4 * npix0)) ||
        (rc = bj->inv.alloc(72 * npix0)) || (rc = bj->W.alloc(72 * npix0)) || (rc = bj->rcond.alloc(8 * npix0)) ||
        (rc = bj->hits.alloc(4 * npix0)))
        return rc;
    MDP_CUDA(cudaMemsetAsync(target.p, 0, 4 * npix0, st));
    const int gb = grid_for(npix0, 256, ctx->sm_count * 8);
    cut_target_kernel<<<gb, 256, 0, st>>>(cut.as<int>(), npix0, A->trash_pix, target.as<uint32_t>());
    MDP_CHECK_LAUNCH(ctx);
    invert_flags_kernel<<<gb, 256, 0, st>>>(target.as<uint32_t>(), keep.as<uint32_t>(), npix0);
    MDP_CHECK_LAUNCH(ctx);
    uint32_t kept_pix = 0;
    MDP_TRY(mdp_exclusive_scan_u32(ctx, keep.as<uint32_t>(), remap.as<uint32_t>(), npix0, &kept_pix));
    rewrite_off_kernel<<<grid_for(m, 256, ctx->sm_count * 16), 256, 0, st>>>(A->off.as<int32_t>(), m,
                                                                            target.as<uint32_t>(), remap.as<uint32_t>());
    MDP_CHECK_LAUNCH(ctx);
    new_lindices_kernel<<<gb, 256, 0, st>>>(A->lindices.as<int32_t>(), A->trash_pix, npix0, target.as<uint32_t>(),
                                            remap.as<uint32_t>(), lind2.as<int32_t>());
    MDP_CHECK_LAUNCH(ctx);
    keep_from_cut_kernel<<<gb, 256, 0, st>>>(cut.as<int>(), keep.as<uint32_t>(), npix0);
    MDP_CHECK_LAUNCH(ctx);
    uint32_t kept_blocks = 0;
    MDP_TRY(mdp_exclusive_scan_u32(ctx, keep.as<uint32_t>(), rankb.as<uint32_t>(), npix0, &kept_blocks));
    MDP_CUDA(cudaMemsetAsync(bj->inv.p, 0, 72 * npix0, st));
    MDP_CUDA(cudaMemsetAsync(bj->W.p, 0, 72 * npix0, st));
    MDP_CUDA(cudaMemsetAsync(bj->rcond.p, 0, 8 * npix0, st));
    MDP_CUDA(cudaMemsetAsync(bj->hits.p, 0, 4 * npix0, st));
    compact_blocks_kernel<<<gb, 256, 0, st>>>(keep.as<uint32_t>(), rankb.as<uint32_t>(), npix0, inv.as<double>(),
                                              rcond.as<double>(), hits.as<int>(), bj->inv.as<double>(),
                                              bj->rcond.as<double>(), bj->hits.as<int32_t>());
    MDP_CHECK_LAUNCH(ctx);
    compact_blocks_kernel<<<gb, 256, 0, st>>>(keep.as<uint32_t>(), rankb.as<uint32_t>(), npix0, W.as<double>(),
                                              rcond.as<double>(), hits.as<int>(), bj->W.as<double>(),
                                              bj->rcond.as<double>(), bj->hits.as<int32_t>());
    MDP_CHECK_LAUNCH(ctx);
    MDP_CUDA(cudaStreamSynchronize(st));
    std::swap(A->lindices.p, lind2.p);
    std::swap(A->lindices.bytes, lind2.bytes);
    A->bins.valid = 0;  // pixels were renumbered
    A->mbins.valid = 0;
    A->trash_pix = 1;
    A->lcount = 3 * (int64_t) kept_pix + 3;
    // the reference pairs kept blocks with kept pixels in order; both counts
    // agree except when, with flagged samples, the last pixel is cut: its
    // target falls past the end, no pixel leaves the map and the reference
    // leaves the last preconditioner rows unset.  Here they are zero blocks.
    bj->npix = kept_pix;
    return MDP_OK;
}

int mdp_pcg_run(mdp_context *ctx, mdp_pointing *A, const mdp_noise *N, const double *inv, int64_t npix,
                const double *d_signal, const double *d_noise, const mdp_solve_params *params, double *d_x,
                double *h_res_rel, mdp_solve_info *info, const mdp_twolevel *tl, const mdp_templates *tpl) {
    cudaStream_t  st = ctx->stream;
    const int64_t m = A->m;
    const int64_t n = 3 * npix;
    const int64_t nmap = A->n_map();  // >= n
    DevBuf &tod_a = ctx->ws[0], &tod_b = ctx->ws[1], &gb1 = ctx->ws[2], &gb2 = ctx->ws[3], &hb = ctx->ws[4],
           &qb = ctx->ws[5], &cgb = ctx->ws[6], &scal = ctx->ws[7];
    int           rc;
    if ((rc = tod_a.alloc(8 * m)) || (rc = tod_b.alloc(8 * m)) || (rc = gb1.alloc(8 * nmap)) ||
        (rc = gb2.alloc(8 * nmap)) || (rc = hb.alloc(8 * nmap)) || (rc = qb.alloc(8 * nmap)) ||
        (rc = cgb.alloc(8 * nmap)) || (rc = scal.alloc(sizeof(Scal))))
        return rc;
    Scal     *S = scal.as<Scal>();
    double   *x = d_x, *g = gb1.as<double>(), *gp = gb2.as<double>(), *h = hb.as<double>();
    double   *q = qb.as<double>(), *Cg = cgb.as<double>();
    double   *ta = tod_a.as<double>(), *tb = tod_b.as<double>();
    const int gm = grid_for(m, 256, ctx->sm_count * 16);
    MDP_CUDA(cudaMemsetAsync(S, 0, sizeof(Scal), st));
    MDP_CUDA(cudaMemsetAsync(x, 0, 8 * nmap, st));
    MDP_CUDA(cudaMemsetAsync(h, 0, 8 * nmap, st));
    MDP_CUDA(cudaMemsetAsync(Cg, 0, 8 * nmap, st));
    rhs_kernel<<<gm, 256, 0, st>>>(A->off.as<int32_t>(), d_signal, d_noise, ta, m);
    MDP_CHECK_LAUNCH(ctx);
    if (tpl)
        MDP_TRY(mdp_templates_filter(ctx, tpl, ta, tb));
    else
        MDP_TRY(mdp_stbmm_impl(ctx, N, ta, tb, nullptr));
    MDP_TRY(mdp_trmatvec_launch(ctx, A, tb, g));
    if (tl) {
        MDP_TRY(mdp_twolevel_qtx(ctx, tl, g));
        pcg_init_tl_kernel<<<RED_BLOCKS, RED_THREADS, 0, st>>>(inv, g, Cg, h, npix, tl->Z.as<double>(),
                                                               tl->AZ.as<double>(), tl->qtx.as<double>(), tl->zn, S);
    } else {
        pcg_init_kernel<<<RED_BLOCKS, RED_THREADS, 0, st>>>(inv, g, Cg, h, npix, S);
    }
    MDP_CHECK_LAUNCH(ctx);
    Scal *hs = reinterpret_cast<Scal *>(ctx->h_pinned);
    MDP_CUDA(cudaMemcpyAsync(hs, S, 8 * 8, cudaMemcpyDeviceToHost, st));
    MDP_CUDA(cudaStreamSynchronize(st));
    const double res0 = hs->res;
    const double tol2rel = params->tol * params->tol * res0;
    if (params->verbose) printf("k = %d, res = %e, g2pix = %e, res_rel = %e\n", 0, hs->res, hs->g2pix, 1.0);
    if (h_res_rel) h_res_rel[0] = 1.0;
    int    k = 1, converged = 0;
    double res = res0;
    if (!std::isfinite(res0)) {
        mdp_set_error("mdp_gls_solve: initial residual is %f", res0);
        return MDP_ENAN;
    }
    if (res <= params->tol) {
        k = params->maxiter;
        converged = 1;
    }
    const bool prof = ctx->profile != 0;
    for (; k < params->maxiter; k++) {
        std::swap(g, gp);
        if (prof) cudaEventRecord(ctx->ev[0], st);
        // P h with the block means of P h fused in when the blocks tile the rows
        const int fused = tpl ? MDP_EUNSUPPORTED : mdp_matvec_blockmeans(ctx, A, N, h, ta);
        if (fused != MDP_OK && fused != MDP_EUNSUPPORTED) return fused;
        if (fused == MDP_EUNSUPPORTED) MDP_TRY(mdp_matvec_launch(ctx, A, h, ta));
        if (prof) cudaEventRecord(ctx->ev[1], st);
        if (tpl)
            MDP_TRY(mdp_templates_filter(ctx, tpl, ta, tb));
        else
            MDP_TRY(mdp_stbmm_impl(ctx, N, ta, tb, fused == MDP_OK ? N->means.as<double>() : nullptr));
        if (prof) cudaEventRecord(ctx->ev[2], st);
        MDP_TRY(mdp_trmatvec_launch(ctx, A, tb, q));
        if (prof) cudaEventRecord(ctx->ev[3], st);
        pcg_coeff_kernel<<<RED_BLOCKS, RED_THREADS, 0, st>>>(h, q, n, S);
        MDP_CHECK_LAUNCH(ctx);
        if (tl) {
            pcg_step_kernel<<<grid_for(n, 256, ctx->sm_count * 8), 256, 0, st>>>(x, h, q, gp, g, n, S);
            MDP_CHECK_LAUNCH(ctx);
            MDP_TRY(mdp_twolevel_qtx(ctx, tl, g));
            pcg_precond_tl_kernel<<<RED_BLOCKS, RED_THREADS, 0, st>>>(inv, g, gp, Cg, npix, tl->Z.as<double>(),
                                                                      tl->AZ.as<double>(), tl->qtx.as<double>(),
                                                                      tl->zn, S);
        } else {
            pcg_update_kernel<<<RED_BLOCKS, RED_THREADS, 0, st>>>(inv, x, h, q, gp, g, Cg, npix, S);
        }
        MDP_CHECK_LAUNCH(ctx);
        if (prof) cudaEventRecord(ctx->ev[4], st);
        MDP_CUDA(cudaMemcpyAsync(hs, S, 8 * 8, cudaMemcpyDeviceToHost, st));
        MDP_CUDA(cudaStreamSynchronize(st));
        if (prof) {
            for (int e = 0; e < 4; e++) {
                float ms = 0.f;
                cudaEventElapsedTime(&ms, ctx->ev[e], ctx->ev[e + 1]);
                ctx->prof_ms[e] += ms;
                ctx->prof_n[e] += 1;
            }
        }
        res = hs->res;
        if (!std::isfinite(res)) {
            mdp_set_error("mdp_gls_solve: residual became %f at iteration %d", res, k);
            return MDP_ENAN;
        }
        if (h_res_rel) h_res_rel[k] = std::sqrt(res) / std::sqrt(res0);
        if (params->verbose)
            printf("k = %d, res = %e, g2pix = %e, res_rel = %e\n", k, res, hs->g2pix_polak, std::sqrt(res) / std::sqrt(res0));
        if (res <= tol2rel) {
            converged = 1;
            break;
        }
        pcg_direction_kernel<<<grid_for(n, 256, ctx->sm_count * 8), 256, 0, st>>>(h, Cg, n, S);
        MDP_CHECK_LAUNCH(ctx);
    }
    MDP_CUDA(cudaStreamSynchronize(st));
    if (info) {
        info->iterations = k;
        info->converged = converged;
        info->res0 = res0;
        info->res = res;
        info->n_map = n;
    }
    return MDP_OK;
}

extern "C" int mdp_gls_solve(mdp_context *ctx, mdp_pointing *A, const mdp_noise *N, const double *d_signal,
                             const double *d_noise, const mdp_solve_params *params, double *d_x, int32_t *d_lstid,
                             double *d_cond, int32_t *d_hits, double *h_res_rel, mdp_solve_info *info) {
    if (!ctx || !A || !N || !d_signal || !d_noise || !params || !d_x) {
        mdp_set_error("mdp_gls_solve: invalid arguments");
        return MDP_EINVAL;
    }
    if (N->nrow_end > A->m) {
        mdp_set_error("mdp_gls_solve: noise blocks extend past the pointing rows");
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
    // two-level preconditioners: Z, AZ and E^+ on the post-cut pointing; the
    // a-posteriori columns start from the first residual (precond.c:1341-1360)
    mdp_twolevel  tl;
    mdp_twolevel *tlp = nullptr;
    if (params->precond != 0) {
        DevBuf g0;
        if (params->precond == 2) {
            MDP_TRY(g0.alloc(8 * (size_t) A->n_map()));
            MDP_TRY(mdp_gls_rhs(ctx, A, N, d_signal, d_noise, g0.as<double>()));
        }
        MDP_TRY(mdp_twolevel_build(ctx, A, N, params->precond, params->z_2lvl, g0.as<double>(), &tl));
        tlp = &tl;
    }
    auto tp1 = std::chrono::steady_clock::now();
    MDP_TRY(mdp_pcg_run(ctx, A, N, bj.inv.as<double>(), bj.npix, d_signal, d_noise, params, d_x, h_res_rel, info,
                        tlp));
    auto tp2 = std::chrono::steady_clock::now();
    if (info) {
        info->n_cut = bj.ncut;
        info->n_map = A->n_map();
        info->precond_seconds = std::chrono::duration<double>(tp1 - tp0).count();
        info->solve_seconds = std::chrono::duration<double>(tp2 - tp1).count();
        info->outer_iterations = 0;
        info->fp64_applications = info->iterations;
    }
    return MDP_OK;
}

// The device-API solves keep the preconditioner with the pointing: the first
// solve builds it and applies the cut to the pointing; a later solve with the
// same noise operator reuses it; another noise operator rebuilds it on the
// already cut pointing.
int mdp_bj_cached(mdp_context *ctx, mdp_pointing *A, const mdp_noise *N, const BJState **out) {
    if (A->bj_cache && A->bj_noise_uid == N->uid) {
        *out = A->bj_cache;
        return MDP_OK;
    }
    delete A->bj_cache;
    A->bj_cache = nullptr;
    BJState *bj = new BJState();
    int      rc = mdp_bj_build(ctx, A, N, bj);
    if (rc != MDP_OK) {
        delete bj;
        return rc;
    }
    A->bj_cache = bj;
    A->bj_noise_uid = N->uid;
    *out = bj;
    return MDP_OK;
}

// ================================================================= mixed precision
extern "C" int mdp_gls_solve_mixed(mdp_context *ctx, mdp_pointing *A, const mdp_noise *Nc, const double *d_signal,
                                   const double *d_noise, const mdp_solve_params *params, double inner_tol,
                                   int inner_maxiter, double *d_x, int32_t *d_lstid, double *d_cond, int32_t *d_hits,
                                   double *h_res_rel, mdp_solve_info *info) {
    if (!ctx || !A || !Nc || !d_signal || !d_noise || !params || !d_x || inner_tol <= 0.0 || inner_maxiter < 1) {
        mdp_set_error("mdp_gls_solve_mixed: invalid arguments");
        return MDP_EINVAL;
    }
    mdp_noise *N = const_cast<mdp_noise *>(Nc);  // the FP32 plan is a cache of the operator
    if (N->nrow_end > A->m) {
        mdp_set_error("mdp_gls_solve_mixed: noise blocks extend past the pointing rows");
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
    MDP_TRY(mdp_pointing_prepare_fp32(ctx, A));
    MDP_TRY(mdp_noise_prepare_fp32(ctx, N));
    MDP_CUDA(cudaStreamSynchronize(st));
    auto tp1 = std::chrono::steady_clock::now();

    const int64_t m = A->m, npix = bj.npix, n = 3 * npix, nmap = A->n_map();
    const double *inv = bj.inv.as<double>();
    DevBuf &tod_a = ctx->ws[0], &tod_b = ctx->ws[1], &f_a = ctx->ws[8], &f_b = ctx->ws[9], &rb = ctx->ws[10],
           &gb1 = ctx->ws[2], &gb2 = ctx->ws[3], &hb = ctx->ws[4], &qb = ctx->ws[5], &cgb = ctx->ws[6],
           &db = ctx->ws[11], &scal = ctx->ws[7];
    int           rc;
    if ((rc = tod_a.alloc(8 * m)) || (rc = tod_b.alloc(8 * m)) || (rc = f_a.alloc(4 * m)) || (rc = f_b.alloc(4 * m)) ||
        (rc = rb.alloc(8 * nmap)) || (rc = gb1.alloc(8 * nmap)) || (rc = gb2.alloc(8 * nmap)) ||
        (rc = hb.alloc(8 * nmap)) || (rc = qb.alloc(8 * nmap)) || (rc = cgb.alloc(8 * nmap)) ||
        (rc = db.alloc(8 * nmap)) || (rc = scal.alloc(sizeof(Scal))))
        return rc;
    Scal     *S = scal.as<Scal>();
    double   *x = d_x, *r = rb.as<double>(), *g = gb1.as<double>(), *gp = gb2.as<double>();
    double   *h = hb.as<double>(), *q = qb.as<double>(), *Cg = cgb.as<double>(), *dl = db.as<double>();
    double   *ta = tod_a.as<double>(), *tb = tod_b.as<double>();
    float    *fa = f_a.as<float>(), *fb = f_b.as<float>();
    const int gm = grid_for(m, 256, ctx->sm_count * 16);
    const int gn = grid_for(nmap, 256, ctx->sm_count * 8);
    Scal     *hs = reinterpret_cast<Scal *>(ctx->h_pinned);
    MDP_CUDA(cudaMemsetAsync(S, 0, sizeof(Scal), st));
    MDP_CUDA(cudaMemsetAsync(x, 0, 8 * nmap, st));
    for (double *v : {r, g, gp, h, q, Cg, dl}) MDP_CUDA(cudaMemsetAsync(v, 0, 8 * nmap, st));

    auto fetch = [&]() -> int {
        MDP_CUDA(cudaMemcpyAsync(hs, S, 8 * 8, cudaMemcpyDeviceToHost, st));
        MDP_CUDA(cudaStreamSynchronize(st));
        return MDP_OK;
    };
    // FP64 residual r = P^T N^-1 (d' - P x)
    int  fp64_apps = 0;
    auto residual = [&](bool x_is_zero) -> int {
        if (x_is_zero) MDP_CUDA(cudaMemsetAsync(ta, 0, 8 * m, st));
        else MDP_TRY(mdp_matvec_launch(ctx, A, x, ta));
        tod_residual_kernel<<<gm, 256, 0, st>>>(A->off.as<int32_t>(), d_signal, d_noise, ta, m);
        MDP_CHECK_LAUNCH(ctx);
        MDP_TRY(mdp_stbmm_impl(ctx, N, ta, tb, nullptr));
        MDP_TRY(mdp_trmatvec_launch(ctx, A, tb, r));
        dot_self_kernel<<<RED_BLOCKS, RED_THREADS, 0, st>>>(r, n, S);
        MDP_CHECK_LAUNCH(ctx);
        fp64_apps++;
        return fetch();
    };
    MDP_TRY(residual(true));
    const double res0 = hs->res;
    if (!std::isfinite(res0)) {
        mdp_set_error("mdp_gls_solve_mixed: initial residual is %f", res0);
        return MDP_ENAN;
    }
    const double tol2rel = params->tol * params->tol * res0;
    if (h_res_rel) h_res_rel[0] = 1.0;
    // two-level preconditioners of the inner PCGs: Z, AZ and E^+ with the FP64
    // operator; the a-posteriori columns start from the first residual r
    mdp_twolevel  tlv;
    mdp_twolevel *tl = nullptr;
    if (params->precond != 0) {
        MDP_TRY(mdp_twolevel_build(ctx, A, N, params->precond, params->z_2lvl, r, &tlv));
        tl = &tlv;
    }
    double res = res0;
    int    outer = 0, inner_total = 0, converged = (res0 <= params->tol);
    const bool prof = ctx->profile != 0;
    while (!converged && inner_total < params->maxiter) {
        // inner PCG on A32 delta = r, delta0 = 0: g = r, Cg = M^-1 g, h = Cg
        MDP_CUDA(cudaMemcpyAsync(g, r, 8 * n, cudaMemcpyDeviceToDevice, st));
        MDP_CUDA(cudaMemsetAsync(dl, 0, 8 * nmap, st));
        if (tl) {
            MDP_TRY(mdp_twolevel_qtx(ctx, tl, g));
            pcg_init_tl_kernel<<<RED_BLOCKS, RED_THREADS, 0, st>>>(inv, g, Cg, h, npix, tl->Z.as<double>(),
                                                                   tl->AZ.as<double>(), tl->qtx.as<double>(), tl->zn,
                                                                   S);
        } else {
            pcg_init_kernel<<<RED_BLOCKS, RED_THREADS, 0, st>>>(inv, g, Cg, h, npix, S);
        }
        MDP_CHECK_LAUNCH(ctx);
        MDP_TRY(fetch());
        const double rin0 = hs->res;
        // inner target: inner_tol, or the reduction still needed (with a
        // factor 2 margin) when that is smaller
        const double need = 0.5 * params->tol / std::sqrt(res / res0);
        const double itol = std::max(inner_tol, std::min(need, 0.5));
        for (int j = 1; j <= inner_maxiter && inner_total < params->maxiter; j++) {
            std::swap(g, gp);
            if (prof) cudaEventRecord(ctx->ev[0], st);
            const int fused = mdp_matvec32_blockmeans(ctx, A, N, h, fa);
            if (fused != MDP_OK && fused != MDP_EUNSUPPORTED) return fused;
            if (fused == MDP_EUNSUPPORTED) MDP_TRY(mdp_matvec32_launch(ctx, A, h, fa));
            if (prof) cudaEventRecord(ctx->ev[1], st);
            MDP_TRY(mdp_stbmm_impl32(ctx, N, fa, fb, fused == MDP_OK ? N->means.as<double>() : nullptr));
            if (prof) cudaEventRecord(ctx->ev[2], st);
            MDP_TRY(mdp_trmatvec32_launch(ctx, A, fb, q));
            if (prof) cudaEventRecord(ctx->ev[3], st);
            pcg_coeff_kernel<<<RED_BLOCKS, RED_THREADS, 0, st>>>(h, q, n, S);
            MDP_CHECK_LAUNCH(ctx);
            if (tl) {
                pcg_step_kernel<<<grid_for(n, 256, ctx->sm_count * 8), 256, 0, st>>>(dl, h, q, gp, g, n, S);
                MDP_CHECK_LAUNCH(ctx);
                MDP_TRY(mdp_twolevel_qtx(ctx, tl, g));
                pcg_precond_tl_kernel<<<RED_BLOCKS, RED_THREADS, 0, st>>>(inv, g, gp, Cg, npix, tl->Z.as<double>(),
                                                                          tl->AZ.as<double>(), tl->qtx.as<double>(),
                                                                          tl->zn, S);
            } else {
                pcg_update_kernel<<<RED_BLOCKS, RED_THREADS, 0, st>>>(inv, dl, h, q, gp, g, Cg, npix, S);
            }
            MDP_CHECK_LAUNCH(ctx);
            if (prof) cudaEventRecord(ctx->ev[4], st);
            MDP_TRY(fetch());
            inner_total++;
            if (prof)
                for (int e = 0; e < 4; e++) {
                    float ms = 0.f;
                    cudaEventElapsedTime(&ms, ctx->ev[e], ctx->ev[e + 1]);
                    ctx->prof_ms[e] += ms;
                    ctx->prof_n[e] += 1;
                }
            if (!std::isfinite(hs->res)) {
                mdp_set_error("mdp_gls_solve_mixed: inner residual became %f", hs->res);
                return MDP_ENAN;
            }
            if (hs->res <= itol * itol * rin0) break;
            pcg_direction_kernel<<<gn, 256, 0, st>>>(h, Cg, n, S);
            MDP_CHECK_LAUNCH(ctx);
        }
        axpy1_kernel<<<gn, 256, 0, st>>>(x, dl, n);
        MDP_CHECK_LAUNCH(ctx);
        outer++;
        MDP_TRY(residual(false));
        res = hs->res;
        if (h_res_rel && outer <= params->maxiter) h_res_rel[outer] = std::sqrt(res / res0);
        if (params->verbose)
            printf("refinement %d: %d inner iterations so far, res_rel = %e\n", outer, inner_total, std::sqrt(res / res0));
        if (!std::isfinite(res)) {
            mdp_set_error("mdp_gls_solve_mixed: residual became %f after refinement %d", res, outer);
            return MDP_ENAN;
        }
        converged = res <= tol2rel;
    }
    MDP_CUDA(cudaStreamSynchronize(st));
    auto tp2 = std::chrono::steady_clock::now();
    if (info) {
        info->iterations = inner_total;
        info->converged = converged;
        info->res0 = res0;
        info->res = res;
        info->n_map = A->n_map();
        info->n_cut = bj.ncut;
        info->precond_seconds = std::chrono::duration<double>(tp1 - tp0).count();
        info->solve_seconds = std::chrono::duration<double>(tp2 - tp1).count();
        info->outer_iterations = outer;
        info->fp64_applications = fp64_apps;
    }
    return MDP_OK;
}

// ================================================================= pieces of a sharded solve
// A solve split over ranks (each rank holding the samples of some detectors
// and stationary intervals) needs the per-rank parts of the steps above with
// the exchanges between them done by the caller: the rank's 3x3 blocks (summed
// over ranks), their inversion and rcond cut, the cut applied to the rank's
// samples, the FP64 residual and one operator application per PCG iteration.

extern "C" int mdp_local_blocks(mdp_context *ctx, mdp_pointing *A, const mdp_noise *N, double *d_W,
                                int32_t *d_hits) {
    if (!ctx || !A || !N || !d_W || !d_hits) return MDP_EINVAL;
    if (!A->triplet) {
        mdp_set_error("mdp_local_blocks: the (I,Q,U) triplet pointing layout is needed");
        return MDP_EUNSUPPORTED;
    }
    MDP_CUDA(cudaSetDevice(ctx->device));
    const int64_t npix = A->n_map() / 3;
    cudaStream_t  st = ctx->stream;
    MDP_TRY(localW_launch(ctx, A, N, d_W, d_hits));
    return MDP_OK;
}

extern "C" int mdp_block_inverse(mdp_context *ctx, int64_t npix, double *d_W, double *d_inv, double *d_rcond,
                                 int32_t *d_cut, int64_t *n_cut) {
    if (!ctx || npix < 0 || (npix > 0 && (!d_W || !d_inv || !d_rcond || !d_cut))) return MDP_EINVAL;
    MDP_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    MDP_TRY(ctx->scratch2.alloc(sizeof(int)));
    MDP_CUDA(cudaMemsetAsync(ctx->scratch2.p, 0, sizeof(int), st));
    if (npix > 0) {
        bj_pixel_kernel<<<grid_for(npix, 128, ctx->sm_count * 8), 128, 0, st>>>(d_W, npix, d_inv, d_rcond, d_cut,
                                                                               ctx->scratch2.as<int>());
        MDP_CHECK_LAUNCH(ctx);
    }
    int h = 0;
    MDP_CUDA(cudaMemcpyAsync(&h, ctx->scratch2.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    MDP_CUDA(cudaStreamSynchronize(st));
    if (n_cut) *n_cut = h;
    return MDP_OK;
}

extern "C" int mdp_pointing_cut(mdp_context *ctx, mdp_pointing *A, const int32_t *d_target, int64_t *kept_pixels) {
    if (!ctx || !A || !d_target) return MDP_EINVAL;
    if (!A->triplet) {
        mdp_set_error("mdp_pointing_cut: the (I,Q,U) triplet pointing layout is needed");
        return MDP_EUNSUPPORTED;
    }
    MDP_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t  st = ctx->stream;
    const int64_t npix0 = A->n_map() / 3;
    if (npix0 == 0) {
        if (kept_pixels) *kept_pixels = 0;
        return MDP_OK;
    }
    const uint32_t *target = reinterpret_cast<const uint32_t *>(d_target);  // 0 / 1 flags
    DevBuf          remap, keep, lind2;
    MDP_TRY(remap.alloc(4 * npix0));
    MDP_TRY(keep.alloc(4 * npix0));
    MDP_TRY(lind2.alloc(4 * (3 * npix0 + 3)));
    const int gb = grid_for(npix0, 256, ctx->sm_count * 8);
    invert_flags_kernel<<<gb, 256, 0, st>>>(target, keep.as<uint32_t>(), npix0);
    MDP_CHECK_LAUNCH(ctx);
    uint32_t kept = 0;
    MDP_TRY(mdp_exclusive_scan_u32(ctx, keep.as<uint32_t>(), remap.as<uint32_t>(), npix0, &kept));
    if (kept_pixels) *kept_pixels = kept;
    if ((int64_t) kept == npix0) return MDP_OK;  // nothing to cut
    rewrite_off_kernel<<<grid_for(A->m, 256, ctx->sm_count * 16), 256, 0, st>>>(A->off.as<int32_t>(), A->m, target,
                                                                               remap.as<uint32_t>());
    MDP_CHECK_LAUNCH(ctx);
    new_lindices_kernel<<<gb, 256, 0, st>>>(A->lindices.as<int32_t>(), A->trash_pix, npix0, target,
                                            remap.as<uint32_t>(), lind2.as<int32_t>());
    MDP_CHECK_LAUNCH(ctx);
    MDP_CUDA(cudaStreamSynchronize(st));
    std::swap(A->lindices.p, lind2.p);
    std::swap(A->lindices.bytes, lind2.bytes);
    A->bins.valid = 0;
    A->mbins.valid = 0;
    A->trash_pix = 1;
    A->lcount = 3 * (int64_t) kept + 3;
    delete A->bj_cache;  // built for the old numbering
    A->bj_cache = nullptr;
    return MDP_OK;
}

// g = P^T N^-1 d' with d' = b (0 on cut rows) + noise: the PCG's first residual for x0 = 0
int mdp_gls_rhs(mdp_context *ctx, mdp_pointing *A, const mdp_noise *N, const double *d_signal, const double *d_noise,
                double *d_g) {
    const int64_t m = A->m;
    MDP_TRY(ctx->ws[0].alloc(8 * m));
    MDP_TRY(ctx->ws[1].alloc(8 * m));
    double *ta = ctx->ws[0].as<double>(), *tb = ctx->ws[1].as<double>();
    rhs_kernel<<<grid_for(m, 256, ctx->sm_count * 16), 256, 0, ctx->stream>>>(A->off.as<int32_t>(), d_signal,
                                                                               d_noise, ta, m);
    MDP_CHECK_LAUNCH(ctx);
    MDP_TRY(mdp_stbmm_impl(ctx, N, ta, tb, nullptr));
    return mdp_trmatvec_launch(ctx, A, tb, d_g);
}

// q = P^T N^-1 P h in FP64, the block means of P h fused into P when the blocks tile the rows
int mdp_apply_op_impl(mdp_context *ctx, mdp_pointing *A, const mdp_noise *N, const double *d_h, double *d_q) {
    const int64_t m = A->m;
    MDP_TRY(ctx->ws[0].alloc(8 * m));
    MDP_TRY(ctx->ws[1].alloc(8 * m));
    double   *ta = ctx->ws[0].as<double>(), *tb = ctx->ws[1].as<double>();
    const int fused = mdp_matvec_blockmeans(ctx, A, N, d_h, ta);
    if (fused != MDP_OK && fused != MDP_EUNSUPPORTED) return fused;
    if (fused == MDP_EUNSUPPORTED) MDP_TRY(mdp_matvec_launch(ctx, A, d_h, ta));
    MDP_TRY(mdp_stbmm_impl(ctx, N, ta, tb, fused == MDP_OK ? N->means.as<double>() : nullptr));
    return mdp_trmatvec_launch(ctx, A, tb, d_q);
}

extern "C" int mdp_gls_residual(mdp_context *ctx, mdp_pointing *A, const mdp_noise *N, const double *d_signal,
                                const double *d_noise, const double *d_x, double *d_r) {
    if (!ctx || !A || !N || !d_signal || !d_noise || !d_r) return MDP_EINVAL;
    if (!A->triplet || N->nrow_end > A->m) {
        mdp_set_error("mdp_gls_residual: triplet pointing and noise blocks within its rows are needed");
        return MDP_EUNSUPPORTED;
    }
    MDP_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const int64_t m = A->m;
    MDP_TRY(ctx->ws[0].alloc(8 * m));
    MDP_TRY(ctx->ws[1].alloc(8 * m));
    double *ta = ctx->ws[0].as<double>(), *tb = ctx->ws[1].as<double>();
    const int gm = grid_for(m, 256, ctx->sm_count * 16);
    if (d_x) MDP_TRY(mdp_matvec_launch(ctx, A, d_x, ta));
    else MDP_CUDA(cudaMemsetAsync(ta, 0, 8 * m, st));
    tod_residual_kernel<<<gm, 256, 0, st>>>(A->off.as<int32_t>(), d_signal, d_noise, ta, m);
    MDP_CHECK_LAUNCH(ctx);
    MDP_TRY(mdp_stbmm_impl(ctx, N, ta, tb, nullptr));
    return mdp_trmatvec_launch(ctx, A, tb, d_r);
}

extern "C" int mdp_apply_op(mdp_context *ctx, mdp_pointing *A, const mdp_noise *Nc, const double *d_h, double *d_q,
                            int fp32) {
    if (!ctx || !A || !Nc || !d_h || !d_q) return MDP_EINVAL;
    mdp_noise *N = const_cast<mdp_noise *>(Nc);  // the FP32 plan is a cache of the operator
    if (N->nrow_end > A->m) {
        mdp_set_error("mdp_apply_op: noise blocks extend past the pointing rows");
        return MDP_EINVAL;
    }
    MDP_CUDA(cudaSetDevice(ctx->device));
    const int64_t m = A->m;
    if (!fp32) return mdp_apply_op_impl(ctx, A, N, d_h, d_q);
    MDP_TRY(mdp_pointing_prepare_fp32(ctx, A));
    MDP_TRY(mdp_noise_prepare_fp32(ctx, N));
    MDP_TRY(ctx->ws[8].alloc(4 * m));
    MDP_TRY(ctx->ws[9].alloc(4 * m));
    float    *fa = ctx->ws[8].as<float>(), *fb = ctx->ws[9].as<float>();
    const int fused = mdp_matvec32_blockmeans(ctx, A, N, d_h, fa);
    if (fused != MDP_OK && fused != MDP_EUNSUPPORTED) return fused;
    if (fused == MDP_EUNSUPPORTED) MDP_TRY(mdp_matvec32_launch(ctx, A, d_h, fa));
    MDP_TRY(mdp_stbmm_impl32(ctx, N, fa, fb, fused == MDP_OK ? N->means.as<double>() : nullptr));
    return mdp_trmatvec32_launch(ctx, A, fb, d_q);
}
