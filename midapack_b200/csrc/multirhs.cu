// Multi-RHS mixed-precision GLS solve: many right-hand sides (Monte-Carlo
// noise realisations, signal + noise) that share one pointing matrix and one
// noise model, e.g. the 128 simulations of a map-making error budget.
//
// Each column is the solve of MAPPRAISER's MLmap/PCG_GLS_true
// (mappraiser/src/mappraiser.c:34-385, pcg_true.c:20-241): block-Jacobi
// preconditioned PCG on (P^T N^-1 P) x = P^T N^-1 d, stopping when
// sum(g^2) <= tol^2 sum(g0^2) with g the unpreconditioned map residual; the
// reference has no multi-RHS solver (it solves one right-hand side per call).
//
// Scheme.  FP64 iterative refinement per column: r = P^T N^-1 (d - P x) in
// FP64, then an inner block-Jacobi PCG on the FP32 operator solves A delta = r
// to a relative residual inner_tol, x += delta, repeat.  The inner solves of
// up to G columns ("slots") advance together: one batched iteration reads the
// pointing once for all slots (P and P^T), runs the FP32 Toeplitz tiles of
// every slot in one launch, and updates the G PCG states with per-slot
// scalars.  A slot whose inner solve stops gets its FP64 refinement step and
// then restarts, or, when its column has converged, takes the next column
// (columns retire independently; the batch stays full while columns remain).
// The batched iteration is captured once as a CUDA graph (two graphs: the
// current and previous gradient buffers alternate) and replayed.
//
// Layout.  The slot vectors are interleaved per pixel, [npix][G][3] FP64, so
// the batched P gathers 3G contiguous values per sample, the batched P^T
// accumulates all slots of a pixel bin in one shared-memory tile, and the
// block-Jacobi apply reads each 3x3 block once for all slots.  The FP32 TODs
// of the slots are column-major [G][m].
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "mdp_internal.cuh"

#define MR_BLOCKS 296
#define MR_THREADS 256
#define MR_MAXG 8
#define MR_BIN_PIX 2048
#define MR_SPLIT 4

struct SlotScal {
    double g2pix, g2pixp, g2pix_polak, coeff, res, ro, gamma, rin0;
    double tol2;     // inner stop: res <= tol2 * rin0
    double dot;      // result of mr_dot_kernel
    int    cont;     // 1 while the inner PCG of the slot continues
    int    stopped;  // set by the device when the inner PCG stops (the slot's run flag drops)
    int    inner_it; // inner iterations since the slot's last (re)start
    int    budget;   // inner iterations the slot may still take (inner cap, column cap)
};

struct MRed {
    double       part[3 * MR_MAXG][MR_BLOCKS];
    unsigned int count[4];
};

// ---------------------------------------------------------------- reductions
// Each block stores K*G partial sums; the last block to finish adds them in
// block order (deterministic).
template <int KG>
__device__ __forceinline__ void mr_block_store(double (&v)[KG], MRed *R) {
    __shared__ double sh[KG][MR_THREADS / 32];
#pragma unroll
    for (int k = 0; k < KG; k++)
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    if ((threadIdx.x & 31) == 0)
#pragma unroll
        for (int k = 0; k < KG; k++) sh[k][threadIdx.x >> 5] = v[k];
    __syncthreads();
    if (threadIdx.x < KG) {
        double s = 0.0;
        for (int w = 0; w < MR_THREADS / 32; w++) s += sh[threadIdx.x][w];
        R->part[threadIdx.x][blockIdx.x] = s;
    }
}

__device__ __forceinline__ bool mr_last_block(MRed *R, int c) {
    __shared__ bool is_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) is_last = (atomicAdd(&R->count[c], 1u) == gridDim.x - 1);
    __syncthreads();
    return is_last;
}

__device__ __forceinline__ double mr_sum(const MRed *R, int k) {
    double s = 0.0;
    for (int b = 0; b < MR_BLOCKS; b++) s += R->part[k][b];
    return s;
}

// ---------------------------------------------------------------- operator kernels
// Y[j] = P h_j (FP32 weights, FP32 copy of h_j) for the running slots, with
// FP64 partial sums per 65536-row chunk (block means of N^-1).  The FP32 copy
// of the slot directions (12 bytes per pixel and slot) keeps the gathered map
// L2-resident for 8 slots of a few million pixels.
template <int G>
__global__ void __launch_bounds__(512) mr_matvec32_kernel(const int32_t *__restrict__ off, const float *__restrict__ w,
                                                          const float *__restrict__ H, const int *__restrict__ run,
                                                          float *__restrict__ Y, int64_t m,
                                                          const int64_t *__restrict__ chunk_start,
                                                          const int32_t *__restrict__ chunk_len, int n_chunks,
                                                          double *__restrict__ partial) {
    bool act[G], any = false;
#pragma unroll
    for (int j = 0; j < G; j++) {
        act[j] = run[j] != 0;
        any = any || act[j];
    }
    if (!any) return;  // every slot has stopped
    const int64_t s = chunk_start[blockIdx.x];
    const int     n = chunk_len[blockIdx.x];
    double        acc[G];
#pragma unroll
    for (int j = 0; j < G; j++) acc[j] = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int64_t t = s + i;
        const int32_t o = off[t];
        float         w0 = 0.f, w1 = 0.f, w2 = 0.f;
        if (o >= 0) {
            w0 = w[3 * t];
            w1 = w[3 * t + 1];
            w2 = w[3 * t + 2];
        }
        const float *h = H + (int64_t) (o >= 0 ? o : 0) * G;  // pixel p = o/3 starts at 3pG = oG
        float        hv[3 * G];
        if (o >= 0) {
            if constexpr (G % 4 == 0) {  // 12G bytes at a 48-byte multiple: float4 loads
#pragma unroll
                for (int q = 0; q < 3 * G / 4; q++) {
                    const float4 f = __ldg(reinterpret_cast<const float4 *>(h) + q);
                    hv[4 * q] = f.x;
                    hv[4 * q + 1] = f.y;
                    hv[4 * q + 2] = f.z;
                    hv[4 * q + 3] = f.w;
                }
            } else if constexpr (G % 2 == 0) {
#pragma unroll
                for (int q = 0; q < 3 * G / 2; q++) {
                    const float2 f = __ldg(reinterpret_cast<const float2 *>(h) + q);
                    hv[2 * q] = f.x;
                    hv[2 * q + 1] = f.y;
                }
            } else {
#pragma unroll
                for (int q = 0; q < 3 * G; q++) hv[q] = __ldg(h + q);
            }
        }
#pragma unroll
        for (int j = 0; j < G; j++) {
            if (!act[j]) continue;
            float v = 0.0f;
            if (o >= 0) v = w0 * hv[3 * j] + w1 * hv[3 * j + 1] + w2 * hv[3 * j + 2];
            Y[(int64_t) j * m + t] = v;
            acc[j] += (double) v;
        }
    }
#pragma unroll
    for (int j = 0; j < G; j++)
        for (int o = 16; o > 0; o >>= 1) acc[j] += __shfl_xor_sync(0xffffffffu, acc[j], o);
    __shared__ double ws[G][16];
    if ((threadIdx.x & 31) == 0)
#pragma unroll
        for (int j = 0; j < G; j++) ws[j][threadIdx.x >> 5] = acc[j];
    __syncthreads();
    if (threadIdx.x < G) {
        double v = 0.0;
        for (int q = 0; q < (int) (blockDim.x >> 5); q++) v += ws[threadIdx.x][q];
        partial[(int64_t) threadIdx.x * n_chunks + blockIdx.x] = v;
    }
}

__global__ void mr_means_kernel(const double *__restrict__ partial, int n_chunks, const int32_t *__restrict__ blk_chunk0,
                                const int32_t *__restrict__ blk_nchunk, const int32_t *__restrict__ blk_len, int nb,
                                double *__restrict__ means) {
    const int j = blockIdx.y;
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int c = 0; c < blk_nchunk[b]; c++) s += partial[(int64_t) j * n_chunks + blk_chunk0[b] + c];
        means[(int64_t) j * nb + b] = s / (double) blk_len[b];
    }
}

// Q (interleaved, zeroed) += P^T Z_j for the running slots: bins of
// MR_BIN_PIX/G pixels, FP64 products and shared-memory sums, one global atomic
// per map entry of the bin.  The shared tile is slot-major, row r = 3j+k holds
// the bin's pixels, with the pixel index XORed by r mod 32: the atomics of a
// warp (consecutive samples, mostly distinct pixels of one row) and the flush
// (consecutive map entries, i.e. consecutive rows at one pixel) both spread
// over the banks.
template <int G>
__device__ __forceinline__ int mr_acc_index(int r, int pl) {
    return r * (MR_BIN_PIX / G) + (pl ^ (r & 31));
}

template <int G>
__global__ void __launch_bounds__(512) mr_trmatvec32_kernel(const int32_t *__restrict__ off,
                                                            const float *__restrict__ w,
                                                            const float *__restrict__ Z, const int *__restrict__ run,
                                                            double *__restrict__ Q, int64_t m,
                                                            const int64_t *__restrict__ bin_start,
                                                            const uint32_t *__restrict__ perm, int64_t npix) {
    constexpr int BP = MR_BIN_PIX / G;
    static_assert(BP % 32 == 0, "bins must hold a multiple of 32 pixels");
    __shared__ double acc[3 * MR_BIN_PIX];
    bool              act[G], any = false;
#pragma unroll
    for (int j = 0; j < G; j++) {
        act[j] = run[j] != 0;
        any = any || act[j];
    }
    if (!any) return;  // every slot has stopped
    const int64_t bin = blockIdx.x / MR_SPLIT;
    const int     part = blockIdx.x % MR_SPLIT;
    for (int i = threadIdx.x; i < 3 * MR_BIN_PIX; i += blockDim.x) acc[i] = 0.0;
    __syncthreads();
    const int64_t s0 = bin_start[bin], s1 = bin_start[bin + 1];
    const int64_t len = s1 - s0;
    const int64_t a = s0 + len * part / MR_SPLIT, b = s0 + len * (part + 1) / MR_SPLIT;
    const int64_t p0 = bin * BP;
    for (int64_t i = a + threadIdx.x; i < b; i += blockDim.x) {
        const int64_t t = perm[i];
        const int     pl = off[t] / 3 - (int) p0;
        const double  w0 = (double) w[3 * t], w1 = (double) w[3 * t + 1], w2 = (double) w[3 * t + 2];
#pragma unroll
        for (int j = 0; j < G; j++) {
            if (!act[j]) continue;
            const double v = (double) Z[(int64_t) j * m + t];
            atomicAdd(acc + mr_acc_index<G>(3 * j, pl), w0 * v);
            atomicAdd(acc + mr_acc_index<G>(3 * j + 1, pl), w1 * v);
            atomicAdd(acc + mr_acc_index<G>(3 * j + 2, pl), w2 * v);
        }
    }
    __syncthreads();
    const int64_t base = p0 * 3 * G;
    const int64_t lim = min((int64_t) 3 * MR_BIN_PIX, npix * 3 * G - base);
    for (int i = threadIdx.x; i < lim; i += blockDim.x) {
        const int    pl = i / (3 * G), r = i - pl * 3 * G;  // map entry (p0 + pl, j, k), r = 3j + k
        const double v = acc[mr_acc_index<G>(r, pl)];
        if (v != 0.0) atomicAdd(Q + base + i, v);
    }
}

// ---------------------------------------------------------------- PCG kernels (interleaved)
// h = gamma_j h + Cg_j for the slots that continue; H32 = FP32 copy of h for
// every running slot
template <int G>
__global__ void mr_direction_kernel(double *__restrict__ H, float *__restrict__ H32, const double *__restrict__ CG,
                                    int64_t npix, const int *__restrict__ run, const SlotScal *__restrict__ S) {
    double gam[G];
    bool   act[G], on[G];
#pragma unroll
    for (int j = 0; j < G; j++) {
        on[j] = run[j] != 0;
        act[j] = on[j] && S[j].cont;
        gam[j] = S[j].gamma;
    }
    const int64_t n = npix * 3 * G;
    for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x) {
        const int j = (int) ((i / 3) % G);
        if (!on[j]) continue;
        double h = H[i];
        if (act[j]) {
            h = h * gam[j] + CG[i];
            H[i] = h;
        }
        H32[i] = (float) h;
    }
}

// coeff_j = (h_j, q_j), ro_j = g2pix_j / coeff_j
template <int G>
__global__ void __launch_bounds__(MR_THREADS) mr_coeff_kernel(const double *__restrict__ H,
                                                             const double *__restrict__ Q, int64_t npix,
                                                             const int *__restrict__ run, SlotScal *S, MRed *R) {
    bool any = false;
#pragma unroll
    for (int j = 0; j < G; j++) any = any || run[j] != 0;
    if (!any) return;  // every slot has stopped: the whole grid returns
    double v[G];
#pragma unroll
    for (int j = 0; j < G; j++) v[j] = 0.0;
    for (int64_t p = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += (int64_t) gridDim.x * blockDim.x) {
        const double *h = H + p * 3 * G, *q = Q + p * 3 * G;
#pragma unroll
        for (int j = 0; j < G; j++) v[j] += h[3 * j] * q[3 * j] + h[3 * j + 1] * q[3 * j + 1] + h[3 * j + 2] * q[3 * j + 2];
    }
    mr_block_store<G>(v, R);
    if (mr_last_block(R, 0) && threadIdx.x == 0) {
        for (int j = 0; j < G; j++)
            if (run[j]) {
                S[j].coeff = mr_sum(R, j);
                S[j].ro = S[j].g2pix / S[j].coeff;
            }
        R->count[0] = 0;
    }
}

// delta += ro h; g = gp - ro q; Cg = M^-1 g; per slot (Cg,g), (Cg,g-gp), (g,g);
// the last block decides whether each slot's inner PCG continues
template <int G>
__global__ void __launch_bounds__(MR_THREADS) mr_update_kernel(const double *__restrict__ inv, double *__restrict__ DL,
                                                              const double *__restrict__ H,
                                                              const double *__restrict__ Q,
                                                              const double *__restrict__ GP, double *__restrict__ Gn,
                                                              double *__restrict__ CG, int64_t npix, int *run,
                                                              SlotScal *S, MRed *R) {
    double ro[G];
    bool   act[G], any = false;
#pragma unroll
    for (int j = 0; j < G; j++) {
        act[j] = run[j] != 0;
        any = any || act[j];
        ro[j] = S[j].ro;
    }
    if (!any) return;  // every slot has stopped: the whole grid returns, no partials
    double v[3 * G];
#pragma unroll
    for (int k = 0; k < 3 * G; k++) v[k] = 0.0;
    for (int64_t p = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += (int64_t) gridDim.x * blockDim.x) {
        const double *I = inv + 9 * p;
        const double  i0 = I[0], i1 = I[1], i2 = I[2], i3 = I[3], i4 = I[4], i5 = I[5], i6 = I[6], i7 = I[7], i8 = I[8];
#pragma unroll
        for (int j = 0; j < G; j++) {
            if (!act[j]) continue;
            const int64_t e = (p * G + j) * 3;
            double        gn[3], go[3];
#pragma unroll
            for (int k = 0; k < 3; k++) {
                DL[e + k] = DL[e + k] + ro[j] * H[e + k];
                go[k] = GP[e + k];
                gn[k] = go[k] - ro[j] * Q[e + k];
                Gn[e + k] = gn[k];
            }
            double c[3];
            c[0] = i0 * gn[0] + i1 * gn[1] + i2 * gn[2];
            c[1] = i3 * gn[0] + i4 * gn[1] + i5 * gn[2];
            c[2] = i6 * gn[0] + i7 * gn[1] + i8 * gn[2];
#pragma unroll
            for (int k = 0; k < 3; k++) {
                CG[e + k] = c[k];
                v[j] += c[k] * gn[k];
                v[G + j] += c[k] * (gn[k] - go[k]);
                v[2 * G + j] += gn[k] * gn[k];
            }
        }
    }
    mr_block_store<3 * G>(v, R);
    if (mr_last_block(R, 1) && threadIdx.x == 0) {
        for (int j = 0; j < G; j++) {
            if (!run[j]) continue;
            SlotScal &s = S[j];
            s.g2pixp = s.g2pix;
            s.g2pix = mr_sum(R, j);
            s.g2pix_polak = mr_sum(R, G + j);
            s.res = mr_sum(R, 2 * G + j);
            s.gamma = s.g2pix_polak / s.g2pixp;
            s.inner_it++;
            s.budget--;
            s.cont = (isfinite(s.res) && s.res > s.tol2 * s.rin0 && s.budget > 0) ? 1 : 0;
            if (!s.cont) {  // the slot stops here: later iterations of the batch skip it
                s.stopped = 1;
                run[j] = 0;
            }
        }
        R->count[1] = 0;
    }
}

// slot j restarts its inner PCG on the residual r (column vector):
// g = r, Cg = M^-1 g, h = Cg, delta = 0, g2pix = (Cg,g), rin0 = res = (g,g)
template <int G>
__global__ void __launch_bounds__(MR_THREADS) mr_slot_init_kernel(const double *__restrict__ inv,
                                                                 const double *__restrict__ r, int j,
                                                                 double *__restrict__ Gn, double *__restrict__ CG,
                                                                 double *__restrict__ H, double *__restrict__ DL,
                                                                 int64_t npix, double tol2, int budget, int *run,
                                                                 SlotScal *S, MRed *R) {
    double v[2] = {0.0, 0.0};
    for (int64_t p = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += (int64_t) gridDim.x * blockDim.x) {
        const double *I = inv + 9 * p;
        const double  g0 = r[3 * p], g1 = r[3 * p + 1], g2 = r[3 * p + 2];
        const double  c0 = I[0] * g0 + I[1] * g1 + I[2] * g2;
        const double  c1 = I[3] * g0 + I[4] * g1 + I[5] * g2;
        const double  c2 = I[6] * g0 + I[7] * g1 + I[8] * g2;
        const int64_t e = (p * G + j) * 3;
        Gn[e] = g0;
        Gn[e + 1] = g1;
        Gn[e + 2] = g2;
        CG[e] = c0;
        CG[e + 1] = c1;
        CG[e + 2] = c2;
        H[e] = c0;
        H[e + 1] = c1;
        H[e + 2] = c2;
        DL[e] = 0.0;
        DL[e + 1] = 0.0;
        DL[e + 2] = 0.0;
        v[0] += c0 * g0 + c1 * g1 + c2 * g2;
        v[1] += g0 * g0 + g1 * g1 + g2 * g2;
    }
    mr_block_store<2>(v, R);
    if (mr_last_block(R, 2) && threadIdx.x == 0) {
        SlotScal &s = S[j];
        s.g2pix = mr_sum(R, 0);
        s.res = mr_sum(R, 1);
        s.rin0 = s.res;
        s.tol2 = tol2;
        s.cont = 0;  // h = Cg already: no direction update before the first iteration
        s.stopped = 0;
        s.inner_it = 0;
        s.budget = budget;
        run[j] = 1;
        R->count[2] = 0;
    }
}

// x (column) += delta_j
template <int G>
__global__ void mr_extract_add_kernel(const double *__restrict__ DL, int j, double *__restrict__ x, int64_t npix) {
    for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < 3 * npix; i += (int64_t) gridDim.x * blockDim.x)
        x[i] += DL[((i / 3) * G + j) * 3 + i % 3];
}

// out = d' - out, d' = signal (0 on cut rows; absent: 0) + noise
template <typename TN>
__global__ void mr_tod_residual_kernel(const int32_t *__restrict__ off, const double *__restrict__ signal,
                                       const TN *__restrict__ noise, double *__restrict__ out, int64_t m) {
    for (int64_t t = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; t < m; t += (int64_t) gridDim.x * blockDim.x) {
        const double s = (signal && off[t] != -2) ? signal[t] : 0.0;
        out[t] = s + (double) noise[t] - out[t];
    }
}

// S[j].dot = (g, g)
__global__ void __launch_bounds__(MR_THREADS) mr_dot_kernel(const double *__restrict__ g, int64_t n, int j,
                                                           SlotScal *S, MRed *R) {
    double v[1] = {0.0};
    for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x)
        v[0] += g[i] * g[i];
    mr_block_store<1>(v, R);
    if (mr_last_block(R, 3) && threadIdx.x == 0) {
        S[j].dot = mr_sum(R, 0);
        R->count[3] = 0;
    }
}

// ---------------------------------------------------------------- host side
namespace {

struct Batch {
    int     G = 0;
    int64_t m = 0, npix = 0, nmap = 0;
    DevBuf  H, Q, G1, G2, CG, DL;  // [npix][G][3]
    DevBuf  H32;                   // FP32 copy of H
    DevBuf  Y, Z;                  // FP32 [G][m]
    DevBuf  partial, means;        // [G][n_chunks], [G][nb]
    DevBuf  run;                   // int [G]
    DevBuf  scal, red;             // SlotScal [G], MRed
    int     n_chunks = 0;
    const int64_t *chunk_start = nullptr;
    const int32_t *chunk_len = nullptr, *blk_chunk0 = nullptr, *blk_nchunk = nullptr;
};

template <int G>
int launch_apply32(mdp_context *ctx, mdp_pointing *A, mdp_noise *N, Batch &B, const float *h) {
    cudaStream_t st = ctx->stream;
    const int   *run = B.run.as<int>();
    mr_matvec32_kernel<G><<<B.n_chunks, 512, 0, st>>>(A->off.as<int32_t>(), A->w32.as<float>(), h, run, B.Y.as<float>(),
                                                      B.m, B.chunk_start, B.chunk_len, B.n_chunks,
                                                      B.partial.as<double>());
    MDP_CHECK_LAUNCH(ctx);
    mr_means_kernel<<<dim3(grid_for(N->nb, 128, 64), G), 128, 0, st>>>(B.partial.as<double>(), B.n_chunks,
                                                                       B.blk_chunk0, B.blk_nchunk,
                                                                       N->blk_len.as<int32_t>(), N->nb,
                                                                       B.means.as<double>());
    MDP_CHECK_LAUNCH(ctx);
    MDP_TRY(mdp_stbmm32_batch(ctx, N, B.Y.as<float>(), B.Z.as<float>(), G, B.m, B.means.as<double>(), run));
    MDP_CUDA(cudaMemsetAsync(B.Q.p, 0, sizeof(double) * B.npix * 3 * G, st));
    if (A->mbins.nbins > 0) {
        mr_trmatvec32_kernel<G><<<(unsigned) (A->mbins.nbins * MR_SPLIT), 512, 0, st>>>(
                A->off.as<int32_t>(), A->w32.as<float>(), B.Z.as<float>(), run, B.Q.as<double>(), B.m,
                A->mbins.start.as<int64_t>(), A->mbins.perm.as<uint32_t>(), B.npix);
        MDP_CHECK_LAUNCH(ctx);
    }
    return MDP_OK;
}

// one batched inner iteration: direction (slots that continue), q = A32 h,
// coeff, update (which stops a slot's inner PCG on the device); with h_scal,
// ends with the slot scalars copied to pinned host memory
template <int G>
int launch_iteration(mdp_context *ctx, mdp_pointing *A, mdp_noise *N, Batch &B, const double *inv, double *g,
                     double *gp, SlotScal *h_scal) {
    cudaStream_t st = ctx->stream;
    int         *run = B.run.as<int>();
    SlotScal    *S = B.scal.as<SlotScal>();
    MRed        *R = B.red.as<MRed>();
    const int    gv = grid_for(B.npix * 3 * G, 256, ctx->sm_count * 8);
    mr_direction_kernel<G><<<gv, 256, 0, st>>>(B.H.as<double>(), B.H32.as<float>(), B.CG.as<double>(), B.npix, run, S);
    MDP_CHECK_LAUNCH(ctx);
    MDP_TRY(launch_apply32<G>(ctx, A, N, B, B.H32.as<float>()));
    mr_coeff_kernel<G><<<MR_BLOCKS, MR_THREADS, 0, st>>>(B.H.as<double>(), B.Q.as<double>(), B.npix, run, S, R);
    MDP_CHECK_LAUNCH(ctx);
    mr_update_kernel<G><<<MR_BLOCKS, MR_THREADS, 0, st>>>(inv, B.DL.as<double>(), B.H.as<double>(), B.Q.as<double>(),
                                                          gp, g, B.CG.as<double>(), B.npix, run, S, R);
    MDP_CHECK_LAUNCH(ctx);
    if (h_scal) MDP_CUDA(cudaMemcpyAsync(h_scal, S, sizeof(SlotScal) * G, cudaMemcpyDeviceToHost, st));
    return MDP_OK;
}

// K batched iterations (K even: the gradient buffers end where they started);
// the slot scalars reach the host after the last
constexpr int MR_K = 4;
template <int G>
int launch_iterations(mdp_context *ctx, mdp_pointing *A, mdp_noise *N, Batch &B, const double *inv,
                      double *const bufs[2], SlotScal *h_scal) {
    for (int k = 0; k < MR_K; k++)
        MDP_TRY(launch_iteration<G>(ctx, A, N, B, inv, bufs[(k & 1) ^ 1], bufs[k & 1], k == MR_K - 1 ? h_scal : nullptr));
    return MDP_OK;
}

int alloc_batch(mdp_context *ctx, mdp_pointing *A, mdp_noise *N, int G, int64_t npix, Batch &B) {
    B.G = G;
    B.m = A->m;
    B.npix = npix;
    B.nmap = 3 * npix;
    int covers = 0;
    MDP_TRY(mdp_noise_chunks(N, &B.n_chunks, &B.chunk_start, &B.chunk_len, &B.blk_chunk0, &B.blk_nchunk, &covers));
    const size_t nv = sizeof(double) * (size_t) std::max<int64_t>(npix, 1) * 3 * G;
    for (DevBuf *b : {&B.H, &B.Q, &B.G1, &B.G2, &B.CG, &B.DL}) MDP_TRY(b->alloc(nv));
    for (DevBuf *b : {&B.H, &B.Q, &B.G1, &B.G2, &B.CG, &B.DL}) MDP_CUDA(cudaMemsetAsync(b->p, 0, nv, ctx->stream));
    MDP_TRY(B.H32.alloc(nv / 2));
    MDP_CUDA(cudaMemsetAsync(B.H32.p, 0, nv / 2, ctx->stream));
    MDP_TRY(B.Y.alloc(sizeof(float) * (size_t) A->m * G));
    MDP_TRY(B.Z.alloc(sizeof(float) * (size_t) A->m * G));
    MDP_TRY(B.partial.alloc(sizeof(double) * (size_t) std::max(B.n_chunks, 1) * G));
    MDP_TRY(B.means.alloc(sizeof(double) * (size_t) N->nb * G));
    MDP_TRY(B.run.alloc(sizeof(int) * G));
    MDP_TRY(B.scal.alloc(sizeof(SlotScal) * (G + 1)));  // entry G: refinement dot products
    MDP_TRY(B.red.alloc(sizeof(MRed)));
    MDP_CUDA(cudaMemsetAsync(B.run.p, 0, sizeof(int) * G, ctx->stream));
    MDP_CUDA(cudaMemsetAsync(B.scal.p, 0, sizeof(SlotScal) * (G + 1), ctx->stream));
    MDP_CUDA(cudaMemsetAsync(B.red.p, 0, sizeof(MRed), ctx->stream));
    if (!A->mbins.valid || A->mbins.bin_pix != MR_BIN_PIX / G)
        MDP_TRY(mdp_build_bins(ctx, A, MR_BIN_PIX / G, &A->mbins));
    return MDP_OK;
}

template <int G>
int time_apply(mdp_context *ctx, mdp_pointing *A, mdp_noise *N, int64_t npix, float *ms_per_column) {
    Batch B;
    MDP_TRY(alloc_batch(ctx, A, N, G, npix, B));
    std::vector<int> ones(G, 1);
    MDP_CUDA(cudaMemcpyAsync(B.run.p, ones.data(), sizeof(int) * G, cudaMemcpyHostToDevice, ctx->stream));
    MDP_TRY(launch_apply32<G>(ctx, A, N, B, B.H32.as<float>()));  // warm-up
    cudaEvent_t e0, e1;
    MDP_CUDA(cudaEventCreate(&e0));
    MDP_CUDA(cudaEventCreate(&e1));
    cudaEventRecord(e0, ctx->stream);
    int rc = MDP_OK;
    for (int r = 0; r < 2 && rc == MDP_OK; r++) rc = launch_apply32<G>(ctx, A, N, B, B.H32.as<float>());
    cudaEventRecord(e1, ctx->stream);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    MDP_TRY(rc);
    *ms_per_column = ms / (2.0f * G);
    return MDP_OK;
}

template <int G>
int run_multi(mdp_context *ctx, mdp_pointing *A, mdp_noise *N, const BJState &bj, int nrhs, const void *d_noise,
              int noise_fp32, int64_t noise_stride, const double *d_signal, int signal_col,
              const mdp_multi_params *prm, double *d_x, mdp_multi_col_info *ci, mdp_multi_info *info) {
    cudaStream_t  st = ctx->stream;
    const int64_t m = A->m, npix = bj.npix, nmap = A->n_map();
    const double *inv = bj.inv.as<double>();
    Batch         B;
    MDP_TRY(alloc_batch(ctx, A, N, G, npix, B));
    DevBuf ta, tb, rv;
    MDP_TRY(ta.alloc(sizeof(double) * m));
    MDP_TRY(tb.alloc(sizeof(double) * m));
    MDP_TRY(rv.alloc(sizeof(double) * std::max<int64_t>(nmap, 1)));
    SlotScal *S = B.scal.as<SlotScal>();
    MRed     *R = B.red.as<MRed>();
    // pinned slot scalars: the ctx pinned block holds at least 4 KiB
    SlotScal *hs = reinterpret_cast<SlotScal *>(ctx->h_pinned);
    static_assert(sizeof(SlotScal) * (MR_MAXG + 1) <= 4096, "slot scalars exceed the pinned block");
    const int gm = grid_for(m, 256, ctx->sm_count * 16);
    const int gn = grid_for(nmap, 256, ctx->sm_count * 8);
    MDP_CUDA(cudaMemsetAsync(d_x, 0, sizeof(double) * (size_t) nmap * nrhs, st));
    int fp64_apps = 0;

    // r = P^T N^-1 (d'_col - P x_col) into rv, returns (r, r) in *res
    auto residual = [&](int col, bool x_zero, double *res) -> int {
        double *x = d_x + (size_t) col * nmap;
        if (x_zero) MDP_CUDA(cudaMemsetAsync(ta.p, 0, sizeof(double) * m, st));
        else MDP_TRY(mdp_matvec_launch(ctx, A, x, ta.as<double>()));
        const double *sig = (col == signal_col) ? d_signal : nullptr;
        if (noise_fp32)
            mr_tod_residual_kernel<float><<<gm, 256, 0, st>>>(
                    A->off.as<int32_t>(), sig, static_cast<const float *>(d_noise) + (size_t) col * noise_stride,
                    ta.as<double>(), m);
        else
            mr_tod_residual_kernel<double><<<gm, 256, 0, st>>>(
                    A->off.as<int32_t>(), sig, static_cast<const double *>(d_noise) + (size_t) col * noise_stride,
                    ta.as<double>(), m);
        MDP_CHECK_LAUNCH(ctx);
        MDP_TRY(mdp_stbmm_impl(ctx, N, ta.as<double>(), tb.as<double>(), nullptr));
        MDP_TRY(mdp_trmatvec_launch(ctx, A, tb.as<double>(), rv.as<double>()));
        mr_dot_kernel<<<MR_BLOCKS, MR_THREADS, 0, st>>>(rv.as<double>(), nmap, G, S, R);
        MDP_CHECK_LAUNCH(ctx);
        MDP_CUDA(cudaMemcpyAsync(hs + G, S + G, sizeof(SlotScal), cudaMemcpyDeviceToHost, st));
        MDP_CUDA(cudaStreamSynchronize(st));
        *res = hs[G].dot;
        fp64_apps++;
        if (!std::isfinite(*res)) {
            mdp_set_error("mdp_gls_solve_multi: residual of column %d became %f", col, *res);
            return MDP_ENAN;
        }
        return MDP_OK;
    };

    std::vector<double> tol2rel(nrhs, 0.0);
    std::vector<int>    slot_col(G, -1), seen_it(G, 0);
    // gradient buffers: an iteration reads the current gradient bufs[k & 1] (as
    // gp) and writes the new one into bufs[(k & 1) ^ 1]; a batch of MR_K (even)
    // iterations leaves the current gradients in bufs[0], where slots start
    double *const       bufs[2] = {B.G1.as<double>(), B.G2.as<double>()};
    const double        itol2 = prm->inner_tol * prm->inner_tol;
    int                 next = 0, batched = 0;
    for (int c = 0; c < nrhs; c++) ci[c] = mdp_multi_col_info{0, 0, 0, 0.0, 0.0};
    auto budget = [&](int col) { return std::max(1, std::min(prm->inner_maxiter, prm->maxiter - ci[col].iterations)); };

    // load the next unconverged column into slot j (or leave it idle)
    auto load = [&](int j) -> int {
        while (next < nrhs) {
            const int col = next++;
            double    res0 = 0.0;
            MDP_TRY(residual(col, true, &res0));
            ci[col].res0 = res0;
            ci[col].res = res0;
            tol2rel[col] = prm->tol * prm->tol * res0;
            if (res0 <= prm->tol) {  // the reference's initial test (pcg_true.c:113-118)
                ci[col].converged = 1;
                continue;
            }
            slot_col[j] = col;
            seen_it[j] = 0;
            mr_slot_init_kernel<G><<<MR_BLOCKS, MR_THREADS, 0, st>>>(inv, rv.as<double>(), j, bufs[0],
                                                                     B.CG.as<double>(), B.H.as<double>(),
                                                                     B.DL.as<double>(), npix, itol2, budget(col),
                                                                     B.run.as<int>(), S, R);
            MDP_CHECK_LAUNCH(ctx);
            return MDP_OK;
        }
        slot_col[j] = -1;
        MDP_CUDA(cudaMemsetAsync(B.run.as<int>() + j, 0, sizeof(int), st));
        return MDP_OK;
    };
    for (int j = 0; j < G; j++) MDP_TRY(load(j));

    // MR_K batched iterations as one CUDA graph: the inner stop test and the
    // stop of a slot run on the device, the host waits once per MR_K iterations
    cudaGraphExec_t gx = nullptr;
    bool            graphs = prm->use_graph != 0;
    uint64_t        graph_launches = 0;  // kernels in one replay
    if (graphs) {
        // captured on a private stream (the context stream may be the legacy
        // default stream, which cannot be captured); replayed on the context stream
        cudaStream_t cap = nullptr;
        if (cudaStreamSynchronize(st) != cudaSuccess || cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking) != cudaSuccess) {
            cudaGetLastError();
            graphs = false;
        }
        if (graphs) {
            cudaGraph_t graph = nullptr;
            if (cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
                if (prm->verbose) printf("graph capture unavailable: %s\n", cudaGetErrorString(cudaGetLastError()));
                cudaGetLastError();
                graphs = false;
            } else {
                const uint64_t l0 = ctx->launches;
                ctx->stream = cap;
                int         rc = launch_iterations<G>(ctx, A, N, B, inv, bufs, hs);
                cudaError_t e = cudaStreamEndCapture(cap, &graph);
                ctx->stream = st;
                graph_launches = ctx->launches - l0;
                ctx->launches = l0;
                cudaError_t ei = (rc == MDP_OK && e == cudaSuccess && graph) ? cudaGraphInstantiate(&gx, graph, 0)
                                                                             : cudaErrorUnknown;
                if (ei != cudaSuccess) {
                    if (prm->verbose)
                        printf("graph capture failed (rc %d): %s / %s\n", rc, cudaGetErrorString(e), cudaGetErrorString(ei));
                    cudaGetLastError();
                    graphs = false;
                    gx = nullptr;
                }
                if (graph) cudaGraphDestroy(graph);
            }
        }
        if (cap) cudaStreamDestroy(cap);
    }
    auto cleanup = [&]() {
        if (gx) cudaGraphExecDestroy(gx);
    };

    int rc = MDP_OK;
    while (rc == MDP_OK) {
        bool any = false;
        for (int j = 0; j < G; j++) any = any || slot_col[j] >= 0;
        if (!any) break;
        if (graphs) {
            if (cudaGraphLaunch(gx, st) != cudaSuccess) {
                mdp_set_error("mdp_gls_solve_multi: graph launch: %s", cudaGetErrorString(cudaGetLastError()));
                rc = MDP_ECUDA;
                break;
            }
            ctx->launches += graph_launches;
        } else if ((rc = launch_iterations<G>(ctx, A, N, B, inv, bufs, hs))) {
            break;
        }
        if (cudaStreamSynchronize(st) != cudaSuccess) {
            mdp_set_error("mdp_gls_solve_multi: %s", cudaGetErrorString(cudaGetLastError()));
            rc = MDP_ECUDA;
            break;
        }
        batched += MR_K;
        for (int j = 0; j < G && rc == MDP_OK; j++) {
            const int col = slot_col[j];
            if (col < 0) continue;
            ci[col].iterations += hs[j].inner_it - seen_it[j];
            seen_it[j] = hs[j].inner_it;
            if (!std::isfinite(hs[j].res)) {
                mdp_set_error("mdp_gls_solve_multi: inner residual of column %d became %f", col, hs[j].res);
                rc = MDP_ENAN;
                break;
            }
            if (!hs[j].stopped) continue;
            // refinement step of this column
            mr_extract_add_kernel<G><<<gn, 256, 0, st>>>(B.DL.as<double>(), j, d_x + (size_t) col * nmap, npix);
            MDP_CHECK_LAUNCH(ctx);
            double res = 0.0;
            if ((rc = residual(col, false, &res))) break;
            ci[col].outer_iterations++;
            ci[col].res = res;
            if (prm->verbose)
                printf("column %d: refinement %d after %d inner iterations, res_rel = %e\n", col,
                       ci[col].outer_iterations, ci[col].iterations, std::sqrt(res / ci[col].res0));
            if (res <= tol2rel[col] || ci[col].iterations >= prm->maxiter) {
                ci[col].converged = res <= tol2rel[col];
                if ((rc = load(j))) break;
            } else {
                seen_it[j] = 0;
                // inner target of this refinement: inner_tol, or the reduction
                // still needed (factor 2 margin) when that is smaller
                const double need = 0.5 * prm->tol / std::sqrt(res / ci[col].res0);
                const double it = std::max(prm->inner_tol, std::min(need, 0.5));
                mr_slot_init_kernel<G><<<MR_BLOCKS, MR_THREADS, 0, st>>>(inv, rv.as<double>(), j, bufs[0],
                                                                         B.CG.as<double>(), B.H.as<double>(),
                                                                         B.DL.as<double>(), npix, it * it, budget(col),
                                                                         B.run.as<int>(), S, R);
                MDP_CHECK_LAUNCH(ctx);
            }
        }
    }
    cleanup();
    if (rc != MDP_OK) return rc;
    if (info) {
        info->batched_iterations = batched;
        info->fp64_applications = fp64_apps;
        info->graph = graphs ? 1 : 0;
    }
    return MDP_OK;
}

}  // namespace

extern "C" int mdp_gls_solve_multi(mdp_context *ctx, mdp_pointing *A, const mdp_noise *Nc, int nrhs,
                                   const void *d_noise, int noise_fp32, int64_t noise_stride, const double *d_signal,
                                   int signal_col, const mdp_multi_params *params, double *d_x, int32_t *d_lstid,
                                   double *d_cond, int32_t *d_hits, mdp_multi_col_info *col_info,
                                   mdp_multi_info *info) {
    if (!ctx || !A || !Nc || nrhs < 1 || !d_noise || noise_stride < A->m || !params || !d_x || !col_info ||
        params->tol <= 0.0 || params->inner_tol <= 0.0 || params->inner_maxiter < 1 || params->maxiter < 1 ||
        (signal_col >= 0 && !d_signal) || signal_col >= nrhs) {
        mdp_set_error("mdp_gls_solve_multi: invalid arguments");
        return MDP_EINVAL;
    }
    int slots = params->slots;
    if (slots != 0 && slots != 1 && slots != 2 && slots != 4 && slots != 8) {
        mdp_set_error("mdp_gls_solve_multi: slots must be 0 (timed), 1, 2, 4 or 8");
        return MDP_EINVAL;
    }
    mdp_noise *N = const_cast<mdp_noise *>(Nc);  // the FP32 plan is a cache of the operator
    if (N->nrow_end != A->m || N->lambda == 1) {
        mdp_set_error("mdp_gls_solve_multi: the noise blocks must cover every pointing row and lambda > 1");
        return MDP_EUNSUPPORTED;
    }
    {
        int            nc = 0, covers = 0;
        const int64_t *a;
        const int32_t *b, *c, *d;
        MDP_TRY(mdp_noise_chunks(N, &nc, &a, &b, &c, &d, &covers));
        if (!covers) {
            mdp_set_error("mdp_gls_solve_multi: the noise blocks must cover every pointing row");
            return MDP_EUNSUPPORTED;
        }
    }
    MDP_CUDA(cudaSetDevice(ctx->device));
    auto    tp0 = std::chrono::steady_clock::now();
    const BJState *bjp = nullptr;
    MDP_TRY(mdp_bj_cached(ctx, A, N, &bjp));
    const BJState &bj = *bjp;
    cudaStream_t st = ctx->stream;
    if (d_lstid)
        MDP_CUDA(cudaMemcpyAsync(d_lstid, A->lindices.as<int32_t>() + 3 * A->trash_pix, 4 * A->n_map(),
                                 cudaMemcpyDeviceToDevice, st));
    if (d_cond) MDP_CUDA(cudaMemcpyAsync(d_cond, bj.rcond.p, 8 * bj.npix, cudaMemcpyDeviceToDevice, st));
    if (d_hits) MDP_CUDA(cudaMemcpyAsync(d_hits, bj.hits.p, 4 * bj.npix, cudaMemcpyDeviceToDevice, st));
    MDP_TRY(mdp_pointing_prepare_fp32(ctx, A));
    MDP_TRY(mdp_noise_prepare_fp32(ctx, N));
    MDP_CUDA(cudaStreamSynchronize(st));
    if (slots == 0) {
        // time one batched operator application per slot count; keep the
        // cheapest per column (no more slots than columns)
        float best = 1e30f;
        for (int G : {1, 2, 4, 8}) {
            if (G > 1 && G > nrhs) break;
            float ms = 0.f;
            switch (G) {
                case 1: MDP_TRY(time_apply<1>(ctx, A, N, bj.npix, &ms)); break;
                case 2: MDP_TRY(time_apply<2>(ctx, A, N, bj.npix, &ms)); break;
                case 4: MDP_TRY(time_apply<4>(ctx, A, N, bj.npix, &ms)); break;
                case 8: MDP_TRY(time_apply<8>(ctx, A, N, bj.npix, &ms)); break;
            }
            if (ms < best * 0.97f) {
                best = ms;
                slots = G;
            }
        }
    }
    auto tp1 = std::chrono::steady_clock::now();
    mdp_multi_info local{};
    int            rc;
    switch (slots) {
        case 1: rc = run_multi<1>(ctx, A, N, bj, nrhs, d_noise, noise_fp32, noise_stride, d_signal, signal_col, params, d_x, col_info, &local); break;
        case 2: rc = run_multi<2>(ctx, A, N, bj, nrhs, d_noise, noise_fp32, noise_stride, d_signal, signal_col, params, d_x, col_info, &local); break;
        case 4: rc = run_multi<4>(ctx, A, N, bj, nrhs, d_noise, noise_fp32, noise_stride, d_signal, signal_col, params, d_x, col_info, &local); break;
        default: rc = run_multi<8>(ctx, A, N, bj, nrhs, d_noise, noise_fp32, noise_stride, d_signal, signal_col, params, d_x, col_info, &local); break;
    }
    MDP_TRY(rc);
    MDP_CUDA(cudaStreamSynchronize(st));
    auto tp2 = std::chrono::steady_clock::now();
    if (info) {
        *info = local;
        info->slots = slots;
        info->n_map = A->n_map();
        info->n_cut = bj.ncut;
        info->precond_seconds = std::chrono::duration<double>(tp1 - tp0).count();
        info->solve_seconds = std::chrono::duration<double>(tp2 - tp1).count();
        int tot = 0;
        for (int c = 0; c < nrhs; c++) tot += col_info[c].iterations;
        info->total_iterations = tot;
    }
    return MDP_OK;
}
