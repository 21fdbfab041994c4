// First rows of the inverse-noise Toeplitz blocks from noise timestreams, on the device.
//
// Restates MAPPRAISER's input-side step compute_invtt / noise2invtt
// (mappraiser/python/TOAST_interface/utils.py:439-481 and 500-602) for a batch of
// stationary intervals at once:
//
//   1. periodogram: scipy.signal.welch(x, fs, window='hann', nperseg=n,
//      detrend='linear') of a block of n samples is ONE segment: remove the
//      least-squares line, multiply by the periodic Hann window, |rfft|^2,
//      one-sided density scaling 1/(fs * sum w^2), doubled except DC and (even n)
//      Nyquist (utils.py:531);
//   2. fit of  a + log10(1 + ((f + fmin)/fknee)^alpha)  to log10(psd[1:]) under the
//      bounds [-20,0] x [-10,0] x [0,20] x [0,1] from (-7, -1, 0.1, 1e-6)
//      (utils.py:534-541): a bounded Levenberg-Marquardt run to the minimum, whose
//      sums over the frequencies are device reductions and whose 4x4 step is solved
//      on the host;
//   3. inverse PSD  10^-a / (1 + ((f + fmin)/fknee)^alpha)  on the block's rfft grid,
//      irfft, times the apodisation window of 2*lambda points after ifftshift, first
//      lambda taps (utils.py:557-584).
//
// Transforms are FP64 complex FFTs of length L = 2^p in shared memory: one pass
// for L <= 4096, else the four-step split L = n1 * n2 (columns of n1 points with a
// twiddle, then rows of n2 points).  The forward transform leaves X[k1 + n1 k2] at
// position n2 k1 + k2 ("split order", FftShape::pos); the inverse reads split order
// and writes natural order, so neither needs a transpose.  Block lengths that are
// not powers of two go through Bluestein's chirp-z convolution of length
// L >= 2n - 1.  Twiddles and chirps take their angles from exact integer
// products reduced modulo the period.
#include "mdp_internal.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace {

constexpr int kTileLog = 12;            // 4096 complex doubles per shared-memory transform
constexpr int kMaxLogL = 24;            // longest transform: 2^12 x 2^12
constexpr int kFftThreads = 512;
constexpr int kFitThreads = 256;
constexpr int kSums = 15;               // J^T J (10), J^T r (4), r^T r (1)
constexpr int kSumThreads = 256;
constexpr int64_t kBatchPoints = int64_t(1) << 27;   // complex points per batch (2 GiB)
constexpr int kMaxEvals = 1000;          // curve_fit's maxfev
constexpr double kLn10 = 2.302585092994045684;
constexpr double kLo[4] = {-20.0, -10.0, 1e-30, 0.0};   // fknee kept > 0: the model divides by it
constexpr double kHi[4] = {0.0, 0.0, 20.0, 1.0};
constexpr double kP0[4] = {-7.0, -1.0, 0.1, 1e-6};

struct FftShape {
    int     logL = 0, log1 = 0, log2 = 0;   // L = 2^logL = 2^log1 * 2^log2; log1 == 0: single pass
    int64_t L = 0;
    __host__ __device__ int64_t pos(int64_t k) const {
        if (log1 == 0) return k;
        return ((k & ((int64_t(1) << log1) - 1)) << log2) | (k >> log1);
    }
};

__host__ __device__ inline double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// exp(sign * i * pi * num / den) for an integer 0 <= num < 2*den
__device__ inline double2 expi_pi(int64_t num, int64_t den, int sign) {
    double s, c;
    sincospi((double) num / (double) den, &s, &c);
    return make_double2(c, sign * s);
}

// chirp exp(sign * i * pi * m^2 / n), m^2 reduced modulo 2n first
__device__ inline double2 chirp(int64_t m, int64_t n, int sign) {
    const int64_t r = (int64_t) (((unsigned long long) m * (unsigned long long) m) % (unsigned long long) (2 * n));
    return expi_pi(r, n, sign);
}

// tw[q] = exp(sign * 2 pi i q / m), q < m/2
__device__ void fill_twiddles(double2 *tw, int logm, int sign) {
    const int m = 1 << logm;
    for (int q = threadIdx.x; q < (m >> 1); q += blockDim.x) tw[q] = expi_pi(2 * q, m, sign);
}

// In-place radix-2 decimation in time over `cnt` sequences of m = 2^logm points,
// stored one after the other in s in bit-reversed order; natural order out.
__device__ void smem_fft(double2 *s, const double2 *tw, int logm, int cnt) {
    const int half_m = 1 << (logm - 1);
    const int nbf = half_m * cnt;
    for (int st = 0; st < logm; ++st) {
        const int half = 1 << st;
        for (int t = threadIdx.x; t < nbf; t += blockDim.x) {
            const int seq = t >> (logm - 1);
            const int b = t & (half_m - 1);
            const int p = b & (half - 1);
            const int i = (seq << logm) + ((b >> st) << (st + 1)) + p;
            const int j = i + half;
            const double2 w = tw[p << (logm - 1 - st)];
            const double2 u = s[i];
            const double2 v = cmul(s[j], w);
            s[i] = make_double2(u.x + v.x, u.y + v.y);
            s[j] = make_double2(u.x - v.x, u.y - v.y);
        }
        __syncthreads();
    }
}

__device__ inline int bitrev(int i, int logm) { return (int) (__brev((unsigned) i) >> (32 - logm)); }

// One CTA per row of n2 = 2^log2 contiguous points (grid.x = n1 rows, grid.y = sequences):
// transform with `sign`, then optionally multiply point j of row k1 by
// exp(sign 2 pi i j k1 / L).
__global__ void __launch_bounds__(kFftThreads) fft_rows_kernel(double2 *buf, FftShape sh, int sign,
                                                               int post_twiddle) {
    extern __shared__ double2 sm[];
    const int n2 = 1 << sh.log2;
    double2 *s = sm;
    double2 *tw = sm + n2;
    const int64_t row = blockIdx.x;
    double2 *p = buf + (int64_t) blockIdx.y * sh.L + (row << sh.log2);
    fill_twiddles(tw, sh.log2, sign);
    for (int j = threadIdx.x; j < n2; j += blockDim.x) s[bitrev(j, sh.log2)] = p[j];
    __syncthreads();
    smem_fft(s, tw, sh.log2, 1);
    for (int j = threadIdx.x; j < n2; j += blockDim.x) {
        double2 v = s[j];
        if (post_twiddle) v = cmul(v, expi_pi(2 * (int64_t) j * row, sh.L, sign));   // j * row < L
        p[j] = v;
    }
}

// One CTA per 2^logc adjacent columns of the n1 x n2 row-major array (a column is n1 =
// 2^log1 points with stride n2): transform with `sign`, then optionally multiply point k1
// of column j2 by exp(sign 2 pi i j2 k1 / L).
__global__ void __launch_bounds__(kFftThreads) fft_cols_kernel(double2 *buf, FftShape sh, int logc, int sign,
                                                               int post_twiddle) {
    extern __shared__ double2 sm[];
    const int n1 = 1 << sh.log1;
    const int C = 1 << logc;
    double2 *s = sm;
    double2 *tw = sm + (n1 << logc);
    const int64_t col0 = (int64_t) blockIdx.x << logc;
    double2 *p = buf + (int64_t) blockIdx.y * sh.L;
    fill_twiddles(tw, sh.log1, sign);
    for (int t = threadIdx.x; t < (n1 << logc); t += blockDim.x) {
        const int c = t & (C - 1), i = t >> logc;
        s[(c << sh.log1) + bitrev(i, sh.log1)] = p[((int64_t) i << sh.log2) + col0 + c];
    }
    __syncthreads();
    smem_fft(s, tw, sh.log1, C);
    for (int t = threadIdx.x; t < (n1 << logc); t += blockDim.x) {
        const int c = t & (C - 1), k1 = t >> logc;
        double2 v = s[(c << sh.log1) + k1];
        if (post_twiddle) v = cmul(v, expi_pi(2 * (col0 + c) * k1, sh.L, sign));   // j2 * k1 < L
        p[((int64_t) k1 << sh.log2) + col0 + c] = v;
    }
}

size_t rows_smem(const FftShape &sh) { return (size_t) 3 * ((size_t) 1 << sh.log2) / 2 * sizeof(double2); }
int cols_logc(const FftShape &sh) { return std::min(sh.log2, kTileLog - sh.log1); }
size_t cols_smem(const FftShape &sh) {
    return (((size_t) 1 << (sh.log1 + cols_logc(sh))) + ((size_t) 1 << (sh.log1 - 1))) * sizeof(double2);
}

int set_fft_smem() {
    // the largest request of either kernel: 4096 points + 2048 twiddles
    const int bytes = (int) ((4096 + 2048) * sizeof(double2));
    MDP_CUDA(cudaFuncSetAttribute(fft_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    MDP_CUDA(cudaFuncSetAttribute(fft_cols_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    return MDP_OK;
}

// natural order in, split order out, unscaled exp(-2 pi i jk/L)
int fft_forward(mdp_context *ctx, double2 *buf, const FftShape &sh, int cnt) {
    if (sh.log1 > 0) {
        const int logc = cols_logc(sh);
        fft_cols_kernel<<<dim3((unsigned) (1u << (sh.log2 - logc)), cnt), kFftThreads, cols_smem(sh), ctx->stream>>>(
            buf, sh, logc, -1, 1);
        MDP_CHECK_LAUNCH(ctx);
    }
    fft_rows_kernel<<<dim3((unsigned) (1u << sh.log1), cnt), kFftThreads, rows_smem(sh), ctx->stream>>>(buf, sh, -1, 0);
    MDP_CHECK_LAUNCH(ctx);
    return MDP_OK;
}

// split order in, natural order out, unscaled exp(+2 pi i jk/L)
int fft_inverse(mdp_context *ctx, double2 *buf, const FftShape &sh, int cnt) {
    fft_rows_kernel<<<dim3((unsigned) (1u << sh.log1), cnt), kFftThreads, rows_smem(sh), ctx->stream>>>(
        buf, sh, +1, sh.log1 > 0 ? 1 : 0);
    MDP_CHECK_LAUNCH(ctx);
    if (sh.log1 > 0) {
        const int logc = cols_logc(sh);
        fft_cols_kernel<<<dim3((unsigned) (1u << (sh.log2 - logc)), cnt), kFftThreads, cols_smem(sh), ctx->stream>>>(
            buf, sh, logc, +1, 0);
        MDP_CHECK_LAUNCH(ctx);
    }
    return MDP_OK;
}

// ------------------------------------------------------------------ periodogram
// Per-chunk sums of x and (t - (n-1)/2) x over each block (grid.x chunks, grid.y blocks).
__global__ void detrend_partial_kernel(const double *noise, const int64_t *off, int64_t n, double *part) {
    __shared__ double red[2][kFitThreads];
    const int b = blockIdx.y;
    const double *x = noise + off[b];
    const double c = 0.5 * (double) (n - 1);
    double s0 = 0.0, s1 = 0.0;
    for (int64_t t = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t) gridDim.x * blockDim.x) {
        const double v = x[t];
        s0 += v;
        s1 += ((double) t - c) * v;
    }
    red[0][threadIdx.x] = s0;
    red[1][threadIdx.x] = s1;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) {
            red[0][threadIdx.x] += red[0][threadIdx.x + h];
            red[1][threadIdx.x] += red[1][threadIdx.x + h];
        }
        __syncthreads();
    }
    if (threadIdx.x < 2) part[((int64_t) b * gridDim.x + blockIdx.x) * 2 + threadIdx.x] = red[threadIdx.x][0];
}

// out[b][s] = sum over chunks of part[b][chunk][s], chunks in order
__global__ void sum_chunks_kernel(const double *part, int cnt, int chunks, int nsum, double *out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= cnt * nsum) return;
    const int b = t / nsum, s = t % nsum;
    const double *p = part + (int64_t) b * chunks * nsum + s;
    double acc = 0.0;
    for (int c = 0; c < chunks; ++c) acc += p[(int64_t) c * nsum];
    out[t] = acc;
}

// buf[b][j] = (x_j - mean - slope (j - (n-1)/2)) * hann_j for j < n, 0 beyond; times the
// chirp exp(-i pi j^2/n) when the block goes through Bluestein.
__global__ void window_load_kernel(const double *noise, const int64_t *off, int64_t n, int64_t L, int blue,
                                   const double *sums, double inv_n, double inv_stt, double2 *buf) {
    const int b = blockIdx.y;
    const double *x = noise + off[b];
    const double mean = sums[2 * b] * inv_n;
    const double slope = sums[2 * b + 1] * inv_stt;
    const double c = 0.5 * (double) (n - 1);
    double2 *o = buf + (int64_t) b * L;
    for (int64_t j = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; j < L; j += (int64_t) gridDim.x * blockDim.x) {
        double2 v = make_double2(0.0, 0.0);
        if (j < n) {
            const double w = 0.5 - 0.5 * cospi((double) (2 * j) / (double) n);
            v.x = (x[j] - mean - slope * ((double) j - c)) * w;
            if (blue) {
                const double2 ch = chirp(j, n, -1);
                v = make_double2(v.x * ch.x, v.x * ch.y);
            }
        }
        o[j] = v;
    }
}

// Bluestein filter b_m = exp(-sign i pi m^2/n) for |m| < n (m < 0 stored at L + m), zero elsewhere
__global__ void chirp_filter_kernel(double2 *bh, int64_t n, int64_t L, int sign) {
    for (int64_t m = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; m < L; m += (int64_t) gridDim.x * blockDim.x) {
        const int64_t mm = m < n ? m : (m > L - n ? L - m : -1);
        bh[m] = mm >= 0 ? chirp(mm, n, -sign) : make_double2(0.0, 0.0);
    }
}

__global__ void cmul_batch_kernel(double2 *buf, const double2 *bh, int64_t L) {
    double2 *o = buf + (int64_t) blockIdx.y * L;
    for (int64_t j = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; j < L; j += (int64_t) gridDim.x * blockDim.x)
        o[j] = cmul(o[j], bh[j]);
}

// psd[k] for k = 0..n/2 (one-sided density); y[k-1] = log10(psd[k]) for k >= 1.
// Non-power-of-two blocks read the Bluestein convolution in natural order (|chirp| = 1).
__global__ void psd_kernel(const double2 *buf, FftShape sh, int blue, int64_t n, double scale, double *y,
                           double *psd, int64_t psd_stride, int *bad) {
    const int b = blockIdx.y;
    const int64_t nf = n / 2;
    const double2 *X = buf + (int64_t) b * sh.L;
    for (int64_t k = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; k <= nf; k += (int64_t) gridDim.x * blockDim.x) {
        const double2 v = X[blue ? k : sh.pos(k)];
        double p = (v.x * v.x + v.y * v.y) * scale;
        if (k > 0 && !((n & 1) == 0 && k == nf)) p *= 2.0;
        if (psd) psd[(int64_t) b * psd_stride + k] = p;
        if (y && k > 0) {
            const double ly = log10(p);
            y[(int64_t) b * nf + k - 1] = ly;
            if (!isfinite(ly)) atomicOr(bad, 1);
        }
    }
}

// ------------------------------------------------------------------ fit
__device__ inline double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Per-chunk sums at params[b] of the model residual r_k = a + log10(1 + u^alpha) - y_k,
// u = (f_k + fmin)/fknee, f_k = k * df (k = 1..nf), and of its Jacobian J_k:
// J^T J (upper triangle, row-major), J^T r, r^T r.
__global__ void __launch_bounds__(kFitThreads) fit_eval_kernel(const double *y, int64_t nf, double df,
                                                               const double *params, const int *active,
                                                               double *part) {
    const int b = blockIdx.y;
    if (!active[b]) return;
    const double a = params[4 * b], al = params[4 * b + 1], fk = params[4 * b + 2], fm = params[4 * b + 3];
    double acc[kSums];
#pragma unroll
    for (int s = 0; s < kSums; ++s) acc[s] = 0.0;
    const double *yb = y + (int64_t) b * nf;
    const double inv_fk = 1.0 / fk;
    // u^alpha as exp(alpha log u), log u being needed for the alpha column anyway: the
    // issue-bound part of the fit (relative change of the residuals ~1e-14)
    for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < nf; i += (int64_t) gridDim.x * blockDim.x) {
        const double f = (double) (i + 1) * df;
        const double fpm = f + fm;
        const double lu = log(fpm / fk);
        const double g = exp(al * lu);
        const double opg = 1.0 + g;
        const double r = a + log10(opg) - yb[i];
        const double q = g / (opg * kLn10);
        const double j1 = q * lu;
        const double j2 = -al * q * inv_fk;
        const double j3 = al * q / fpm;
        acc[0] += 1.0;      acc[1] += j1;       acc[2] += j2;       acc[3] += j3;
        acc[4] += j1 * j1;  acc[5] += j1 * j2;  acc[6] += j1 * j3;
        acc[7] += j2 * j2;  acc[8] += j2 * j3;  acc[9] += j3 * j3;
        acc[10] += r;       acc[11] += j1 * r;  acc[12] += j2 * r;  acc[13] += j3 * r;
        acc[14] += r * r;
    }
    __shared__ double red[kFitThreads / 32][kSums];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int s = 0; s < kSums; ++s) {
        const double v = warp_sum(acc[s]);
        if (lane == 0) red[warp][s] = v;
    }
    __syncthreads();
    if (threadIdx.x < kSums) {
        double v = 0.0;
        for (int w = 0; w < kFitThreads / 32; ++w) v += red[w][threadIdx.x];
        part[((int64_t) b * gridDim.x + blockIdx.x) * kSums + threadIdx.x] = v;
    }
}

// Levenberg-Marquardt state of one block (host).
struct Lm {
    double p[4], F = 0, H[4][4], g[4], D[4], mu = 1e-3, pt[4];
    int evals = 0;
    bool done = false, converged = false;
};

void lm_load(const double *s, double H[4][4], double g[4], double *F) {
    const int up[4][4] = {{0, 1, 2, 3}, {1, 4, 5, 6}, {2, 5, 7, 8}, {3, 6, 8, 9}};
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) H[i][j] = s[up[i][j]];
    for (int i = 0; i < 4; ++i) g[i] = s[10 + i];
    *F = 0.5 * s[14];
}

// Trial point of a damped Gauss-Newton step on the variables that are not held at a bound
// by the gradient; false when no step can be formed (singular system or no change).
bool lm_trial(Lm &s) {
    int fr[4], nf = 0;
    for (int i = 0; i < 4; ++i) {
        const bool held = (s.p[i] <= kLo[i] && s.g[i] > 0) || (s.p[i] >= kHi[i] && s.g[i] < 0);
        if (!held) fr[nf++] = i;
    }
    if (nf == 0) return false;
    double A[4][5];
    for (int r = 0; r < nf; ++r) {
        for (int c = 0; c < nf; ++c) A[r][c] = s.H[fr[r]][fr[c]];
        A[r][r] += s.mu * s.D[fr[r]];
        A[r][nf] = -s.g[fr[r]];
    }
    for (int c = 0; c < nf; ++c) {   // Gaussian elimination, partial pivoting
        int piv = c;
        for (int r = c + 1; r < nf; ++r)
            if (std::fabs(A[r][c]) > std::fabs(A[piv][c])) piv = r;
        if (!(std::fabs(A[piv][c]) > 0.0) || !std::isfinite(A[piv][c])) return false;
        if (piv != c)
            for (int k = 0; k <= nf; ++k) std::swap(A[c][k], A[piv][k]);
        for (int r = c + 1; r < nf; ++r) {
            const double m = A[r][c] / A[c][c];
            for (int k = c; k <= nf; ++k) A[r][k] -= m * A[c][k];
        }
    }
    double d[4] = {0, 0, 0, 0};
    for (int r = nf - 1; r >= 0; --r) {
        double v = A[r][nf];
        for (int k = r + 1; k < nf; ++k) v -= A[r][k] * d[fr[k]];
        d[fr[r]] = v / A[r][r];
    }
    bool moved = false;
    for (int i = 0; i < 4; ++i) {
        double v = s.p[i] + d[i];
        if (!std::isfinite(v)) return false;
        v = std::min(std::max(v, kLo[i]), kHi[i]);
        s.pt[i] = v;
        moved |= (v != s.p[i]);
    }
    return moved;
}

struct Batch {
    int     first = 0, cnt = 0;
    int64_t n = 0;
};

int shape_for(int64_t n, FftShape *sh, int *blue) {
    int64_t L = 1;
    int logL = 0;
    const bool pow2 = (n & (n - 1)) == 0;
    const int64_t need = pow2 ? n : 2 * n - 1;
    while (L < need) {
        L <<= 1;
        ++logL;
    }
    if (logL > kMaxLogL) return MDP_EUNSUPPORTED;
    sh->L = L;
    sh->logL = logL;
    sh->log2 = std::min(logL, kTileLog);
    sh->log1 = logL - sh->log2;
    *blue = pow2 ? 0 : 1;
    return MDP_OK;
}

int chunks_for(int64_t points, int threads, int per_thread, int max_chunks) {
    int64_t c = (points + (int64_t) threads * per_thread - 1) / ((int64_t) threads * per_thread);
    return (int) std::max<int64_t>(1, std::min<int64_t>(c, max_chunks));
}

// Bluestein filters for a length: bh[0] for forward (sign -1), bh[1] for inverse (sign +1),
// each already transformed (split order).
int bluestein_filters(mdp_context *ctx, int64_t n, const FftShape &sh, double2 *bh0, double2 *bh1) {
    const int g = grid_for(sh.L, 256);
    chirp_filter_kernel<<<g, 256, 0, ctx->stream>>>(bh0, n, sh.L, -1);
    MDP_CHECK_LAUNCH(ctx);
    chirp_filter_kernel<<<g, 256, 0, ctx->stream>>>(bh1, n, sh.L, +1);
    MDP_CHECK_LAUNCH(ctx);
    MDP_TRY(fft_forward(ctx, bh0, sh, 1));
    MDP_TRY(fft_forward(ctx, bh1, sh, 1));
    return MDP_OK;
}

// Periodogram of one batch of equal-length blocks into y (log10 psd[1..n/2]) and/or psd.
int periodogram_batch(mdp_context *ctx, const double *d_noise, const int64_t *d_off, int cnt, int64_t n,
                      const FftShape &sh, int blue, const double2 *bh0, double2 *buf, DevBuf &part, DevBuf &sums,
                      double fsamp, double *y, double *psd, int64_t psd_stride, int *d_bad) {
    const int chunks = chunks_for(n, kFitThreads, 16, 256);
    MDP_TRY(part.alloc((size_t) cnt * chunks * kSums * sizeof(double)));
    MDP_TRY(sums.alloc((size_t) cnt * kSums * sizeof(double)));
    detrend_partial_kernel<<<dim3(chunks, cnt), kFitThreads, 0, ctx->stream>>>(d_noise, d_off, n, part.as<double>());
    MDP_CHECK_LAUNCH(ctx);
    sum_chunks_kernel<<<(cnt * 2 + kSumThreads - 1) / kSumThreads, kSumThreads, 0, ctx->stream>>>(
        part.as<double>(), cnt, chunks, 2, sums.as<double>());
    MDP_CHECK_LAUNCH(ctx);
    const double dn = (double) n;
    const double stt = dn * (dn * dn - 1.0) / 12.0;   // sum of (t - (n-1)/2)^2
    const int gl = (int) std::min<int64_t>((sh.L + 255) / 256, 1024);
    window_load_kernel<<<dim3(gl, cnt), 256, 0, ctx->stream>>>(d_noise, d_off, n, sh.L, blue, sums.as<double>(),
                                                                1.0 / dn, 1.0 / stt, buf);
    MDP_CHECK_LAUNCH(ctx);
    MDP_TRY(fft_forward(ctx, buf, sh, cnt));
    // periodic Hann: sum of w^2 = 3n/8 (n >= 3)
    double scale = 1.0 / (fsamp * (3.0 * dn / 8.0));
    if (blue) {
        cmul_batch_kernel<<<dim3(gl, cnt), 256, 0, ctx->stream>>>(buf, bh0, sh.L);
        MDP_CHECK_LAUNCH(ctx);
        MDP_TRY(fft_inverse(ctx, buf, sh, cnt));
        const double il = 1.0 / (double) sh.L;   // exact: L is a power of two
        scale *= il * il;
    }
    const int gp = (int) std::min<int64_t>((n / 2 + 256) / 256, 1024);
    psd_kernel<<<dim3(gp, cnt), 256, 0, ctx->stream>>>(buf, sh, blue, n, scale, y, psd, psd_stride, d_bad);
    MDP_CHECK_LAUNCH(ctx);
    return MDP_OK;
}

// ------------------------------------------------------------------ inverse autocorrelation
// Inverse PSD sig / (1 + ((f_kk + fmin)/fknee)^alpha) at kk = min(k, n-k), k < n (the
// Hermitian extension irfft uses), written in split order; Bluestein blocks get it times
// the chirp exp(+i pi k^2/n) in natural order, zero padded to L.
__global__ void invpsd_kernel(double2 *buf, FftShape sh, int blue, int64_t n, double df, const double *params,
                              const double *sig) {
    const int b = blockIdx.y;
    const double al = params[4 * b + 1], fk = params[4 * b + 2], fm = params[4 * b + 3], sg = sig[b];
    double2 *o = buf + (int64_t) b * sh.L;
    const int64_t lim = blue ? sh.L : n;
    for (int64_t k = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; k < lim; k += (int64_t) gridDim.x * blockDim.x) {
        if (k >= n) {
            o[k] = make_double2(0.0, 0.0);
            continue;
        }
        const int64_t kk = k <= n - k ? k : n - k;
        const double f = (double) kk * df;
        const double S = sg / (1.0 + pow((f + fm) / fk, al));
        if (blue) {
            const double2 ch = chirp(k, n, +1);
            o[k] = make_double2(S * ch.x, S * ch.y);
        } else {
            o[sh.pos(k)] = make_double2(S, 0.0);
        }
    }
}

// invtt[b][j] = window[j] * Re(x_j) / n, j < lambda; x in natural order (Bluestein: the
// convolution / L times the chirp exp(+i pi j^2/n)).
__global__ void invtt_out_kernel(const double2 *buf, int64_t L, int blue, int64_t n, int lam, const double *win,
                                 double *invtt) {
    const int b = blockIdx.y;
    const double2 *x = buf + (int64_t) b * L;
    const double inv_n = 1.0 / (double) n;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < lam; j += gridDim.x * blockDim.x) {
        double re;
        if (blue) {
            const double2 ch = chirp(j, n, +1);
            const double2 c = make_double2(x[j].x / (double) L, x[j].y / (double) L);
            re = c.x * ch.x - c.y * ch.y;
        } else {
            re = x[j].x;
        }
        invtt[(int64_t) b * lam + j] = win[j] * (re * inv_n);
    }
}

// ------------------------------------------------------------------ apodisation windows
// Dolph-Chebyshev window of M = 2 lam + 1 points (scipy.signal.windows.chebwin, odd M):
// p_k = T_{M-1}(x_k), x_k = beta cos(pi k / M), w_n = sum_k p_k cos(2 pi n k / M)
// (p_k = p_{M-k}).  Near x = 1, T_{M-1} amplifies the rounding of x by up to (M-1)^2,
// so x - 1 is formed directly, (beta - 1) - 2 beta sin^2(pi k / 2M) with
// beta - 1 = 2 sinh^2(t/2), and T_{M-1}(x) = cos((M-1) 2 asin(sqrt((1-x)/2))) for
// |x| <= 1, cosh((M-1) 2 asinh(sqrt((x-1)/2))) for x > 1.  (scipy evaluates
// cos((M-1) acos(x)) of a rounded x: its window is off by up to 5e-9 at lam = 2^14;
// this form is exact to about 1e-15.)
__global__ void cheb_p_kernel(double *p, int lam, double beta, double beta_m1) {
    const int64_t M = 2 * (int64_t) lam + 1;
    const double order = (double) (M - 1);
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k <= lam; k += gridDim.x * blockDim.x) {
        const double s = sinpi((double) k / (double) (2 * M));
        const double d = beta_m1 - 2.0 * beta * s * s;   // x - 1
        double v;
        if (d > 0.0) v = cosh(order * 2.0 * asinh(sqrt(0.5 * d)));
        else if (d >= -2.0) v = cos(order * 2.0 * asin(sqrt(-0.5 * d)));
        else v = cosh(order * acosh(-1.0 - d));   // x < -1: not reached for k <= lam, M odd
        p[k] = v;
    }
}

// Chebyshev samples p_{min(j, M-j)} times the chirp exp(-i pi j^2/M) for j < M, zero to L
// (the Bluestein input of the length-M DFT of p)
__global__ void cheb_load_kernel(const double *p, int lam, int64_t L, double2 *buf) {
    const int64_t M = 2 * (int64_t) lam + 1;
    for (int64_t j = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; j < L; j += (int64_t) gridDim.x * blockDim.x) {
        double2 v = make_double2(0.0, 0.0);
        if (j < M) {
            const double pk = p[j <= M - j ? j : M - j];
            const double2 ch = chirp(j, M, -1);
            v = make_double2(pk * ch.x, pk * ch.y);
        }
        buf[j] = v;
    }
}

// w[n] = Re(DFT(p))_n for n <= lam from the Bluestein convolution (natural order, times L)
__global__ void cheb_out_kernel(const double2 *conv, int lam, int64_t L, double *w) {
    const int64_t M = 2 * (int64_t) lam + 1;
    for (int64_t nn = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; nn <= lam;
         nn += (int64_t) gridDim.x * blockDim.x) {
        const double2 c = make_double2(conv[nn].x / (double) L, conv[nn].y / (double) L);
        const double2 ch = chirp(nn, M, -1);
        w[nn] = c.x * ch.x - c.y * ch.y;
    }
}

// window[j] = w[j] / max_{n <= lam} w[n], j < lam (one CTA)
__global__ void cheb_norm_kernel(const double *w, int lam, double *win) {
    __shared__ double red[256];
    double m = -INFINITY;
    for (int i = threadIdx.x; i <= lam; i += blockDim.x) m = fmax(m, w[i]);
    red[threadIdx.x] = m;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + h]);
        __syncthreads();
    }
    const double mx = red[0];
    for (int j = threadIdx.x; j < lam; j += blockDim.x) win[j] = w[j] / mx;
}

// general_gaussian(2 lam, p=1, sig) after ifftshift: exp(-0.5 (j/sig)^2), j < lam
__global__ void gauss_window_kernel(int lam, double sig, double *win) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < lam; j += gridDim.x * blockDim.x) {
        const double v = (double) j / sig;
        win[j] = exp(-0.5 * (v * v));
    }
}

int window_impl(mdp_context *ctx, int lam, int apod, double *d_win) {
    if (apod == MDP_APOD_GAUSSIAN) {
        gauss_window_kernel<<<grid_for(lam, 256), 256, 0, ctx->stream>>>(lam, (1.0 / 3.0) * lam, d_win);
        MDP_CHECK_LAUNCH(ctx);
        return MDP_OK;
    }
    // chebwin: DFT of length M = 2 lam + 1 (odd) through Bluestein
    const int64_t M = 2 * (int64_t) lam + 1;
    FftShape sh;
    int blue;
    if (shape_for(M, &sh, &blue) != MDP_OK) {
        mdp_set_error("chebwin of %lld points needs a transform longer than 2^%d points", (long long) M, kMaxLogL);
        return MDP_EUNSUPPORTED;
    }
    DevBuf pw, cbuf, cbh;
    MDP_TRY(pw.alloc((size_t) 2 * (lam + 1) * sizeof(double)));
    MDP_TRY(cbuf.alloc((size_t) sh.L * sizeof(double2)));
    MDP_TRY(cbh.alloc((size_t) sh.L * sizeof(double2)));
    double *p = pw.as<double>(), *w = p + lam + 1;
    const double order = 2.0 * lam;
    const double t = 1.0 / order * std::acosh(std::pow(10.0, 150.0 / 20.0));
    const double sht = std::sinh(0.5 * t);
    cheb_p_kernel<<<grid_for(lam + 1, 256), 256, 0, ctx->stream>>>(p, lam, std::cosh(t), 2.0 * sht * sht);
    MDP_CHECK_LAUNCH(ctx);
    const int g = grid_for(sh.L, 256);
    chirp_filter_kernel<<<g, 256, 0, ctx->stream>>>(cbh.as<double2>(), M, sh.L, -1);
    MDP_CHECK_LAUNCH(ctx);
    MDP_TRY(fft_forward(ctx, cbh.as<double2>(), sh, 1));
    cheb_load_kernel<<<g, 256, 0, ctx->stream>>>(p, lam, sh.L, cbuf.as<double2>());
    MDP_CHECK_LAUNCH(ctx);
    MDP_TRY(fft_forward(ctx, cbuf.as<double2>(), sh, 1));
    cmul_batch_kernel<<<dim3(g, 1), 256, 0, ctx->stream>>>(cbuf.as<double2>(), cbh.as<double2>(), sh.L);
    MDP_CHECK_LAUNCH(ctx);
    MDP_TRY(fft_inverse(ctx, cbuf.as<double2>(), sh, 1));
    cheb_out_kernel<<<grid_for(lam + 1, 256), 256, 0, ctx->stream>>>(cbuf.as<double2>(), lam, sh.L, w);
    MDP_CHECK_LAUNCH(ctx);
    cheb_norm_kernel<<<1, 256, 0, ctx->stream>>>(w, lam, d_win);
    MDP_CHECK_LAUNCH(ctx);
    // the temporaries are freed on return: finish with them first
    MDP_CUDA(cudaStreamSynchronize(ctx->stream));
    return MDP_OK;
}

// Validates the blocks and groups runs of equal lengths into batches of at most
// kBatchPoints transform points (and 65535 blocks).
int make_batches(int nb, const int32_t *h_n, int64_t min_n, std::vector<Batch> *out, std::vector<int64_t> *offs) {
    out->clear();
    offs->assign(nb, 0);
    int64_t o = 0;
    for (int b = 0; b < nb; ++b) {
        const int64_t n = h_n[b];
        if (n < min_n) {
            mdp_set_error("block %d has %lld samples (at least %lld needed)", b, (long long) n, (long long) min_n);
            return MDP_EINVAL;
        }
        FftShape sh;
        int blue;
        if (shape_for(n, &sh, &blue) != MDP_OK) {
            mdp_set_error("block %d: %lld samples need a transform longer than 2^%d points", b, (long long) n,
                          kMaxLogL);
            return MDP_EUNSUPPORTED;
        }
        (*offs)[b] = o;
        o += n;
        const int64_t cap = std::max<int64_t>(1, std::min<int64_t>(65535, kBatchPoints / sh.L));
        if (!out->empty() && out->back().n == n && out->back().cnt < cap) {
            out->back().cnt++;
        } else {
            Batch bt;
            bt.first = b;
            bt.cnt = 1;
            bt.n = n;
            out->push_back(bt);
        }
    }
    return MDP_OK;
}

double rfft_step(int64_t n, double fsamp) {
    // numpy/scipy rfftfreq(n, d=1/fs): k * (1 / (n * d))
    const double d = 1.0 / fsamp;
    return 1.0 / ((double) n * d);
}

}  // namespace

// ====================================================================== C API
extern "C" int mdp_apod_window(mdp_context *ctx, int lambda, int apod, double *d_window) {
    if (!ctx || !d_window || lambda < 1 || (apod != MDP_APOD_CHEBWIN && apod != MDP_APOD_GAUSSIAN)) {
        mdp_set_error("mdp_apod_window: bad argument");
        return MDP_EINVAL;
    }
    MDP_TRY(set_fft_smem());
    MDP_TRY(window_impl(ctx, lambda, apod, d_window));
    MDP_CUDA(cudaStreamSynchronize(ctx->stream));
    return MDP_OK;
}

extern "C" int mdp_periodogram(mdp_context *ctx, int nb, const int32_t *h_n, const double *d_noise, double fsamp,
                               double *d_psd) {
    if (!ctx || nb < 1 || !h_n || !d_noise || !d_psd || !(fsamp > 0.0) || !std::isfinite(fsamp)) {
        mdp_set_error("mdp_periodogram: bad argument");
        return MDP_EINVAL;
    }
    std::vector<Batch> batches;
    std::vector<int64_t> offs;
    MDP_TRY(make_batches(nb, h_n, 4, &batches, &offs));
    MDP_TRY(set_fft_smem());
    DevBuf buf, bh, part, sums, doff, flag;
    MDP_TRY(flag.alloc(sizeof(int)));
    int64_t psd_at = 0;
    int64_t bh_n = -1;
    for (const Batch &bt : batches) {
        FftShape sh;
        int blue;
        MDP_TRY(shape_for(bt.n, &sh, &blue));
        MDP_TRY(buf.alloc((size_t) bt.cnt * sh.L * sizeof(double2)));
        MDP_TRY(doff.alloc((size_t) bt.cnt * sizeof(int64_t)));
        MDP_CUDA(cudaMemcpyAsync(doff.p, offs.data() + bt.first, bt.cnt * sizeof(int64_t), cudaMemcpyHostToDevice,
                                 ctx->stream));
        if (blue && bh_n != bt.n) {
            MDP_TRY(bh.alloc((size_t) 2 * sh.L * sizeof(double2)));
            MDP_TRY(bluestein_filters(ctx, bt.n, sh, bh.as<double2>(), bh.as<double2>() + sh.L));
            bh_n = bt.n;
        }
        MDP_TRY(periodogram_batch(ctx, d_noise, doff.as<int64_t>(), bt.cnt, bt.n, sh, blue, bh.as<double2>(),
                                  buf.as<double2>(), part, sums, fsamp, nullptr, d_psd + psd_at, bt.n / 2 + 1,
                                  flag.as<int>()));
        psd_at += (int64_t) bt.cnt * (bt.n / 2 + 1);
        // buffers are reused by the next batch: finish this one first
        MDP_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    return MDP_OK;
}

extern "C" int mdp_noise2invtt(mdp_context *ctx, int nb, const int32_t *h_n, const double *d_noise, int lambda,
                               double fsamp, int apod, double *d_invtt, double *h_params, int32_t *h_evals) {
    if (!ctx || nb < 1 || !h_n || !d_noise || !d_invtt || lambda < 1 || !(fsamp > 0.0) || !std::isfinite(fsamp)) {
        mdp_set_error("mdp_noise2invtt: bad argument");
        return MDP_EINVAL;
    }
    if (apod != MDP_APOD_CHEBWIN && apod != MDP_APOD_GAUSSIAN) {
        mdp_set_error("mdp_noise2invtt: apodisation window %d is not supported", apod);
        return MDP_EINVAL;
    }
    for (int b = 0; b < nb; ++b)
        if (lambda > h_n[b] / 2) {
            mdp_set_error("Bandwidth cannot be larger than timestream (block %d: %d samples, lambda %d)", b, h_n[b],
                          lambda);
            return MDP_EINVAL;
        }
    std::vector<Batch> batches;
    std::vector<int64_t> offs;
    MDP_TRY(make_batches(nb, h_n, 8, &batches, &offs));   // >= 4 frequencies for 4 parameters
    MDP_TRY(set_fft_smem());

    DevBuf win, buf, bh, part, sums, doff, y, prm, act, sig, flag;
    MDP_TRY(win.alloc((size_t) lambda * sizeof(double)));
    MDP_TRY(window_impl(ctx, lambda, apod, win.as<double>()));
    MDP_TRY(flag.alloc(sizeof(int)));
    int nonconv = 0;
    int64_t bh_n = -1;
    std::vector<Lm> st;
    std::vector<double> h_prm, h_sums, h_sig;
    std::vector<int> h_act;
    for (const Batch &bt : batches) {
        const int cnt = bt.cnt;
        const int64_t n = bt.n, nf = n / 2;
        FftShape sh;
        int blue;
        MDP_TRY(shape_for(n, &sh, &blue));
        MDP_TRY(buf.alloc((size_t) cnt * sh.L * sizeof(double2)));
        MDP_TRY(y.alloc((size_t) cnt * nf * sizeof(double)));
        MDP_TRY(doff.alloc((size_t) cnt * sizeof(int64_t)));
        MDP_TRY(prm.alloc((size_t) cnt * 4 * sizeof(double)));
        MDP_TRY(act.alloc((size_t) cnt * sizeof(int)));
        MDP_TRY(sig.alloc((size_t) cnt * sizeof(double)));
        MDP_CUDA(cudaMemsetAsync(flag.p, 0, sizeof(int), ctx->stream));
        MDP_CUDA(cudaMemcpyAsync(doff.p, offs.data() + bt.first, cnt * sizeof(int64_t), cudaMemcpyHostToDevice,
                                 ctx->stream));
        if (blue && bh_n != n) {
            MDP_TRY(bh.alloc((size_t) 2 * sh.L * sizeof(double2)));
            MDP_TRY(bluestein_filters(ctx, n, sh, bh.as<double2>(), bh.as<double2>() + sh.L));
            bh_n = n;
        }
        MDP_TRY(periodogram_batch(ctx, d_noise, doff.as<int64_t>(), cnt, n, sh, blue, bh.as<double2>(),
                                  buf.as<double2>(), part, sums, fsamp, y.as<double>(), nullptr, 0, flag.as<int>()));
        int bad = 0;
        MDP_CUDA(cudaMemcpyAsync(&bad, flag.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        MDP_CUDA(cudaStreamSynchronize(ctx->stream));
        if (bad) {
            mdp_set_error("a periodogram of blocks %d..%d has a zero or non-finite value", bt.first,
                          bt.first + cnt - 1);
            return MDP_ENAN;
        }

        // ---- fit: all blocks of the batch iterate together
        const double df = rfft_step(n, fsamp);
        const int chunks = chunks_for(nf, kFitThreads, 16, 256);
        MDP_TRY(part.alloc((size_t) cnt * chunks * kSums * sizeof(double)));
        MDP_TRY(sums.alloc((size_t) cnt * kSums * sizeof(double)));
        st.assign(cnt, Lm());
        h_prm.assign((size_t) cnt * 4, 0.0);
        h_sums.assign((size_t) cnt * kSums, 0.0);
        h_act.assign(cnt, 1);
        for (int b = 0; b < cnt; ++b)
            for (int i = 0; i < 4; ++i) st[b].p[i] = st[b].pt[i] = kP0[i];
        bool first = true;
        for (;;) {
            int nact = 0;
            for (int b = 0; b < cnt; ++b) {
                h_act[b] = 0;
                if (st[b].done) continue;
                if (!first) {
                    // damp until a step can be formed
                    while (!lm_trial(st[b])) {
                        st[b].mu *= 4.0;
                        if (st[b].mu > 1e20) {
                            st[b].done = st[b].converged = true;
                            break;
                        }
                    }
                    if (st[b].done) continue;
                }
                h_act[b] = 1;
                ++nact;
                for (int i = 0; i < 4; ++i) h_prm[4 * b + i] = st[b].pt[i];
            }
            if (nact == 0) break;
            MDP_CUDA(cudaMemcpyAsync(prm.p, h_prm.data(), cnt * 4 * sizeof(double), cudaMemcpyHostToDevice,
                                     ctx->stream));
            MDP_CUDA(cudaMemcpyAsync(act.p, h_act.data(), cnt * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
            fit_eval_kernel<<<dim3(chunks, cnt), kFitThreads, 0, ctx->stream>>>(
                y.as<double>(), nf, df, prm.as<double>(), act.as<int>(), part.as<double>());
            MDP_CHECK_LAUNCH(ctx);
            sum_chunks_kernel<<<(cnt * kSums + kSumThreads - 1) / kSumThreads, kSumThreads, 0, ctx->stream>>>(
                part.as<double>(), cnt, chunks, kSums, sums.as<double>());
            MDP_CHECK_LAUNCH(ctx);
            MDP_CUDA(cudaMemcpyAsync(h_sums.data(), sums.p, cnt * kSums * sizeof(double), cudaMemcpyDeviceToHost,
                                     ctx->stream));
            MDP_CUDA(cudaStreamSynchronize(ctx->stream));
            for (int b = 0; b < cnt; ++b) {
                if (!h_act[b]) continue;
                Lm &s = st[b];
                double H[4][4], g[4], F;
                lm_load(&h_sums[(size_t) b * kSums], H, g, &F);
                ++s.evals;
                bool finite = std::isfinite(F);
                for (int i = 0; i < 4; ++i) {
                    finite = finite && std::isfinite(g[i]);
                    for (int j = 0; j < 4; ++j) finite = finite && std::isfinite(H[i][j]);
                }
                if (first) {
                    if (!finite) {
                        mdp_set_error("block %d: the model is not finite at the starting point", bt.first + b);
                        return MDP_ENAN;
                    }
                    s.F = F;
                    std::memcpy(s.H, H, sizeof(H));
                    std::memcpy(s.g, g, sizeof(g));
                    for (int i = 0; i < 4; ++i) s.D[i] = std::max(H[i][i], 1e-300);
                } else if (finite && F < s.F) {
                    const double rel = (s.F - F) / s.F;
                    std::memcpy(s.p, s.pt, sizeof(s.p));
                    s.F = F;
                    std::memcpy(s.H, H, sizeof(H));
                    std::memcpy(s.g, g, sizeof(g));
                    for (int i = 0; i < 4; ++i) s.D[i] = std::max(s.D[i], H[i][i]);
                    s.mu = std::max(s.mu / 3.0, 1e-20);
                    if (rel <= 1e-16) s.done = s.converged = true;
                } else {
                    s.mu *= 4.0;
                    if (s.mu > 1e20) s.done = s.converged = true;
                }
                if (!s.done && s.evals >= kMaxEvals) s.done = true;   // not converged
            }
            first = false;
        }

        // ---- inverse PSD, irfft, window
        h_sig.assign(cnt, 0.0);
        for (int b = 0; b < cnt; ++b) {
            for (int i = 0; i < 4; ++i) h_prm[4 * b + i] = st[b].p[i];
            h_sig[b] = std::pow(10.0, -st[b].p[0]);
            if (h_params)
                for (int i = 0; i < 4; ++i) h_params[4 * (int64_t) (bt.first + b) + i] = st[b].p[i];
            if (h_evals) h_evals[bt.first + b] = st[b].converged ? st[b].evals : -1;
            if (!st[b].converged) ++nonconv;
        }
        MDP_CUDA(cudaMemcpyAsync(prm.p, h_prm.data(), cnt * 4 * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
        MDP_CUDA(cudaMemcpyAsync(sig.p, h_sig.data(), cnt * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
        const int gi = (int) std::min<int64_t>(((blue ? sh.L : n) + 255) / 256, 1024);
        invpsd_kernel<<<dim3(gi, cnt), 256, 0, ctx->stream>>>(buf.as<double2>(), sh, blue, n, df, prm.as<double>(),
                                                              sig.as<double>());
        MDP_CHECK_LAUNCH(ctx);
        if (blue) {
            MDP_TRY(fft_forward(ctx, buf.as<double2>(), sh, cnt));
            const int gl = (int) std::min<int64_t>((sh.L + 255) / 256, 1024);
            cmul_batch_kernel<<<dim3(gl, cnt), 256, 0, ctx->stream>>>(buf.as<double2>(), bh.as<double2>() + sh.L,
                                                                       sh.L);
            MDP_CHECK_LAUNCH(ctx);
        }
        MDP_TRY(fft_inverse(ctx, buf.as<double2>(), sh, cnt));
        invtt_out_kernel<<<dim3(grid_for(lambda, 256, 64), cnt), 256, 0, ctx->stream>>>(
            buf.as<double2>(), sh.L, blue, n, lambda, win.as<double>(), d_invtt + (int64_t) bt.first * lambda);
        MDP_CHECK_LAUNCH(ctx);
        // buffers are reused by the next batch: finish this one first
        MDP_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    if (nonconv) {
        mdp_set_error("Optimal parameters not found: %d block(s) reached %d evaluations", nonconv, kMaxEvals);
        return MDP_ENOCONV;
    }
    return MDP_OK;
}
