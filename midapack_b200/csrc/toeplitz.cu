// Inverse-noise operator N^-1 on the device: per stationary block, remove the
// block mean and apply the symmetric banded Toeplitz block.
//
// Reference: algebra/src/toeplitz/toeplitz_wizard.c:80-111 (stbmmProd: mean
// removal then mpi_stbmm), toeplitz_block.c:115-636 (per-block dispatch),
// toeplitz.c:298-367 (tpltz_init), 441-470 (circ_init_fftw: circulant
// embedding c[0]=T[0], c[i]=c[bs-i]=T[i]), 731-865 (stmm_core overlap-save:
// tile stride bs - 2(lambda-1), zero padding outside the block),
// 569-616 (scmm_direct: forward FFT, spectrum product, inverse FFT).
//
// B200 design.  All tiles of all blocks run in one launch: one CTA (or one
// thread-block cluster of C CTAs sharing the FFT through distributed shared
// memory) per overlap-save tile.  A tile of N real samples is packed as N/2
// complex points z[j] = x[2j] + i x[2j+1]; the complex FFT is an in-place
// radix-2 decimation-in-frequency transform executed as radix-16 register
// passes over shared memory (natural order in, bit-reversed out).  The real
// FFT untangling, the product with the block's real even spectrum H and the
// re-tangling for the inverse are fused into one pass over bit-reversed
// pairs (k, M-k); the inverse is the mirror decimation-in-time transform with
// conjugate twiddles (bit-reversed in, natural out).  No bit-reversal pass and
// no global-memory round trip exist between the forward and inverse
// transforms.  Spectra (N/2+1 doubles per distinct block row) and twiddles
// (exp(-2 pi i k/N), computed on the host in long double) are built once.
#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>

#include "mdp_internal.cuh"

namespace cg = cooperative_groups;

// ------------------------------------------------------------------ complex helpers
// The FFT runs on double2 (FP64 path) or float2 (FP32 operator of the mixed
// precision solver); the helpers are overloaded on both.
template <typename T> struct CT;
template <> struct CT<double> { using V = double2; };
template <> struct CT<float> { using V = float2; };

__device__ __forceinline__ double2 mkv(double2, double x, double y) { return make_double2(x, y); }
__device__ __forceinline__ float2 mkv(float2, float x, float y) { return make_float2(x, y); }

template <typename V> __device__ __forceinline__ V cadd(V a, V b) { return mkv(a, a.x + b.x, a.y + b.y); }
template <typename V> __device__ __forceinline__ V csub(V a, V b) { return mkv(a, a.x - b.x, a.y - b.y); }
template <typename V> __device__ __forceinline__ V cmul(V a, V b) {
    return mkv(a, a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename V> __device__ __forceinline__ V cmulc(V a, V b) {  // a * conj(b)
    return mkv(a, a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
template <typename V> __device__ __forceinline__ V csq(V a) {  // a^2
    return mkv(a, a.x * a.x - a.y * a.y, 2 * a.x * a.y);
}

// 16th roots of unity exp(-2 pi i k / 16), k < 8, correctly rounded
__constant__ double2 c_w16[8] = {
    {0x1.0000000000000p+0, 0.0},
    {0x1.d906bcf328d46p-1, -0x1.87de2a6aea963p-2},
    {0x1.6a09e667f3bcdp-1, -0x1.6a09e667f3bcdp-1},
    {0x1.87de2a6aea963p-2, -0x1.d906bcf328d46p-1},
    {0.0, -0x1.0000000000000p+0},
    {-0x1.87de2a6aea963p-2, -0x1.d906bcf328d46p-1},
    {-0x1.6a09e667f3bcdp-1, -0x1.6a09e667f3bcdp-1},
    {-0x1.d906bcf328d46p-1, -0x1.87de2a6aea963p-2},
};
__constant__ float2 c_w16f[8] = {
    {0x1.000000p+0f, 0.0f},
    {0x1.d906bcp-1f, -0x1.87de2ap-2f},
    {0x1.6a09e6p-1f, -0x1.6a09e6p-1f},
    {0x1.87de2ap-2f, -0x1.d906bcp-1f},
    {0.0f, -0x1.000000p+0f},
    {-0x1.87de2ap-2f, -0x1.d906bcp-1f},
    {-0x1.6a09e6p-1f, -0x1.6a09e6p-1f},
    {-0x1.d906bcp-1f, -0x1.87de2ap-2f},
};
__device__ __forceinline__ double2 w16(double2, int i) { return c_w16[i]; }
__device__ __forceinline__ float2 w16(float2, int i) { return c_w16f[i]; }

// Shared-memory index swizzle: XOR the low 3 bits of a complex index with
// bits 5-7.  Every pass below reads sets of elements at a stride of L/R; the
// swizzle spreads those over all 8 bank groups of a 128-byte row (16-byte
// elements; for 8-byte elements it halves the conflicts of the small-group
// passes), so no FP64 pass has bank conflicts.
__device__ __forceinline__ int swz(int i) { return i ^ ((i >> 5) & 7); }
// 8-byte elements (float2): 16 per 128-byte row, XOR 4 bits
__device__ __forceinline__ int swzv(double2, int i) { return swz(i); }
__device__ __forceinline__ int swzv(float2, int i) { return i ^ ((i >> 5) & 15); }

// DIF stages of a radix-R register set.  Element i of the set sits at group
// position q + i*(L/R) inside a DIF group of size L; w = W_L^q is loaded by
// the caller.  Stage j (group L/2^j, span L/2^(j+1)) pairs i and i + R/2^(j+1)
// (i mod R/2^j < R/2^(j+1)); the difference is multiplied by
// W_{L/2^j}^{q + r L/R} = w^(2^j) * W_16^(r 2^j 16/R), r = i mod R/2^j.
template <typename V, int R>
__device__ __forceinline__ void dif_set(V (&v)[R], V w) {
    V wj = w;
#pragma unroll
    for (int j = 0, sub = R; sub > 1; j++, sub >>= 1) {
        const int half = sub >> 1;
#pragma unroll
        for (int i = 0; i < R; i++) {
            const int r = i % sub;
            if (r < half) {
                const V a = v[i], b = v[i + half];
                v[i] = cadd(a, b);
                const V tw = (r == 0) ? wj : cmul(wj, w16(wj, (r << j) * (16 / R)));
                v[i + half] = cmul(csub(a, b), tw);
            }
        }
        wj = csq(wj);
    }
}

// exact mirror of dif_set with conjugate twiddles (decimation in time)
template <typename V, int R>
__device__ __forceinline__ void dit_set(V (&v)[R], V w) {
    constexpr int NS = (R >= 16) ? 4 : (R >= 8) ? 3 : (R >= 4) ? 2 : 1;
    V             wpow[NS];
    wpow[0] = w;
#pragma unroll
    for (int j = 1; j < NS; j++) wpow[j] = csq(wpow[j - 1]);
#pragma unroll
    for (int j = NS - 1; j >= 0; j--) {
        const int sub = R >> j, half = sub >> 1;
#pragma unroll
        for (int i = 0; i < R; i++) {
            const int r = i % sub;
            if (r < half) {
                const V tw = (r == 0) ? wpow[j] : cmul(wpow[j], w16(w, (r << j) * (16 / R)));
                const V a = v[i];
                const V t = cmulc(v[i + half], tw);
                v[i] = cadd(a, t);
                v[i + half] = csub(a, t);
            }
        }
    }
}

// one local pass of R = 2^k stages starting at group size L over smem s[0..ML);
// tw[k] = exp(-2 pi i k / N) with N = 2^logN
template <typename V, int R, bool INVERSE>
__device__ __forceinline__ void local_pass(V *s, int ML, int L, int logN_over_L, const V *__restrict__ tw) {
    const int nsets = ML / R;
    const int stride = L / R;
    for (int set = threadIdx.x; set < nsets; set += blockDim.x) {
        const int g = set / stride, q = set - g * stride;
        const int base = g * L + q;
        const V   w = __ldg(tw + ((int64_t) q << logN_over_L));  // W_L^q
        V         v[R];
#pragma unroll
        for (int i = 0; i < R; i++) v[i] = s[swzv(V{}, base + i * stride)];
        if (INVERSE) dit_set<V, R>(v, w);
        else dif_set<V, R>(v, w);
#pragma unroll
        for (int i = 0; i < R; i++) s[swzv(V{}, base + i * stride)] = v[i];
    }
    __syncthreads();
}

// all local stages of the per-CTA transform, 4 per pass; the schedule is
// resolved at compile time (no local-memory tables)
template <typename V, int LOG_ML, bool INVERSE>
__device__ __forceinline__ void local_fft(V *s, int logN, const V *__restrict__ tw) {
    constexpr int NP = (LOG_ML + 3) / 4;
    constexpr int ML = 1 << LOG_ML;
#pragma unroll
    for (int pi = 0; pi < NP; pi++) {
        const int p = INVERSE ? (NP - 1 - pi) : pi;
        const int rem = LOG_ML - 4 * p;
        const int k = rem >= 4 ? 4 : rem;
        const int logL = LOG_ML - 4 * p;
        const int L = 1 << logL;
        const int lno = logN - logL;
        if (k == 4) local_pass<V, 16, INVERSE>(s, ML, L, lno, tw);
        else if (k == 3) local_pass<V, 8, INVERSE>(s, ML, L, lno, tw);
        else if (k == 2) local_pass<V, 4, INVERSE>(s, ML, L, lno, tw);
        else local_pass<V, 2, INVERSE>(s, ML, L, lno, tw);
    }
}

// ------------------------------------------------------------------ the tile kernel
template <typename T>
struct TileArgsT {
    const T                  *vin;
    T                        *vout;
    const int64_t            *tile_start;  // first output row of the tile (global)
    const int32_t            *tile_block;
    const int64_t            *blk_start;
    const int32_t            *blk_len;
    const int32_t            *blk_spec;
    const T                  *spectra;     // [n_spec][M+1]
    const typename CT<T>::V  *tw;          // [M]
    const double             *means;       // [nb] or nullptr
    int                       lambda;
};
typedef TileArgsT<double> TileArgs;

template <typename T, int LOG_ML, int C>
__global__ void __launch_bounds__(512) toeplitz_tile_kernel(TileArgsT<T> a) {
    using V = typename CT<T>::V;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V            *smem = reinterpret_cast<V *>(smem_raw);
    constexpr int ML = 1 << LOG_ML;
    constexpr int M = ML * C;       // complex points per tile
    constexpr int N = 2 * M;        // real samples per tile
    int           logM = LOG_ML;
    for (int c = C; c > 1; c >>= 1) logM++;
    const int logN = logM + 1;

    const int     rank = (C > 1) ? (int) (blockIdx.x % C) : 0;
    const int64_t tile = (C > 1) ? (int64_t) (blockIdx.x / C) : (int64_t) blockIdx.x;
    const int     blk = a.tile_block[tile];
    const int64_t bs = a.blk_start[blk];
    const int64_t be = bs + a.blk_len[blk];
    const int64_t t0 = a.tile_start[tile];
    const int     halo = a.lambda - 1;
    const int64_t ws = t0 - halo;               // window start (row of x[0])
    const int     E = N - 2 * halo;            // outputs per tile
    const T       mu = a.means ? (T) a.means[blk] : (T) 0;

    // ---- load this CTA's 2*ML real samples of the window (zero outside the block)
    T            *sd = reinterpret_cast<T *>(smem);
    const int64_t r0 = ws + (int64_t) rank * 2 * ML;
    // batches of 8 independent loads per thread keep many HBM requests in flight
    for (int j0 = threadIdx.x; j0 < 2 * ML; j0 += 8 * blockDim.x) {
        T v[8];
#pragma unroll
        for (int u = 0; u < 8; u++) {
            const int     j = j0 + u * blockDim.x;
            const int64_t row = r0 + j;
            v[u] = (j < 2 * ML && row >= bs && row < be) ? __ldg(a.vin + row) : mu;
        }
#pragma unroll
        for (int u = 0; u < 8; u++) {
            const int j = j0 + u * blockDim.x;
            if (j < 2 * ML) sd[2 * swzv(V{}, j >> 1) + (j & 1)] = v[u] - mu;
        }
    }

    if constexpr (C > 1) {
        cg::cluster_group cluster = cg::this_cluster();
        cluster.sync();
        // cross-CTA DIF stages: set q holds element c of CTA c at local q
        for (int q = rank * (ML / C) + threadIdx.x; q < (rank + 1) * (ML / C); q += blockDim.x) {
            V         v[C];
            const int sq = swzv(V{}, q);
#pragma unroll
            for (int c = 0; c < C; c++) v[c] = cluster.map_shared_rank(smem, c)[sq];
            dif_set<V, C>(v, __ldg(a.tw + 2 * q));  // W_M^q = W_N^(2q)
#pragma unroll
            for (int c = 0; c < C; c++) cluster.map_shared_rank(smem, c)[sq] = v[c];
        }
        cluster.sync();
    } else {
        __syncthreads();
    }

    local_fft<V, LOG_ML, false>(smem, logN, a.tw);

    if constexpr (C > 1) cg::this_cluster().sync();

    // ---- real-FFT untangle, spectrum product, re-tangle (bit-reversed storage)
    const T *H = a.spectra + (int64_t) a.blk_spec[blk] * (M + 1);
    // Position P holds Z[rev(P)]; pairs (k, M-k) with k <= M/2 are handled by the
    // owner of rev(k).  k <= M/2 exactly for even local positions plus the single
    // position of k = M/2 (local index 1 of rank 0), so each thread walks even
    // positions in batches of 4 with the spectrum and twiddle loads issued first.
    constexpr int NPAIR = ML / 2;
    const T       half = (T) 0.5;
    for (int i0 = threadIdx.x; i0 < NPAIR + 1; i0 += 4 * blockDim.x) {
        int  p1[4], p2[4];
        T    hk[4], hm[4];
        V    wk[4];
        bool act[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int i = i0 + u * blockDim.x;
            int       p = 2 * i;
            act[u] = i < NPAIR;
            if (i == NPAIR) {  // the k = M/2 pair: local position 1 of rank 0
                p = 1;
                act[u] = (rank == 0);
            }
            const int P1 = rank * ML + p;
            const int k = act[u] ? (int) (__brev((unsigned) P1) >> (32 - logM)) : 0;
            const int k2 = (M - k) & (M - 1);
            p1[u] = p;
            p2[u] = (int) (__brev((unsigned) k2) >> (32 - logM));
            hk[u] = act[u] ? __ldg(H + k) : (T) 0;
            hm[u] = act[u] ? __ldg(H + (M - k)) : (T) 0;
            wk[u] = act[u] ? __ldg(a.tw + k) : mkv(wk[u], (T) 1, (T) 0);
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
            if (!act[u]) continue;
            const int P2 = p2[u];
            V        *s1 = smem + swzv(V{}, p1[u]);
            V        *s2;
            if constexpr (C > 1) s2 = cg::this_cluster().map_shared_rank(smem, P2 / ML) + swzv(V{}, P2 % ML);
            else s2 = smem + swzv(V{}, P2);
            const V Z1 = *s1, Z2 = *s2;
            const V E0 = mkv(Z1, half * (Z1.x + Z2.x), half * (Z1.y - Z2.y));
            const V O0 = mkv(Z1, half * (Z1.y + Z2.y), -half * (Z1.x - Z2.x));
            const T ca = half * (hk[u] + hm[u]), cb = half * (hk[u] - hm[u]);
            const V wO = cmul(wk[u], O0);
            const V Ep = mkv(Z1, ca * E0.x + cb * wO.x, ca * E0.y + cb * wO.y);
            const V cE = cmulc(E0, wk[u]);  // conj(w) * E
            const V Op = mkv(Z1, cb * cE.x + ca * O0.x, cb * cE.y + ca * O0.y);
            *s1 = mkv(Z1, Ep.x - Op.y, Ep.y + Op.x);
            if (P2 != rank * ML + p1[u]) *s2 = mkv(Z1, Ep.x + Op.y, -Ep.y + Op.x);
        }
    }

    if constexpr (C > 1) cg::this_cluster().sync();
    else __syncthreads();

    local_fft<V, LOG_ML, true>(smem, logN, a.tw);

    if constexpr (C > 1) {
        cg::cluster_group cluster = cg::this_cluster();
        cluster.sync();
        for (int q = rank * (ML / C) + threadIdx.x; q < (rank + 1) * (ML / C); q += blockDim.x) {
            V         v[C];
            const int sq = swzv(V{}, q);
#pragma unroll
            for (int c = 0; c < C; c++) v[c] = cluster.map_shared_rank(smem, c)[sq];
            dit_set<V, C>(v, __ldg(a.tw + 2 * q));  // W_M^q = W_N^(2q)
#pragma unroll
            for (int c = 0; c < C; c++) cluster.map_shared_rank(smem, c)[sq] = v[c];
        }
        cluster.sync();
    }

    // ---- store the tile's central outputs, scaled by 1/M
    const T       scale = (T) 1 / (T) M;
    const int64_t out_end = min(t0 + (int64_t) E, be);
    for (int j = threadIdx.x; j < 2 * ML; j += blockDim.x) {
        const int64_t row = r0 + j;
        if (row >= t0 && row < out_end) a.vout[row] = sd[2 * swzv(V{}, j >> 1) + (j & 1)] * scale;
    }
}

// ------------------------------------------------------------------ spectra
// H[k] = T0 + 2 sum_{i<lambda} T[i] cos(2 pi i k / N), k = 0..N/2: the DFT of
// the circulant embedding, which is real and even.
__global__ void spectrum_kernel(const double *__restrict__ T, int lambda, int N, const double2 *__restrict__ tw,
                                double *__restrict__ H) {
    const int M = N / 2;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k <= M; k += gridDim.x * blockDim.x) {
        double acc = 0.0, comp = 0.0;  // Kahan-compensated sum of the cosine terms
        for (int i = 1; i < lambda; i++) {
            const int64_t e = ((int64_t) i * k) % N;
            // cos(2 pi e / N) from the half-period table (tw covers e < N/2)
            const double  c = (e < M) ? tw[e].x : -tw[e - M].x;
            const double  y = T[i] * c - comp;
            const double  t = acc + y;
            comp = (t - acc) - y;
            acc = t;
        }
        H[k] = T[0] + 2.0 * acc;
    }
}

// ------------------------------------------------------------------ block means and white noise
template <typename T>
__global__ void block_partial_sums(const T *__restrict__ v, const int64_t *__restrict__ chunk_start,
                                   const int32_t *__restrict__ chunk_len, double *__restrict__ partial) {
    const int64_t s = chunk_start[blockIdx.x];
    const int     n = chunk_len[blockIdx.x];
    double        acc = 0.0;
    for (int j = threadIdx.x; j < n; j += blockDim.x) acc += (double) v[s + j];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    __shared__ double ws[32];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double x = (threadIdx.x < (blockDim.x >> 5)) ? ws[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (threadIdx.x == 0) partial[blockIdx.x] = x;
    }
}

__global__ void block_means_final(const double *__restrict__ partial, const int32_t *__restrict__ blk_chunk0,
                                  const int32_t *__restrict__ blk_nchunk, const int32_t *__restrict__ blk_len,
                                  int nb, double *__restrict__ means) {
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int c = 0; c < blk_nchunk[b]; c++) s += partial[blk_chunk0[b] + c];
        means[b] = s / (double) blk_len[b];
    }
}

__global__ void white_kernel(const double *__restrict__ vin, double *__restrict__ vout, const int64_t *__restrict__ bstart,
                             const int32_t *__restrict__ blen, const double *__restrict__ t0, int nb) {
    const int b = blockIdx.y;
    const int64_t s = bstart[b];
    const int n = blen[b];
    const double d = t0[b];
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) vout[s + j] = d * vin[s + j];
}

// ------------------------------------------------------------------ plan
struct NoiseExtra {
    DevBuf chunk_start, chunk_len, blk_chunk0, blk_nchunk, partial;
    int    n_chunks = 0;
    bool   covers_all = true;
};
static std::map<const mdp_noise *, NoiseExtra *> g_extra;

static int choose_fft(int lambda, int64_t max_block, int *log_ml, int *cluster) {
    const char *env = getenv("MDP_TOEPLITZ_FFT");  // force the real tile size N (power of two)
    int         forced = env ? atoi(env) : 0;
    double      best = 1e300;
    int         bl = -1, bc = 1;
    for (int C = 1; C <= 8; C <<= 1)
        for (int lml = 6; lml <= 13; lml++) {
            if (C > 1 && lml != 13) continue;
            const int64_t N = 2LL * C * (1LL << lml);
            const int64_t E = N - 2LL * (lambda - 1);
            if (E < 1) continue;
            if (forced && N != forced) continue;
            int logN = lml + 1;
            for (int c = C; c > 1; c >>= 1) logN++;
            // FFT work per useful output, a penalty for cluster traffic, and a
            // penalty when a tile is much larger than the blocks it covers
            double eff = (double) std::min<int64_t>(E, max_block);
            double cost = (double) N / eff * (logN + 3) + (C > 1 ? 3.0 * std::log2((double) C) : 0.0);
            if (E < N / 4 && !forced) cost *= 1.5;
            if (cost < best) {
                best = cost;
                bl = lml;
                bc = C;
            }
        }
    if (bl < 0) return MDP_EUNSUPPORTED;
    *log_ml = bl;
    *cluster = bc;
    return MDP_OK;
}

typedef void (*tile_fn)(TileArgs);
static tile_fn pick_kernel(int log_ml, int C) {
    if (C == 1) switch (log_ml) {
            case 6: return toeplitz_tile_kernel<double, 6, 1>;
            case 7: return toeplitz_tile_kernel<double, 7, 1>;
            case 8: return toeplitz_tile_kernel<double, 8, 1>;
            case 9: return toeplitz_tile_kernel<double, 9, 1>;
            case 10: return toeplitz_tile_kernel<double, 10, 1>;
            case 11: return toeplitz_tile_kernel<double, 11, 1>;
            case 12: return toeplitz_tile_kernel<double, 12, 1>;
            case 13: return toeplitz_tile_kernel<double, 13, 1>;
        }
    if (log_ml == 13) switch (C) {
            case 2: return toeplitz_tile_kernel<double, 13, 2>;
            case 4: return toeplitz_tile_kernel<double, 13, 4>;
            case 8: return toeplitz_tile_kernel<double, 13, 8>;
        }
    return nullptr;
}

extern "C" int mdp_noise_create(mdp_context *ctx, int nb_blocks, const int64_t *h_idv, const int32_t *h_n, int lambda,
                                const double *h_T, mdp_noise **out) {
    if (!ctx || !out || nb_blocks <= 0 || !h_idv || !h_n || !h_T || lambda < 1) {
        mdp_set_error("mdp_noise_create: invalid arguments");
        return MDP_EINVAL;
    }
    *out = nullptr;
    MDP_CUDA(cudaSetDevice(ctx->device));
    int64_t max_block = 0;
    for (int b = 0; b < nb_blocks; b++) {
        if (h_n[b] < 0 || h_idv[b] < 0) {
            mdp_set_error("mdp_noise_create: negative block size or offset (block %d)", b);
            return MDP_EINVAL;
        }
        if (b > 0 && h_idv[b] < h_idv[b - 1] + h_n[b - 1]) {
            mdp_set_error("mdp_noise_create: blocks must be sorted and disjoint (block %d)", b);
            return MDP_EINVAL;
        }
        if (lambda > 1 && h_n[b] > 0 && h_n[b] < lambda - 1) {
            // the reference rejects this case in stmm_main (toeplitz.c:948-949, error 1)
            mdp_set_error("mdp_noise_create: Toeplitz band width > block size (block %d: n=%d, lambda=%d)", b, h_n[b],
                          lambda);
            return MDP_EINVAL;
        }
        max_block = std::max<int64_t>(max_block, h_n[b]);
    }
    mdp_noise *N = new mdp_noise();
    NoiseExtra *X = new NoiseExtra();
    N->nb = nb_blocks;
    N->lambda = lambda;
    N->h_idv.assign(h_idv, h_idv + nb_blocks);
    N->h_n.assign(h_n, h_n + nb_blocks);
    N->h_T0.resize(nb_blocks);
    int64_t expect = 0;
    for (int b = 0; b < nb_blocks; b++) {
        N->h_T0[b] = h_T[(size_t) b * lambda];
        if (h_idv[b] != expect) X->covers_all = false;
        expect = h_idv[b] + h_n[b];
    }
    N->nrow_end = expect;
    auto fail = [&](int rc) {
        delete X;
        delete N;
        return rc;
    };
    int rc;
    std::vector<int32_t> h_len(N->h_n);
    if ((rc = N->blk_start.alloc(8 * nb_blocks)) || (rc = N->blk_len.alloc(4 * nb_blocks)) ||
        (rc = N->blk_t0.alloc(8 * nb_blocks)) || (rc = N->means.alloc(8 * nb_blocks)) ||
        (rc = N->blk_spec.alloc(4 * nb_blocks)))
        return fail(rc);
    cudaMemcpy(N->blk_start.p, h_idv, 8 * nb_blocks, cudaMemcpyHostToDevice);
    cudaMemcpy(N->blk_len.p, h_n, 4 * nb_blocks, cudaMemcpyHostToDevice);
    cudaMemcpy(N->blk_t0.p, N->h_T0.data(), 8 * nb_blocks, cudaMemcpyHostToDevice);

    // chunks for the deterministic block-mean reduction
    const int            CH = 1 << 16;
    std::vector<int64_t> cs;
    std::vector<int32_t> cl, c0(nb_blocks), cn(nb_blocks);
    for (int b = 0; b < nb_blocks; b++) {
        c0[b] = (int32_t) cs.size();
        for (int64_t o = 0; o < h_n[b]; o += CH) {
            cs.push_back(h_idv[b] + o);
            cl.push_back((int32_t) std::min<int64_t>(CH, h_n[b] - o));
        }
        cn[b] = (int32_t) cs.size() - c0[b];
    }
    X->n_chunks = (int) cs.size();
    if ((rc = X->chunk_start.alloc(8 * std::max<size_t>(cs.size(), 1))) ||
        (rc = X->chunk_len.alloc(4 * std::max<size_t>(cl.size(), 1))) || (rc = X->blk_chunk0.alloc(4 * nb_blocks)) ||
        (rc = X->blk_nchunk.alloc(4 * nb_blocks)) || (rc = X->partial.alloc(8 * std::max<size_t>(cs.size(), 1))))
        return fail(rc);
    if (!cs.empty()) {
        cudaMemcpy(X->chunk_start.p, cs.data(), 8 * cs.size(), cudaMemcpyHostToDevice);
        cudaMemcpy(X->chunk_len.p, cl.data(), 4 * cl.size(), cudaMemcpyHostToDevice);
    }
    cudaMemcpy(X->blk_chunk0.p, c0.data(), 4 * nb_blocks, cudaMemcpyHostToDevice);
    cudaMemcpy(X->blk_nchunk.p, cn.data(), 4 * nb_blocks, cudaMemcpyHostToDevice);

    if (lambda > 1) {
        if ((rc = choose_fft(lambda, max_block, &N->log2_ml, &N->cluster))) {
            mdp_set_error("mdp_noise_create: no FFT tile fits lambda=%d", lambda);
            return fail(rc);
        }
        const int M = N->cluster << N->log2_ml;
        N->fft_n = 2 * M;
        const int64_t E = (int64_t) N->fft_n - 2LL * (lambda - 1);
        std::vector<int64_t> ts;
        std::vector<int32_t> tb;
        for (int b = 0; b < nb_blocks; b++)
            for (int64_t o = 0; o < h_n[b]; o += E) {
                ts.push_back(h_idv[b] + o);
                tb.push_back(b);
            }
        N->n_tiles = (int64_t) ts.size();
        if ((rc = N->tile_start.alloc(8 * std::max<size_t>(ts.size(), 1))) ||
            (rc = N->tile_block.alloc(4 * std::max<size_t>(tb.size(), 1))))
            return fail(rc);
        if (!ts.empty()) {
            cudaMemcpy(N->tile_start.p, ts.data(), 8 * ts.size(), cudaMemcpyHostToDevice);
            cudaMemcpy(N->tile_block.p, tb.data(), 4 * tb.size(), cudaMemcpyHostToDevice);
        }
        // twiddles exp(-2 pi i k / N), k < N/2, in long double then rounded
        std::vector<double2> tw(M);
        for (int k = 0; k < M; k++) {
            long double ang = -2.0L * 3.14159265358979323846264338327950288L * (long double) k / (long double) N->fft_n;
            tw[k] = make_double2((double) cosl(ang), (double) sinl(ang));
        }
        if ((rc = N->twiddle.alloc(sizeof(double2) * M))) return fail(rc);
        cudaMemcpy(N->twiddle.p, tw.data(), sizeof(double2) * M, cudaMemcpyHostToDevice);
        // distinct block rows share one spectrum
        std::vector<int32_t> spec_of(nb_blocks);
        std::vector<int>     uniq;
        for (int b = 0; b < nb_blocks; b++) {
            int found = -1;
            for (size_t u = 0; u < uniq.size(); u++)
                if (!memcmp(h_T + (size_t) uniq[u] * lambda, h_T + (size_t) b * lambda, sizeof(double) * lambda)) {
                    found = (int) u;
                    break;
                }
            if (found < 0) {
                found = (int) uniq.size();
                uniq.push_back(b);
            }
            spec_of[b] = found;
        }
        N->n_spec = (int) uniq.size();
        N->h_Tuniq.resize((size_t) N->n_spec * lambda);
        for (int u = 0; u < N->n_spec; u++)
            memcpy(N->h_Tuniq.data() + (size_t) u * lambda, h_T + (size_t) uniq[u] * lambda, sizeof(double) * lambda);
        cudaMemcpy(N->blk_spec.p, spec_of.data(), 4 * nb_blocks, cudaMemcpyHostToDevice);
        if ((rc = N->spectra.alloc(sizeof(double) * (size_t) N->n_spec * (M + 1)))) return fail(rc);
        DevBuf dT;
        if ((rc = dT.alloc(sizeof(double) * lambda))) return fail(rc);
        for (int u = 0; u < N->n_spec; u++) {
            cudaMemcpy(dT.p, h_T + (size_t) uniq[u] * lambda, sizeof(double) * lambda, cudaMemcpyHostToDevice);
            spectrum_kernel<<<grid_for(M + 1, 128, 4096), 128, 0, ctx->stream>>>(
                    dT.as<double>(), lambda, N->fft_n, N->twiddle.as<double2>(),
                    N->spectra.as<double>() + (size_t) u * (M + 1));
            ctx->launches++;
            cudaStreamSynchronize(ctx->stream);
        }
        tile_fn fn = pick_kernel(N->log2_ml, N->cluster);
        size_t  smem = sizeof(double2) << N->log2_ml;
        cudaFuncSetAttribute((const void *) fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
        if (N->cluster > 1) cudaFuncSetAttribute((const void *) fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    }
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        mdp_set_error("mdp_noise_create: %s", cudaGetErrorString(e));
        return fail(MDP_ECUDA);
    }
    g_extra[N] = X;
    *out = N;
    return MDP_OK;
}

extern "C" void mdp_noise_destroy(mdp_noise *N) {
    if (!N) return;
    auto it = g_extra.find(N);
    if (it != g_extra.end()) {
        delete it->second;
        g_extra.erase(it);
    }
    delete N;
}

extern "C" int mdp_noise_tile(const mdp_noise *N, int *fft_size, int *cluster_ctas, int64_t *n_tiles) {
    if (!N) return MDP_EINVAL;
    if (fft_size) *fft_size = N->fft_n;
    if (cluster_ctas) *cluster_ctas = N->cluster;
    if (n_tiles) *n_tiles = N->n_tiles;
    return MDP_OK;
}

int mdp_block_means(mdp_context *ctx, const mdp_noise *N, const double *d_v, double *d_means) {
    NoiseExtra *X = g_extra.at(N);
    if (X->n_chunks == 0) {
        MDP_CUDA(cudaMemsetAsync(d_means, 0, 8 * N->nb, ctx->stream));
        return MDP_OK;
    }
    block_partial_sums<double><<<X->n_chunks, 512, 0, ctx->stream>>>(d_v, X->chunk_start.as<int64_t>(),
                                                             X->chunk_len.as<int32_t>(), X->partial.as<double>());
    MDP_CHECK_LAUNCH(ctx);
    block_means_final<<<grid_for(N->nb, 128, 1024), 128, 0, ctx->stream>>>(
            X->partial.as<double>(), X->blk_chunk0.as<int32_t>(), X->blk_nchunk.as<int32_t>(), N->blk_len.as<int32_t>(),
            N->nb, d_means);
    MDP_CHECK_LAUNCH(ctx);
    return MDP_OK;
}

// out = N^-1 in (in != out required); d_means: precomputed block means or nullptr to compute here
int mdp_stbmm_impl(mdp_context *ctx, const mdp_noise *N, const double *d_in, double *d_out, const double *d_means) {
    NoiseExtra *X = g_extra.at(N);
    if (!X->covers_all)
        MDP_CUDA(cudaMemcpyAsync(d_out, d_in, sizeof(double) * N->nrow_end, cudaMemcpyDeviceToDevice, ctx->stream));
    if (N->lambda == 1) {
        dim3 grid(std::max(1, std::min(64, (int) ((N->h_n.empty() ? 1 : N->h_n[0]) / 256 + 1))), N->nb);
        white_kernel<<<grid, 256, 0, ctx->stream>>>(d_in, d_out, N->blk_start.as<int64_t>(), N->blk_len.as<int32_t>(),
                                                    N->blk_t0.as<double>(), N->nb);
        MDP_CHECK_LAUNCH(ctx);
        return MDP_OK;
    }
    if (!d_means) {
        MDP_TRY(mdp_block_means(ctx, N, d_in, N->means.as<double>()));
        d_means = N->means.as<double>();
    }
    if (N->n_tiles == 0) return MDP_OK;
    TileArgs a;
    a.vin = d_in;
    a.vout = d_out;
    a.tile_start = N->tile_start.as<int64_t>();
    a.tile_block = N->tile_block.as<int32_t>();
    a.blk_start = N->blk_start.as<int64_t>();
    a.blk_len = N->blk_len.as<int32_t>();
    a.blk_spec = N->blk_spec.as<int32_t>();
    a.spectra = N->spectra.as<double>();
    a.tw = N->twiddle.as<double2>();
    a.means = d_means;
    a.lambda = N->lambda;
    tile_fn  fn = pick_kernel(N->log2_ml, N->cluster);
    size_t   smem = sizeof(double2) << N->log2_ml;
    int      threads = std::min(512, std::max(64, (1 << N->log2_ml) / 16));
    if (N->n_tiles * N->cluster > 0x7fffffffLL) return MDP_EUNSUPPORTED;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned) (N->n_tiles * N->cluster));
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = ctx->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = N->cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    MDP_CUDA(cudaLaunchKernelEx(&cfg, fn, a));
    MDP_CHECK_LAUNCH(ctx);
    return MDP_OK;
}

// y = P x fused with the block-mean partial sums of y: one CTA per 65536-row
// chunk of a block, so the mean-removal pass of N^-1 needs no second read of y.
__global__ void __launch_bounds__(512) matvec_chunk_sums_kernel(const int32_t *__restrict__ off,
                                                                const double *__restrict__ w,
                                                                const double *__restrict__ x, double *__restrict__ y,
                                                                const int64_t *__restrict__ chunk_start,
                                                                const int32_t *__restrict__ chunk_len,
                                                                double *__restrict__ partial) {
    const int64_t s = chunk_start[blockIdx.x];
    const int     n = chunk_len[blockIdx.x];
    double        acc = 0.0;
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        const int64_t t = s + j;
        const int32_t o = off[t];
        double        v = 0.0;
        if (o >= 0) v = w[3 * t] * __ldg(x + o) + w[3 * t + 1] * __ldg(x + o + 1) + w[3 * t + 2] * __ldg(x + o + 2);
        y[t] = v;
        acc += v;
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    __shared__ double ws[16];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = (threadIdx.x < (blockDim.x >> 5)) ? ws[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) partial[blockIdx.x] = v;
    }
}

// y = P x and the block means of y into N->means.  Returns MDP_EUNSUPPORTED
// (and does nothing) when the blocks do not cover every row or the pointing is
// not in the triplet layout; the caller then runs P and N^-1 separately.
int mdp_matvec_blockmeans(mdp_context *ctx, const mdp_pointing *A, const mdp_noise *N, const double *d_x,
                          double *d_y) {
    NoiseExtra *X = g_extra.at(N);
    if (!A->triplet || !X->covers_all || N->lambda == 1 || N->nrow_end != A->m || X->n_chunks == 0)
        return MDP_EUNSUPPORTED;
    matvec_chunk_sums_kernel<<<X->n_chunks, 512, 0, ctx->stream>>>(A->off.as<int32_t>(), A->values, d_x, d_y,
                                                                   X->chunk_start.as<int64_t>(),
                                                                   X->chunk_len.as<int32_t>(), X->partial.as<double>());
    MDP_CHECK_LAUNCH(ctx);
    block_means_final<<<grid_for(N->nb, 128, 1024), 128, 0, ctx->stream>>>(
            X->partial.as<double>(), X->blk_chunk0.as<int32_t>(), X->blk_nchunk.as<int32_t>(), N->blk_len.as<int32_t>(),
            N->nb, N->means.as<double>());
    MDP_CHECK_LAUNCH(ctx);
    return MDP_OK;
}

// ------------------------------------------------------------------ FP32 operator
typedef void (*tile_fn32)(TileArgsT<float>);
static tile_fn32 pick_kernel32(int log_ml, int C) {
    if (C == 1) switch (log_ml) {
            case 6: return toeplitz_tile_kernel<float, 6, 1>;
            case 7: return toeplitz_tile_kernel<float, 7, 1>;
            case 8: return toeplitz_tile_kernel<float, 8, 1>;
            case 9: return toeplitz_tile_kernel<float, 9, 1>;
            case 10: return toeplitz_tile_kernel<float, 10, 1>;
            case 11: return toeplitz_tile_kernel<float, 11, 1>;
            case 12: return toeplitz_tile_kernel<float, 12, 1>;
            case 13: return toeplitz_tile_kernel<float, 13, 1>;
            case 14: return toeplitz_tile_kernel<float, 14, 1>;
        }
    if (log_ml == 14) switch (C) {
            case 2: return toeplitz_tile_kernel<float, 14, 2>;
            case 4: return toeplitz_tile_kernel<float, 14, 4>;
            case 8: return toeplitz_tile_kernel<float, 14, 8>;
        }
    return nullptr;
}

// FP32 tiles hold 2^14 complex points per CTA (128 KiB); same cost model as FP64
static int choose_fft32(int lambda, int64_t max_block, int *log_ml, int *cluster) {
    const char *env = getenv("MDP_TOEPLITZ_FFT32");
    int         forced = env ? atoi(env) : 0;
    double      best = 1e300;
    int         bl = -1, bc = 1;
    for (int C = 1; C <= 8; C <<= 1)
        for (int lml = 6; lml <= 14; lml++) {
            if (C > 1 && lml != 14) continue;
            const int64_t N = 2LL * C * (1LL << lml);
            const int64_t E = N - 2LL * (lambda - 1);
            if (E < 1) continue;
            if (forced && N != forced) continue;
            int logN = lml + 1;
            for (int c = C; c > 1; c >>= 1) logN++;
            double eff = (double) std::min<int64_t>(E, max_block);
            double cost = (double) N / eff * (logN + 3) + (C > 1 ? 3.0 * std::log2((double) C) : 0.0);
            if (E < N / 4 && !forced) cost *= 1.5;
            if (cost < best) {
                best = cost;
                bl = lml;
                bc = C;
            }
        }
    if (bl < 0) return MDP_EUNSUPPORTED;
    *log_ml = bl;
    *cluster = bc;
    return MDP_OK;
}

__global__ void to_float_kernel(const double *__restrict__ in, float *__restrict__ out, int64_t n) {
    for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x)
        out[i] = (float) in[i];
}

int mdp_noise_prepare_fp32(mdp_context *ctx, mdp_noise *N) {
    if (N->f32.ready) return MDP_OK;
    if (N->lambda == 1) {
        N->f32.ready = 1;
        return MDP_OK;
    }
    int64_t max_block = 0;
    for (int b = 0; b < N->nb; b++) max_block = std::max<int64_t>(max_block, N->h_n[b]);
    MDP_TRY(choose_fft32(N->lambda, max_block, &N->f32.log2_ml, &N->f32.cluster));
    const int     M = N->f32.cluster << N->f32.log2_ml;
    const int     Nn = 2 * M;
    const int64_t E = (int64_t) Nn - 2LL * (N->lambda - 1);
    N->f32.fft_n = Nn;
    std::vector<int64_t> ts;
    std::vector<int32_t> tb;
    for (int b = 0; b < N->nb; b++)
        for (int64_t o = 0; o < N->h_n[b]; o += E) {
            ts.push_back(N->h_idv[b] + o);
            tb.push_back(b);
        }
    N->f32.n_tiles = (int64_t) ts.size();
    MDP_TRY(N->f32.tile_start.alloc(8 * std::max<size_t>(ts.size(), 1)));
    MDP_TRY(N->f32.tile_block.alloc(4 * std::max<size_t>(tb.size(), 1)));
    if (!ts.empty()) {
        MDP_CUDA(cudaMemcpy(N->f32.tile_start.p, ts.data(), 8 * ts.size(), cudaMemcpyHostToDevice));
        MDP_CUDA(cudaMemcpy(N->f32.tile_block.p, tb.data(), 4 * tb.size(), cudaMemcpyHostToDevice));
    }
    // twiddles: long double on the host, FP64 copy for the spectra, FP32 copy for the tiles
    std::vector<double2> tw(M);
    std::vector<float2>  twf(M);
    for (int k = 0; k < M; k++) {
        long double ang = -2.0L * 3.14159265358979323846264338327950288L * (long double) k / (long double) Nn;
        tw[k] = make_double2((double) cosl(ang), (double) sinl(ang));
        twf[k] = make_float2((float) cosl(ang), (float) sinl(ang));
    }
    DevBuf tw64, spec64, dT;
    MDP_TRY(tw64.alloc(sizeof(double2) * M));
    MDP_TRY(N->f32.twiddle.alloc(sizeof(float2) * M));
    MDP_CUDA(cudaMemcpy(tw64.p, tw.data(), sizeof(double2) * M, cudaMemcpyHostToDevice));
    MDP_CUDA(cudaMemcpy(N->f32.twiddle.p, twf.data(), sizeof(float2) * M, cudaMemcpyHostToDevice));
    MDP_TRY(spec64.alloc(sizeof(double) * (size_t) N->n_spec * (M + 1)));
    MDP_TRY(N->f32.spectra.alloc(sizeof(float) * (size_t) N->n_spec * (M + 1)));
    MDP_TRY(dT.alloc(sizeof(double) * N->lambda));
    for (int u = 0; u < N->n_spec; u++) {
        MDP_CUDA(cudaMemcpy(dT.p, N->h_Tuniq.data() + (size_t) u * N->lambda, sizeof(double) * N->lambda,
                            cudaMemcpyHostToDevice));
        spectrum_kernel<<<grid_for(M + 1, 128, 4096), 128, 0, ctx->stream>>>(
                dT.as<double>(), N->lambda, Nn, tw64.as<double2>(), spec64.as<double>() + (size_t) u * (M + 1));
        MDP_CHECK_LAUNCH(ctx);
    }
    const int64_t ns = (int64_t) N->n_spec * (M + 1);
    to_float_kernel<<<grid_for(ns, 256, 1024), 256, 0, ctx->stream>>>(spec64.as<double>(), N->f32.spectra.as<float>(), ns);
    MDP_CHECK_LAUNCH(ctx);
    MDP_CUDA(cudaStreamSynchronize(ctx->stream));
    tile_fn32 fn = pick_kernel32(N->f32.log2_ml, N->f32.cluster);
    const int smem = (int) (sizeof(float2) << N->f32.log2_ml);
    MDP_CUDA(cudaFuncSetAttribute((const void *) fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    if (N->f32.cluster > 1)
        MDP_CUDA(cudaFuncSetAttribute((const void *) fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    N->f32.ready = 1;
    return MDP_OK;
}

__global__ void white32_kernel(const float *__restrict__ vin, float *__restrict__ vout,
                               const int64_t *__restrict__ bstart, const int32_t *__restrict__ blen,
                               const double *__restrict__ t0) {
    const int     b = blockIdx.y;
    const int64_t s = bstart[b];
    const int     n = blen[b];
    const float   d = (float) t0[b];
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) vout[s + j] = d * vin[s + j];
}

// out = N^-1 in with the FP32 tile kernels; d_means (FP64 block means of in)
// may be given (fused into the producer of in) or nullptr
int mdp_stbmm_impl32(mdp_context *ctx, mdp_noise *N, const float *d_in, float *d_out, const double *d_means) {
    NoiseExtra *X = g_extra.at(N);
    MDP_TRY(mdp_noise_prepare_fp32(ctx, N));
    if (!X->covers_all)
        MDP_CUDA(cudaMemcpyAsync(d_out, d_in, sizeof(float) * N->nrow_end, cudaMemcpyDeviceToDevice, ctx->stream));
    if (N->lambda == 1) {
        dim3 grid(64, N->nb);
        white32_kernel<<<grid, 256, 0, ctx->stream>>>(d_in, d_out, N->blk_start.as<int64_t>(), N->blk_len.as<int32_t>(),
                                                      N->blk_t0.as<double>());
        MDP_CHECK_LAUNCH(ctx);
        return MDP_OK;
    }
    if (!d_means) {
        if (X->n_chunks > 0) {
            block_partial_sums<float><<<X->n_chunks, 512, 0, ctx->stream>>>(
                    d_in, X->chunk_start.as<int64_t>(), X->chunk_len.as<int32_t>(), X->partial.as<double>());
            MDP_CHECK_LAUNCH(ctx);
            block_means_final<<<grid_for(N->nb, 128, 1024), 128, 0, ctx->stream>>>(
                    X->partial.as<double>(), X->blk_chunk0.as<int32_t>(), X->blk_nchunk.as<int32_t>(),
                    N->blk_len.as<int32_t>(), N->nb, N->means.as<double>());
            MDP_CHECK_LAUNCH(ctx);
        }
        d_means = N->means.as<double>();
    }
    if (N->f32.n_tiles == 0) return MDP_OK;
    TileArgsT<float> a;
    a.vin = d_in;
    a.vout = d_out;
    a.tile_start = N->f32.tile_start.as<int64_t>();
    a.tile_block = N->f32.tile_block.as<int32_t>();
    a.blk_start = N->blk_start.as<int64_t>();
    a.blk_len = N->blk_len.as<int32_t>();
    a.blk_spec = N->blk_spec.as<int32_t>();
    a.spectra = N->f32.spectra.as<float>();
    a.tw = N->f32.twiddle.as<float2>();
    a.means = d_means;
    a.lambda = N->lambda;
    tile_fn32 fn = pick_kernel32(N->f32.log2_ml, N->f32.cluster);
    if (N->f32.n_tiles * N->f32.cluster > 0x7fffffffLL) return MDP_EUNSUPPORTED;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned) (N->f32.n_tiles * N->f32.cluster));
    cfg.blockDim = dim3(std::min(512, std::max(64, (1 << N->f32.log2_ml) / 16)));
    cfg.dynamicSmemBytes = sizeof(float2) << N->f32.log2_ml;
    cfg.stream = ctx->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = N->f32.cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    MDP_CUDA(cudaLaunchKernelEx(&cfg, fn, a));
    MDP_CHECK_LAUNCH(ctx);
    return MDP_OK;
}

// y32 = P x (x FP64, weights FP32) fused with FP64 block-mean partial sums
__global__ void __launch_bounds__(512) matvec32_chunk_sums_kernel(const int32_t *__restrict__ off,
                                                                  const float *__restrict__ w,
                                                                  const double *__restrict__ x, float *__restrict__ y,
                                                                  const int64_t *__restrict__ chunk_start,
                                                                  const int32_t *__restrict__ chunk_len,
                                                                  double *__restrict__ partial) {
    const int64_t s = chunk_start[blockIdx.x];
    const int     n = chunk_len[blockIdx.x];
    double        acc = 0.0;
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        const int64_t t = s + j;
        const int32_t o = off[t];
        float         v = 0.0f;
        if (o >= 0)
            v = w[3 * t] * (float) __ldg(x + o) + w[3 * t + 1] * (float) __ldg(x + o + 1) +
                w[3 * t + 2] * (float) __ldg(x + o + 2);
        y[t] = v;
        acc += (double) v;
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    __shared__ double ws[16];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = (threadIdx.x < (blockDim.x >> 5)) ? ws[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) partial[blockIdx.x] = v;
    }
}

int mdp_matvec32_blockmeans(mdp_context *ctx, const mdp_pointing *A, const mdp_noise *N, const double *d_x,
                            float *d_y) {
    NoiseExtra *X = g_extra.at(N);
    if (!A->triplet || !A->w32.p || !X->covers_all || N->lambda == 1 || N->nrow_end != A->m || X->n_chunks == 0)
        return MDP_EUNSUPPORTED;
    matvec32_chunk_sums_kernel<<<X->n_chunks, 512, 0, ctx->stream>>>(A->off.as<int32_t>(), A->w32.as<float>(), d_x, d_y,
                                                                     X->chunk_start.as<int64_t>(),
                                                                     X->chunk_len.as<int32_t>(), X->partial.as<double>());
    MDP_CHECK_LAUNCH(ctx);
    block_means_final<<<grid_for(N->nb, 128, 1024), 128, 0, ctx->stream>>>(
            X->partial.as<double>(), X->blk_chunk0.as<int32_t>(), X->blk_nchunk.as<int32_t>(), N->blk_len.as<int32_t>(),
            N->nb, N->means.as<double>());
    MDP_CHECK_LAUNCH(ctx);
    return MDP_OK;
}

extern "C" int mdp_noise_tile_fp32(mdp_context *ctx, mdp_noise *N, int *fft_size, int *cluster_ctas,
                                   int64_t *n_tiles) {
    if (!ctx || !N) return MDP_EINVAL;
    MDP_CUDA(cudaSetDevice(ctx->device));
    MDP_TRY(mdp_noise_prepare_fp32(ctx, N));
    if (fft_size) *fft_size = N->f32.fft_n;
    if (cluster_ctas) *cluster_ctas = N->f32.cluster;
    if (n_tiles) *n_tiles = N->f32.n_tiles;
    return MDP_OK;
}

extern "C" int mdp_stbmm_fp32(mdp_context *ctx, mdp_noise *N, const float *d_in, float *d_out) {
    if (!ctx || !N || !d_in || !d_out || d_in == d_out) {
        mdp_set_error("mdp_stbmm_fp32: invalid arguments (in-place is not supported)");
        return MDP_EINVAL;
    }
    MDP_CUDA(cudaSetDevice(ctx->device));
    return mdp_stbmm_impl32(ctx, N, d_in, d_out, nullptr);
}

extern "C" int mdp_stbmm(mdp_context *ctx, const mdp_noise *N, const double *d_in, double *d_out) {
    if (!ctx || !N || !d_in || !d_out) return MDP_EINVAL;
    const double *src = d_in;
    if (d_in == d_out) {
        MDP_TRY(ctx->scratch.alloc(sizeof(double) * N->nrow_end));
        MDP_CUDA(cudaMemcpyAsync(ctx->scratch.p, d_in, sizeof(double) * N->nrow_end, cudaMemcpyDeviceToDevice,
                                 ctx->stream));
        src = ctx->scratch.as<double>();
    }
    return mdp_stbmm_impl(ctx, N, src, d_out, nullptr);
}

// ------------------------------------------------------------------ allocation-free N^-1
// Some callers cannot allocate device memory at the moment they apply the
// noise operator: code running inside a fixed memory arena or pool that owns
// all device memory, callers that forbid cudaMalloc/cudaFree in their solve
// loop because those calls synchronise the device, and plugins loaded into a
// host that hands them only the buffers it owns.  mdp_stbmm_noalloc serves
// them: the per-chunk partial sums and per-block means of the mean-removal
// pass live in the file-scope array below instead of buffers of the noise
// object, and the call allocates nothing.  The array holds
// MDP_NOALLOC_SCRATCH_DOUBLES doubles (1 MiB) on every device that loads this
// library, until the process exits.
#define MDP_NOALLOC_SCRATCH_DOUBLES (1 << 17)
static __device__ __align__(256) double g_stbmm_scratch[MDP_NOALLOC_SCRATCH_DOUBLES];

static std::mutex g_noalloc_mu;
static double    *g_noalloc_ptr[64] = {nullptr};

// The host-side name g_stbmm_scratch is only a stand-in for the symbol, not a
// device address: the address is looked up once per device, with that device
// current, and cached.
static int noalloc_scratch(int device, double **out) {
    if (device < 0 || device >= 64) return MDP_EINVAL;
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[device]) {
        void       *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_stbmm_scratch);
        if (e != cudaSuccess) {
            mdp_set_error("mdp_stbmm_noalloc: cudaGetSymbolAddress failed on device %d: %s", device,
                          cudaGetErrorString(e));
            return MDP_ECUDA;
        }
        g_noalloc_ptr[device] = static_cast<double *>(p);
    }
    *out = g_noalloc_ptr[device];
    return MDP_OK;
}

extern "C" int mdp_stbmm_noalloc(mdp_context *ctx, const mdp_noise *N, const double *d_in, double *d_out) {
    if (!ctx || !N || !d_in || !d_out) {
        mdp_set_error("mdp_stbmm_noalloc: invalid arguments");
        return MDP_EINVAL;
    }
    if (d_in == d_out) {
        mdp_set_error("mdp_stbmm_noalloc: in-place application needs a copy of the input; pass d_out != d_in");
        return MDP_EINVAL;
    }
    NoiseExtra   *X = g_extra.at(N);
    const int64_t need = (int64_t) X->n_chunks + N->nb;
    if (N->lambda > 1 && need > MDP_NOALLOC_SCRATCH_DOUBLES) {
        mdp_set_error("mdp_stbmm_noalloc: %lld scratch doubles needed (%d blocks, %d 65536-row chunks), limit %d",
                      (long long) need, N->nb, X->n_chunks, MDP_NOALLOC_SCRATCH_DOUBLES);
        return MDP_EINVAL;
    }
    MDP_CUDA(cudaSetDevice(ctx->device));
    double *scratch = nullptr;
    MDP_TRY(noalloc_scratch(ctx->device, &scratch));
    if (N->lambda == 1) return mdp_stbmm_impl(ctx, N, d_in, d_out, nullptr);  // no mean removal, no scratch
    double *partial = scratch;                 // [n_chunks], each written before it is read
    double *means = scratch + X->n_chunks;     // [nb], each written before it is read
    if (X->n_chunks > 0) {
        block_partial_sums<double><<<X->n_chunks, 512, 0, ctx->stream>>>(d_in, X->chunk_start.as<int64_t>(),
                                                                 X->chunk_len.as<int32_t>(), partial);
        MDP_CHECK_LAUNCH(ctx);
        block_means_final<<<grid_for(N->nb, 128, 1024), 128, 0, ctx->stream>>>(
                partial, X->blk_chunk0.as<int32_t>(), X->blk_nchunk.as<int32_t>(), N->blk_len.as<int32_t>(), N->nb,
                means);
        MDP_CHECK_LAUNCH(ctx);
    } else {
        MDP_CUDA(cudaMemsetAsync(means, 0, sizeof(double) * N->nb, ctx->stream));
    }
    return mdp_stbmm_impl(ctx, N, d_in, d_out, means);
}
