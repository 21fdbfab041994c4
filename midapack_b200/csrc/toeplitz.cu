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
#include <atomic>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>

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

// Complex FP32 arithmetic on Blackwell's paired FP32 instructions (add / sub /
// mul / fma .f32x2): one instruction for both components, each lane rounded as
// the scalar instruction would round it (6-8 % faster FP32 N^-1 than scalar).
__device__ __forceinline__ unsigned long long f2b(float x, float y) {
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(x), "f"(y));
    return r;
}
__device__ __forceinline__ float2 b2f(unsigned long long r) {
    float2 v;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(v.x), "=f"(v.y) : "l"(r));
    return v;
}
template <> __device__ __forceinline__ float2 cadd<float2>(float2 a, float2 b) {
    unsigned long long r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(f2b(a.x, a.y)), "l"(f2b(b.x, b.y)));
    return b2f(r);
}
template <> __device__ __forceinline__ float2 csub<float2>(float2 a, float2 b) {
    unsigned long long r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(f2b(a.x, a.y)), "l"(f2b(b.x, b.y)));
    return b2f(r);
}
// a b = (a.x b.x - a.y b.y, a.x b.y + a.y b.x) = (a.x, a.x) (b.x, b.y) + (a.y, a.y) (-b.y, b.x)
template <> __device__ __forceinline__ float2 cmul<float2>(float2 a, float2 b) {
    unsigned long long t, r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(t) : "l"(f2b(a.x, a.x)), "l"(f2b(b.x, b.y)));
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(f2b(a.y, a.y)), "l"(f2b(-b.y, b.x)), "l"(t));
    return b2f(r);
}
// a conj(b) = (a.x b.x + a.y b.y, a.y b.x - a.x b.y) = (a.x, a.y) (b.x, b.x) + (a.y, a.x) (b.y, -b.y)
template <> __device__ __forceinline__ float2 cmulc<float2>(float2 a, float2 b) {
    unsigned long long t, r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(t) : "l"(f2b(a.x, a.y)), "l"(f2b(b.x, b.x)));
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(f2b(a.y, a.x)), "l"(f2b(b.y, -b.y)), "l"(t));
    return b2f(r);
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
// wl[q] = W_L^q = exp(-2 pi i q / L), q < L/R, staged in shared memory
template <typename V, int R, bool INVERSE>
__device__ __forceinline__ void local_pass(V *s, int ML, int L, const V *wl) {
    const int nsets = ML / R;
    const int stride = L / R;
    for (int set = threadIdx.x; set < nsets; set += blockDim.x) {
        const int g = set / stride, q = set - g * stride;
        const int base = g * L + q;
        const V   w = wl[q];
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

// Pass p of the local transform starts at group size L = 2^(LOG_ML - 4p) and
// needs W_L^q for q < L/R.  The per-pass twiddle tables are packed one after
// the other (they depend on L only, not on the tile size); ltw_offset(l, p) is
// where pass p's table starts and ltw_offset(l, passes) the packed size.
__host__ __device__ constexpr int ltw_passes(int log_ml) { return (log_ml + 3) / 4; }
__host__ __device__ constexpr int ltw_offset(int log_ml, int p) {
    int off = 0;
    for (int i = 0; i < p; i++) {
        const int logL = log_ml - 4 * i;
        off += 1 << (logL - (logL >= 4 ? 4 : logL));
    }
    return off;
}
__host__ __device__ constexpr int ltw_size(int log_ml) { return ltw_offset(log_ml, ltw_passes(log_ml)); }

// all local stages of the per-CTA transform, 4 per pass; the schedule is
// resolved at compile time (no local-memory tables); stw = packed tables in
// shared memory
template <typename V, int LOG_ML, bool INVERSE>
__device__ __forceinline__ void local_fft(V *s, const V *stw) {
    constexpr int NP = ltw_passes(LOG_ML);
    constexpr int ML = 1 << LOG_ML;
#pragma unroll
    for (int pi = 0; pi < NP; pi++) {
        const int p = INVERSE ? (NP - 1 - pi) : pi;
        const int logL = LOG_ML - 4 * p;
        const int k = logL >= 4 ? 4 : logL;
        const int L = 1 << logL;
        const V  *wl = stw + ltw_offset(LOG_ML, p);
        if (k == 4) local_pass<V, 16, INVERSE>(s, ML, L, wl);
        else if (k == 3) local_pass<V, 8, INVERSE>(s, ML, L, wl);
        else if (k == 2) local_pass<V, 4, INVERSE>(s, ML, L, wl);
        else local_pass<V, 2, INVERSE>(s, ML, L, wl);
    }
}

// ------------------------------------------------------------------ the tile kernel
// The twist tables are in the order the product pass visits the spectrum:
// entry e = rank * ML/2 + i is the pair (k, M-k) of position P = rank*ML + 2i,
// k = bitrev(P); entry C*ML/2 is k = M/2.  Reading them is one coalesced
// stream instead of three scattered gathers per pair.
template <typename T>
struct TileArgsT {
    using V = typename CT<T>::V;
    const T       *vin;
    T             *vout;
    const int64_t *tile_start;  // first output row of the tile (global)
    const int32_t *tile_block;
    const int64_t *blk_start;
    const int32_t *blk_len;
    const int32_t *blk_spec;
    const V       *hpair;       // [n_spec][M/2+1]: ((H[k]+H[M-k])/2, (H[k]-H[M-k])/2)
    const V       *ttw;         // [M/2+1]: W_N^k
    const V       *ltw;         // packed local-pass twiddles W_L^q
    const V       *twm;         // [ML]: W_M^q for the cross-CTA stages
    const double  *means;       // [nb] or nullptr; [ncols][nb] for a column batch
    int            lambda;
    int            nb;          // blocks (stride of the per-column means)
    int64_t        col_stride;  // rows between the columns of a batch (blockIdx.y = column)
    const int     *active;      // [ncols] nonzero for the columns to apply, or nullptr (all)
};

// FP32 tiles of up to 2^13 points per CTA (64 KB of shared memory, two CTAs
// fit an SM) are held to 64 registers so that two 512-thread CTAs are resident
// (15-25 % faster despite ~100 bytes of spills); larger FP32 tiles and FP64
// tiles (one CTA per SM by shared memory) keep 128.
template <typename T, int LOG_ML, int C>
__global__ void __launch_bounds__(512, (sizeof(T) == 4 && LOG_ML <= 13) ? 2 : 1) toeplitz_tile_kernel(TileArgsT<T> a) {
    using V = typename CT<T>::V;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V            *smem = reinterpret_cast<V *>(smem_raw);
    constexpr int ML = 1 << LOG_ML;
    constexpr int M = ML * C;       // complex points per tile
    constexpr int N = 2 * M;        // real samples per tile
    int           logM = LOG_ML;
    for (int c = C; c > 1; c >>= 1) logM++;

    const int     rank = (C > 1) ? (int) (blockIdx.x % C) : 0;
    const int64_t tile = (C > 1) ? (int64_t) (blockIdx.x / C) : (int64_t) blockIdx.x;
    // column of a batch: every CTA of a cluster has the same blockIdx.y, so a
    // skipped column leaves whole clusters before their first barrier
    if (a.active && !a.active[blockIdx.y]) return;
    if (blockIdx.y) {
        a.vin += (int64_t) blockIdx.y * a.col_stride;
        a.vout += (int64_t) blockIdx.y * a.col_stride;
        if (a.means) a.means += (int64_t) blockIdx.y * a.nb;
    }
    const int     blk = a.tile_block[tile];
    const int64_t bs = a.blk_start[blk];
    const int64_t be = bs + a.blk_len[blk];
    const int64_t t0 = a.tile_start[tile];
    const int     halo = a.lambda - 1;
    const int64_t ws = t0 - halo;               // window start (row of x[0])
    const int     E = N - 2 * halo;            // outputs per tile
    const T       mu = a.means ? (T) a.means[blk] : (T) 0;

    // ---- stage the local-pass twiddles behind the tile
    constexpr int NLTW = ltw_size(LOG_ML);
    V            *stw = smem + ML;
    for (int i = threadIdx.x; i < NLTW; i += blockDim.x) stw[i] = __ldg(a.ltw + i);

    // ---- load this CTA's 2*ML real samples of the window (zero outside the block)
    T            *sd = reinterpret_cast<T *>(smem);
    const int64_t r0 = ws + (int64_t) rank * 2 * ML;
    // Asynchronous element copies global -> shared (no register staging, the
    // whole part in flight at once), zero-filled outside the block, into the
    // swizzled layout; then the block mean is removed in place.
    {
        const uint32_t sbase = static_cast<uint32_t>(__cvta_generic_to_shared(sd));
        for (int j = threadIdx.x; j < 2 * ML; j += blockDim.x) {
            const int64_t  row = r0 + j;
            const bool     in = row >= bs && row < be;
            const T       *src = in ? a.vin + row : a.vin;
            const uint32_t dst = sbase + (uint32_t) (sizeof(T) * (2 * swzv(V{}, j >> 1) + (j & 1)));
            if constexpr (sizeof(T) == 4)
                asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(dst), "l"(src), "r"(in ? 4 : 0)
                             : "memory");
            else
                asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(dst), "l"(src), "r"(in ? 8 : 0)
                             : "memory");
        }
        asm volatile("cp.async.wait_all;\n" ::: "memory");
        if (mu != (T) 0)
            for (int j = threadIdx.x; j < 2 * ML; j += blockDim.x) {
                const int64_t row = r0 + j;
                if (row >= bs && row < be) sd[2 * swzv(V{}, j >> 1) + (j & 1)] -= mu;
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
            dif_set<V, C>(v, __ldg(a.twm + q));
#pragma unroll
            for (int c = 0; c < C; c++) cluster.map_shared_rank(smem, c)[sq] = v[c];
        }
        cluster.sync();
    } else {
        __syncthreads();
    }

    local_fft<V, LOG_ML, false>(smem, stw);

    if constexpr (C > 1) cg::this_cluster().sync();

    // ---- real-FFT untangle, spectrum product, re-tangle (bit-reversed storage)
    // Position P holds Z[rev(P)]; pairs (k, M-k) with k <= M/2 are handled by the
    // owner of rev(k).  k <= M/2 exactly for even local positions plus the single
    // position of k = M/2 (local index 1 of rank 0), so each thread walks even
    // positions in batches of 4 with the table loads issued first.
    constexpr int NPAIR = ML / 2;
    const T       half = (T) 0.5;
    const V      *HP = a.hpair + (int64_t) a.blk_spec[blk] * (C * NPAIR + 1);
    for (int i0 = threadIdx.x; i0 < NPAIR + 1; i0 += 4 * blockDim.x) {
        int  p1[4], p2[4];
        V    hc[4], wk[4];
        bool act[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int i = i0 + u * blockDim.x;
            int       p = 2 * i, e = rank * NPAIR + i;
            act[u] = i < NPAIR;
            if (i == NPAIR) {  // the k = M/2 pair: local position 1 of rank 0
                p = 1;
                e = C * NPAIR;
                act[u] = (rank == 0);
            }
            const int P1 = rank * ML + p;
            const int k = act[u] ? (int) (__brev((unsigned) P1) >> (32 - logM)) : 0;
            const int k2 = (M - k) & (M - 1);
            p1[u] = p;
            p2[u] = (int) (__brev((unsigned) k2) >> (32 - logM));
            hc[u] = act[u] ? __ldg(HP + e) : mkv(hc[u], (T) 0, (T) 0);
            wk[u] = act[u] ? __ldg(a.ttw + e) : mkv(wk[u], (T) 1, (T) 0);
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
            const T ca = hc[u].x, cb = hc[u].y;
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

    local_fft<V, LOG_ML, true>(smem, stw);

    if constexpr (C > 1) {
        cg::cluster_group cluster = cg::this_cluster();
        cluster.sync();
        for (int q = rank * (ML / C) + threadIdx.x; q < (rank + 1) * (ML / C); q += blockDim.x) {
            V         v[C];
            const int sq = swzv(V{}, q);
#pragma unroll
            for (int c = 0; c < C; c++) v[c] = cluster.map_shared_rank(smem, c)[sq];
            dit_set<V, C>(v, __ldg(a.twm + q));
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

// ------------------------------------------------------------------ split tiles
// The same overlap-save tile product as toeplitz_tile_kernel, as a four-step
// FFT in three kernels with the tile's spectrum in a global scratch array
// (M = M1*M2 complex points per tile, z[M2*j1 + j2] = x[2j] + i x[2j+1]):
//   split_cols_kernel  (forward)  per column j2: M1-point DFT over j1, times
//                      W_M^(j2 k1) -> Y[k1][j2]
//   split_rows_kernel  per row pair (k1, M1-k1): M2-point DFT of both rows,
//                      the real-FFT untangle / spectrum product / re-tangle of
//                      the pairs (k, M-k) (k = k1 + M1 k2 and M-k lie in the
//                      paired rows), inverse DFT of both rows, times W_M^(-j2 k1)
//   split_cols_kernel  (inverse)  per column: inverse M1-point DFT over k1
//                      (as conj(DFT(conj)) ), store of the tile's central
//                      outputs scaled by 1/M
// Every CTA is small (tens of KiB of shared memory, several per SM) and none
// waits on another CTA: the latency of one CTA's loads is hidden by the others.
// Shared layout of a batch of sequences: element i of sequence b at
// b*L + (i ^ (b & min(L,32)-1)), so that a warp working on 32 sequences at the
// same position spreads over all banks.
template <int L>
__device__ __forceinline__ int sq_idx(int b, int i) {
    constexpr int XM = (L < 32 ? L : 32) - 1;
    return b * L + (i ^ (b & XM));
}

// one DIF (or DIT) pass of radix R at group size G over nseq sequences of length L
template <typename V, int R, int L, bool INVERSE>
__device__ __forceinline__ void seq_pass(V *s, int nseq, int G, const V *wl) {
    const int stride = G / R;
    const int nsets = nseq * (L / R);
    for (int t = threadIdx.x; t < nsets; t += blockDim.x) {
        const int b = t % nseq;
        const int r = t / nseq;
        const int g = r / stride, q = r - g * stride;
        const int base = g * G + q;
        const V   w = wl[q];
        V         v[R];
#pragma unroll
        for (int i = 0; i < R; i++) v[i] = s[sq_idx<L>(b, base + i * stride)];
        if (INVERSE) dit_set<V, R>(v, w);
        else dif_set<V, R>(v, w);
#pragma unroll
        for (int i = 0; i < R; i++) s[sq_idx<L>(b, base + i * stride)] = v[i];
    }
    __syncthreads();
}

// full length-L transform of nseq sequences (DIF: natural in, bit-reversed out;
// INVERSE: DIT with conjugate twiddles, bit-reversed in, natural out)
template <typename V, int LOG_L, bool INVERSE>
__device__ __forceinline__ void seq_fft(V *s, int nseq, const V *stw) {
    constexpr int NP = ltw_passes(LOG_L);
    constexpr int L = 1 << LOG_L;
#pragma unroll
    for (int pi = 0; pi < NP; pi++) {
        const int p = INVERSE ? (NP - 1 - pi) : pi;
        const int logG = LOG_L - 4 * p;
        const int k = logG >= 4 ? 4 : logG;
        const int G = 1 << logG;
        const V  *wl = stw + ltw_offset(LOG_L, p);
        if (k == 4) seq_pass<V, 16, L, INVERSE>(s, nseq, G, wl);
        else if (k == 3) seq_pass<V, 8, L, INVERSE>(s, nseq, G, wl);
        else if (k == 2) seq_pass<V, 4, L, INVERSE>(s, nseq, G, wl);
        else seq_pass<V, 2, L, INVERSE>(s, nseq, G, wl);
    }
}

// the passes of seq_fft but the innermost one (group size 2^(LOG_L - 4(NP-1)),
// sets of consecutive positions): DIF passes 0..NP-2, or the DIT passes
// NP-2..0 that follow an innermost pass done by the caller
template <typename V, int LOG_L, bool INVERSE>
__device__ __forceinline__ void seq_fft_outer(V *s, int nseq, const V *stw) {
    constexpr int NP = ltw_passes(LOG_L);
    constexpr int L = 1 << LOG_L;
#pragma unroll
    for (int pi = 0; pi < NP - 1; pi++) {
        const int p = INVERSE ? (NP - 2 - pi) : pi;
        const int logG = LOG_L - 4 * p;  // >= 5: radix-16 passes only
        const int G = 1 << logG;
        seq_pass<V, 16, L, INVERSE>(s, nseq, G, stw + ltw_offset(LOG_L, p));
    }
}

// real-FFT untangle, product with the real even spectrum, re-tangle of one
// pair (Z1 = Z[k], Z2 = Z[M-k]); hc = ((H[k]+H[M-k])/2, (H[k]-H[M-k])/2), wk = W_N^k
template <typename V, typename T>
__device__ __forceinline__ void twist_pair(V &Z1, V &Z2, V hc, V wk) {
    const T half = (T) 0.5;
    const V E0 = mkv(Z1, half * (Z1.x + Z2.x), half * (Z1.y - Z2.y));
    const V O0 = mkv(Z1, half * (Z1.y + Z2.y), -half * (Z1.x - Z2.x));
    const T ca = hc.x, cb = hc.y;
    const V wO = cmul(wk, O0);
    const V Ep = mkv(Z1, ca * E0.x + cb * wO.x, ca * E0.y + cb * wO.y);
    const V cE = cmulc(E0, wk);
    const V Op = mkv(Z1, cb * cE.x + ca * O0.x, cb * cE.y + ca * O0.y);
    Z1 = mkv(Z1, Ep.x - Op.y, Ep.y + Op.x);
    Z2 = mkv(Z1, Ep.x + Op.y, -Ep.y + Op.x);
}

template <typename T>
struct SplitArgsT {
    using V = typename CT<T>::V;
    const T       *vin;
    T             *vout;
    V             *Y;           // [n_tiles][M1][M2] scratch
    const int64_t *tile_start;
    const int32_t *tile_block;
    const int64_t *blk_start;
    const int32_t *blk_len;
    const int32_t *blk_spec;
    const V       *hpair;       // [n_spec][M/2+1] in split pair order
    const V       *ttw;         // [M/2+1] W_N^k in split pair order
    const V       *ltw1, *ltw2; // packed pass twiddles of the M1- and M2-point transforms
    const V       *wa, *wb;     // W_M^e = wa[e >> 8] * wb[e & 255]
    const double  *means;
    int            lambda;
    int            nb;
    int64_t        col_stride;
    const int     *active;
    int            log_m1, log_m2;
    int            E;           // outputs per tile
    int            vec2;        // vin aligned to two samples: pair loads
};

template <typename V>
__device__ __forceinline__ V split_tw(const V *wa, const V *wb, int e) {  // W_M^e
    return cmul(wa[e >> 8], wb[e & 255]);
}

// threads of a split kernel working on `work` complex points (one radix-16 set each)
__host__ __device__ constexpr int split_nt(int work) { return work / 16 < 64 ? 64 : (work / 16 > 512 ? 512 : work / 16); }
// resident CTAs per SM asked of the compiler for a split kernel of nt threads:
// FP32 kernels are held to 64 registers (1024 threads per SM; a few bytes of
// spills, 10-13 % faster than 80-90 registers at a third fewer warps); FP64
// kernels keep their registers (their 16 complex points take 64 by themselves)
__host__ __device__ constexpr int split_minb(int nt, int elem) { return elem == 4 ? (1024 / nt > 1 ? 1024 / nt : 1) : 1; }

// forward (INV = false) or inverse (INV = true) column transforms of one tile:
// CW consecutive columns per CTA
template <typename T, int LOG_M1, int CW, bool INV>
__global__ void __launch_bounds__(split_nt(CW << LOG_M1), split_minb(split_nt(CW << LOG_M1), sizeof(T)))
        split_cols_kernel(SplitArgsT<T> a) {
    using V = typename CT<T>::V;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V            *s = reinterpret_cast<V *>(smem_raw);
    constexpr int M1 = 1 << LOG_M1;
    constexpr int NT = split_nt(CW * M1);      // == blockDim.x
    constexpr int EPT = (CW * M1 + NT - 1) / NT;  // elements per thread
    const int     M2 = 1 << a.log_m2;
    const int     M = M1 * M2;
    const int     ncg = M2 / CW;
    const int64_t tile = blockIdx.x / ncg;
    const int     c0 = (int) (blockIdx.x % ncg) * CW;
    if (a.active && !a.active[blockIdx.y]) return;
    if (blockIdx.y) {
        a.vin += (int64_t) blockIdx.y * a.col_stride;
        a.vout += (int64_t) blockIdx.y * a.col_stride;
        if (a.means) a.means += (int64_t) blockIdx.y * a.nb;
    }
    V *Y = a.Y + (tile * M);
    // stage the pass twiddles and the W_M factor tables
    constexpr int NLTW = ltw_size(LOG_M1);
    V            *stw = s + CW * M1;
    V            *swa = stw + NLTW;
    V            *swb = swa + ((M >> 8) > 0 ? (M >> 8) : 1);
    for (int i = threadIdx.x; i < NLTW; i += blockDim.x) stw[i] = __ldg(a.ltw1 + i);
    for (int i = threadIdx.x; i < (M >> 8); i += blockDim.x) swa[i] = __ldg(a.wa + i);
    for (int i = threadIdx.x; i < 256; i += blockDim.x) swb[i] = __ldg(a.wb + i);
    const int     blk = a.tile_block[tile];
    const int64_t bs = a.blk_start[blk];
    const int64_t be = bs + a.blk_len[blk];
    const int64_t t0 = a.tile_start[tile];
    // the window starts on an even row (split tiles keep one output fewer
    // than the band allows, so the window can move down by one)
    const int64_t ws = (t0 - (a.lambda - 1)) & ~(int64_t) 1;
    // all loads of a thread are issued before its shared-memory stores
    if (!INV) {
        const T mu = a.means ? (T) a.means[blk] : (T) 0;
        // element (j1, c): samples ws + 2(M2 j1 + c0 + c) + {0, 1}, one aligned
        // pair load where both lie in the block
        T x0[EPT], x1[EPT];
#pragma unroll
        for (int u = 0; u < EPT; u++) {
            const int     e = threadIdx.x + u * NT;
            const int     c = e % CW, j1 = e / CW;
            const int64_t row = ws + 2 * (M2 * j1 + c0 + c);  // in-tile offsets fit in 32 bits (M <= 2^18)
            const bool    ok = e < CW * M1;
            if (a.vec2 && ok && row >= bs && row + 1 < be) {
                const V z = __ldg(reinterpret_cast<const V *>(a.vin + row));
                x0[u] = z.x - mu;
                x1[u] = z.y - mu;
            } else {
                x0[u] = (ok && row >= bs && row < be) ? __ldg(a.vin + row) - mu : (T) 0;
                x1[u] = (ok && row + 1 >= bs && row + 1 < be) ? __ldg(a.vin + row + 1) - mu : (T) 0;
            }
        }
#pragma unroll
        for (int u = 0; u < EPT; u++) {
            const int e = threadIdx.x + u * NT;
            if (e < CW * M1) s[sq_idx<M1>(e % CW, e / CW)] = mkv(V{}, x0[u], x1[u]);
        }
    } else {
        // Y'[k1][c0 + c], conjugated: the inverse DFT is conj(DFT(conj(.)))
        V y[EPT];
#pragma unroll
        for (int u = 0; u < EPT; u++) {
            const int e = threadIdx.x + u * NT;
            if (e < CW * M1) y[u] = Y[(e / CW) * M2 + c0 + e % CW];
        }
#pragma unroll
        for (int u = 0; u < EPT; u++) {
            const int e = threadIdx.x + u * NT;
            if (e < CW * M1) s[sq_idx<M1>(e % CW, e / CW)] = mkv(y[u], y[u].x, -y[u].y);
        }
    }
    __syncthreads();
    seq_fft<V, LOG_M1, false>(s, CW, stw);
    if (!INV) {
        // position p holds k1 = rev(p): Y[k1][j2] = W_M^(j2 k1) * value
        for (int e = threadIdx.x; e < CW * M1; e += blockDim.x) {
            const int c = e % CW, p = e / CW;
            const int k1 = (int) (__brev((unsigned) p) >> (32 - LOG_M1));
            const int j2 = c0 + c;
            const V   v = s[sq_idx<M1>(c, p)];
            Y[k1 * M2 + j2] = cmul(v, split_tw(swa, swb, (j2 * k1) & (M - 1)));
        }
    } else {
        // position p holds j1 = rev(p): z'[M2 j1 + j2] = conj(value) / M, samples 2(M2 j1 + j2) + {0, 1}
        const int64_t out_end = min(t0 + (int64_t) a.E, be);
        const T       scale = (T) 1 / (T) M;
        for (int e = threadIdx.x; e < CW * M1; e += blockDim.x) {
            const int     c = e % CW, p = e / CW;
            const int     j1 = (int) (__brev((unsigned) p) >> (32 - LOG_M1));
            const V       v = s[sq_idx<M1>(c, p)];
            const int64_t row = ws + 2 * (M2 * j1 + c0 + c);
            if (row >= t0 && row < out_end) a.vout[row] = v.x * scale;
            if (row + 1 >= t0 && row + 1 < out_end) a.vout[row + 1] = -v.y * scale;
        }
    }
}

// row pairs of one tile: pair rp = 0 holds the self-paired rows 0 and M1/2,
// pair rp > 0 the rows rp and M1 - rp; RP pairs (2 RP rows) per CTA
template <typename T, int LOG_M2, int RP>
__global__ void __launch_bounds__(split_nt(2 * RP << LOG_M2), split_minb(split_nt(2 * RP << LOG_M2), sizeof(T)))
        split_rows_kernel(SplitArgsT<T> a) {
    using V = typename CT<T>::V;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V            *s = reinterpret_cast<V *>(smem_raw);
    constexpr int M2 = 1 << LOG_M2;
    constexpr int NT = split_nt(2 * RP * M2);          // == blockDim.x
    constexpr int EPT = (2 * RP * M2 + NT - 1) / NT;  // elements per thread
    const int     M1 = 1 << a.log_m1;
    const int     M = M1 * M2;
    const int     npg = (M1 / 2) / RP;  // CTAs per tile
    const int64_t tile = blockIdx.x / npg;
    const int     rp0 = (int) (blockIdx.x % npg) * RP;
    if (a.active && !a.active[blockIdx.y]) return;
    V *Y = a.Y + (tile * M);
    constexpr int NLTW = ltw_size(LOG_M2);
    V            *stw = s + 2 * RP * M2;
    V            *swa = stw + NLTW;
    V            *swb = swa + ((M >> 8) > 0 ? (M >> 8) : 1);
    for (int i = threadIdx.x; i < NLTW; i += blockDim.x) stw[i] = __ldg(a.ltw2 + i);
    for (int i = threadIdx.x; i < (M >> 8); i += blockDim.x) swa[i] = __ldg(a.wa + i);
    for (int i = threadIdx.x; i < 256; i += blockDim.x) swb[i] = __ldg(a.wb + i);
    const V *HP = a.hpair + (int64_t) a.blk_spec[a.tile_block[tile]] * (M / 2 + 1);
    // slot r = 2 (rp - rp0) + {0: row A, 1: row B}
    auto row_of = [&](int r) {
        const int rp = rp0 + (r >> 1);
        if (rp == 0) return (r & 1) ? M1 / 2 : 0;
        return (r & 1) ? M1 - rp : rp;
    };
    {
        V y[EPT];
#pragma unroll
        for (int u = 0; u < EPT; u++) {
            const int e = threadIdx.x + u * NT;
            if (e < 2 * RP * M2) y[u] = Y[row_of(e / M2) * M2 + e % M2];
        }
#pragma unroll
        for (int u = 0; u < EPT; u++) {
            const int e = threadIdx.x + u * NT;
            if (e < 2 * RP * M2) s[sq_idx<M2>(e / M2, e % M2)] = y[u];
        }
    }
    __syncthreads();
    constexpr int RL_ = 1 << (LOG_M2 - 4 * (ltw_passes(LOG_M2) - 1));
    if (RL_ <= 4 && rp0 > 0) {
        // Rows k1 and M1-k1: the innermost forward pass works on sets of RL
        // consecutive positions, and position p of row A pairs with position
        // M2-1-p of row B, so set g of row A pairs element i <-> RL-1-i with
        // set NSET-1-g of row B.  That pass, the spectrum product of the pairs
        // and the first inverse pass run on the two sets in registers: one
        // shared-memory round trip instead of three (for small innermost
        // passes; with radix-16 sets the per-thread work is too long and the
        // three separate passes are faster).
        constexpr int NP = ltw_passes(LOG_M2);
        constexpr int RL = 1 << (LOG_M2 - 4 * (NP - 1));
        constexpr int NSET = M2 / RL;
        seq_fft_outer<V, LOG_M2, false>(s, 2 * RP, stw);
        const V one = mkv(V{}, (T) 1, (T) 0);
        for (int it = threadIdx.x; it < RP * NSET; it += blockDim.x) {
            const int rl = it / NSET, g = it - rl * NSET, gb = NSET - 1 - g;
            V         va[RL], vb[RL];
#pragma unroll
            for (int i = 0; i < RL; i++) {
                va[i] = s[sq_idx<M2>(2 * rl, g * RL + i)];
                vb[i] = s[sq_idx<M2>(2 * rl + 1, gb * RL + i)];
            }
            dif_set<V, RL>(va, one);
            dif_set<V, RL>(vb, one);
            const int pr0 = (M2 + 1) + (rp0 + rl - 1) * M2 + g * RL;
#pragma unroll
            for (int i = 0; i < RL; i++)
                twist_pair<V, T>(va[i], vb[RL - 1 - i], __ldg(HP + pr0 + i), __ldg(a.ttw + pr0 + i));
            dit_set<V, RL>(va, one);
            dit_set<V, RL>(vb, one);
#pragma unroll
            for (int i = 0; i < RL; i++) {
                s[sq_idx<M2>(2 * rl, g * RL + i)] = va[i];
                s[sq_idx<M2>(2 * rl + 1, gb * RL + i)] = vb[i];
            }
        }
        __syncthreads();
        seq_fft_outer<V, LOG_M2, true>(s, 2 * RP, stw);
        for (int e = threadIdx.x; e < 2 * RP * M2; e += blockDim.x) {
            const int r = e / M2, j2 = e % M2;
            const int k1 = row_of(r);
            const V   v = s[sq_idx<M2>(r, j2)];
            Y[k1 * M2 + j2] = cmulc(v, split_tw(swa, swb, (j2 * k1) & (M - 1)));
        }
        return;
    }
    seq_fft<V, LOG_M2, false>(s, 2 * RP, stw);
    // pairs (k, M-k): position p of row A with position M2-1-p of row B, or
    // inside rows 0 and M1/2 for rp = 0 (table entries in the same order)
    const T   half = (T) 0.5;
    const int npairs = RP * M2 + (rp0 == 0 ? 1 : 0);
    for (int i = threadIdx.x; i < npairs; i += blockDim.x) {
        int pr, pa, pb, ra, rb;  // table entry, positions, slots
        if (rp0 == 0 && i < M2 + 1) {
            pr = i;
            if (i < M2 / 2 + 1) {  // row 0: like a single tile of M2 points
                ra = rb = 0;
                int p = 2 * i;
                if (i == M2 / 2) p = 1;
                const int k2 = (int) (__brev((unsigned) p) >> (32 - LOG_M2));
                pa = p;
                pb = (int) (__brev((unsigned) ((M2 - k2) & (M2 - 1))) >> (32 - LOG_M2));
            } else {  // row M1/2: k2 with M2-1-k2
                ra = rb = 1;
                pa = i - (M2 / 2 + 1);
                pb = M2 - 1 - pa;
            }
        } else {
            const int ii = (rp0 == 0) ? i - (M2 + 1) : i;
            const int rl = (rp0 == 0 ? 1 : 0) + ii / M2;  // pair within the CTA
            pa = ii % M2;
            pb = M2 - 1 - pa;
            ra = 2 * rl;
            rb = 2 * rl + 1;
            pr = (rp0 + rl == 0) ? 0 : (M2 + 1) + (rp0 + rl - 1) * M2 + pa;
        }
        const V hc = __ldg(HP + pr), wk = __ldg(a.ttw + pr);
        V      *s1 = s + sq_idx<M2>(ra, pa), *s2 = s + sq_idx<M2>(rb, pb);
        const V Z1 = *s1, Z2 = *s2;
        const V E0 = mkv(Z1, half * (Z1.x + Z2.x), half * (Z1.y - Z2.y));
        const V O0 = mkv(Z1, half * (Z1.y + Z2.y), -half * (Z1.x - Z2.x));
        const T ca = hc.x, cb = hc.y;
        const V wO = cmul(wk, O0);
        const V Ep = mkv(Z1, ca * E0.x + cb * wO.x, ca * E0.y + cb * wO.y);
        const V cE = cmulc(E0, wk);
        const V Op = mkv(Z1, cb * cE.x + ca * O0.x, cb * cE.y + ca * O0.y);
        *s1 = mkv(Z1, Ep.x - Op.y, Ep.y + Op.x);
        if (s2 != s1) *s2 = mkv(Z1, Ep.x + Op.y, -Ep.y + Op.x);
    }
    __syncthreads();
    seq_fft<V, LOG_M2, true>(s, 2 * RP, stw);
    for (int e = threadIdx.x; e < 2 * RP * M2; e += blockDim.x) {
        const int r = e / M2, j2 = e % M2;
        const int k1 = row_of(r);
        const V   v = s[sq_idx<M2>(r, j2)];
        Y[k1 * M2 + j2] = cmulc(v, split_tw(swa, swb, (j2 * k1) & (M - 1)));
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

int mdp_spectrum_H(mdp_context *ctx, const double *h_T, int lambda, int Nn, const double2 *d_tw, double *d_H) {
    DevBuf dT;
    MDP_TRY(dT.alloc(sizeof(double) * lambda));
    MDP_CUDA(cudaMemcpyAsync(dT.p, h_T, sizeof(double) * lambda, cudaMemcpyHostToDevice, ctx->stream));
    spectrum_kernel<<<grid_for(Nn / 2 + 1, 128, 4096), 128, 0, ctx->stream>>>(dT.as<double>(), lambda, Nn, d_tw, d_H);
    MDP_CHECK_LAUNCH(ctx);
    MDP_CUDA(cudaStreamSynchronize(ctx->stream));  // dT is released on return
    return MDP_OK;
}

// Spectrum of the circulant embedding exactly as the reference builds it
// (circ_init_fftw, toeplitz.c:441-470: c[0] = T[0], then for i = 1..lambda-1
// c[i] = T[i] and c[bs-i] = T[i], later writes winning), for any bs:
// F[k] = sum_j c[j] exp(-2 pi i j k / bs), k = 0..bs/2, summed over the nonzero
// entries only (Kahan-compensated FP64), twiddles exp(-2 pi i e / bs), e < bs,
// from long double on the host.
__global__ void circ_spectrum_kernel(const int32_t *__restrict__ jidx, const double *__restrict__ cval, int nnz,
                                     int bs, const double2 *__restrict__ tw, double2 *__restrict__ F) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k <= bs / 2; k += gridDim.x * blockDim.x) {
        double re = 0.0, im = 0.0, cre = 0.0, cim = 0.0;
        for (int t = 0; t < nnz; t++) {
            const double2 w = tw[((int64_t) jidx[t] * k) % bs];
            const double  yr = cval[t] * w.x - cre, yi = cval[t] * w.y - cim;
            const double  tr = re + yr, ti = im + yi;
            cre = (tr - re) - yr;
            cim = (ti - im) - yi;
            re = tr;
            im = ti;
        }
        F[k] = make_double2(re, im);
    }
}

// Twist table of one spectrum in tile position order (see TileArgsT); the
// halves are formed in the tile's precision T from H rounded to T.
template <typename T>
__global__ void twist_pairs_kernel(const double *__restrict__ H, int M, int logM, int ML, int C,
                                   typename CT<T>::V *__restrict__ out) {
    const int npair = ML / 2, n = C * npair + 1;
    const T   half = (T) 0.5;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        int k = M / 2;
        if (e < C * npair) {
            const int r = e / npair, i = e - r * npair;
            k = (int) (__brev((unsigned) (r * ML + 2 * i)) >> (32 - logM));
        }
        const T hk = (T) H[k], hm = (T) H[M - k];
        out[e] = mkv(out[e], half * (hk + hm), half * (hk - hm));
    }
}

// spectrum pairs of the split tiles in their pair order: kidx[e] = k of the
// first element of pair e
template <typename T>
__global__ void split_pairs_kernel(const double *__restrict__ H, int M, const int32_t *__restrict__ kidx, int n,
                                   typename CT<T>::V *__restrict__ out) {
    const T half = (T) 0.5;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const int k = kidx[e];
        const T   hk = (T) H[k], hm = (T) H[M - k];
        out[e] = mkv(out[e], half * (hk + hm), half * (hk - hm));
    }
}

// exp(-2 pi i num / den) in long double, rounded to V
// exp(-2 pi i k / 2^LOG_ROOTS), k < 2^LOG_ROOTS, in long double: computed once per
// process, so that plan tables (all of them W_den^num with den a power of two
// up to 2^LOG_ROOTS) are lookups.  The angle 2 pi num/den equals 2 pi k/2^LOG_ROOTS
// exactly for k = num 2^LOG_ROOTS / den, so a lookup returns the same value
// as evaluating cosl/sinl directly.
constexpr int LOG_ROOTS = 19;
struct RootTable {
    std::vector<long double> re, im;
    RootTable() : re(1u << LOG_ROOTS), im(1u << LOG_ROOTS) {
        const long double two_pi = 2.0L * 3.14159265358979323846264338327950288L;
        for (uint32_t k = 0; k < (1u << LOG_ROOTS); k++) {
            const long double ang = -two_pi * (long double) k / (long double) (1u << LOG_ROOTS);
            re[k] = cosl(ang);
            im[k] = sinl(ang);
        }
    }
};
static const RootTable &root_table() {
    static const RootTable t;  // thread-safe one-time initialisation
    return t;
}
static inline void host_cexp_ld(long double num, long double den, long double *re, long double *im) {
    if (den >= 1.0L && den <= (long double) (1u << LOG_ROOTS) && num >= 0.0L && num == floorl(num)) {
        const uint64_t d = (uint64_t) den, n = (uint64_t) num;
        if ((long double) d == den && (d & (d - 1)) == 0) {
            const uint64_t   k = (n % d) * ((1ull << LOG_ROOTS) / d);
            const RootTable &t = root_table();
            *re = t.re[k];
            *im = t.im[k];
            return;
        }
    }
    const long double ang = -2.0L * 3.14159265358979323846264338327950288L * num / den;
    *re = cosl(ang);
    *im = sinl(ang);
}
void mdp_host_cexp(long double num, long double den, double *re, double *im) {
    long double r, i;
    host_cexp_ld(num, den, &r, &i);
    *re = (double) r;
    *im = (double) i;
}
static inline void host_cexp(long double num, long double den, double2 *o) {
    long double re, im;
    host_cexp_ld(num, den, &re, &im);
    *o = make_double2((double) re, (double) im);
}
static inline void host_cexp(long double num, long double den, float2 *o) {
    long double re, im;
    host_cexp_ld(num, den, &re, &im);
    *o = make_float2((float) re, (float) im);
}

int mdp_circulant_spectrum(mdp_context *ctx, const double *h_T, int lambda, int bs, double *h_F) {
    if (bs < 1 || lambda < 1 || !h_T || !h_F) return MDP_EINVAL;
    std::vector<double> c(bs, 0.0);
    c[0] = h_T[0];
    for (int i = 1; i < lambda; i++) {
        if (i < bs) c[i] = h_T[i];
        if (bs - i >= 0 && bs - i < bs) c[bs - i] = h_T[i];
    }
    std::vector<int32_t> jn;
    std::vector<double>  cn;
    for (int j = 0; j < bs; j++)
        if (c[j] != 0.0) {
            jn.push_back(j);
            cn.push_back(c[j]);
        }
    std::vector<double2> tw(bs);
    for (int e = 0; e < bs; e++) host_cexp(e, bs, &tw[e]);
    const int nf = bs / 2 + 1;
    DevBuf    dj, dc, dt, dF;
    MDP_TRY(dj.alloc(4 * std::max<size_t>(jn.size(), 1)));
    MDP_TRY(dc.alloc(8 * std::max<size_t>(cn.size(), 1)));
    MDP_TRY(dt.alloc(sizeof(double2) * bs));
    MDP_TRY(dF.alloc(sizeof(double2) * nf));
    if (!jn.empty()) {
        MDP_CUDA(cudaMemcpyAsync(dj.p, jn.data(), 4 * jn.size(), cudaMemcpyHostToDevice, ctx->stream));
        MDP_CUDA(cudaMemcpyAsync(dc.p, cn.data(), 8 * cn.size(), cudaMemcpyHostToDevice, ctx->stream));
    }
    MDP_CUDA(cudaMemcpyAsync(dt.p, tw.data(), sizeof(double2) * bs, cudaMemcpyHostToDevice, ctx->stream));
    circ_spectrum_kernel<<<grid_for(nf, 128, 4096), 128, 0, ctx->stream>>>(dj.as<int32_t>(), dc.as<double>(),
                                                                         (int) jn.size(), bs, dt.as<double2>(),
                                                                         dF.as<double2>());
    MDP_CHECK_LAUNCH(ctx);
    MDP_CUDA(cudaMemcpyAsync(h_F, dF.p, sizeof(double2) * nf, cudaMemcpyDeviceToHost, ctx->stream));
    MDP_CUDA(cudaStreamSynchronize(ctx->stream));
    return MDP_OK;
}

// Twiddle tables of a tile plan (ML = 2^log_ml points per CTA, C CTAs, M = C*ML,
// N = 2M): packed local-pass tables, W_M^q for q < ML, and the twist twiddles
// W_N^k in tile position order.
template <typename V>
static int build_tile_twiddles(int log_ml, int C, DevBuf &ltw, DevBuf &twm, DevBuf &ttw) {
    const int ML = 1 << log_ml, M = C * ML, N = 2 * M, npair = ML / 2;
    int       logM = log_ml;
    for (int c = C; c > 1; c >>= 1) logM++;
    std::vector<V> l(ltw_size(log_ml)), m(ML), t(C * npair + 1);
    for (int p = 0; p < ltw_passes(log_ml); p++) {
        const int logL = log_ml - 4 * p, k = logL >= 4 ? 4 : logL, off = ltw_offset(log_ml, p);
        for (int q = 0; q < (1 << (logL - k)); q++) host_cexp(q, (long double) (1 << logL), &l[off + q]);
    }
    for (int q = 0; q < ML; q++) host_cexp(q, M, &m[q]);
    for (int e = 0; e < C * npair + 1; e++) {
        int k = M / 2;
        if (e < C * npair) {
            const unsigned P = (unsigned) ((e / npair) * ML + 2 * (e % npair));
            unsigned       r = 0;
            for (int b = 0; b < logM; b++) r |= ((P >> b) & 1u) << (logM - 1 - b);
            k = (int) r;
        }
        host_cexp(k, N, &t[e]);
    }
    MDP_TRY(ltw.alloc(sizeof(V) * l.size()));
    MDP_TRY(twm.alloc(sizeof(V) * m.size()));
    MDP_TRY(ttw.alloc(sizeof(V) * t.size()));
    MDP_CUDA(cudaMemcpy(ltw.p, l.data(), sizeof(V) * l.size(), cudaMemcpyHostToDevice));
    MDP_CUDA(cudaMemcpy(twm.p, m.data(), sizeof(V) * m.size(), cudaMemcpyHostToDevice));
    MDP_CUDA(cudaMemcpy(ttw.p, t.data(), sizeof(V) * t.size(), cudaMemcpyHostToDevice));
    return MDP_OK;
}

// dynamic shared memory of a tile kernel: the tile plus the staged twiddles
template <typename V>
static size_t tile_smem(int log_ml) {
    return sizeof(V) * ((size_t) (1 << log_ml) + (size_t) ltw_size(log_ml));
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
// Tile kernels that exist, per precision: one CTA of 2^6 .. 2^LMAX complex
// points, or clusters of 2, 4 or 8 CTAs of 2^(LMAX-1) or 2^LMAX points each
// (LMAX = 13 for FP64 and 14 for FP32: 128 KiB of tile per CTA).
template <typename T> struct TileLimits;
template <> struct TileLimits<double> { static constexpr int LMAX = 13; };
template <> struct TileLimits<float> { static constexpr int LMAX = 14; };

template <typename T>
using tile_fn_t = void (*)(TileArgsT<T>);

template <typename T, int L>
static tile_fn_t<T> pick_cluster(int C) {
    switch (C) {
        case 1: return toeplitz_tile_kernel<T, L, 1>;
        case 2: return toeplitz_tile_kernel<T, L, 2>;
        case 4: return toeplitz_tile_kernel<T, L, 4>;
        case 8: return toeplitz_tile_kernel<T, L, 8>;
    }
    return nullptr;
}

template <typename T>
static tile_fn_t<T> pick_kernel(int log_ml, int C) {
    constexpr int LMAX = TileLimits<T>::LMAX;
    if (log_ml == LMAX) return pick_cluster<T, LMAX>(C);
    if (log_ml == LMAX - 1) return pick_cluster<T, LMAX - 1>(C);
    if (C != 1) return nullptr;
    switch (log_ml) {
        case 6: return toeplitz_tile_kernel<T, 6, 1>;
        case 7: return toeplitz_tile_kernel<T, 7, 1>;
        case 8: return toeplitz_tile_kernel<T, 8, 1>;
        case 9: return toeplitz_tile_kernel<T, 9, 1>;
        case 10: return toeplitz_tile_kernel<T, 10, 1>;
        case 11: return toeplitz_tile_kernel<T, 11, 1>;
        case 12: return toeplitz_tile_kernel<T, 12, 1>;
    }
    return nullptr;
}

// split plans: columns per CTA (CW), row pairs per CTA (RP), largest column length
template <typename T> struct SplitShape;
template <> struct SplitShape<float> { static constexpr int CW = 16, RP = 8, M1MAX = 9; };
template <> struct SplitShape<double> { static constexpr int CW = 16, RP = 2, M1MAX = 8; };

struct TileCand {
    int log_ml, C, threads;
    int split = 0, log_m1 = 0, log_m2 = 0;  // split plan: M = 2^log_m1 * 2^log_m2
                                            // (split 2: cluster four-step, M = 2C x 4096)
};

static int64_t cand_N(const TileCand &c) {
    if (c.split == 2) return 2LL * (2 * c.C) * 4096;
    return c.split ? (2LL << (c.log_m1 + c.log_m2)) : 2LL * c.C * (1LL << c.log_ml);
}
// the split plans (1 and 2) keep one output fewer than the band allows, so that
// every window starts on an even row
static int64_t cand_E(const TileCand &c, int lambda) { return cand_N(c) - 2LL * (lambda - 1) - (c.split ? 1 : 0); }

// split plans: columns of 16 <= M1 <= 2^m1max points, rows of 32 <= M2 <= 512
// points; shapes whose transforms end in a lone radix-2 pass (5 or 9 bits) are
// kept only when no other shape gives the same M
static std::vector<std::pair<int, int>> split_shapes(int logM, int m1max) {
    std::vector<std::pair<int, int>> all, good;
    for (int a = 4; a <= m1max; a++) {
        const int b = logM - a;
        if (b < 5 || b > 9) continue;
        all.push_back({a, b});
        if (a % 4 != 1 && b % 4 != 1) good.push_back({a, b});
    }
    return good.empty() ? all : good;
}

static int default_threads(int log_ml) { return std::min(512, std::max(64, (1 << log_ml) / 16)); }

static int ceil_log2_i(int64_t v) {
    int b = 0;
    while ((1LL << b) < v) b++;
    return b;
}

// The cluster four-step tiles are candidates of the automatic choice (the
// autotuner times them with the others).
static const bool g_cluster4_auto = true;

// every launchable configuration whose tile holds the band (E >= 1)
template <typename T>
static std::vector<TileCand> tile_candidates(int lambda) {
    constexpr int         LMAX = TileLimits<T>::LMAX;
    std::vector<TileCand> out;
    for (int lml = 6; lml <= LMAX; lml++)
        for (int C = 1; C <= 8; C <<= 1) {
            if (C > 1 && lml < LMAX - 1) continue;
            const int64_t N = 2LL * C * (1LL << lml);
            if (N - 2LL * (lambda - 1) < 1) continue;
            out.push_back({lml, C, default_threads(lml)});
            if (default_threads(lml) == 512) out.push_back({lml, C, 256});  // 2 CTAs per SM when registers allow
        }
    for (int logM = 9; logM <= 17; logM++)
        for (auto ab : split_shapes(logM, SplitShape<T>::M1MAX)) {
            TileCand c{0, 0, 0, 1, ab.first, ab.second};
            if (cand_E(c, lambda) < 1) continue;
            out.push_back(c);
        }
    if (g_cluster4_auto)
        for (int C = 2; C <= 8; C <<= 1) {  // cluster four-step tiles of 2C x 4096 points
            TileCand c{13, C, 256, 2, 0, 12};
            if (cand_E(c, lambda) < 1 || ninv4_smem<T>(C) > NINV4_SMEM_MAX) continue;
            out.push_back(c);
        }
    return out;
}

// cost model: FFT work per useful output, a penalty for cluster traffic, and
// a penalty when a tile is much larger than the blocks it covers
static double tile_model_cost(const TileCand &c, int lambda, int64_t max_block) {
    const int64_t N = cand_N(c);
    const int64_t E = N - 2LL * (lambda - 1);
    const int     logN = ceil_log2_i(N);
    const double  eff = (double) std::min<int64_t>(E, std::max<int64_t>(max_block, 1));
    double        cost = (double) N / eff * (logN + 3);
    if (c.split == 2) {
        cost *= 0.6;  // the tile stays on chip; paired-lane arithmetic
    } else if (c.split) {
        cost *= 1.3;  // scratch round trips; the timed choice decides
    } else {
        if (c.C > 1) cost += 3.0 * std::log2((double) c.C);
        if (c.threads != default_threads(c.log_ml)) cost *= 1.01;  // ties go to the default launch shape
    }
    if (E < N / 4) cost *= 1.5;
    return cost;
}

template <typename T>
static int build_plan(mdp_context *ctx, mdp_noise *N, mdp_tile_plan &P, const TileCand &c, bool spectra);
template <typename T>
static int launch_tiles(mdp_context *ctx, const mdp_noise *N, const mdp_tile_plan &P, const T *d_in, T *d_out,
                        const double *d_means, int ncols = 1, int64_t col_stride = 0, const int *d_active = nullptr);

// Autotuner.  The plans of a precision are keyed by the band (ceil log2 of
// lambda) and the block length (ceil log2); the first noise operator with a
// new key times every candidate kept by the screen below on a sample of its
// own blocks (at most 2^24 rows, zero data: the tile kernels do the same work
// whatever the values) and the fastest per useful row is kept for the process.
struct TuneKey {
    int prec, lam_bits, blk_bits, device;
    bool operator<(const TuneKey &o) const {
        return std::tie(prec, lam_bits, blk_bits, device) < std::tie(o.prec, o.lam_bits, o.blk_bits, o.device);
    }
};
static std::mutex                   g_tune_mu;
static std::map<TuneKey, TileCand> g_tuned;

static int ceil_log2(int64_t v) {
    int b = 0;
    while ((1LL << b) < v) b++;
    return b;
}

template <typename T>
static int tune_plan(mdp_context *ctx, const mdp_noise *N, const std::vector<TileCand> &cands, TileCand *best) {
    // sample: whole blocks from the start, at most 2^24 rows (one long block is cut there)
    const int64_t    cap = 1LL << 24;
    std::vector<int64_t> idv;
    std::vector<int32_t> len;
    int64_t              rows = 0;
    for (int b = 0; b < N->nb && rows < cap; b++) {
        if (N->h_n[b] <= 0) continue;
        const int64_t n = std::min<int64_t>(N->h_n[b], cap - rows);
        if (n < N->h_n[b] && !idv.empty()) break;
        idv.push_back(rows);
        len.push_back((int32_t) n);
        rows += n;
    }
    if (idv.empty()) return MDP_EUNSUPPORTED;
    mdp_noise S;
    S.nb = (int) idv.size();
    S.lambda = N->lambda;
    S.nrow_end = rows;
    S.h_idv = idv;
    S.h_n = len;
    S.n_spec = 1;
    std::vector<int32_t> spec(S.nb, 0);
    MDP_TRY(S.blk_start.alloc(8 * S.nb));
    MDP_TRY(S.blk_len.alloc(4 * S.nb));
    MDP_TRY(S.blk_spec.alloc(4 * S.nb));
    MDP_TRY(S.means.alloc(8 * S.nb));
    MDP_CUDA(cudaMemcpy(S.blk_start.p, idv.data(), 8 * S.nb, cudaMemcpyHostToDevice));
    MDP_CUDA(cudaMemcpy(S.blk_len.p, len.data(), 4 * S.nb, cudaMemcpyHostToDevice));
    MDP_CUDA(cudaMemcpy(S.blk_spec.p, spec.data(), 4 * S.nb, cudaMemcpyHostToDevice));
    MDP_CUDA(cudaMemset(S.means.p, 0, 8 * S.nb));
    DevBuf in, out;
    MDP_TRY(in.alloc(sizeof(T) * rows));
    MDP_TRY(out.alloc(sizeof(T) * rows));
    MDP_CUDA(cudaMemset(in.p, 0, sizeof(T) * rows));
    cudaEvent_t e0, e1;
    MDP_CUDA(cudaEventCreate(&e0));
    MDP_CUDA(cudaEventCreate(&e1));
    double bestt = 1e300;
    int    rc = MDP_OK;
    for (const TileCand &c : cands) {
        mdp_tile_plan P;
        if ((rc = build_plan<T>(ctx, &S, P, c, false))) break;
        if ((rc = launch_tiles<T>(ctx, &S, P, in.as<T>(), out.as<T>(), S.means.as<double>()))) break;  // warm-up
        float ms = 1e30f;  // best of three trials of two applications
        for (int trial = 0; trial < 3 && rc == MDP_OK; trial++) {
            float t = 0.f;
            cudaEventRecord(e0, ctx->stream);
            for (int r = 0; r < 2 && rc == MDP_OK; r++)
                rc = launch_tiles<T>(ctx, &S, P, in.as<T>(), out.as<T>(), S.means.as<double>());
            cudaEventRecord(e1, ctx->stream);
            if (rc == MDP_OK && (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&t, e0, e1) != cudaSuccess)) {
                rc = MDP_ECUDA;
                mdp_set_error("tile autotuner: %s", cudaGetErrorString(cudaGetLastError()));
            }
            ms = std::min(ms, t);
        }
        if (rc) break;
        if (ms < bestt) {
            bestt = ms;
            *best = c;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return rc;
}

// A plan given by name (mdp_noise_set_plan): "log2_ml,cluster,threads"
// (one-kernel tiles), "s,log_m1,log_m2" (split tiles) or "c,cluster" (cluster
// four-step tiles).
template <typename T>
static int parse_plan(const char *plan, int lambda, TileCand *out) {
    TileCand c{0, 0, 0};
    bool     ok;
    if (plan[0] == 's') {
        c.split = 1;
        ok = sscanf(plan + 1, ",%d,%d", &c.log_m1, &c.log_m2) == 2 && c.log_m1 >= 4 &&
             c.log_m1 <= SplitShape<T>::M1MAX && c.log_m2 >= 5 && c.log_m2 <= 9;
    } else if (plan[0] == 'c') {
        c = TileCand{13, 0, 256, 2, 0, 12};
        ok = sscanf(plan + 1, ",%d", &c.C) == 1 && (c.C == 2 || c.C == 4 || c.C == 8) &&
             ninv4_smem<T>(c.C) <= NINV4_SMEM_MAX;
    } else {
        ok = sscanf(plan, "%d,%d,%d", &c.log_ml, &c.C, &c.threads) == 3 && pick_kernel<T>(c.log_ml, c.C) &&
             c.threads >= 32 && c.threads <= 512 && !(c.threads & 31);
    }
    if (!ok || cand_E(c, lambda) < 1 || 8 * cand_E(c, lambda) < cand_N(c)) {
        mdp_set_error("invalid tile plan '%s' for lambda=%d (or under an eighth of its tile useful)", plan, lambda);
        return MDP_EINVAL;
    }
    *out = c;
    return MDP_OK;
}

// The plan of a precision: the cheapest candidate by the cost model, or
// (tune) the fastest of the screened candidates timed on the device, cached
// per key for the process.  forced > 0 keeps the one-kernel tiles of forced
// real samples only (cost model).
template <typename T>
static int choose_plan(mdp_context *ctx, const mdp_noise *N, TileCand *out, int *tuned, bool tune = true,
                       int64_t forced = 0) {
    const bool f32 = sizeof(T) == 4;
    *tuned = 0;
    std::vector<TileCand> cands = tile_candidates<T>(N->lambda);
    if (forced) {
        std::vector<TileCand> keep;
        for (const TileCand &c : cands)
            if (cand_N(c) == forced && !c.split) keep.push_back(c);
        cands.swap(keep);
    }
    if (cands.empty()) return MDP_EUNSUPPORTED;
    std::sort(cands.begin(), cands.end(), [&](const TileCand &a, const TileCand &b) {
        return tile_model_cost(a, N->lambda, N->max_block) < tile_model_cost(b, N->lambda, N->max_block);
    });
    *out = cands[0];
    if (forced || !tune || cands.size() == 1) return MDP_OK;
    // screen: tiles at least a quarter useful and not longer than twice the block plus the halo
    std::vector<TileCand> screen;
    for (const TileCand &c : cands) {
        const int64_t Nn = cand_N(c), E = cand_E(c, N->lambda);
        if (E * 4 >= Nn && E <= 2 * std::max<int64_t>(N->max_block, 1) + 2LL * N->lambda) screen.push_back(c);
    }
    if (screen.size() <= 1) return MDP_OK;
    const TuneKey key{f32 ? 32 : 64, ceil_log2(N->lambda), ceil_log2(std::max<int64_t>(N->max_block, 1)),
                      ctx->device};
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto                        it = g_tuned.find(key);
    if (it != g_tuned.end()) {
        const TileCand &c = it->second;
        if (cand_E(c, N->lambda) >= 1) {
            *out = c;
            *tuned = 1;
            return MDP_OK;
        }
    }
    TileCand best = screen[0];
    MDP_TRY(tune_plan<T>(ctx, N, screen, &best));
    g_tuned[key] = best;
    *out = best;
    *tuned = 1;
    return MDP_OK;
}

// ---- split plans: kernels, shapes and tables

template <typename T, bool INV>
static const void *pick_cols(int log_m1) {
    constexpr int CW = SplitShape<T>::CW;
    switch (log_m1) {
        case 4: return (const void *) split_cols_kernel<T, 4, CW, INV>;
        case 5: return (const void *) split_cols_kernel<T, 5, CW, INV>;
        case 6: return (const void *) split_cols_kernel<T, 6, CW, INV>;
        case 7: return (const void *) split_cols_kernel<T, 7, CW, INV>;
        case 8: return (const void *) split_cols_kernel<T, 8, CW, INV>;
        case 9:
            if constexpr (SplitShape<T>::M1MAX >= 9) return (const void *) split_cols_kernel<T, 9, CW, INV>;
    }
    return nullptr;
}

template <typename T>
static const void *pick_rows(int log_m2) {
    constexpr int RP = SplitShape<T>::RP;
    switch (log_m2) {
        case 5: return (const void *) split_rows_kernel<T, 5, RP>;
        case 6: return (const void *) split_rows_kernel<T, 6, RP>;
        case 7: return (const void *) split_rows_kernel<T, 7, RP>;
        case 8: return (const void *) split_rows_kernel<T, 8, RP>;
        case 9: return (const void *) split_rows_kernel<T, 9, RP>;
    }
    return nullptr;
}

template <typename V>
static size_t split_cols_smem(int log_m1, int log_m2, int CW) {
    const int M = 1 << (log_m1 + log_m2);
    return sizeof(V) * ((size_t) CW * (1 << log_m1) + ltw_size(log_m1) + std::max(1, M >> 8) + 256);
}
template <typename V>
static size_t split_rows_smem(int log_m1, int log_m2, int RP) {
    const int M = 1 << (log_m1 + log_m2);
    return sizeof(V) * ((size_t) 2 * RP * (1 << log_m2) + ltw_size(log_m2) + std::max(1, M >> 8) + 256);
}

static int rev_bits(int v, int bits) {
    int r = 0;
    for (int b = 0; b < bits; b++) r |= ((v >> b) & 1) << (bits - 1 - b);
    return r;
}

// k of the first element of each pair, in the order split_rows_kernel visits them
static std::vector<int32_t> split_pair_k(int log_m1, int log_m2) {
    const int            M1 = 1 << log_m1, M2 = 1 << log_m2;
    std::vector<int32_t> k;
    k.reserve((size_t) M1 * M2 / 2 + 1);
    for (int i = 0; i < M2 / 2 + 1; i++) {  // row 0
        const int p = (i == M2 / 2) ? 1 : 2 * i;
        k.push_back(M1 * rev_bits(p, log_m2));
    }
    for (int pa = 0; pa < M2 / 2; pa++) k.push_back(M1 / 2 + M1 * rev_bits(pa, log_m2));  // row M1/2
    for (int rp = 1; rp < M1 / 2; rp++)
        for (int pa = 0; pa < M2; pa++) k.push_back(rp + M1 * rev_bits(pa, log_m2));
    return k;
}

template <typename T>
static int build_split_tables(mdp_context *ctx, mdp_noise *N, mdp_tile_plan &P, bool spectra) {
    using V = typename CT<T>::V;
    const int M = 1 << (P.log_m1 + P.log_m2), Nn = 2 * M;
    std::vector<V> l1(ltw_size(P.log_m1)), l2(ltw_size(P.log_m2)), wa(std::max(1, M >> 8)), wb(256);
    auto           pack = [](std::vector<V> &l, int log_l) {
        for (int p = 0; p < ltw_passes(log_l); p++) {
            const int logG = log_l - 4 * p, k = logG >= 4 ? 4 : logG, off = ltw_offset(log_l, p);
            for (int q = 0; q < (1 << (logG - k)); q++) host_cexp(q, (long double) (1 << logG), &l[off + q]);
        }
    };
    pack(l1, P.log_m1);
    pack(l2, P.log_m2);
    for (size_t i = 0; i < wa.size(); i++) host_cexp((long double) (256 * i), M, &wa[i]);
    for (int j = 0; j < 256; j++) host_cexp(j, M, &wb[j]);
    const std::vector<int32_t> kidx = split_pair_k(P.log_m1, P.log_m2);
    const int                  npair = (int) kidx.size();
    std::vector<V>             tt(npair);
    for (int e = 0; e < npair; e++) host_cexp(kidx[e], Nn, &tt[e]);
    MDP_TRY(P.ltw.alloc(sizeof(V) * l1.size()));
    MDP_TRY(P.ltw2.alloc(sizeof(V) * l2.size()));
    MDP_TRY(P.wa.alloc(sizeof(V) * wa.size()));
    MDP_TRY(P.wb.alloc(sizeof(V) * wb.size()));
    MDP_TRY(P.ttw.alloc(sizeof(V) * npair));
    MDP_CUDA(cudaMemcpy(P.ltw.p, l1.data(), sizeof(V) * l1.size(), cudaMemcpyHostToDevice));
    MDP_CUDA(cudaMemcpy(P.ltw2.p, l2.data(), sizeof(V) * l2.size(), cudaMemcpyHostToDevice));
    MDP_CUDA(cudaMemcpy(P.wa.p, wa.data(), sizeof(V) * wa.size(), cudaMemcpyHostToDevice));
    MDP_CUDA(cudaMemcpy(P.wb.p, wb.data(), sizeof(V) * wb.size(), cudaMemcpyHostToDevice));
    MDP_CUDA(cudaMemcpy(P.ttw.p, tt.data(), sizeof(V) * npair, cudaMemcpyHostToDevice));
    MDP_TRY(P.spectra.alloc(sizeof(V) * (size_t) N->n_spec * npair));
    MDP_TRY(P.scratch.alloc(sizeof(V) * (size_t) std::max<int64_t>(P.n_tiles, 1) * M));
    if (spectra) {
        std::vector<double2> tw(M);
        for (int k = 0; k < M; k++) host_cexp(k, Nn, &tw[k]);
        DevBuf tw64, dH, dT, dk;
        MDP_TRY(tw64.alloc(sizeof(double2) * M));
        MDP_TRY(dH.alloc(sizeof(double) * (M + 1)));
        MDP_TRY(dT.alloc(sizeof(double) * N->lambda));
        MDP_TRY(dk.alloc(sizeof(int32_t) * npair));
        MDP_CUDA(cudaMemcpy(tw64.p, tw.data(), sizeof(double2) * M, cudaMemcpyHostToDevice));
        MDP_CUDA(cudaMemcpy(dk.p, kidx.data(), sizeof(int32_t) * npair, cudaMemcpyHostToDevice));
        for (int u = 0; u < N->n_spec; u++) {
            MDP_CUDA(cudaMemcpy(dT.p, N->h_Tuniq.data() + (size_t) u * N->lambda, sizeof(double) * N->lambda,
                                cudaMemcpyHostToDevice));
            spectrum_kernel<<<grid_for(M + 1, 128, 4096), 128, 0, ctx->stream>>>(dT.as<double>(), N->lambda, Nn,
                                                                                tw64.as<double2>(), dH.as<double>());
            MDP_CHECK_LAUNCH(ctx);
            split_pairs_kernel<T><<<grid_for(npair, 256, 1024), 256, 0, ctx->stream>>>(
                    dH.as<double>(), M, dk.as<int32_t>(), npair, P.spectra.as<V>() + (size_t) u * npair);
            MDP_CHECK_LAUNCH(ctx);
            MDP_CUDA(cudaStreamSynchronize(ctx->stream));
        }
    } else {
        MDP_CUDA(cudaMemset(P.spectra.p, 0, sizeof(V) * (size_t) N->n_spec * npair));
    }
    constexpr int CW = SplitShape<T>::CW, RP = SplitShape<T>::RP;
    const size_t  sc = split_cols_smem<V>(P.log_m1, P.log_m2, CW), sr = split_rows_smem<V>(P.log_m1, P.log_m2, RP);
    // A split kernel's shared memory depends on both factors while the kernel
    // only fixes one of them: plans of other operators launch the same kernel
    // with other sizes.  The per-kernel limit is therefore raised to the
    // device's opt-in maximum once, never lowered to this plan's need (which
    // would make the launches of a larger plan built earlier fail).
    int optin = 0;
    MDP_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device));
    if (sc > (size_t) optin || sr > (size_t) optin) return MDP_EUNSUPPORTED;
    for (const void *fn : {pick_cols<T, false>(P.log_m1), pick_cols<T, true>(P.log_m1)}) {
        if (!fn) return MDP_EUNSUPPORTED;
        MDP_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    }
    const void *fr = pick_rows<T>(P.log_m2);
    if (!fr) return MDP_EUNSUPPORTED;
    MDP_CUDA(cudaFuncSetAttribute(fr, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    return MDP_OK;
}

template <typename T>
static int launch_split(mdp_context *ctx, const mdp_noise *N, const mdp_tile_plan &P, const T *d_in, T *d_out,
                        const double *d_means, int ncols, int64_t col_stride, const int *d_active) {
    using V = typename CT<T>::V;
    constexpr int CW = SplitShape<T>::CW, RP = SplitShape<T>::RP;
    const int     M1 = 1 << P.log_m1, M2 = 1 << P.log_m2;
    const int64_t gc = P.n_tiles * (M2 / CW), gr = P.n_tiles * (M1 / 2 / RP);
    if (gc > 0x7fffffffLL || gr > 0x7fffffffLL) return MDP_EUNSUPPORTED;
    const int    tc = split_nt(CW * M1), tr = split_nt(2 * RP * M2);  // the kernels' compile-time thread counts
    const size_t sc = split_cols_smem<V>(P.log_m1, P.log_m2, CW), sr = split_rows_smem<V>(P.log_m1, P.log_m2, RP);
    // the columns of a batch share the scratch array: one column after the other
    for (int c = 0; c < ncols; c++) {
        SplitArgsT<T> a;
        a.vin = d_in + (int64_t) c * col_stride;
        a.vout = d_out + (int64_t) c * col_stride;
        a.Y = P.scratch.as<V>();
        a.tile_start = P.tile_start.as<int64_t>();
        a.tile_block = P.tile_block.as<int32_t>();
        a.blk_start = N->blk_start.as<int64_t>();
        a.blk_len = N->blk_len.as<int32_t>();
        a.blk_spec = N->blk_spec.as<int32_t>();
        a.hpair = P.spectra.as<V>();
        a.ttw = P.ttw.as<V>();
        a.ltw1 = P.ltw.as<V>();
        a.ltw2 = P.ltw2.as<V>();
        a.wa = P.wa.as<V>();
        a.wb = P.wb.as<V>();
        a.means = d_means ? d_means + (int64_t) c * N->nb : nullptr;
        a.lambda = N->lambda;
        a.nb = N->nb;
        a.col_stride = 0;
        a.active = d_active ? d_active + c : nullptr;
        a.log_m1 = P.log_m1;
        a.log_m2 = P.log_m2;
        a.E = P.fft_n - 2 * (N->lambda - 1) - 1;
        a.vec2 = reinterpret_cast<uintptr_t>(a.vin) % (2 * sizeof(T)) == 0;
        void *args[] = {&a};
        MDP_CUDA(cudaLaunchKernel(pick_cols<T, false>(P.log_m1), dim3((unsigned) gc), dim3(tc), args, sc, ctx->stream));
        MDP_CHECK_LAUNCH(ctx);
        MDP_CUDA(cudaLaunchKernel(pick_rows<T>(P.log_m2), dim3((unsigned) gr), dim3(tr), args, sr, ctx->stream));
        MDP_CHECK_LAUNCH(ctx);
        MDP_CUDA(cudaLaunchKernel(pick_cols<T, true>(P.log_m1), dim3((unsigned) gc), dim3(tc), args, sc, ctx->stream));
        MDP_CHECK_LAUNCH(ctx);
    }
    return MDP_OK;
}

// Builds a tile plan: the tile table over the operator's blocks, the twiddle
// tables and (spectra = true) the spectrum pairs of every distinct block row.
template <typename T>
static int build_plan(mdp_context *ctx, mdp_noise *N, mdp_tile_plan &P, const TileCand &c, bool spectra) {
    using V = typename CT<T>::V;
    P.split = c.split;
    P.log_m1 = c.log_m1;
    P.log_m2 = c.log_m2;
    P.log2_ml = c.log_ml;
    P.cluster = c.C;
    P.threads = c.threads;
    const int M = (int) (cand_N(c) / 2);
    P.fft_n = 2 * M;
    // split tiles: one output fewer, so that every window can start on an even row
    const int64_t        E = cand_E(c, N->lambda);
    if (E < 1) return MDP_EUNSUPPORTED;
    std::vector<int64_t> ts;
    std::vector<int32_t> tb;
    for (int b = 0; b < N->nb; b++)
        for (int64_t o = 0; o < N->h_n[b]; o += E) {
            ts.push_back(N->h_idv[b] + o);
            tb.push_back(b);
        }
    P.n_tiles = (int64_t) ts.size();
    if (P.n_tiles * std::max(P.cluster, 1) > 0x7fffffffLL) {
        mdp_set_error("noise operator: %lld tiles exceed one launch", (long long) P.n_tiles);
        return MDP_EUNSUPPORTED;
    }
    MDP_TRY(P.tile_start.alloc(8 * std::max<size_t>(ts.size(), 1)));
    MDP_TRY(P.tile_block.alloc(4 * std::max<size_t>(tb.size(), 1)));
    if (!ts.empty()) {
        MDP_CUDA(cudaMemcpy(P.tile_start.p, ts.data(), 8 * ts.size(), cudaMemcpyHostToDevice));
        MDP_CUDA(cudaMemcpy(P.tile_block.p, tb.data(), 4 * tb.size(), cudaMemcpyHostToDevice));
    }
    if (c.split == 2) {
        MDP_TRY(ninv4_build<T>(ctx, N, P, spectra));
        P.ready = 1;
        return MDP_OK;
    }
    if (c.split) {
        P.cluster = 0;
        P.threads = 0;
        MDP_TRY(build_split_tables<T>(ctx, N, P, spectra));
        P.ready = 1;
        return MDP_OK;
    }
    MDP_TRY(build_tile_twiddles<V>(c.log_ml, c.C, P.ltw, P.twm, P.ttw));
    const int64_t npair = (int64_t) M / 2 + 1;
    MDP_TRY(P.spectra.alloc(sizeof(V) * (size_t) N->n_spec * npair));
    if (spectra) {
        // H[k], k <= M, in FP64 from the twiddles exp(-2 pi i k / N) (long double on the host)
        std::vector<double2> tw(M);
        for (int k = 0; k < M; k++) host_cexp(k, P.fft_n, &tw[k]);
        DevBuf tw64, dH, dT;
        MDP_TRY(tw64.alloc(sizeof(double2) * M));
        MDP_TRY(dH.alloc(sizeof(double) * (M + 1)));
        MDP_TRY(dT.alloc(sizeof(double) * N->lambda));
        MDP_CUDA(cudaMemcpy(tw64.p, tw.data(), sizeof(double2) * M, cudaMemcpyHostToDevice));
        int logM = c.log_ml;
        for (int k = c.C; k > 1; k >>= 1) logM++;
        for (int u = 0; u < N->n_spec; u++) {
            MDP_CUDA(cudaMemcpy(dT.p, N->h_Tuniq.data() + (size_t) u * N->lambda, sizeof(double) * N->lambda,
                                cudaMemcpyHostToDevice));
            spectrum_kernel<<<grid_for(M + 1, 128, 4096), 128, 0, ctx->stream>>>(
                    dT.as<double>(), N->lambda, P.fft_n, tw64.as<double2>(), dH.as<double>());
            MDP_CHECK_LAUNCH(ctx);
            twist_pairs_kernel<T><<<grid_for(npair, 256, 1024), 256, 0, ctx->stream>>>(
                    dH.as<double>(), M, logM, 1 << c.log_ml, c.C, P.spectra.as<V>() + (size_t) u * npair);
            MDP_CHECK_LAUNCH(ctx);
            MDP_CUDA(cudaStreamSynchronize(ctx->stream));
        }
    } else {
        MDP_CUDA(cudaMemset(P.spectra.p, 0, sizeof(V) * (size_t) N->n_spec * npair));
    }
    tile_fn_t<T> fn = pick_kernel<T>(c.log_ml, c.C);
    if (!fn) return MDP_EUNSUPPORTED;
    MDP_CUDA(cudaFuncSetAttribute((const void *) fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int) tile_smem<V>(c.log_ml)));
    if (c.C > 1) MDP_CUDA(cudaFuncSetAttribute((const void *) fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    P.ready = 1;
    return MDP_OK;
}

template <typename T>
static int launch_tiles(mdp_context *ctx, const mdp_noise *N, const mdp_tile_plan &P, const T *d_in, T *d_out,
                        const double *d_means, int ncols, int64_t col_stride, const int *d_active) {
    using V = typename CT<T>::V;
    if (P.n_tiles == 0 || ncols < 1) return MDP_OK;
    if (ncols > 65535) return MDP_EUNSUPPORTED;
    if (P.split == 2) return ninv4_launch<T>(ctx, N, P, d_in, d_out, d_means, ncols, col_stride, d_active);
    if (P.split) return launch_split<T>(ctx, N, P, d_in, d_out, d_means, ncols, col_stride, d_active);
    TileArgsT<T> a;
    a.vin = d_in;
    a.vout = d_out;
    a.tile_start = P.tile_start.as<int64_t>();
    a.tile_block = P.tile_block.as<int32_t>();
    a.blk_start = N->blk_start.as<int64_t>();
    a.blk_len = N->blk_len.as<int32_t>();
    a.blk_spec = N->blk_spec.as<int32_t>();
    a.hpair = P.spectra.as<V>();
    a.ttw = P.ttw.as<V>();
    a.ltw = P.ltw.as<V>();
    a.twm = P.twm.as<V>();
    a.means = d_means;
    a.lambda = N->lambda;
    a.nb = N->nb;
    a.col_stride = col_stride;
    a.active = d_active;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned) (P.n_tiles * P.cluster), (unsigned) ncols);
    cfg.blockDim = dim3(P.threads);
    cfg.dynamicSmemBytes = tile_smem<V>(P.log2_ml);
    cfg.stream = ctx->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = P.cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    MDP_CUDA(cudaLaunchKernelEx(&cfg, pick_kernel<T>(P.log2_ml, P.cluster), a));
    MDP_CHECK_LAUNCH(ctx);
    return MDP_OK;
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
    static std::atomic<uint64_t> next_uid{1};
    mdp_noise  *N = new mdp_noise();
    N->uid = next_uid++;
    N->nb = nb_blocks;
    N->lambda = lambda;
    N->max_block = max_block;
    N->h_idv.assign(h_idv, h_idv + nb_blocks);
    N->h_n.assign(h_n, h_n + nb_blocks);
    N->h_T0.resize(nb_blocks);
    int64_t expect = 0;
    for (int b = 0; b < nb_blocks; b++) {
        N->h_T0[b] = h_T[(size_t) b * lambda];
        if (h_idv[b] != expect) N->covers_all = false;
        expect = h_idv[b] + h_n[b];
    }
    N->nrow_end = expect;
    auto fail = [&](int rc) {
        delete N;
        return rc;
    };
    int rc;
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
    N->n_chunks = (int) cs.size();
    if ((rc = N->chunk_start.alloc(8 * std::max<size_t>(cs.size(), 1))) ||
        (rc = N->chunk_len.alloc(4 * std::max<size_t>(cl.size(), 1))) || (rc = N->blk_chunk0.alloc(4 * nb_blocks)) ||
        (rc = N->blk_nchunk.alloc(4 * nb_blocks)) || (rc = N->partial.alloc(8 * std::max<size_t>(cs.size(), 1))))
        return fail(rc);
    if (!cs.empty()) {
        cudaMemcpy(N->chunk_start.p, cs.data(), 8 * cs.size(), cudaMemcpyHostToDevice);
        cudaMemcpy(N->chunk_len.p, cl.data(), 4 * cl.size(), cudaMemcpyHostToDevice);
    }
    cudaMemcpy(N->blk_chunk0.p, c0.data(), 4 * nb_blocks, cudaMemcpyHostToDevice);
    cudaMemcpy(N->blk_nchunk.p, cn.data(), 4 * nb_blocks, cudaMemcpyHostToDevice);

    if (lambda > 1) {
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
        TileCand c;
        if ((rc = choose_plan<double>(ctx, N, &c, &N->p64.tuned))) {
            if (rc == MDP_EUNSUPPORTED) mdp_set_error("mdp_noise_create: no FFT tile fits lambda=%d", lambda);
            return fail(rc);
        }
        if ((rc = build_plan<double>(ctx, N, N->p64, c, true))) return fail(rc);
    }
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        mdp_set_error("mdp_noise_create: %s", cudaGetErrorString(e));
        return fail(MDP_ECUDA);
    }
    *out = N;
    return MDP_OK;
}

extern "C" void mdp_noise_destroy(mdp_noise *N) { delete N; }

extern "C" int mdp_noise_tile(const mdp_noise *N, int *fft_size, int *cluster_ctas, int64_t *n_tiles) {
    if (!N) return MDP_EINVAL;
    if (fft_size) *fft_size = N->p64.fft_n;
    if (cluster_ctas) *cluster_ctas = N->p64.cluster;
    if (n_tiles) *n_tiles = N->p64.n_tiles;
    return MDP_OK;
}

int mdp_block_means(mdp_context *ctx, const mdp_noise *N, const double *d_v, double *d_means) {
    if (N->n_chunks == 0) {
        MDP_CUDA(cudaMemsetAsync(d_means, 0, 8 * N->nb, ctx->stream));
        return MDP_OK;
    }
    block_partial_sums<double><<<N->n_chunks, 512, 0, ctx->stream>>>(d_v, N->chunk_start.as<int64_t>(),
                                                             N->chunk_len.as<int32_t>(), N->partial.as<double>());
    MDP_CHECK_LAUNCH(ctx);
    block_means_final<<<grid_for(N->nb, 128, 1024), 128, 0, ctx->stream>>>(
            N->partial.as<double>(), N->blk_chunk0.as<int32_t>(), N->blk_nchunk.as<int32_t>(), N->blk_len.as<int32_t>(),
            N->nb, d_means);
    MDP_CHECK_LAUNCH(ctx);
    return MDP_OK;
}

// out = N^-1 in (in != out required); d_means: precomputed block means or nullptr to compute here
int mdp_stbmm_impl(mdp_context *ctx, const mdp_noise *N, const double *d_in, double *d_out, const double *d_means) {
    if (!N->covers_all)
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
    return launch_tiles<double>(ctx, N, N->p64, d_in, d_out, d_means);
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
    if (!A->triplet || !N->covers_all || N->lambda == 1 || N->nrow_end != A->m || N->n_chunks == 0)
        return MDP_EUNSUPPORTED;
    matvec_chunk_sums_kernel<<<N->n_chunks, 512, 0, ctx->stream>>>(A->off.as<int32_t>(), A->values, d_x, d_y,
                                                                   N->chunk_start.as<int64_t>(),
                                                                   N->chunk_len.as<int32_t>(), N->partial.as<double>());
    MDP_CHECK_LAUNCH(ctx);
    block_means_final<<<grid_for(N->nb, 128, 1024), 128, 0, ctx->stream>>>(
            N->partial.as<double>(), N->blk_chunk0.as<int32_t>(), N->blk_nchunk.as<int32_t>(), N->blk_len.as<int32_t>(),
            N->nb, N->means.as<double>());
    MDP_CHECK_LAUNCH(ctx);
    return MDP_OK;
}

// ------------------------------------------------------------------ FP32 operator
int mdp_noise_prepare_fp32(mdp_context *ctx, mdp_noise *N) {
    if (N->p32.ready) return MDP_OK;
    if (N->lambda == 1) {
        N->p32.ready = 1;
        return MDP_OK;
    }
    TileCand c;
    MDP_TRY(choose_plan<float>(ctx, N, &c, &N->p32.tuned));
    return build_plan<float>(ctx, N, N->p32, c, true);
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
    MDP_TRY(mdp_noise_prepare_fp32(ctx, N));
    if (!N->covers_all)
        MDP_CUDA(cudaMemcpyAsync(d_out, d_in, sizeof(float) * N->nrow_end, cudaMemcpyDeviceToDevice, ctx->stream));
    if (N->lambda == 1) {
        dim3 grid(64, N->nb);
        white32_kernel<<<grid, 256, 0, ctx->stream>>>(d_in, d_out, N->blk_start.as<int64_t>(), N->blk_len.as<int32_t>(),
                                                      N->blk_t0.as<double>());
        MDP_CHECK_LAUNCH(ctx);
        return MDP_OK;
    }
    if (!d_means) {
        if (N->n_chunks > 0) {
            block_partial_sums<float><<<N->n_chunks, 512, 0, ctx->stream>>>(
                    d_in, N->chunk_start.as<int64_t>(), N->chunk_len.as<int32_t>(), N->partial.as<double>());
            MDP_CHECK_LAUNCH(ctx);
            block_means_final<<<grid_for(N->nb, 128, 1024), 128, 0, ctx->stream>>>(
                    N->partial.as<double>(), N->blk_chunk0.as<int32_t>(), N->blk_nchunk.as<int32_t>(),
                    N->blk_len.as<int32_t>(), N->nb, N->means.as<double>());
            MDP_CHECK_LAUNCH(ctx);
        }
        d_means = N->means.as<double>();
    }
    return launch_tiles<float>(ctx, N, N->p32, d_in, d_out, d_means);
}

// FP32 N^-1 over a batch of columns (column c at in + c*col_stride, its
// block means at d_means + c*nb, all given); columns with d_active[c] == 0
// are left untouched.  The blocks must cover rows [0, nrow_end) and lambda > 1.
int mdp_stbmm32_batch(mdp_context *ctx, mdp_noise *N, const float *d_in, float *d_out, int ncols,
                      int64_t col_stride, const double *d_means, const int *d_active) {
    if (!N->covers_all || N->lambda == 1 || !d_means) return MDP_EUNSUPPORTED;
    MDP_TRY(mdp_noise_prepare_fp32(ctx, N));
    return launch_tiles<float>(ctx, N, N->p32, d_in, d_out, d_means, ncols, col_stride, d_active);
}

// chunks of the block-mean reduction (65536 rows each, in block order)
int mdp_noise_chunks(const mdp_noise *N, int *n_chunks, const int64_t **d_chunk_start, const int32_t **d_chunk_len,
                     const int32_t **d_blk_chunk0, const int32_t **d_blk_nchunk, int *covers_all) {
    *n_chunks = N->n_chunks;
    *d_chunk_start = N->chunk_start.as<int64_t>();
    *d_chunk_len = N->chunk_len.as<int32_t>();
    *d_blk_chunk0 = N->blk_chunk0.as<int32_t>();
    *d_blk_nchunk = N->blk_nchunk.as<int32_t>();
    *covers_all = N->covers_all ? 1 : 0;
    return MDP_OK;
}

// x4[q] = ((float) x[3q], (float) x[3q+1], (float) x[3q+2], 0): one aligned
// 16-byte gather per sample in the FP32 P instead of three 8-byte ones
__global__ void map_to_float4_kernel(const double *__restrict__ x, float4 *__restrict__ x4, int64_t npix) {
    for (int64_t q = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; q < npix; q += (int64_t) gridDim.x * blockDim.x)
        x4[q] = make_float4((float) x[3 * q], (float) x[3 * q + 1], (float) x[3 * q + 2], 0.0f);
}

__device__ __forceinline__ float p32_row(int32_t o, float w0, float w1, float w2, const float4 *__restrict__ x4) {
    if (o < 0) return 0.0f;
    const float4 m = __ldg(x4 + o / 3);
    return w0 * m.x + w1 * m.y + w2 * m.z;
}

// y32 = P x with the map as FP32 quadruples, fused with FP64 block-mean
// partial sums; four consecutive samples per thread with 16-byte loads of
// their offsets and weights (the chunk's unaligned head and tail one by one)
__global__ void __launch_bounds__(512) matvec32_chunk_sums4_kernel(const int32_t *__restrict__ off,
                                                                   const float *__restrict__ w,
                                                                   const float4 *__restrict__ x4,
                                                                   float *__restrict__ y,
                                                                   const int64_t *__restrict__ chunk_start,
                                                                   const int32_t *__restrict__ chunk_len,
                                                                   double *__restrict__ partial) {
    const int64_t s = chunk_start[blockIdx.x];
    const int64_t e = s + chunk_len[blockIdx.x];
    const int64_t a = min((s + 3) & ~(int64_t) 3, e);  // first multiple of 4 in [s, e]
    const int64_t b = max(e & ~(int64_t) 3, a);         // end of the aligned body
    double        acc = 0.0;
    for (int64_t t = a + 4 * (int64_t) threadIdx.x; t < b; t += 4 * (int64_t) blockDim.x) {
        const int4    o = __ldg(reinterpret_cast<const int4 *>(off + t));
        const float4 *wv = reinterpret_cast<const float4 *>(w + 3 * t);  // 48-byte aligned
        const float4  w0 = __ldg(wv), w1 = __ldg(wv + 1), w2 = __ldg(wv + 2);
        float4        v;
        v.x = p32_row(o.x, w0.x, w0.y, w0.z, x4);
        v.y = p32_row(o.y, w0.w, w1.x, w1.y, x4);
        v.z = p32_row(o.z, w1.z, w1.w, w2.x, x4);
        v.w = p32_row(o.w, w2.y, w2.z, w2.w, x4);
        *reinterpret_cast<float4 *>(y + t) = v;
        acc += (double) v.x + (double) v.y + (double) v.z + (double) v.w;
    }
    // head [s, a) and tail [b, e): fewer than 4 rows each
    const int64_t rest = (a - s) + (e - b);
    if (threadIdx.x < rest) {
        const int64_t t = threadIdx.x < a - s ? s + threadIdx.x : b + (threadIdx.x - (a - s));
        const float   v = p32_row(off[t], w[3 * t], w[3 * t + 1], w[3 * t + 2], x4);
        y[t] = v;
        acc += (double) v;
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    __shared__ double wsum[16];
    if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = (threadIdx.x < (blockDim.x >> 5)) ? wsum[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) partial[blockIdx.x] = v;
    }
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
    if (!A->triplet || !A->w32.p || !N->covers_all || N->lambda == 1 || N->nrow_end != A->m || N->n_chunks == 0)
        return MDP_EUNSUPPORTED;
    const int64_t npix = A->n_map() / 3;
    // the vector loads need 16-byte aligned offsets, weights and output
    const bool vec = (reinterpret_cast<uintptr_t>(A->off.p) % 16 == 0) &&
                     (reinterpret_cast<uintptr_t>(A->w32.p) % 16 == 0) && (reinterpret_cast<uintptr_t>(d_y) % 16 == 0);
    if (vec) {
        MDP_TRY(ctx->ws[12].alloc(sizeof(float4) * (size_t) std::max<int64_t>(npix, 1)));
        float4 *x4 = ctx->ws[12].as<float4>();
        map_to_float4_kernel<<<grid_for(npix, 256, ctx->sm_count * 8), 256, 0, ctx->stream>>>(d_x, x4, npix);
        MDP_CHECK_LAUNCH(ctx);
        matvec32_chunk_sums4_kernel<<<N->n_chunks, 512, 0, ctx->stream>>>(
                A->off.as<int32_t>(), A->w32.as<float>(), x4, d_y, N->chunk_start.as<int64_t>(),
                N->chunk_len.as<int32_t>(), N->partial.as<double>());
    } else {
        matvec32_chunk_sums_kernel<<<N->n_chunks, 512, 0, ctx->stream>>>(
                A->off.as<int32_t>(), A->w32.as<float>(), d_x, d_y, N->chunk_start.as<int64_t>(),
                N->chunk_len.as<int32_t>(), N->partial.as<double>());
    }
    MDP_CHECK_LAUNCH(ctx);
    block_means_final<<<grid_for(N->nb, 128, 1024), 128, 0, ctx->stream>>>(
            N->partial.as<double>(), N->blk_chunk0.as<int32_t>(), N->blk_nchunk.as<int32_t>(), N->blk_len.as<int32_t>(),
            N->nb, N->means.as<double>());
    MDP_CHECK_LAUNCH(ctx);
    return MDP_OK;
}

extern "C" int mdp_noise_set_plan(mdp_context *ctx, mdp_noise *N, int fp32, const char *plan) {
    if (!ctx || !N || !plan) {
        mdp_set_error("mdp_noise_set_plan: invalid arguments");
        return MDP_EINVAL;
    }
    MDP_CUDA(cudaSetDevice(ctx->device));
    if (N->lambda == 1) return MDP_OK;  // white noise: no tiles
    mdp_tile_plan &P = fp32 ? N->p32 : N->p64;
    TileCand       c;
    int            tuned = 0;
    if (!strcmp(plan, "auto") || !strcmp(plan, "model")) {
        MDP_TRY(fp32 ? choose_plan<float>(ctx, N, &c, &tuned, plan[0] == 'a')
                     : choose_plan<double>(ctx, N, &c, &tuned, plan[0] == 'a'));
    } else if (!strncmp(plan, "fft:", 4)) {
        const int64_t n = atoll(plan + 4);
        const int     rc = fp32 ? choose_plan<float>(ctx, N, &c, &tuned, false, n)
                                : choose_plan<double>(ctx, N, &c, &tuned, false, n);
        if (rc) {
            mdp_set_error("mdp_noise_set_plan: no one-kernel tile of %lld samples holds lambda=%d", (long long) n,
                          N->lambda);
            return rc;
        }
    } else {
        MDP_TRY(fp32 ? parse_plan<float>(plan, N->lambda, &c) : parse_plan<double>(plan, N->lambda, &c));
    }
    MDP_CUDA(cudaStreamSynchronize(ctx->stream));  // no launch of the old plan is in flight
    P.reset();
    const int rc = fp32 ? build_plan<float>(ctx, N, P, c, true) : build_plan<double>(ctx, N, P, c, true);
    P.tuned = tuned;
    return rc;
}

extern "C" int mdp_noise_tile_fp32(mdp_context *ctx, mdp_noise *N, int *fft_size, int *cluster_ctas,
                                   int64_t *n_tiles) {
    if (!ctx || !N) return MDP_EINVAL;
    MDP_CUDA(cudaSetDevice(ctx->device));
    MDP_TRY(mdp_noise_prepare_fp32(ctx, N));
    if (fft_size) *fft_size = N->p32.fft_n;
    if (cluster_ctas) *cluster_ctas = N->p32.cluster;
    if (n_tiles) *n_tiles = N->p32.n_tiles;
    return MDP_OK;
}

extern "C" int mdp_prepare_fp32(mdp_context *ctx, mdp_pointing *A, mdp_noise *N) {
    if (!ctx || !A || !N) return MDP_EINVAL;
    MDP_CUDA(cudaSetDevice(ctx->device));
    MDP_TRY(mdp_pointing_prepare_fp32(ctx, A));
    MDP_TRY(mdp_noise_prepare_fp32(ctx, N));
    MDP_CUDA(cudaStreamSynchronize(ctx->stream));
    return MDP_OK;
}

extern "C" int mdp_noise_plan(mdp_context *ctx, mdp_noise *N, int fp32, int *log2_cta_points, int *cluster_ctas,
                              int *threads, int *tuned, int *split_log_m1, int *split_log_m2) {
    if (!ctx || !N) return MDP_EINVAL;
    MDP_CUDA(cudaSetDevice(ctx->device));
    if (fp32) MDP_TRY(mdp_noise_prepare_fp32(ctx, N));
    const mdp_tile_plan &P = fp32 ? N->p32 : N->p64;
    if (log2_cta_points) *log2_cta_points = P.log2_ml;
    if (cluster_ctas) *cluster_ctas = P.cluster;
    if (threads) *threads = P.threads;
    if (tuned) *tuned = P.tuned;
    if (split_log_m1) *split_log_m1 = P.split ? (P.split == 2 ? 1 + (P.cluster == 8 ? 3 : P.cluster == 4 ? 2 : 1) : P.log_m1) : 0;
    if (split_log_m2) *split_log_m2 = P.split ? P.log_m2 : 0;
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
// current, and cached.  It belongs to the device's primary context, the one
// the runtime API uses; another context on the device or a cudaDeviceReset
// would need a new lookup, and neither is supported (documented in the header).
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
    const int64_t need = (int64_t) N->n_chunks + N->nb;
    if (N->lambda > 1 && need > MDP_NOALLOC_SCRATCH_DOUBLES) {
        mdp_set_error("mdp_stbmm_noalloc: %lld scratch doubles needed (%d blocks, %d 65536-row chunks), limit %d",
                      (long long) need, N->nb, N->n_chunks, MDP_NOALLOC_SCRATCH_DOUBLES);
        return MDP_EINVAL;
    }
    MDP_CUDA(cudaSetDevice(ctx->device));
    double *scratch = nullptr;
    MDP_TRY(noalloc_scratch(ctx->device, &scratch));
    if (N->lambda == 1) return mdp_stbmm_impl(ctx, N, d_in, d_out, nullptr);  // no mean removal, no scratch
    double *partial = scratch;                 // [n_chunks], each written before it is read
    double *means = scratch + N->n_chunks;     // [nb], each written before it is read
    if (N->n_chunks > 0) {
        block_partial_sums<double><<<N->n_chunks, 512, 0, ctx->stream>>>(d_in, N->chunk_start.as<int64_t>(),
                                                                 N->chunk_len.as<int32_t>(), partial);
        MDP_CHECK_LAUNCH(ctx);
        block_means_final<<<grid_for(N->nb, 128, 1024), 128, 0, ctx->stream>>>(
                partial, N->blk_chunk0.as<int32_t>(), N->blk_nchunk.as<int32_t>(), N->blk_len.as<int32_t>(), N->nb,
                means);
        MDP_CHECK_LAUNCH(ctx);
    } else {
        MDP_CUDA(cudaMemsetAsync(means, 0, sizeof(double) * N->nb, ctx->stream));
    }
    return mdp_stbmm_impl(ctx, N, d_in, d_out, means);
}
