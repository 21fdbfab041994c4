// Inverse-noise tiles as one thread-block cluster per overlap-save tile: a
// four-step FFT whose two data exchanges go through distributed shared memory,
// so a tile never leaves the chip between its load and its store.
//
// Reference: algebra/src/toeplitz/toeplitz.c:731-865 (stmm_core overlap-save
// tiles), 569-616 (scmm_direct: forward FFT, spectrum product, inverse FFT),
// 441-470 (circ_init_fftw: the circulant embedding whose spectrum H is used).
//
// A tile of N = 2M real samples is packed as M complex points z[j] = x[2j] +
// i x[2j+1], M = M1*M2 with M1 = 2C (C = CTAs of the cluster) and M2 = 4096,
// j = M2*n1 + n2.  Step A (per column n2): the M1-point DFT over n1 in
// registers, times W_M^(n2 k1).  CTA c owns the columns n2 of one M2/C range
// for step A and the two rows k1 = c and M1 - c (rows 0 and C on CTA 0) for
// step B: the M2-point DFT over n2 of each row, as three radix-16 DIF passes
// over shared memory (bit-reversed out).  The rows (k1, M1 - k1) hold every
// pair (k, M - k) of the real-FFT untangle: the untangle, the product with
// the block's real even spectrum and the re-tangle run in one pass, then the
// inverse passes mirror the forward ones.
//
// The two rows of a CTA are the two lanes of every register: one Blackwell
// paired FP32 instruction (add/sub/mul/fma .f32x2) works on both rows (FP64
// runs the same code on pairs of doubles).  A shared-memory position holds
// (x_A, x_B, y_A, y_B): one 16-byte load gives both lanes' real parts and
// both lanes' imaginary parts.  Positions are padded by one entry per 16, so
// the strided accesses of every pass spread over all banks.
//
// Exchanges: after step A each CTA writes the values of row k1 into the CTA
// owning k1 (st through the cluster-mapped address of the owner's shared
// memory); after the inverse row passes each CTA writes each column's values
// back into the CTA owning that column.  Cluster barriers order them.  No TMA
// and no multicast are used; every CTA reads only its own shared memory.
#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <type_traits>
#include <vector>

#include "mdp_internal.cuh"

namespace cg = cooperative_groups;

namespace {

// ------------------------------------------------------------------ lane pairs
template <typename T> struct Pr;
template <> struct Pr<float> {
    unsigned long long v;
};
template <> struct Pr<double> {
    double a, b;
};

__device__ __forceinline__ Pr<float> pmk(float a, float b) {
    Pr<float> r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r.v) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ float plo(Pr<float> p) {
    float a;
    asm("{.reg .f32 t; mov.b64 {%0, t}, %1;}" : "=f"(a) : "l"(p.v));
    return a;
}
__device__ __forceinline__ float phi(Pr<float> p) {
    float b;
    asm("{.reg .f32 t; mov.b64 {t, %0}, %1;}" : "=f"(b) : "l"(p.v));
    return b;
}
__device__ __forceinline__ Pr<float> padd(Pr<float> a, Pr<float> b) {
    Pr<float> r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
    return r;
}
__device__ __forceinline__ Pr<float> psub(Pr<float> a, Pr<float> b) {
    Pr<float> r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
    return r;
}
__device__ __forceinline__ Pr<float> pmul(Pr<float> a, Pr<float> b) {
    Pr<float> r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
    return r;
}
__device__ __forceinline__ Pr<float> pfma(Pr<float> a, Pr<float> b, Pr<float> c) {  // a*b + c
    Pr<float> r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r.v) : "l"(a.v), "l"(b.v), "l"(c.v));
    return r;
}
__device__ __forceinline__ Pr<float> pswap(Pr<float> p) { return pmk(phi(p), plo(p)); }

__device__ __forceinline__ Pr<double> pmk(double a, double b) { return Pr<double>{a, b}; }
__device__ __forceinline__ double plo(Pr<double> p) { return p.a; }
__device__ __forceinline__ double phi(Pr<double> p) { return p.b; }
__device__ __forceinline__ Pr<double> padd(Pr<double> x, Pr<double> y) { return {x.a + y.a, x.b + y.b}; }
__device__ __forceinline__ Pr<double> psub(Pr<double> x, Pr<double> y) { return {x.a - y.a, x.b - y.b}; }
__device__ __forceinline__ Pr<double> pmul(Pr<double> x, Pr<double> y) { return {x.a * y.a, x.b * y.b}; }
__device__ __forceinline__ Pr<double> pfma(Pr<double> x, Pr<double> y, Pr<double> z) {
    return {fma(x.a, y.a, z.a), fma(x.b, y.b, z.b)};
}
__device__ __forceinline__ Pr<double> pswap(Pr<double> p) { return {p.b, p.a}; }

template <typename T> __device__ __forceinline__ Pr<T> pdup(T s) { return pmk(s, s); }
// a compile-time constant on both lanes: plain integer bits for FP32 (the
// compiler may rematerialise it at each use instead of keeping it live)
template <typename T> __device__ __forceinline__ Pr<T> pcst(double v);
template <> __device__ __forceinline__ Pr<float> pcst<float>(double v) {
    const unsigned long long u = __float_as_uint((float) v);
    return Pr<float>{(u << 32) | u};
}
template <> __device__ __forceinline__ Pr<double> pcst<double>(double v) { return Pr<double>{v, v}; }

// complex values on both lanes: x = real parts (lane A, lane B), y = imaginary parts
template <typename T> struct CP {
    Pr<T> x, y;
};

template <typename T> __device__ __forceinline__ CP<T> cpadd(CP<T> a, CP<T> b) { return {padd(a.x, b.x), padd(a.y, b.y)}; }
template <typename T> __device__ __forceinline__ CP<T> cpsub(CP<T> a, CP<T> b) { return {psub(a.x, b.x), psub(a.y, b.y)}; }
// a * w
template <typename T> __device__ __forceinline__ CP<T> cpmul(CP<T> a, CP<T> w) {
    return {psub(pmul(a.x, w.x), pmul(a.y, w.y)), pfma(a.x, w.y, pmul(a.y, w.x))};
}
// a * conj(w)
template <typename T> __device__ __forceinline__ CP<T> cpmulc(CP<T> a, CP<T> w) {
    return {pfma(a.x, w.x, pmul(a.y, w.y)), psub(pmul(a.y, w.x), pmul(a.x, w.y))};
}

// ------------------------------------------------------------------ W_16^m, m < 8
// cos and -sin of 2 pi m / 16 (exact decimal expansions rounded by the compiler)
__host__ __device__ constexpr double w16c(int m) {
    return m == 0 ? 1.0 : m == 1 ? 0.92387953251128675613 : m == 2 ? 0.70710678118654752440
         : m == 3 ? 0.38268343236508977173 : m == 4 ? 0.0 : m == 5 ? -0.38268343236508977173
         : m == 6 ? -0.70710678118654752440 : -0.92387953251128675613;
}
__host__ __device__ constexpr double w16s(int m) {  // imaginary part of W_16^m = -sin(2 pi m / 16)
    return m == 0 ? 0.0 : m == 1 ? -0.38268343236508977173 : m == 2 ? -0.70710678118654752440
         : m == 3 ? -0.92387953251128675613 : m == 4 ? -1.0 : m == 5 ? -0.92387953251128675613
         : m == 6 ? -0.70710678118654752440 : -0.38268343236508977173;
}

// cos and -sin of 2 pi m / 32, m < 16
__host__ __device__ constexpr double w32c(int m) {
    return m == 0 ? 1.0 : m == 1 ? 0.98078528040323044913 : m == 2 ? 0.92387953251128675613
         : m == 3 ? 0.83146961230254523708 : m == 4 ? 0.70710678118654752440 : m == 5 ? 0.55557023301960222474
         : m == 6 ? 0.38268343236508977173 : m == 7 ? 0.19509032201612826785 : m == 8 ? 0.0
         : m == 9 ? -0.19509032201612826785 : m == 10 ? -0.38268343236508977173 : m == 11 ? -0.55557023301960222474
         : m == 12 ? -0.70710678118654752440 : m == 13 ? -0.83146961230254523708 : m == 14 ? -0.92387953251128675613
         : -0.98078528040323044913;
}
__host__ __device__ constexpr double w32s(int m) { return -w32c((m + 24) % 32 < 16 ? (m + 24) % 32 : 32 - (m + 24) % 32); }

// d * W_16^m (CONJ: d * conj(W_16^m)), m known at compile time
template <typename T, int M, bool CONJ>
__device__ __forceinline__ CP<T> mulw16(CP<T> d) {
    if constexpr (M == 0) {
        return d;
    } else if constexpr (M == 4) {
        if constexpr (!CONJ) return {d.y, psub(pcst<T>(0.0), d.x)};  // * -i
        else return {psub(pcst<T>(0.0), d.y), d.x};                   // * i
    } else if constexpr (M == 2 || M == 6) {
        const Pr<T> r = pcst<T>(0.70710678118654752440);
        // W^2 = (1 - i) r, W^6 = (-1 - i) r; conjugates (1 + i) r, (-1 + i) r
        if constexpr (M == 2 && !CONJ) return {pmul(padd(d.x, d.y), r), pmul(psub(d.y, d.x), r)};
        else if constexpr (M == 2 && CONJ) return {pmul(psub(d.x, d.y), r), pmul(padd(d.x, d.y), r)};
        else if constexpr (M == 6 && !CONJ) return {pmul(psub(d.y, d.x), r), pmul(padd(d.x, d.y), pcst<T>(-0.70710678118654752440))};
        else return {pmul(padd(d.x, d.y), pcst<T>(-0.70710678118654752440)), pmul(psub(d.x, d.y), r)};
    } else {
        const CP<T> w{pcst<T>(w16c(M)), pcst<T>(w16s(M))};
        return CONJ ? cpmulc(d, w) : cpmul(d, w);
    }
}

// In-register radix-2 decimation in frequency over R = 2^L points (natural in;
// v[i] = DFT_R(v)[rev_L(i)] out).  Stage j: span h = R/2^(j+1), the difference
// of (i, i + h) times W_{2h}^(i mod 2h) = W_16^((i mod 2h) * 8/h) (R <= 16).
template <typename T, int R, int H>
__device__ __forceinline__ void dif_stage(CP<T> (&v)[R]) {
#pragma unroll
    for (int i = 0; i < R; i++) {
        if ((i % (2 * H)) < H) {
            const CP<T> a = v[i], b = v[i + H];
            v[i] = cpadd(a, b);
            const CP<T> d = cpsub(a, b);
            constexpr int S = 8 / H;
            switch ((i % (2 * H)) * S) {
                case 0: v[i + H] = d; break;
                case 1: v[i + H] = mulw16<T, 1, false>(d); break;
                case 2: v[i + H] = mulw16<T, 2, false>(d); break;
                case 3: v[i + H] = mulw16<T, 3, false>(d); break;
                case 4: v[i + H] = mulw16<T, 4, false>(d); break;
                case 5: v[i + H] = mulw16<T, 5, false>(d); break;
                case 6: v[i + H] = mulw16<T, 6, false>(d); break;
                default: v[i + H] = mulw16<T, 7, false>(d); break;
            }
        }
    }
}
template <typename T, int R>
__device__ __forceinline__ void dif_reg(CP<T> (&v)[R]) {
    if constexpr (R >= 16) dif_stage<T, R, 8>(v);
    if constexpr (R >= 8) dif_stage<T, R, 4>(v);
    if constexpr (R >= 4) dif_stage<T, R, 2>(v);
    if constexpr (R >= 2) dif_stage<T, R, 1>(v);
}
// the mirror: decimation in time with conjugate twiddles, v[i] = X[rev_L(i)]
// in, the unnormalised inverse DFT in natural order out
template <typename T, int R, int H>
__device__ __forceinline__ void dit_stage(CP<T> (&v)[R]) {
#pragma unroll
    for (int i = 0; i < R; i++) {
        if ((i % (2 * H)) < H) {
            const CP<T> a = v[i];
            CP<T>       b;
            constexpr int S = 8 / H;
            switch ((i % (2 * H)) * S) {
                case 0: b = v[i + H]; break;
                case 1: b = mulw16<T, 1, true>(v[i + H]); break;
                case 2: b = mulw16<T, 2, true>(v[i + H]); break;
                case 3: b = mulw16<T, 3, true>(v[i + H]); break;
                case 4: b = mulw16<T, 4, true>(v[i + H]); break;
                case 5: b = mulw16<T, 5, true>(v[i + H]); break;
                case 6: b = mulw16<T, 6, true>(v[i + H]); break;
                default: b = mulw16<T, 7, true>(v[i + H]); break;
            }
            v[i] = cpadd(a, b);
            v[i + H] = cpsub(a, b);
        }
    }
}
template <typename T, int R>
__device__ __forceinline__ void dit_reg(CP<T> (&v)[R]) {
    if constexpr (R >= 2) dit_stage<T, R, 1>(v);
    if constexpr (R >= 4) dit_stage<T, R, 2>(v);
    if constexpr (R >= 8) dit_stage<T, R, 4>(v);
    if constexpr (R >= 16) dit_stage<T, R, 8>(v);
}

__host__ __device__ constexpr int rev_bits_c(int v, int bits) {
    int r = 0;
    for (int b = 0; b < bits; b++) r |= ((v >> b) & 1) << (bits - 1 - b);
    return r;
}
__host__ __device__ constexpr int ilog2_c(int v) { return v <= 1 ? 0 : 1 + ilog2_c(v >> 1); }

// v[i] *= w^rev(i) (CONJ: times conj(w^rev(i))), i = 1..R-1, R = 2^L <= 16,
// the powers from w^1 by a product tree of depth <= 4 (w^2k = (w^k)^2,
// w^(8+j) = w^8 w^j), each applied as soon as it is formed.  The powers are
// named registers, not an array, so that nothing is placed in local memory.
template <typename T, int R, bool CONJ, int K>
__device__ __forceinline__ void apply_pow(CP<T> (&v)[R], const CP<T> &w) {
    constexpr int i = rev_bits_c(K, ilog2_c(R));
    v[i] = CONJ ? cpmulc(v[i], w) : cpmul(v[i], w);
}
template <typename T, int R, bool CONJ>
__device__ __forceinline__ void apply_powers(CP<T> (&v)[R], CP<T> w1) {
    static_assert(R == 2 || R == 4 || R == 8 || R == 16, "radix 2, 4, 8 or 16");
    apply_pow<T, R, CONJ, 1>(v, w1);
    if constexpr (R >= 4) {
        const CP<T> w2 = cpmul(w1, w1);
        apply_pow<T, R, CONJ, 2>(v, w2);
        const CP<T> w3 = cpmul(w2, w1);
        apply_pow<T, R, CONJ, 3>(v, w3);
        if constexpr (R >= 8) {
            const CP<T> w4 = cpmul(w2, w2);
            apply_pow<T, R, CONJ, 4>(v, w4);
            const CP<T> w5 = cpmul(w4, w1);
            apply_pow<T, R, CONJ, 5>(v, w5);
            const CP<T> w6 = cpmul(w4, w2);
            apply_pow<T, R, CONJ, 6>(v, w6);
            const CP<T> w7 = cpmul(w4, w3);
            apply_pow<T, R, CONJ, 7>(v, w7);
            if constexpr (R >= 16) {
                const CP<T> w8 = cpmul(w4, w4);
                apply_pow<T, R, CONJ, 8>(v, w8);
                apply_pow<T, R, CONJ, 9>(v, cpmul(w8, w1));
                apply_pow<T, R, CONJ, 10>(v, cpmul(w8, w2));
                apply_pow<T, R, CONJ, 11>(v, cpmul(w8, w3));
                apply_pow<T, R, CONJ, 12>(v, cpmul(w8, w4));
                apply_pow<T, R, CONJ, 13>(v, cpmul(w8, w5));
                apply_pow<T, R, CONJ, 14>(v, cpmul(w8, w6));
                apply_pow<T, R, CONJ, 15>(v, cpmul(w8, w7));
            }
        }
    }
}

// ------------------------------------------------------------------ geometry
constexpr int LOGM2 = 12;
constexpr int M2 = 1 << LOGM2;  // row length
constexpr int NT = 256;         // threads per CTA
constexpr int NSET = M2 / 16;   // radix-16 sets per row pass (== NT)
static_assert(NSET == NT, "one radix-16 set per thread in the row passes");

__host__ __device__ constexpr int rpos(int p) { return p + (p >> 4); }  // padded row position
__host__ __device__ constexpr int row_entries() { return M2 + M2 / 16; }
template <int C> __host__ __device__ constexpr int col_entries() { return (M2 / C / 2) * (2 * C + 1); }
template <int C> __host__ __device__ constexpr int buf_entries() {
    return row_entries() > col_entries<C>() ? row_entries() : col_entries<C>();
}
// the spectrum values of a CTA's two rows staged in shared memory as lane
// pairs (H[rA + M1 k2], H[rB + M1 k2]), k2 = rev(p), position p at entry
// hpos(p) = p + p / 16 (spread over all banks for the pass's strided reads)
__host__ __device__ constexpr int hpos(int p) { return p + (p >> 4); }
constexpr int HENT = M2 + M2 / 16;  // staged pairs

template <typename T>
struct alignas(16) Ent {  // one shared-memory position: (x_A, x_B), (y_A, y_B)
    Pr<T> x, y;
};

template <typename T>
struct Ninv4Args {
    const T       *vin;
    T             *vout;
    const int64_t *tile_start;  // first output row of each tile
    const int32_t *tile_block;
    const int64_t *blk_start;
    const int32_t *blk_len;
    const int32_t *blk_spec;
    const T       *hrow;        // [n_spec][M + 4]: pairs (H[rA + M1 rev(p)], H[rB + M1 rev(p)]) / (4M) of CTA c
                                //   at 2 (c M2 + p), then H[M] / (4M)
    const Ent<T>  *wbase;       // [C]: (W_N^rA, W_N^rB) of CTA c's rows, as ((re_A, re_B), (im_A, im_B))
    const typename std::conditional<sizeof(T) == 4, float2, double2>::type *wlo;  // [256]: W_2M2^rev8(t)
    const double2 *twM;         // [M2]: W_M^n2 (FP64; rounded to T on use)
    const double2 *tw4096;      // [256]: W_4096^q
    const double  *means;       // [nb] or [ncols][nb]
    int64_t        n_tiles;
    int64_t        ahead;       // tiles between this one and the one whose input is prefetched
    int            lambda;
    int            nb;
    int            E;           // outputs per tile
    int            vec2;        // vin and vout aligned to two samples
    int64_t        col_stride;  // rows between the columns of a batch (blockIdx.y)
    const int     *active;      // [ncols] or nullptr
};

// read-only global loads of table entries
__device__ __forceinline__ Ent<float> ldg_ent(const Ent<float> *p) {
    const ulonglong2 u = __ldg(reinterpret_cast<const ulonglong2 *>(p));
    return Ent<float>{Pr<float>{u.x}, Pr<float>{u.y}};
}
__device__ __forceinline__ Ent<double> ldg_ent(const Ent<double> *p) {
    const double2 a = __ldg(reinterpret_cast<const double2 *>(p)), b = __ldg(reinterpret_cast<const double2 *>(p) + 1);
    return Ent<double>{Pr<double>{a.x, a.y}, Pr<double>{b.x, b.y}};
}
template <typename T>
__device__ __forceinline__ CP<T> ent2cp(Ent<T> e) {
    return {e.x, e.y};
}

// a staged spectrum pair from shared memory, in program order (the untangle
// pass reads one position at a time; letting the compiler hoist all sixteen
// costs registers the kernel does not have)
__device__ __forceinline__ Pr<float> lds_pair(const Pr<float> *p) {
    Pr<float>      r;
    const unsigned a = (unsigned) __cvta_generic_to_shared(p);
    asm volatile("ld.shared.b64 %0, [%1];" : "=l"(r.v) : "r"(a) : "memory");
    return r;
}
__device__ __forceinline__ Pr<double> lds_pair(const Pr<double> *p) {
    Pr<double>     r;
    const unsigned a = (unsigned) __cvta_generic_to_shared(p);
    asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(r.a), "=d"(r.b) : "r"(a) : "memory");
    return r;
}

// cluster barriers (all threads of every CTA of the cluster)
__device__ __forceinline__ void cluster_arrive_relaxed() { asm volatile("barrier.cluster.arrive.relaxed.aligned;\n" ::: "memory"); }
__device__ __forceinline__ void cluster_arrive() { asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory"); }
__device__ __forceinline__ void cluster_wait() { asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory"); }

// forward row pass (radix-16 DIF) at group size G over this CTA's two rows
template <typename T, int G>
__device__ __forceinline__ void row_pass_fwd(Ent<T> *buf, const double2 *tw4096) {
    constexpr int S = G / 16;
    const int     t = threadIdx.x;
    const int     g = t / S, q = t % S;
    const int     base = g * G + q;
    CP<T>         v[16];
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = ent2cp(buf[rpos(base + i * S)]);
    dif_reg<T, 16>(v);
    if constexpr (G > 16) {
        const double2 w = __ldg(tw4096 + q * (4096 / G));
        apply_powers<T, 16, false>(v, CP<T>{pdup<T>((T) w.x), pdup<T>((T) w.y)});
    }
#pragma unroll
    for (int i = 0; i < 16; i++) buf[rpos(base + i * S)] = Ent<T>{v[i].x, v[i].y};
}

// inverse row pass (radix-16 DIT, conjugate twiddles) at group size G; the
// values stay in registers (the caller stores them)
template <typename T, int G>
__device__ __forceinline__ void row_pass_inv_load(const Ent<T> *buf, const double2 *tw4096, CP<T> (&v)[16]) {
    constexpr int S = G / 16;
    const int     t = threadIdx.x;
    const int     g = t / S, q = t % S;
    const int     base = g * G + q;
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = ent2cp(buf[rpos(base + i * S)]);
    if constexpr (G > 16) {
        const double2 w = __ldg(tw4096 + q * (4096 / G));
        apply_powers<T, 16, true>(v, CP<T>{pdup<T>((T) w.x), pdup<T>((T) w.y)});
    }
    dit_reg<T, 16>(v);
}

// ------------------------------------------------------------------ the kernel
template <typename T, int C>
__global__ void __cluster_dims__(C, 1, 1) __launch_bounds__(NT, sizeof(T) == 4 ? 2 : 1) ninv4_kernel(Ninv4Args<T> a) {
    constexpr int M1 = 2 * C;
    constexpr int LOGM1 = ilog2_c(M1);
    constexpr int M = M1 * M2;
    constexpr int NC = M2 / C;       // step-A columns of this CTA
    constexpr int NP = NC / 2;       // column pairs (lanes: u, u + NC/2)
    constexpr int CS = M1 + 1;       // padded stride of a column pair in the column layout
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Ent<T>       *buf = reinterpret_cast<Ent<T> *>(smem_raw);
    cg::cluster_group cluster = cg::this_cluster();
    const int     c = (int) cluster.block_rank();
    if (a.active && !a.active[blockIdx.y]) return;  // uniform over the cluster
    const T      *vin = a.vin + (int64_t) blockIdx.y * a.col_stride;
    T            *vout = a.vout + (int64_t) blockIdx.y * a.col_stride;
    const double *means = a.means ? a.means + (int64_t) blockIdx.y * a.nb : nullptr;
    // every CTA of the cluster is running before any writes into another's shared memory
    cluster_arrive_relaxed();
    // One cluster per tile.  Each CTA asks L2 for its share of the input of the
    // tile one wave later (a.ahead = the clusters resident at once), which a
    // cluster of the next wave will load.
    {
    const int64_t tile = blockIdx.x / C;
    const int     blk = a.tile_block[tile];
    const int64_t bs = a.blk_start[blk];
    const int64_t be = bs + a.blk_len[blk];
    const int64_t t0 = a.tile_start[tile];
    const int64_t ws = (t0 - (a.lambda - 1)) & ~(int64_t) 1;  // even window start
    const bool    inside = ws >= bs && ws + 2LL * M <= be;
    const T       mu = means ? (T) means[blk] : (T) 0;
    if (tile + a.ahead < a.n_tiles) {
        const int64_t nt = tile + a.ahead;
        const int     nblk = a.tile_block[nt];
        const int64_t nbs = a.blk_start[nblk], nbe = nbs + a.blk_len[nblk];
        const int64_t nws = (a.tile_start[nt] - (a.lambda - 1)) & ~(int64_t) 1;
        // M1 runs of 2 NC samples, 128-byte lines; rows kept inside the next tile's block
        constexpr int LINE = 128 / (int) sizeof(T), PER_RUN = 2 * NC / LINE;
        for (int e = threadIdx.x; e < M1 * PER_RUN; e += NT) {
            const int64_t r = nws + 2LL * (M2 * (e / PER_RUN) + c * NC) + (int64_t) (e % PER_RUN) * LINE;
            if (r >= nbs && r < nbe) asm volatile("prefetch.global.L2 [%0];" ::"l"(vin + r));
        }
    }

    // ---- step A: columns (u, u + NC/2) of this CTA, M1-point DFT over n1, times W_M^(n2 k1)
    for (int u = threadIdx.x; u < NP; u += NT) {
        const int n2a = c * NC + u, n2b = n2a + NP;
        CP<T>     v[M1];
#pragma unroll
        for (int n1 = 0; n1 < M1; n1++) {
            const int64_t ra = ws + 2LL * (M2 * n1 + n2a), rb = ws + 2LL * (M2 * n1 + n2b);
            T             xa, ya, xb, yb;
            if (inside && a.vec2) {
                const auto za = __ldg(reinterpret_cast<const typename std::conditional<sizeof(T) == 4, float2, double2>::type *>(vin + ra));
                const auto zb = __ldg(reinterpret_cast<const typename std::conditional<sizeof(T) == 4, float2, double2>::type *>(vin + rb));
                xa = za.x - mu;
                ya = za.y - mu;
                xb = zb.x - mu;
                yb = zb.y - mu;
            } else {
                xa = (ra >= bs && ra < be) ? __ldg(vin + ra) - mu : (T) 0;
                ya = (ra + 1 >= bs && ra + 1 < be) ? __ldg(vin + ra + 1) - mu : (T) 0;
                xb = (rb >= bs && rb < be) ? __ldg(vin + rb) - mu : (T) 0;
                yb = (rb + 1 >= bs && rb + 1 < be) ? __ldg(vin + rb + 1) - mu : (T) 0;
            }
            v[n1] = CP<T>{pmk(xa, xb), pmk(ya, yb)};
        }
        dif_reg<T, M1>(v);  // v[i] = A[k1 = rev(i)]
        {
            const double2 wa = __ldg(a.twM + n2a), wb = __ldg(a.twM + n2b);
            apply_powers<T, M1, false>(v, CP<T>{pmk((T) wa.x, (T) wb.x), pmk((T) wa.y, (T) wb.y)});
        }
        if (u == threadIdx.x) cluster_wait();  // (first iteration) all CTAs started
        // row k1 goes to CTA owner(k1): rows d and M1 - d on CTA d, rows 0 and C on CTA 0
#pragma unroll
        for (int d = 0; d < C; d++) {
            const int     kA = d, kB = (d == 0) ? C : M1 - d;
            const CP<T>   A = v[rev_bits_c(kA, LOGM1)], B = v[rev_bits_c(kB, LOGM1)];
            Ent<T>       *rb = cluster.map_shared_rank(buf, d);
            rb[rpos(n2a)] = Ent<T>{pmk(plo(A.x), plo(B.x)), pmk(plo(A.y), plo(B.y))};
            rb[rpos(n2b)] = Ent<T>{pmk(phi(A.x), phi(B.x)), pmk(phi(A.y), phi(B.y))};
        }
    }
    if (NP <= threadIdx.x) cluster_wait();  // threads without a column pair (none for NP >= NT)
    cluster_arrive();
    cluster_wait();  // every row of this CTA is in place

    // this CTA's two spectrum rows (rA, rB) into shared memory, in flight
    // during the forward row passes
    // (after the row layout: the column layout's tail, used only once the
    // untangle pass has read the spectrum)
    Pr<T> *sH = reinterpret_cast<Pr<T> *>(smem_raw + sizeof(Ent<T>) * row_entries());
    {
        const T *hs = a.hrow + (size_t) a.blk_spec[blk] * (M + 4) + (size_t) 2 * c * M2;
#pragma unroll 1
        for (int p = threadIdx.x; p < M2; p += NT) {
            const unsigned dst = (unsigned) __cvta_generic_to_shared(sH + hpos(p));
            if constexpr (sizeof(T) == 4)
                asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(hs + 2 * p) : "memory");
            else
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(hs + 2 * p) : "memory");
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    }

    // ---- step B forward: three radix-16 DIF passes per row (both rows on the lanes)
    row_pass_fwd<T, 4096>(buf, a.tw4096);
    __syncthreads();
    row_pass_fwd<T, 256>(buf, a.tw4096);
    __syncthreads();
    row_pass_fwd<T, 16>(buf, a.tw4096);
    asm volatile("cp.async.wait_all;\n" ::: "memory");  // this thread's spectrum copies
    __syncthreads();

    // ---- untangle, spectrum product, re-tangle; then the first inverse pass
    {
        const int   t = threadIdx.x;
        // W_N^k of lane r = W_N^r W_2M2^k2, k2 = rev4(i) 2^8 + rev8(t): W_N^r W_2M2^rev8(t) once per
        // thread, times the constant W_32^rev4(i) per position
        const Ent<T> wb = ldg_ent(a.wbase + c);
        const auto   wl = __ldg(a.wlo + t);
        const CP<T>  wt = cpmul(CP<T>{wb.x, wb.y}, CP<T>{pdup<T>(wl.x), pdup<T>(wl.y)});
        const T      hM = (c == 0) ? a.hrow[(size_t) a.blk_spec[blk] * (M + 4) + M] : (T) 0;
        CP<T>        v[16];
#pragma unroll
        for (int i = 0; i < 16; i++) v[i] = ent2cp(buf[rpos(16 * t + i)]);
#pragma unroll
        for (int i = 0; i < 16; i++) {
            const int p = 16 * t + i;
            CP<T>     z2;
            // (H[kA], H[kB]) and (H[M - kA], H[M - kB]): M - k of one lane lies
            // in the other lane's row at position M2-1-p (rows c and M1 - c);
            // on CTA 0 lane B (row C) pairs with itself there, and lane A (row
            // 0) with row 0 at rev(M2 - k2), or H[M] for k2 = 0
            const Pr<T> hk = lds_pair(sH + hpos(p));
            Pr<T>       hm;
            if (c != 0) {
                // lane A pairs with lane B of position M2-1-p and vice versa
                const Ent<T> e = buf[rpos(M2 - 1 - p)];
                z2 = CP<T>{pswap(e.x), pswap(e.y)};
                hm = pswap(lds_pair(sH + hpos(M2 - 1 - p)));
            } else {
                // row 0 (lane A): k2 = rev(p) pairs with M2 - k2; row C (lane B): position M2-1-p
                const int k2 = (int) (__brev((unsigned) p) >> (32 - LOGM2));
                const int pp = (int) (__brev((unsigned) ((M2 - k2) & (M2 - 1))) >> (32 - LOGM2));
                const Ent<T> ea = buf[rpos(pp)], eb = buf[rpos(M2 - 1 - p)];
                z2 = CP<T>{pmk(plo(ea.x), phi(eb.x)), pmk(plo(ea.y), phi(eb.y))};
                hm = pmk(k2 == 0 ? hM : plo(lds_pair(sH + hpos(pp))), phi(lds_pair(sH + hpos(M2 - 1 - p))));
            }
            // (ca, cb) = (H[k] + H[M-k], H[k] - H[M-k]), already / (4M)
            const Ent<T> h{padd(hk, hm), psub(hk, hm)};
            const int    m = rev_bits_c(i, 4);
            const CP<T>  wp = cpmul(wt, CP<T>{pcst<T>(w32c(m)), pcst<T>(w32s(m))});
            const Ent<T> w{wp.x, wp.y};  // W_N^k
            const CP<T>  z1 = v[i];
            const Pr<T>  e0x = padd(z1.x, z2.x), e0y = psub(z1.y, z2.y);
            const Pr<T>  o0x = padd(z1.y, z2.y), o0y = psub(z2.x, z1.x);
            const Pr<T>  wox = psub(pmul(w.x, o0x), pmul(w.y, o0y));
            const Pr<T>  woy = pfma(w.x, o0y, pmul(w.y, o0x));
            const Pr<T>  epx = pfma(h.x, e0x, pmul(h.y, wox));
            const Pr<T>  epy = pfma(h.x, e0y, pmul(h.y, woy));
            const Pr<T>  cex = pfma(w.x, e0x, pmul(w.y, e0y));
            const Pr<T>  cey = psub(pmul(w.x, e0y), pmul(w.y, e0x));
            const Pr<T>  opx = pfma(h.y, cex, pmul(h.x, o0x));
            const Pr<T>  opy = pfma(h.y, cey, pmul(h.x, o0y));
            v[i] = CP<T>{psub(epx, opy), padd(epy, opx)};
        }
        __syncthreads();  // every partner value has been read
        dit_reg<T, 16>(v);
#pragma unroll
        for (int i = 0; i < 16; i++) buf[rpos(16 * t + i)] = Ent<T>{v[i].x, v[i].y};
    }
    __syncthreads();
    {
        CP<T> v[16];
        row_pass_inv_load<T, 256>(buf, a.tw4096, v);
        const int t = threadIdx.x, g = t / 16, q = t % 16;
#pragma unroll
        for (int i = 0; i < 16; i++) buf[rpos(g * 256 + q + i * 16)] = Ent<T>{v[i].x, v[i].y};
    }
    __syncthreads();
    {
        CP<T> v[16];
        row_pass_inv_load<T, 4096>(buf, a.tw4096, v);
        cluster_arrive();
        cluster_wait();  // every CTA has read its rows: the buffers take the column layout
        // value n2 = q + 256 n of rows (kA, kB) -> column n2 of CTA n2 / NC.
        // Columns u and u + NP (the two lanes of the destination's entry) are
        // values n and n + NP/256 of this thread: one 16-byte store per row.
        const int     q = threadIdx.x;
        const int     kA = c, kB = (c == 0) ? C : M1 - c;
        constexpr int DN = NP / 256;
#pragma unroll
        for (int n = 0; n < 16; n++) {
            if ((n / DN) % 2 != 0) continue;  // the upper half of a pair: stored with its lower half
            const int n2 = q + 256 * n;
            const int d = n2 / NC, up = (n2 % NC) % NP;
            Ent<T>   *cb = cluster.map_shared_rank(buf, d);
            const CP<T> lo = v[n], hi = v[n + DN];
            cb[up * CS + kA] = Ent<T>{pmk(plo(lo.x), plo(hi.x)), pmk(plo(lo.y), plo(hi.y))};
            cb[up * CS + kB] = Ent<T>{pmk(phi(lo.x), phi(hi.x)), pmk(phi(lo.y), phi(hi.y))};
        }
    }
    cluster_arrive();
    cluster_wait();  // every column of this CTA is in place

    // ---- step A inverse: times W_M^(-n2 k1), inverse M1-point DFT over k1, store
    const int64_t out_end = min(t0 + (int64_t) a.E, be);
    for (int u = threadIdx.x; u < NP; u += NT) {
        const int n2a = c * NC + u, n2b = n2a + NP;
        CP<T>     v[M1];
        {
            // DIT input order: v[i] holds k1 = rev(i), times conj(W_M^(n2 k1))
#pragma unroll
            for (int i = 0; i < M1; i++) v[i] = ent2cp(buf[u * CS + rev_bits_c(i, LOGM1)]);
            // (last column pair of the thread) this CTA's buffer may take the next tile's rows
            if (u + NT >= NP) cluster_arrive();
            const double2 wa = __ldg(a.twM + n2a), wb = __ldg(a.twM + n2b);
            apply_powers<T, M1, true>(v, CP<T>{pmk((T) wa.x, (T) wb.x), pmk((T) wa.y, (T) wb.y)});
        }
        dit_reg<T, M1>(v);  // v[n1] natural
#pragma unroll
        for (int n1 = 0; n1 < M1; n1++) {
            const int64_t ra = ws + 2LL * (M2 * n1 + n2a), rb = ws + 2LL * (M2 * n1 + n2b);
            const T       xa = plo(v[n1].x), ya = plo(v[n1].y), xb = phi(v[n1].x), yb = phi(v[n1].y);
            if (a.vec2 && ra >= t0 && ra + 1 < out_end) {
                using V2 = typename std::conditional<sizeof(T) == 4, float2, double2>::type;
                *reinterpret_cast<V2 *>(vout + ra) = V2{xa, ya};
            } else {
                if (ra >= t0 && ra < out_end) vout[ra] = xa;
                if (ra + 1 >= t0 && ra + 1 < out_end) vout[ra + 1] = ya;
            }
            if (a.vec2 && rb >= t0 && rb + 1 < out_end) {
                using V2 = typename std::conditional<sizeof(T) == 4, float2, double2>::type;
                *reinterpret_cast<V2 *>(vout + rb) = V2{xb, yb};
            } else {
                if (rb >= t0 && rb < out_end) vout[rb] = xb;
                if (rb + 1 >= t0 && rb + 1 < out_end) vout[rb + 1] = yb;
            }
        }
    }
    }
    cluster_wait();  // matches the arrive after the column reads
}

// ------------------------------------------------------------------ tables
// the staged spectrum table of one spectrum H[0..M] (FP64, N = 2M point
// circulant spectrum), scaled by 1/(4M) (a power of two, exact): for CTA c,
// position p, the lane pair (H[rA + M1 k2], H[rB + M1 k2]), k2 = rev(p), rows
// (rA, rB) = (c, M1 - c), (0, C) on CTA 0, in the order the untangle pass
// reads them; H[M] follows
template <typename T>
__global__ void ninv4_hrow_kernel(const double *__restrict__ H, int C, T *__restrict__ out) {
    const int    M1 = 2 * C, M = M1 * M2;
    const double s = 1.0 / (4.0 * (double) M);
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e <= C * M2; e += gridDim.x * blockDim.x) {
        if (e == C * M2) {
            out[M] = (T) (H[M] * s);
            continue;
        }
        const int c = e / M2, p = e % M2;
        const int rA = c, rB = (c == 0) ? C : M1 - c;
        const int k2 = (int) (__brev((unsigned) p) >> (32 - LOGM2));
        out[2 * e] = (T) (H[rA + M1 * k2] * s);
        out[2 * e + 1] = (T) (H[rB + M1 * k2] * s);
    }
}

}  // namespace

// ------------------------------------------------------------------ host side
static void cexp_ld(long double num, long double den, double *re, double *im) { mdp_host_cexp(num, den, re, im); }

// sets the kernel's shared-memory limit and returns how many clusters fit on the device at once
template <typename T, int C>
static constexpr size_t ninv4_smem_c() {
    const size_t rows = sizeof(Ent<T>) * row_entries() + sizeof(Pr<T>) * HENT;
    return rows > sizeof(Ent<T>) * buf_entries<C>() ? rows : sizeof(Ent<T>) * buf_entries<C>();
}

template <typename T, int C>
static int ninv4_setup_kernel(int *max_clusters) {
    constexpr size_t smem = ninv4_smem_c<T, C>();
    MDP_CUDA(cudaFuncSetAttribute((const void *) ninv4_kernel<T, C>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int) smem));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(C * 256);
    cfg.blockDim = dim3(NT);
    cfg.dynamicSmemBytes = smem;
    int n = 0;
    MDP_CUDA(cudaOccupancyMaxActiveClusters(&n, (void *) ninv4_kernel<T, C>, &cfg));
    if (n < 1) {
        mdp_set_error("cluster four-step tiles: no %d-CTA cluster fits on this device", C);
        return MDP_EUNSUPPORTED;
    }
    *max_clusters = n;
    return MDP_OK;
}

template <typename T>
size_t ninv4_smem(int C) {
    switch (C) {
        case 2: return ninv4_smem_c<T, 2>();
        case 4: return ninv4_smem_c<T, 4>();
        case 8: return ninv4_smem_c<T, 8>();
    }
    return 0;
}

// The plan's tables: P.ttw = the per-CTA twist factors [C] Ent<T>, P.wa = W_{2 M2}^rev8(t) [256]
// (T2), P.twm = W_M^n2 [M2] double2, P.ltw = W_4096^q [256] double2, P.spectra = the staged
// spectrum tables [n_spec][M + 4] T (ninv4_hrow_kernel, from the FP64 spectra H of each
// distinct row when `spectra`, else zero).  Tiles are laid as for the split plans (one
// output fewer than the band allows, even window starts).
template <typename T>
int ninv4_build(mdp_context *ctx, mdp_noise *N, mdp_tile_plan &P, bool spectra) {
    const int C = P.cluster, M1 = 2 * C, M = M1 * M2, Nn = 2 * M;
    if (C != 2 && C != 4 && C != 8) return MDP_EUNSUPPORTED;
    const size_t ne = (size_t) M + 4;  // staged spectrum table entries per spectrum
    // W_N^k of lane r at position p = 16 t + i (k = r + M1 rev(p)) = W_N^r W_{2 M2}^rev8(t) W_32^rev4(i):
    // the per-CTA factors (ttw) and W_{2 M2}^rev8(t) by thread (wa; W_32 are constants)
    {
        std::vector<T> base(4 * C);
        for (int c = 0; c < C; c++) {
            const int rA = c, rB = (c == 0) ? C : M1 - c;
            double    ar, ai, br, bi;
            cexp_ld(rA, Nn, &ar, &ai);
            cexp_ld(rB, Nn, &br, &bi);
            base[4 * c + 0] = (T) ar;
            base[4 * c + 1] = (T) br;
            base[4 * c + 2] = (T) ai;
            base[4 * c + 3] = (T) bi;
        }
        MDP_TRY(P.ttw.alloc(sizeof(Ent<T>) * C));
        MDP_CUDA(cudaMemcpy(P.ttw.p, base.data(), sizeof(T) * base.size(), cudaMemcpyHostToDevice));
        std::vector<T> w(2 * NSET);
        for (int t = 0; t < NSET; t++) {
            double re, im;
            cexp_ld(rev_bits_c(t, 8), 2 * M2, &re, &im);
            w[2 * t] = (T) re;
            w[2 * t + 1] = (T) im;
        }
        MDP_TRY(P.wa.alloc(sizeof(T) * w.size()));
        MDP_CUDA(cudaMemcpy(P.wa.p, w.data(), sizeof(T) * w.size(), cudaMemcpyHostToDevice));
    }
    {
        std::vector<double2> tm(M2), t4(256);
        for (int j = 0; j < M2; j++) cexp_ld(j, M, &tm[j].x, &tm[j].y);
        for (int q = 0; q < 256; q++) cexp_ld(q, 4096, &t4[q].x, &t4[q].y);
        MDP_TRY(P.twm.alloc(sizeof(double2) * M2));
        MDP_TRY(P.ltw.alloc(sizeof(double2) * 256));
        MDP_CUDA(cudaMemcpy(P.twm.p, tm.data(), sizeof(double2) * M2, cudaMemcpyHostToDevice));
        MDP_CUDA(cudaMemcpy(P.ltw.p, t4.data(), sizeof(double2) * 256, cudaMemcpyHostToDevice));
    }
    MDP_TRY(P.spectra.alloc(sizeof(T) * ne * std::max(N->n_spec, 1)));
    if (spectra) {
        // H[k], k <= M, in FP64 from exp(-2 pi i k / N), k < M (long double on the host)
        std::vector<double2> tw(M);
        for (int k = 0; k < M; k++) cexp_ld(k, Nn, &tw[k].x, &tw[k].y);
        DevBuf dH, dtw;
        MDP_TRY(dH.alloc(sizeof(double) * (M + 1)));
        MDP_TRY(dtw.alloc(sizeof(double2) * M));
        MDP_CUDA(cudaMemcpy(dtw.p, tw.data(), sizeof(double2) * M, cudaMemcpyHostToDevice));
        for (int u = 0; u < N->n_spec; u++) {
            MDP_TRY(mdp_spectrum_H(ctx, N->h_Tuniq.data() + (size_t) u * N->lambda, N->lambda, Nn,
                                   dtw.as<double2>(), dH.as<double>()));
            ninv4_hrow_kernel<T><<<grid_for((int64_t) ne, 256, 1024), 256, 0, ctx->stream>>>(
                    dH.as<double>(), C, P.spectra.as<T>() + (size_t) u * ne);
            MDP_CHECK_LAUNCH(ctx);
            MDP_CUDA(cudaStreamSynchronize(ctx->stream));
        }
    } else {
        MDP_CUDA(cudaMemset(P.spectra.p, 0, sizeof(T) * ne * std::max(N->n_spec, 1)));
    }
    switch (C) {
        case 2: MDP_TRY((ninv4_setup_kernel<T, 2>(&P.threads))); break;
        case 4: MDP_TRY((ninv4_setup_kernel<T, 4>(&P.threads))); break;
        case 8: MDP_TRY((ninv4_setup_kernel<T, 8>(&P.threads))); break;
    }
    return MDP_OK;
}

template <typename T>
int ninv4_launch(mdp_context *ctx, const mdp_noise *N, const mdp_tile_plan &P, const T *d_in, T *d_out,
                 const double *d_means, int ncols, int64_t col_stride, const int *d_active) {
    if (P.n_tiles == 0 || ncols < 1) return MDP_OK;
    const int C = P.cluster;
    Ninv4Args<T> a;
    a.vin = d_in;
    a.vout = d_out;
    a.tile_start = P.tile_start.as<int64_t>();
    a.tile_block = P.tile_block.as<int32_t>();
    a.blk_start = N->blk_start.as<int64_t>();
    a.blk_len = N->blk_len.as<int32_t>();
    a.blk_spec = N->blk_spec.as<int32_t>();
    a.hrow = P.spectra.as<T>();
    a.wbase = P.ttw.as<Ent<T>>();
    a.wlo = static_cast<const typename std::conditional<sizeof(T) == 4, float2, double2>::type *>(P.wa.p);
    a.twM = P.twm.as<double2>();
    a.tw4096 = P.ltw.as<double2>();
    a.means = d_means;
    a.n_tiles = P.n_tiles;
    a.lambda = N->lambda;
    a.nb = N->nb;
    a.E = P.fft_n - 2 * (N->lambda - 1) - 1;
    a.vec2 = (reinterpret_cast<uintptr_t>(d_in) % (2 * sizeof(T)) == 0) &&
             (reinterpret_cast<uintptr_t>(d_out) % (2 * sizeof(T)) == 0) && (col_stride % 2 == 0);
    a.col_stride = col_stride;
    a.active = d_active;
    // one cluster per tile; P.threads holds how many clusters are resident at once
    a.ahead = std::max(P.threads, 1);
    const int64_t nblk = P.n_tiles * C;
    if (nblk > 0x7fffffffLL) return MDP_EUNSUPPORTED;
    dim3 grid((unsigned) nblk, (unsigned) ncols);
    size_t smem = ninv4_smem<T>(C);
    switch (C) {
        case 2: ninv4_kernel<T, 2><<<grid, NT, smem, ctx->stream>>>(a); break;
        case 4: ninv4_kernel<T, 4><<<grid, NT, smem, ctx->stream>>>(a); break;
        case 8: ninv4_kernel<T, 8><<<grid, NT, smem, ctx->stream>>>(a); break;
        default: return MDP_EUNSUPPORTED;
    }
    MDP_CHECK_LAUNCH(ctx);
    return MDP_OK;
}

template int    ninv4_build<float>(mdp_context *, mdp_noise *, mdp_tile_plan &, bool);
template int    ninv4_build<double>(mdp_context *, mdp_noise *, mdp_tile_plan &, bool);
template int    ninv4_launch<float>(mdp_context *, const mdp_noise *, const mdp_tile_plan &, const float *, float *,
                                    const double *, int, int64_t, const int *);
template int    ninv4_launch<double>(mdp_context *, const mdp_noise *, const mdp_tile_plan &, const double *, double *,
                                     const double *, int, int64_t, const int *);
template size_t ninv4_smem<float>(int);
template size_t ninv4_smem<double>(int);
