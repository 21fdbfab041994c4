// Internal declarations shared by the midapack_b200 CUDA sources.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <string>
#include <vector>

#include "midapack_b200.h"

#define MDP_SM_COUNT_HINT 148

// ---------------------------------------------------------------- errors
void mdp_set_error(const char *fmt, ...);

#define MDP_CUDA(call)                                                                       \
    do {                                                                                     \
        cudaError_t e__ = (call);                                                            \
        if (e__ != cudaSuccess) {                                                            \
            mdp_set_error("%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e__)); \
            return MDP_ECUDA;                                                                \
        }                                                                                    \
    } while (0)

#define MDP_CHECK_LAUNCH(ctx)                                                                \
    do {                                                                                     \
        (ctx)->launches++;                                                                   \
        cudaError_t e__ = cudaGetLastError();                                                \
        if (e__ != cudaSuccess) {                                                            \
            mdp_set_error("%s:%d kernel launch: %s", __FILE__, __LINE__, cudaGetErrorString(e__)); \
            return MDP_ECUDA;                                                                \
        }                                                                                    \
    } while (0)

#define MDP_TRY(expr)                                                                        \
    do {                                                                                     \
        int rc__ = (expr);                                                                   \
        if (rc__ != MDP_OK) return rc__;                                                     \
    } while (0)

// ---------------------------------------------------------------- device buffer
struct DevBuf {
    void  *p     = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p     = nullptr;
        bytes = 0;
    }
    int alloc(size_t nbytes) {  // (re)allocate when too small; contents are not kept
        if (nbytes <= bytes && p) return MDP_OK;
        release();
        if (nbytes == 0) nbytes = 16;
        cudaError_t e = cudaMalloc(&p, nbytes);
        if (e != cudaSuccess) {
            p = nullptr;
            cudaGetLastError();
            mdp_set_error("cudaMalloc(%zu bytes): %s", nbytes, cudaGetErrorString(e));
            return MDP_ENOMEM;
        }
        bytes = nbytes;
        return MDP_OK;
    }
    template <class T> T *as() const { return static_cast<T *>(p); }
};

// ---------------------------------------------------------------- context
struct mdp_context {
    int          device = 0;
    int          sm_count = MDP_SM_COUNT_HINT;
    cudaStream_t stream = nullptr;
    bool         own_stream = false;
    uint64_t     launches = 0;
    // small reusable scratch
    DevBuf       red;       // reduction partials
    DevBuf       scalars;   // device scalars of the solver
    DevBuf       scratch;   // large temporary (stbmm in place, scans)
    DevBuf       scratch2;
    // work buffers of the solves, kept for the context's next solve (a context
    // runs one solve at a time): no cudaMalloc/cudaFree, which would
    // synchronise the device, in the solves of a serving loop
    DevBuf       ws[13];    // [12]: FP32 (x, y, z, 0) copy of the map gathered by the FP32 P
    double      *h_pinned = nullptr;  // pinned host scalars
    // optional per-operator timing inside the solver (CUDA events on the stream)
    int          profile = 0;
    double       prof_ms[4] = {0, 0, 0, 0};   // P, N^-1, P^T, vector/dot kernels
    int64_t      prof_n[4] = {0, 0, 0, 0};
    cudaEvent_t  ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
};

// ---------------------------------------------------------------- block Jacobi state (solver.cu)
// Kept blocks after the rcond cut, in their original order; block k pairs
// with pixel k of the re-initialised pointing.
struct BJState {
    DevBuf  inv;    // [npix][9] inverse blocks, row-major
    DevBuf  W;      // [npix][9] P^T diag(N^-1) P blocks
    DevBuf  rcond;  // [npix]
    DevBuf  hits;   // [npix]
    int64_t npix = 0;
    int64_t ncut = 0;
};
// ---------------------------------------------------------------- pointing
struct mdp_pt_bins {
    int     valid = 0;
    int     bin_pix = 0;
    int64_t nbins = 0;
    DevBuf  start;   // int64 [nbins+1] offsets into perm
    DevBuf  perm;    // uint32 [valid rows] sample index, grouped by bin
    // slices of the bins' lists (P^T): every bin's list cut into runs of at
    // most slice_len rows (one run for an empty bin); a bin of one slice is
    // written by it, the slices of a longer bin write partial maps that are
    // then summed in slice order.  The partial buffer belongs to the pointing:
    // two P^T of one pointing must not run at the same time.
    int64_t nslices = 0, nmulti = 0, slice_len = 0;
    DevBuf  slice_bin;    // int32 [nslices]
    DevBuf  slice_lo;     // uint32 [nslices] first list entry
    DevBuf  slice_hi;     // uint32 [nslices] one past the last
    DevBuf  slice_out;    // int32 [nslices] -1: the bin's map entries, else its row of `partial`
    DevBuf  multi_bin;    // int32 [nmulti] bins of several slices
    DevBuf  multi_first;  // int32 [nmulti] their first row of `partial`
    DevBuf  multi_n;      // int32 [nmulti] and how many
    DevBuf  partial;      // double [rows][3 bin_pix]
};

struct mdp_pointing {
    int64_t       m = 0;
    int           nnz = 0;
    int           trash_pix = 0;
    int64_t       lcount = 0;
    int           triplet = 0;        // fast layout: one map offset per row
    const double *values = nullptr;   // borrowed [m*nnz]
    DevBuf        lindices;           // int32 [lcount]
    DevBuf        local;              // int32 [m*nnz] (general layout only)
    DevBuf        off;                // int32 [m]: map offset 3q, -1 trash row, -2 cut row (triplet layout)
    // P^T by map bins (triplet layout): samples grouped by bins of bin_pix
    // pixels; bins for one map, and finer bins for the column batches of the
    // multi-RHS solver (bin_pix / columns)
    mdp_pt_bins   bins;
    mdp_pt_bins   mbins;
    DevBuf        w32;                // float [m*3] weights for the FP32 operator (built on first use)
    // block-Jacobi preconditioner of the device-API solves, kept with the
    // pointing: built (and the rcond cut applied) by the first solve, reused
    // by later solves with the same noise operator
    BJState      *bj_cache = nullptr;
    uint64_t      bj_noise_uid = 0;
    ~mdp_pointing() { delete bj_cache; }
    int64_t n_map() const { return lcount - (int64_t) nnz * trash_pix; }
};

// ---------------------------------------------------------------- noise
// One tile plan of the inverse-noise operator: FP64 tiles (the operator of
// the reference) or FP32 tiles (the inner operator of the mixed-precision
// solver).  V = double2 or float2.
struct mdp_tile_plan {
    int     ready = 0;
    int     split = 0;     // 0: one kernel (one CTA or cluster per tile); 1: three-kernel four-step FFT;
                           // 2: cluster four-step (ninv4.cu: C = cluster CTAs, M = 2C x 4096 points)
    int     log_m1 = 0, log_m2 = 0;  // split: M = 2^log_m1 * 2^log_m2 complex points per tile
    DevBuf  scratch;       // split: [n_tiles][M] complex work array
    DevBuf  ltw2, wa, wb;  // split: row-pass twiddles, W_M factor tables
    int     log2_ml = 0;   // per-CTA complex points = 2^log2_ml
    int     cluster = 1;   // CTAs per tile
    int     threads = 0;   // threads per CTA
    int     fft_n = 0;     // real FFT size N = 2 * cluster * 2^log2_ml
    int     tuned = 0;     // 1 when picked by timing the candidates on the device
    int64_t n_tiles = 0;
    DevBuf  tile_start;    // int64 [n_tiles] first output row (global)
    DevBuf  tile_block;    // int32 [n_tiles]
    DevBuf  spectra;       // V [n_spec][N/4+1]: spectrum pairs in tile position order
    DevBuf  ltw, twm, ttw; // packed local-pass, cross-CTA and twist twiddles
    void reset() {         // back to an unbuilt plan, device buffers released
        ready = split = log_m1 = log_m2 = log2_ml = threads = fft_n = tuned = 0;
        cluster = 1;
        n_tiles = 0;
        for (DevBuf *b : {&scratch, &ltw2, &wa, &wb, &tile_start, &tile_block, &spectra, &ltw, &twm, &ttw})
            b->release();
    }
};

struct mdp_noise {
    uint64_t             uid = 0;        // unique per created operator
    int                  nb = 0;
    int                  lambda = 0;
    int64_t              nrow_end = 0;   // max(idv+n)
    int64_t              max_block = 0;
    std::vector<int64_t> h_idv;
    std::vector<int32_t> h_n;
    std::vector<double>  h_T0;           // diagonal of each block
    DevBuf               blk_start;      // int64 [nb]
    DevBuf               blk_len;        // int32 [nb]
    DevBuf               blk_spec;       // int32 [nb] index of the block's spectrum
    DevBuf               blk_t0;         // double [nb] T_block[0]
    DevBuf               means;          // double [nb]
    int                  n_spec = 0;
    std::vector<double>  h_Tuniq;        // [n_spec][lambda] distinct first rows
    mdp_tile_plan        p64;            // built at creation
    mdp_tile_plan        p32;            // built on first FP32 use
    // 65536-row chunks of the deterministic block-mean reduction
    int                  n_chunks = 0;
    bool                 covers_all = true;  // blocks tile rows [0, nrow_end) without holes
    DevBuf               chunk_start;    // int64 [n_chunks]
    DevBuf               chunk_len;      // int32 [n_chunks]
    DevBuf               blk_chunk0;     // int32 [nb] first chunk of each block
    DevBuf               blk_nchunk;     // int32 [nb]
    DevBuf               partial;        // double [n_chunks] chunk sums
};

// ---------------------------------------------------------------- two-level preconditioner (twolevel.cu)
// M g = BJ_inv (g - AZ qtx) + Z qtx with qtx = Em1 Z^T g, Em1 the pseudo-inverse
// of E = Z^T AZ and AZ = P^T N^-1 P Z.
#define MDP_TL_MAX_ZN 128
#define MDP_TL_BLOCKS 296
struct mdp_twolevel {
    int     precond = 0;   // 1: a priori columns (build_Z), 2: Ritz vectors (Lanczos)
    int     zn = 0;        // deflation columns
    int64_t n = 0;         // map unknowns
    DevBuf  Z, AZ;         // double [zn][n]
    DevBuf  Em1;           // double [zn][zn] row-major
    DevBuf  qtx;           // double [zn]
    DevBuf  part;          // double [zn][MDP_TL_BLOCKS] partial dot products
    std::vector<double> h_Em1;
};
int mdp_twolevel_build(mdp_context *ctx, mdp_pointing *A, const mdp_noise *N, int precond, int zn,
                       const double *d_g0, mdp_twolevel *tl);
int mdp_twolevel_qtx(mdp_context *ctx, const mdp_twolevel *tl, const double *d_g);
int mdp_apply_op_impl(mdp_context *ctx, mdp_pointing *A, const mdp_noise *N, const double *d_h, double *d_q);
int mdp_gls_rhs(mdp_context *ctx, mdp_pointing *A, const mdp_noise *N, const double *d_signal, const double *d_noise,
                double *d_g);
int mdp_bj_build(mdp_context *ctx, mdp_pointing *A, const mdp_noise *N, BJState *bj);
int mdp_ecg_run(mdp_context *ctx, mdp_pointing *A, const mdp_noise *N, const double *inv, int64_t npix,
                const double *d_signal, const double *d_noise, const mdp_ecg_params *prm, double *d_x,
                double *h_res_rel, mdp_solve_info *info);
int mdp_bj_cached(mdp_context *ctx, mdp_pointing *A, const mdp_noise *N, const BJState **bj);
// tpl != nullptr: MTmap's weighting W - W T B T^T W (templates.cu) in place of N^-1
int mdp_pcg_run(mdp_context *ctx, mdp_pointing *A, const mdp_noise *N, const double *inv, int64_t npix,
                const double *d_signal, const double *d_noise, const mdp_solve_params *params, double *d_x,
                double *h_res_rel, mdp_solve_info *info, const mdp_twolevel *tl = nullptr,
                const mdp_templates *tpl = nullptr);
int mdp_pointing_create_ex(mdp_context *ctx, int64_t m, int nnz, const int32_t *d_g, const double *d_values,
                           int32_t *d_local_out, mdp_pointing **out);
int mdp_matvec_launch(mdp_context *ctx, const mdp_pointing *A, const double *d_x, double *d_y);
int mdp_trmatvec_launch(mdp_context *ctx, const mdp_pointing *A, const double *d_y, double *d_x);

// ---------------------------------------------------------------- helpers (pointing.cu / reduce)
int mdp_exclusive_scan_u32(mdp_context *ctx, const uint32_t *d_in, uint32_t *d_out, int64_t n,
                           uint32_t *h_total);
int mdp_stbmm_impl(mdp_context *ctx, const mdp_noise *N, const double *d_in, double *d_out,
                   const double *d_means_or_null);
int mdp_block_means(mdp_context *ctx, const mdp_noise *N, const double *d_v, double *d_means);
// spectrum of the reference's circulant embedding of T (circ_init_fftw), bs/2+1 complex into h_F
int mdp_circulant_spectrum(mdp_context *ctx, const double *h_T, int lambda, int bs, double *h_F);
// H[k], k = 0..Nn/2, of the Nn-point circulant embedding of the band T (device,
// FP64); d_tw = exp(-2 pi i k / Nn), k < Nn/2
int mdp_spectrum_H(mdp_context *ctx, const double *h_T, int lambda, int Nn, const double2 *d_tw, double *d_H);
// exp(-2 pi i num / den) from long double (a table lookup for power-of-two den <= 2^19)
void mdp_host_cexp(long double num, long double den, double *re, double *im);
// cluster four-step tiles of N^-1 (ninv4.cu): tables of a plan, launch
template <typename T>
int ninv4_build(mdp_context *ctx, mdp_noise *N, mdp_tile_plan &P, bool spectra);
template <typename T>
int ninv4_launch(mdp_context *ctx, const mdp_noise *N, const mdp_tile_plan &P, const T *d_in, T *d_out,
                 const double *d_means, int ncols, int64_t col_stride, const int *d_active);
// dynamic shared memory of a cluster four-step CTA, and the largest a B200 CTA may use
template <typename T>
size_t ninv4_smem(int C);
#define NINV4_SMEM_MAX ((size_t) 227 * 1024)
int mdp_matvec_blockmeans(mdp_context *ctx, const mdp_pointing *A, const mdp_noise *N, const double *d_x,
                          double *d_y);
// FP32 operator pieces (mixed precision)
int mdp_noise_prepare_fp32(mdp_context *ctx, mdp_noise *N);
int mdp_stbmm_impl32(mdp_context *ctx, mdp_noise *N, const float *d_in, float *d_out, const double *d_means);
int mdp_stbmm32_batch(mdp_context *ctx, mdp_noise *N, const float *d_in, float *d_out, int ncols,
                      int64_t col_stride, const double *d_means, const int *d_active);
int mdp_noise_chunks(const mdp_noise *N, int *n_chunks, const int64_t **d_chunk_start, const int32_t **d_chunk_len,
                     const int32_t **d_blk_chunk0, const int32_t **d_blk_nchunk, int *covers_all);
int mdp_pointing_prepare_fp32(mdp_context *ctx, mdp_pointing *A);
int mdp_matvec32_blockmeans(mdp_context *ctx, const mdp_pointing *A, const mdp_noise *N, const double *d_x,
                            float *d_y);
int mdp_trmatvec32_launch(mdp_context *ctx, mdp_pointing *A, const float *d_y, double *d_x);
int mdp_matvec32_launch(mdp_context *ctx, mdp_pointing *A, const double *d_x, float *d_y);

inline int grid_for(int64_t n, int threads, int max_blocks = 148 * 16) {
    int64_t b = (n + threads - 1) / threads;
    if (b > max_blocks) b = max_blocks;
    if (b < 1) b = 1;
    return (int) b;
}

// sample lists of the pointing's rows grouped by bins of bin_pix pixels
int mdp_build_bins(mdp_context *ctx, mdp_pointing *A, int bin_pix, mdp_pt_bins *B, bool slices = false);
// P^T and the block-Jacobi sums run over bins of MDP_PT_BIN_PIX pixels when the
// pointing is a triplet pointing of 2^20 rows or more (pointing.cu)
#define MDP_PT_BIN_PIX 256
bool mdp_pointing_binned(const mdp_pointing *A);
int  mdp_pointing_bins(mdp_context *ctx, mdp_pointing *A);  // builds A->bins when missing
