// Pointing matrix P on the device: index compression (MatInit/MatLocalShape),
// y = P x (MatVecProd) and x = P^T y (TrMatVecProd), plus the context, error
// handling and the device-wide scan they use.
//
// Reference: algebra/src/mapmat/mapmat.c:54-73 (MatInit), 496-521
// (MatLocalShape), 704-729 (MatVecProd), 819-859 (TrMatVecProd);
// algebra/src/mapmat/csort.c:111-135 (counting_sort), cindex.c:34-42,102-116
// (sindex/dichotomy).
#include <cstdarg>
#include <cstring>

#include "mdp_internal.cuh"

// ============================================================== errors
static thread_local char g_err[512] = "";

void mdp_set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

extern "C" const char *mdp_last_error(void) { return g_err; }

extern "C" const char *mdp_strerror(int code) {
    switch (code) {
        case MDP_OK: return "ok";
        case MDP_EINVAL: return "invalid argument";
        case MDP_ENOMEM: return "out of memory";
        case MDP_ECUDA: return "CUDA error";
        case MDP_EUNSUPPORTED: return "unsupported input";
        case MDP_ENAN: return "NaN or Inf in a reduction";
        case MDP_ETIMEOUT: return "device wait timed out";
        case MDP_ENOCONV: return "fit did not converge";
        default: return "unknown error";
    }
}

// ============================================================== context
extern "C" int mdp_context_create(int device, mdp_context **out) {
    if (!out) return MDP_EINVAL;
    *out = nullptr;
    int ndev = 0;
    MDP_CUDA(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) {
        mdp_set_error("device %d not present (%d devices)", device, ndev);
        return MDP_EINVAL;
    }
    MDP_CUDA(cudaSetDevice(device));
    mdp_context *ctx = new mdp_context();
    ctx->device = device;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) == cudaSuccess) ctx->sm_count = prop.multiProcessorCount;
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete ctx;
        mdp_set_error("cudaStreamCreate failed");
        return MDP_ECUDA;
    }
    ctx->own_stream = true;
    if (cudaMallocHost(&ctx->h_pinned, 4096) != cudaSuccess) {
        cudaStreamDestroy(ctx->stream);
        delete ctx;
        mdp_set_error("cudaMallocHost failed");
        return MDP_ENOMEM;
    }
    *out = ctx;
    return MDP_OK;
}

extern "C" int mdp_context_trim(mdp_context *ctx) {
    if (!ctx) return MDP_EINVAL;
    MDP_CUDA(cudaSetDevice(ctx->device));
    MDP_CUDA(cudaStreamSynchronize(ctx->stream));
    for (DevBuf &b : ctx->ws) b.release();
    ctx->scratch.release();
    ctx->scratch2.release();
    return MDP_OK;
}

extern "C" void mdp_context_destroy(mdp_context *ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
    if (ctx->h_pinned) cudaFreeHost(ctx->h_pinned);
    for (int i = 0; i < 5; i++)
        if (ctx->ev[i]) cudaEventDestroy(ctx->ev[i]);
    delete ctx;
}

extern "C" int mdp_context_set_stream(mdp_context *ctx, void *cuda_stream) {
    if (!ctx) return MDP_EINVAL;
    MDP_CUDA(cudaStreamSynchronize(ctx->stream));
    if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
    if (cuda_stream) {
        ctx->stream     = (cudaStream_t) cuda_stream;
        ctx->own_stream = false;
    } else {
        MDP_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
        ctx->own_stream = true;
    }
    return MDP_OK;
}

extern "C" void *mdp_context_stream(mdp_context *ctx) { return ctx ? (void *) ctx->stream : nullptr; }

extern "C" int mdp_synchronize(mdp_context *ctx) {
    if (!ctx) return MDP_EINVAL;
    MDP_CUDA(cudaStreamSynchronize(ctx->stream));
    return MDP_OK;
}

extern "C" uint64_t mdp_launch_count(const mdp_context *ctx) { return ctx ? ctx->launches : 0; }

extern "C" int mdp_profile_enable(mdp_context *ctx, int enable) {
    if (!ctx) return MDP_EINVAL;
    if (enable && !ctx->ev[0])
        for (int i = 0; i < 5; i++) MDP_CUDA(cudaEventCreate(&ctx->ev[i]));
    ctx->profile = enable ? 1 : 0;
    for (int i = 0; i < 4; i++) {
        ctx->prof_ms[i] = 0.0;
        ctx->prof_n[i] = 0;
    }
    return MDP_OK;
}

extern "C" int mdp_profile_read(const mdp_context *ctx, double *ms, int64_t *count) {
    if (!ctx) return MDP_EINVAL;
    for (int i = 0; i < 4; i++) {
        if (ms) ms[i] = ctx->prof_ms[i];
        if (count) count[i] = ctx->prof_n[i];
    }
    return MDP_OK;
}

// ============================================================== device-wide exclusive scan (uint32)
// Three phases: per-tile totals, scan of the totals (recursively), rescan of
// each tile with its offset.  Tiles of SCAN_TILE elements, one CTA per tile.
#define SCAN_THREADS 256
#define SCAN_ITEMS 16
#define SCAN_TILE (SCAN_THREADS * SCAN_ITEMS)

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t *total) {
    __shared__ uint32_t warp_tot[SCAN_THREADS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t  x    = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = (lane < SCAN_THREADS / 32) ? warp_tot[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < SCAN_THREADS / 32) warp_tot[lane] = w;
    }
    __syncthreads();
    uint32_t before = (warp > 0 ? warp_tot[warp - 1] : 0u) + x - v;
    if (total) *total = warp_tot[SCAN_THREADS / 32 - 1];
    __syncthreads();
    return before;
}

__global__ void scan_tile_sums(const uint32_t *__restrict__ in, uint32_t *__restrict__ sums, int64_t n) {
    int64_t  base = (int64_t) blockIdx.x * SCAN_TILE + (int64_t) threadIdx.x * SCAN_ITEMS;
    uint32_t s    = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++)
        if (base + i < n) s += in[base + i];
    uint32_t tot;
    block_exclusive_scan(s, &tot);
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

__global__ void scan_tile_apply(const uint32_t *__restrict__ in, uint32_t *__restrict__ out,
                                const uint32_t *__restrict__ offs, int64_t n) {
    int64_t  base = (int64_t) blockIdx.x * SCAN_TILE + (int64_t) threadIdx.x * SCAN_ITEMS;
    uint32_t v[SCAN_ITEMS];
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++) {
        v[i] = (base + i < n) ? in[base + i] : 0u;
        s += v[i];
    }
    uint32_t run = block_exclusive_scan(s, nullptr) + (offs ? offs[blockIdx.x] : 0u);
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++) {
        if (base + i < n) out[base + i] = run;
        run += v[i];
    }
}

int mdp_exclusive_scan_u32(mdp_context *ctx, const uint32_t *d_in, uint32_t *d_out, int64_t n,
                           uint32_t *h_total) {
    if (n <= 0) {
        if (h_total) *h_total = 0;
        return MDP_OK;
    }
    int64_t ntiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (ntiles == 1) {
        scan_tile_apply<<<1, SCAN_THREADS, 0, ctx->stream>>>(d_in, d_out, nullptr, n);
        MDP_CHECK_LAUNCH(ctx);
    } else {
        DevBuf sums, sums_scan;
        MDP_TRY(sums.alloc(sizeof(uint32_t) * ntiles));
        MDP_TRY(sums_scan.alloc(sizeof(uint32_t) * ntiles));
        scan_tile_sums<<<(unsigned) ntiles, SCAN_THREADS, 0, ctx->stream>>>(d_in, sums.as<uint32_t>(), n);
        MDP_CHECK_LAUNCH(ctx);
        MDP_TRY(mdp_exclusive_scan_u32(ctx, sums.as<uint32_t>(), sums_scan.as<uint32_t>(), ntiles, nullptr));
        scan_tile_apply<<<(unsigned) ntiles, SCAN_THREADS, 0, ctx->stream>>>(d_in, d_out, sums_scan.as<uint32_t>(),
                                                                              n);
        MDP_CHECK_LAUNCH(ctx);
        MDP_CUDA(cudaStreamSynchronize(ctx->stream));  // sums freed at scope exit
    }
    if (h_total) {
        uint32_t last_out = 0, last_in = 0;
        MDP_CUDA(cudaMemcpyAsync(&last_out, d_out + n - 1, 4, cudaMemcpyDeviceToHost, ctx->stream));
        MDP_CUDA(cudaMemcpyAsync(&last_in, d_in + n - 1, 4, cudaMemcpyDeviceToHost, ctx->stream));
        MDP_CUDA(cudaStreamSynchronize(ctx->stream));
        *h_total = last_out + last_in;
    }
    return MDP_OK;
}

// ============================================================== index compression
__global__ void minmax_kernel(const int32_t *__restrict__ g, int64_t n, int32_t *__restrict__ out_min,
                              int32_t *__restrict__ out_max) {
    int32_t mn = INT32_MAX, mx = INT32_MIN;
    for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x) {
        int32_t v = g[i];
        mn        = min(mn, v);
        mx        = max(mx, v);
    }
    for (int o = 16; o > 0; o >>= 1) {
        mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    __shared__ int32_t smn[32], smx[32];
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        smn[warp] = mn;
        smx[warp] = mx;
    }
    __syncthreads();
    if (warp == 0) {
        int nw = blockDim.x >> 5;
        mn     = lane < nw ? smn[lane] : INT32_MAX;
        mx     = lane < nw ? smx[lane] : INT32_MIN;
        for (int o = 16; o > 0; o >>= 1) {
            mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
            mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        }
        if (lane == 0) {
            out_min[blockIdx.x] = mn;
            out_max[blockIdx.x] = mx;
        }
    }
}

__global__ void mark_kernel(const int32_t *__restrict__ g, int64_t n, int32_t gmin, uint32_t *__restrict__ flags) {
    for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x)
        flags[(int64_t) g[i] - gmin] = 1u;
}

__global__ void lindices_kernel(const uint32_t *__restrict__ flags, const uint32_t *__restrict__ rank, int64_t range,
                                int32_t gmin, int32_t *__restrict__ lind) {
    for (int64_t v = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; v < range; v += (int64_t) gridDim.x * blockDim.x)
        if (flags[v]) lind[rank[v]] = (int32_t) (v + gmin);
}

__global__ void localize_kernel(const int32_t *__restrict__ g, int64_t n, int32_t gmin,
                                const uint32_t *__restrict__ rank, int32_t *__restrict__ local) {
    for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x)
        local[i] = (int32_t) rank[(int64_t) g[i] - gmin];
}

// one map offset per row when every row is a consecutive triplet (3q, 3q+1, 3q+2)
// of local indices, or a trash row (first local index 0 with a trash pixel)
__global__ void triplet_kernel(const int32_t *__restrict__ g, int64_t m, int32_t gmin, const uint32_t *__restrict__ rank,
                               int trash, int32_t *__restrict__ off, int *__restrict__ bad) {
    int local_bad = 0;
    for (int64_t t = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; t < m; t += (int64_t) gridDim.x * blockDim.x) {
        int32_t l0 = (int32_t) rank[(int64_t) g[3 * t] - gmin];
        if (trash && l0 == 0) {
            off[t] = -1;
            continue;
        }
        int32_t l1 = (int32_t) rank[(int64_t) g[3 * t + 1] - gmin];
        int32_t l2 = (int32_t) rank[(int64_t) g[3 * t + 2] - gmin];
        if (l1 != l0 + 1 || l2 != l0 + 2 || (l0 % 3) != 0) local_bad = 1;
        off[t] = l0 - 3 * trash;
    }
    if (local_bad) atomicOr(bad, 1);
}

// In trash mode the reference reads x[local - nnz] for every entry of a row
// whose first local index is not 0 (mapmat.c:711-719): an entry with local
// index < nnz there would read before the map.  Such pointings are rejected.
__global__ void validate_general_kernel(const int32_t *__restrict__ local, int64_t m, int nnz, int *__restrict__ bad) {
    int local_bad = 0;
    for (int64_t t = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; t < m; t += (int64_t) gridDim.x * blockDim.x) {
        if (local[t * nnz] == 0) continue;
        for (int j = 0; j < nnz; j++)
            if (local[t * nnz + j] < nnz) local_bad = 1;
    }
    if (local_bad) atomicOr(bad, 1);
}

int mdp_pointing_create_ex(mdp_context *ctx, int64_t m, int nnz, const int32_t *d_g, const double *d_values,
                           int32_t *d_local_out, mdp_pointing **out) {
    if (!ctx || !out || m < 0 || nnz <= 0 || (m > 0 && (!d_g || !d_values))) {
        mdp_set_error("mdp_pointing_create: invalid arguments");
        return MDP_EINVAL;
    }
    *out = nullptr;
    if (m == 0) {
        mdp_set_error("mdp_pointing_create: empty pointing (m == 0)");
        return MDP_EINVAL;
    }
    MDP_CUDA(cudaSetDevice(ctx->device));
    const int64_t n = m * (int64_t) nnz;
    // 1. min / max
    const int nb = 2 * ctx->sm_count;
    DevBuf    mm;
    MDP_TRY(mm.alloc(sizeof(int32_t) * 2 * nb));
    minmax_kernel<<<nb, 512, 0, ctx->stream>>>(d_g, n, mm.as<int32_t>(), mm.as<int32_t>() + nb);
    MDP_CHECK_LAUNCH(ctx);
    std::vector<int32_t> hmm(2 * nb);
    MDP_CUDA(cudaMemcpyAsync(hmm.data(), mm.p, sizeof(int32_t) * 2 * nb, cudaMemcpyDeviceToHost, ctx->stream));
    MDP_CUDA(cudaStreamSynchronize(ctx->stream));
    int32_t gmin = INT32_MAX, gmax = INT32_MIN;
    for (int i = 0; i < nb; i++) {
        gmin = std::min(gmin, hmm[i]);
        gmax = std::max(gmax, hmm[nb + i]);
    }
    const int64_t range = (int64_t) gmax - gmin + 1;
    // 2. presence flags over [min, max] (the counting sort's bitmap) and their ranks
    DevBuf flags, rank;
    MDP_TRY(flags.alloc(sizeof(uint32_t) * range));
    MDP_TRY(rank.alloc(sizeof(uint32_t) * range));
    MDP_CUDA(cudaMemsetAsync(flags.p, 0, sizeof(uint32_t) * range, ctx->stream));
    mark_kernel<<<grid_for(n, 256, ctx->sm_count * 32), 256, 0, ctx->stream>>>(d_g, n, gmin, flags.as<uint32_t>());
    MDP_CHECK_LAUNCH(ctx);
    uint32_t lcount = 0;
    MDP_TRY(mdp_exclusive_scan_u32(ctx, flags.as<uint32_t>(), rank.as<uint32_t>(), range, &lcount));

    mdp_pointing *A = new mdp_pointing();
    A->m            = m;
    A->nnz          = nnz;
    A->values       = d_values;
    A->lcount       = lcount;
    int rc          = A->lindices.alloc(sizeof(int32_t) * (size_t) lcount);
    if (rc) {
        delete A;
        return rc;
    }
    lindices_kernel<<<grid_for(range, 256, ctx->sm_count * 32), 256, 0, ctx->stream>>>(
            flags.as<uint32_t>(), rank.as<uint32_t>(), range, gmin, A->lindices.as<int32_t>());
    A->trash_pix = gmin < 0 ? 1 : 0;  // lindices[0] == gmin
    ctx->launches++;
    // 3. per-row map offsets (triplet layout) or full local indices (general layout)
    bool triplet = false;
    if (nnz == 3) {
        DevBuf bad;
        if ((rc = A->off.alloc(sizeof(int32_t) * m)) || (rc = bad.alloc(sizeof(int)))) {
            delete A;
            return rc;
        }
        cudaMemsetAsync(bad.p, 0, sizeof(int), ctx->stream);
        triplet_kernel<<<grid_for(m, 256, ctx->sm_count * 32), 256, 0, ctx->stream>>>(
                d_g, m, gmin, rank.as<uint32_t>(), A->trash_pix, A->off.as<int32_t>(), bad.as<int>());
        ctx->launches++;
        int hbad = 1;
        cudaMemcpyAsync(&hbad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
        if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
            delete A;
            mdp_set_error("pointing compression failed: %s", cudaGetErrorString(cudaGetLastError()));
            return MDP_ECUDA;
        }
        triplet = (hbad == 0);
        if (!triplet) A->off.release();
    }
    A->triplet = triplet ? 1 : 0;
    int32_t *local = d_local_out;
    if (!triplet) {
        if ((rc = A->local.alloc(sizeof(int32_t) * n))) {
            delete A;
            return rc;
        }
        localize_kernel<<<grid_for(n, 256, ctx->sm_count * 32), 256, 0, ctx->stream>>>(d_g, n, gmin, rank.as<uint32_t>(),
                                                                                      A->local.as<int32_t>());
        ctx->launches++;
        if (A->trash_pix) {
            DevBuf bad;
            if ((rc = bad.alloc(sizeof(int)))) {
                delete A;
                return rc;
            }
            cudaMemsetAsync(bad.p, 0, sizeof(int), ctx->stream);
            validate_general_kernel<<<grid_for(m, 256, ctx->sm_count * 32), 256, 0, ctx->stream>>>(
                    A->local.as<int32_t>(), m, nnz, bad.as<int>());
            ctx->launches++;
            int hbad = 0;
            cudaMemcpyAsync(&hbad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
            cudaStreamSynchronize(ctx->stream);
            if (hbad) {
                delete A;
                mdp_set_error("mdp_pointing_create: a row that is not a trash row holds a negative (flagged) index");
                return MDP_EINVAL;
            }
        }
        if (d_local_out)
            cudaMemcpyAsync(d_local_out, A->local.p, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, ctx->stream);
    } else if (local) {
        localize_kernel<<<grid_for(n, 256, ctx->sm_count * 32), 256, 0, ctx->stream>>>(d_g, n, gmin, rank.as<uint32_t>(),
                                                                                      local);
        ctx->launches++;
    }
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        delete A;
        mdp_set_error("pointing compression: %s", cudaGetErrorString(e));
        return MDP_ECUDA;
    }
    *out = A;
    return MDP_OK;
}

extern "C" int mdp_pointing_create(mdp_context *ctx, int64_t m, int nnz, const int32_t *d_gindices,
                                   const double *d_values, mdp_pointing **out) {
    return mdp_pointing_create_ex(ctx, m, nnz, d_gindices, d_values, nullptr, out);
}

extern "C" void mdp_pointing_destroy(mdp_pointing *A) { delete A; }

extern "C" int mdp_pointing_shape(const mdp_pointing *A, int64_t *lcount, int *trash_pix, int64_t *n_map,
                                  int *triplet_layout) {
    if (!A) return MDP_EINVAL;
    if (lcount) *lcount = A->lcount;
    if (trash_pix) *trash_pix = A->trash_pix;
    if (n_map) *n_map = A->n_map();
    if (triplet_layout) *triplet_layout = A->triplet;
    return MDP_OK;
}

extern "C" int mdp_pointing_lindices(mdp_context *ctx, const mdp_pointing *A, int32_t *d_lindices) {
    if (!ctx || !A || !d_lindices) return MDP_EINVAL;
    MDP_CUDA(cudaMemcpyAsync(d_lindices, A->lindices.p, sizeof(int32_t) * A->lcount, cudaMemcpyDeviceToDevice,
                             ctx->stream));
    return MDP_OK;
}

// local indices of the triplet layout: 3q+j for valid rows, 0,1,2 for trash rows
__global__ void expand_local_kernel(const int32_t *__restrict__ off, int64_t m, int trash, int32_t *__restrict__ local) {
    for (int64_t t = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; t < m; t += (int64_t) gridDim.x * blockDim.x) {
        int32_t o  = off[t];
        int32_t l0 = (o < 0) ? 0 : o + 3 * trash;
        local[3 * t] = l0;
        local[3 * t + 1] = l0 + 1;
        local[3 * t + 2] = l0 + 2;
    }
}

extern "C" int mdp_pointing_local_indices(mdp_context *ctx, const mdp_pointing *A, int32_t *d_local) {
    if (!ctx || !A || !d_local) return MDP_EINVAL;
    if (!A->triplet) {
        MDP_CUDA(cudaMemcpyAsync(d_local, A->local.p, sizeof(int32_t) * A->m * A->nnz, cudaMemcpyDeviceToDevice,
                                 ctx->stream));
        return MDP_OK;
    }
    expand_local_kernel<<<grid_for(A->m, 256, ctx->sm_count * 32), 256, 0, ctx->stream>>>(A->off.as<int32_t>(), A->m,
                                                                                          A->trash_pix, d_local);
    MDP_CHECK_LAUNCH(ctx);
    return MDP_OK;
}

// ============================================================== y = P x
// Triplet layout: 2 rows per thread so the 6 weights load as 3 aligned double2.
__global__ void __launch_bounds__(256) matvec_triplet_kernel(const int32_t *__restrict__ off,
                                                             const double *__restrict__ w,
                                                             const double *__restrict__ x, double *__restrict__ y,
                                                             int64_t m) {
    const int64_t npair = m >> 1;
    for (int64_t p = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; p < npair; p += (int64_t) gridDim.x * blockDim.x) {
        const int2    o  = reinterpret_cast<const int2 *>(off)[p];
        const double2 a  = reinterpret_cast<const double2 *>(w)[3 * p];
        const double2 b  = reinterpret_cast<const double2 *>(w)[3 * p + 1];
        const double2 c  = reinterpret_cast<const double2 *>(w)[3 * p + 2];
        double        y0 = 0.0, y1 = 0.0;
        if (o.x >= 0) y0 = a.x * __ldg(x + o.x) + a.y * __ldg(x + o.x + 1) + b.x * __ldg(x + o.x + 2);
        if (o.y >= 0) y1 = b.y * __ldg(x + o.y) + c.x * __ldg(x + o.y + 1) + c.y * __ldg(x + o.y + 2);
        reinterpret_cast<double2 *>(y)[p] = make_double2(y0, y1);
    }
    if ((m & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
        int64_t t = m - 1;
        int32_t o = off[t];
        y[t]      = (o >= 0) ? w[3 * t] * x[o] + w[3 * t + 1] * x[o + 1] + w[3 * t + 2] * x[o + 2] : 0.0;
    }
}

// General layout: the reference loop, row by row (mapmat.c:711-727)
__global__ void matvec_general_kernel(const int32_t *__restrict__ local, const double *__restrict__ w,
                                      const double *__restrict__ x, double *__restrict__ y, int64_t m, int nnz,
                                      int trash) {
    for (int64_t t = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; t < m; t += (int64_t) gridDim.x * blockDim.x) {
        double acc = 0.0;
        if (trash) {
            if (local[t * nnz] != 0)
                for (int j = 0; j < nnz; j++) acc += w[t * nnz + j] * x[local[t * nnz + j] - nnz];
        } else {
            for (int j = 0; j < nnz; j++) acc += w[t * nnz + j] * x[local[t * nnz + j]];
        }
        y[t] = acc;
    }
}

// Triplet layout, one row per thread, any alignment of w / y.
__global__ void matvec_triplet_scalar_kernel(const int32_t *__restrict__ off, const double *__restrict__ w,
                                             const double *__restrict__ x, double *__restrict__ y, int64_t m) {
    for (int64_t t = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; t < m; t += (int64_t) gridDim.x * blockDim.x) {
        const int32_t o = off[t];
        y[t] = (o >= 0) ? w[3 * t] * x[o] + w[3 * t + 1] * x[o + 1] + w[3 * t + 2] * x[o + 2] : 0.0;
    }
}

__global__ void trmatvec_triplet_scalar_kernel(const int32_t *__restrict__ off, const double *__restrict__ w,
                                               const double *__restrict__ y, double *__restrict__ x, int64_t m) {
    for (int64_t t = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; t < m; t += (int64_t) gridDim.x * blockDim.x) {
        const int32_t o = off[t];
        if (o < 0) continue;
        const double v = y[t];
        atomicAdd(x + o, w[3 * t] * v);
        atomicAdd(x + o + 1, w[3 * t + 1] * v);
        atomicAdd(x + o + 2, w[3 * t + 2] * v);
    }
}

static inline bool aligned16(const void *a, const void *b) {
    return (((uintptr_t) a | (uintptr_t) b) & 15u) == 0;
}

int mdp_matvec_launch(mdp_context *ctx, const mdp_pointing *A, const double *d_x, double *d_y) {
    if (A->triplet && !aligned16(A->values, d_y)) {
        matvec_triplet_scalar_kernel<<<grid_for(A->m, 256, ctx->sm_count * 16), 256, 0, ctx->stream>>>(
                A->off.as<int32_t>(), A->values, d_x, d_y, A->m);
    } else if (A->triplet) {
        int64_t npair = A->m >> 1;
        matvec_triplet_kernel<<<grid_for(npair > 0 ? npair : 1, 256, ctx->sm_count * 16), 256, 0, ctx->stream>>>(
                A->off.as<int32_t>(), A->values, d_x, d_y, A->m);
    } else {
        matvec_general_kernel<<<grid_for(A->m, 256, ctx->sm_count * 16), 256, 0, ctx->stream>>>(
                A->local.as<int32_t>(), A->values, d_x, d_y, A->m, A->nnz, A->trash_pix);
    }
    MDP_CHECK_LAUNCH(ctx);
    return MDP_OK;
}

extern "C" int mdp_matvec(mdp_context *ctx, const mdp_pointing *A, const double *d_x, double *d_y) {
    if (!ctx || !A || !d_x || !d_y) return MDP_EINVAL;
    return mdp_matvec_launch(ctx, A, d_x, d_y);
}

// ============================================================== x = P^T y
// FP64 atomics into the (L2-resident) map.
__global__ void __launch_bounds__(256) trmatvec_triplet_kernel(const int32_t *__restrict__ off,
                                                               const double *__restrict__ w,
                                                               const double *__restrict__ y, double *__restrict__ x,
                                                               int64_t m) {
    const int64_t npair = m >> 1;
    for (int64_t p = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; p < npair; p += (int64_t) gridDim.x * blockDim.x) {
        const int2    o  = reinterpret_cast<const int2 *>(off)[p];
        const double2 yy = reinterpret_cast<const double2 *>(y)[p];
        const double2 a  = reinterpret_cast<const double2 *>(w)[3 * p];
        const double2 b  = reinterpret_cast<const double2 *>(w)[3 * p + 1];
        const double2 c  = reinterpret_cast<const double2 *>(w)[3 * p + 2];
        if (o.x >= 0) {
            atomicAdd(x + o.x, a.x * yy.x);
            atomicAdd(x + o.x + 1, a.y * yy.x);
            atomicAdd(x + o.x + 2, b.x * yy.x);
        }
        if (o.y >= 0) {
            atomicAdd(x + o.y, b.y * yy.y);
            atomicAdd(x + o.y + 1, c.x * yy.y);
            atomicAdd(x + o.y + 2, c.y * yy.y);
        }
    }
    if ((m & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
        int64_t t = m - 1;
        int32_t o = off[t];
        if (o >= 0)
            for (int j = 0; j < 3; j++) atomicAdd(x + o + j, w[3 * t + j] * y[t]);
    }
}

__global__ void trmatvec_general_kernel(const int32_t *__restrict__ local, const double *__restrict__ w,
                                        const double *__restrict__ y, double *__restrict__ x, int64_t m, int nnz,
                                        int trash) {
    for (int64_t t = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; t < m; t += (int64_t) gridDim.x * blockDim.x) {
        if (trash && local[t * nnz] == 0) continue;
        for (int j = 0; j < nnz; j++) atomicAdd(x + local[t * nnz + j] - nnz * trash, w[t * nnz + j] * y[t]);
    }
}

// ---- P^T by map bins.  The samples of each bin of PT_BIN_PIX consecutive
// pixels are listed once per pointing, in time order (a stable partition of
// the rows by bin, so the list is the same on every build): counts per
// (row chunk, bin), bin totals, an exclusive scan over the bins, per-chunk
// offsets within each bin, then one warp per row chunk writes its rows in
// order.  Each bin's list is cut into slices of a fixed length (a function of
// the row and bin counts only), and one warp owns one slice: it walks the
// slice in order, 32 rows a step, and adds each row's three products into its
// shared-memory copy of the bin's map.  A step whose offsets run strictly up
// or down the lanes hits distinct pixels; in any other step the rows that hit
// the same pixel are summed in lane order by the group's lowest lane, which
// adds the sum.  A bin of one slice is written by that warp;
// the slices of a longer bin write partial maps, summed in slice order by one
// thread per map entry.  The order of every addition is fixed, so the sums
// are reproducible bit for bit, and no atomic operation touches the map.
// Slicing keeps the work per warp bounded: small maps (few bins) still fill
// the device.
#define PT_BIN_PIX MDP_PT_BIN_PIX
#define PT_WARPS 8

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

// count[c][b] += rows of chunk c (rows [c*chunk, (c+1)*chunk)) in bin b
__global__ void bin_chunk_count_kernel(const int32_t *__restrict__ off, int64_t m, int bin3, int64_t chunk,
                                       int64_t nbins, uint32_t *__restrict__ count) {
    const int64_t c = blockIdx.x;
    const int64_t r0 = c * chunk, r1 = min(m, r0 + chunk);
    uint32_t     *row = count + c * nbins;
    for (int64_t t0 = r0; t0 < r1; t0 += blockDim.x) {
        const int64_t t = t0 + threadIdx.x;
        const int32_t o = (t < r1) ? off[t] : -1;
        const int     b = (o >= 0) ? o / bin3 : -1;
        const unsigned peers = __match_any_sync(0xffffffffu, b);
        if (b >= 0 && lane_id() == __ffs(peers) - 1) atomicAdd(row + b, (uint32_t) __popc(peers));
    }
}

// tot[b] = sum_c count[c][b]
__global__ void bin_total_kernel(const uint32_t *__restrict__ count, int64_t nchunks, int64_t nbins,
                                 uint32_t *__restrict__ tot) {
    for (int64_t b = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; b < nbins; b += (int64_t) gridDim.x * blockDim.x) {
        uint32_t s = 0;
        for (int64_t c = 0; c < nchunks; c++) s += count[c * nbins + b];
        tot[b] = s;
    }
}

// count[c][b] <- start[b] + sum_{c' < c} count[c'][b]: where chunk c's rows of bin b begin
__global__ void bin_offsets_kernel(uint32_t *__restrict__ count, int64_t nchunks, int64_t nbins,
                                   const uint32_t *__restrict__ start) {
    for (int64_t b = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; b < nbins; b += (int64_t) gridDim.x * blockDim.x) {
        uint32_t run = start[b];
        for (int64_t c = 0; c < nchunks; c++) {
            const uint32_t n = count[c * nbins + b];
            count[c * nbins + b] = run;
            run += n;
        }
    }
}

// one warp per chunk: its rows in order into their bins' lists (cursor row of
// the chunk in shared memory when it fits, else in place in global memory)
__global__ void __launch_bounds__(32) bin_chunk_scatter_kernel(const int32_t *__restrict__ off, int64_t m, int bin3,
                                                               int64_t chunk, int64_t nbins,
                                                               uint32_t *__restrict__ offs, uint32_t *__restrict__ perm,
                                                               int use_smem) {
    extern __shared__ uint32_t cur_s[];
    const int64_t c = blockIdx.x;
    const int64_t r0 = c * chunk, r1 = min(m, r0 + chunk);
    uint32_t     *cur = use_smem ? cur_s : offs + c * nbins;
    if (use_smem) {
        for (int64_t b = lane_id(); b < nbins; b += 32) cur_s[b] = offs[c * nbins + b];
        __syncwarp();
    }
    const unsigned below = (1u << lane_id()) - 1u;
    constexpr int  U = 8;  // steps of 32 rows whose offsets are loaded ahead
    for (int64_t t0 = r0; t0 < r1; t0 += 32 * U) {
        int32_t o[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int64_t t = t0 + 32 * u + lane_id();
            o[u] = (t < r1) ? off[t] : -1;
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int64_t  t = t0 + 32 * u + lane_id();
            const int      b = (o[u] >= 0) ? o[u] / bin3 : -1;
            const unsigned peers = __match_any_sync(0xffffffffu, b);
            const int      leader = __ffs(peers) - 1;
            uint32_t       base = 0;
            if (b >= 0 && lane_id() == leader) {
                base = cur[b];
                cur[b] = base + (uint32_t) __popc(peers);
            }
            base = __shfl_sync(0xffffffffu, base, leader);
            if (b >= 0) perm[base + __popc(peers & below)] = (uint32_t) t;
            __syncwarp();
        }
    }
}

// rows per slice of the P^T bin lists: about 2^14 slices, enough to fill the
// device whatever the map size, at least 512 and at most 2^16 rows each; a
// function of the pointing alone (rows and bins), so that the sums are the
// same on every device.  Longer slices would leave a small map's few bins to a few warps;
// shorter ones write more partial maps (3 bin_pix doubles per slice of a bin
// cut in several).
static int64_t pt_slice_len(int64_t m, int64_t nbins) {
    int64_t len = 512;
    while (len < (1 << 16) && m / len > (1 << 14)) len <<= 1;
    // bins enough to fill the device by themselves: cut only the bins longer
    // than the average (fewer partial maps to write and sum)
    if (nbins >= 4096)
        while (len < (1 << 16) && len < m / nbins) len <<= 1;
    return len;
}

int mdp_build_bins(mdp_context *ctx, mdp_pointing *A, int bin_pix, mdp_pt_bins *B, bool slices) {
    const int64_t npix = A->n_map() / 3;
    const int     bin3 = 3 * bin_pix;
    const int64_t nb = (npix + bin_pix - 1) / bin_pix;
    B->valid = 0;
    if (A->m > 0xffffffffLL) {
        mdp_set_error("P^T bins: %lld rows exceed 32-bit row indices", (long long) A->m);
        return MDP_EUNSUPPORTED;
    }
    // row chunks (one warp each for the scatter): at least 2^14 rows, at most
    // 2^26 (chunk, bin) counters
    int64_t chunk = 1 << 14;
    while (((A->m + chunk - 1) / chunk) * std::max<int64_t>(nb, 1) > (1LL << 26)) chunk <<= 1;
    const int64_t nch = std::max<int64_t>((A->m + chunk - 1) / chunk, 1);
    DevBuf        count, tot, start;
    MDP_TRY(count.alloc(4 * (size_t) nch * std::max<int64_t>(nb, 1)));
    MDP_TRY(tot.alloc(4 * (nb + 1)));
    MDP_TRY(start.alloc(4 * (nb + 1)));
    MDP_CUDA(cudaMemsetAsync(count.p, 0, 4 * (size_t) nch * std::max<int64_t>(nb, 1), ctx->stream));
    MDP_CUDA(cudaMemsetAsync(tot.p, 0, 4 * (nb + 1), ctx->stream));
    if (nb > 0) {
        bin_chunk_count_kernel<<<(unsigned) nch, 256, 0, ctx->stream>>>(A->off.as<int32_t>(), A->m, bin3, chunk, nb,
                                                                       count.as<uint32_t>());
        MDP_CHECK_LAUNCH(ctx);
        bin_total_kernel<<<grid_for(nb, 256, 1024), 256, 0, ctx->stream>>>(count.as<uint32_t>(), nch, nb,
                                                                           tot.as<uint32_t>());
        MDP_CHECK_LAUNCH(ctx);
    }
    uint32_t total = 0;
    MDP_TRY(mdp_exclusive_scan_u32(ctx, tot.as<uint32_t>(), start.as<uint32_t>(), nb + 1, &total));
    MDP_TRY(B->perm.alloc(4 * std::max<int64_t>(total, 1)));
    if (nb > 0) {
        bin_offsets_kernel<<<grid_for(nb, 256, 1024), 256, 0, ctx->stream>>>(count.as<uint32_t>(), nch, nb,
                                                                             start.as<uint32_t>());
        MDP_CHECK_LAUNCH(ctx);
        int optin = 0;
        MDP_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device));
        const size_t sm = 4 * (size_t) nb;
        const int    use_smem = sm <= (size_t) optin ? 1 : 0;
        if (use_smem)
            MDP_CUDA(cudaFuncSetAttribute((const void *) bin_chunk_scatter_kernel,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int) sm));
        bin_chunk_scatter_kernel<<<(unsigned) nch, 32, use_smem ? sm : 0, ctx->stream>>>(
                A->off.as<int32_t>(), A->m, bin3, chunk, nb, count.as<uint32_t>(), B->perm.as<uint32_t>(), use_smem);
        MDP_CHECK_LAUNCH(ctx);
    }
    std::vector<uint32_t> hs(nb + 1);
    MDP_CUDA(cudaMemcpyAsync(hs.data(), start.p, 4 * (nb + 1), cudaMemcpyDeviceToHost, ctx->stream));
    MDP_CUDA(cudaStreamSynchronize(ctx->stream));
    std::vector<int64_t> hs64(nb + 1);
    for (int64_t i = 0; i <= nb; i++) hs64[i] = hs[i];
    MDP_TRY(B->start.alloc(8 * (nb + 1)));
    MDP_CUDA(cudaMemcpy(B->start.p, hs64.data(), 8 * (nb + 1), cudaMemcpyHostToDevice));
    B->nslices = B->nmulti = 0;
    if (slices && nb > 0) {
        const int64_t        len = pt_slice_len(A->m, nb);
        std::vector<int32_t> sb, so, mb, mf, mn;
        std::vector<uint32_t> lo, hi;
        int32_t              rows = 0;
        for (int64_t b = 0; b < nb; b++) {
            const int64_t n = hs64[b + 1] - hs64[b];
            const int64_t k = std::max<int64_t>((n + len - 1) / len, 1);
            if (k > 1) {
                mb.push_back((int32_t) b);
                mf.push_back(rows);
                mn.push_back((int32_t) k);
            }
            for (int64_t j = 0; j < k; j++) {
                sb.push_back((int32_t) b);
                lo.push_back((uint32_t) (hs64[b] + j * len));
                hi.push_back((uint32_t) std::min<int64_t>(hs64[b] + (j + 1) * len, hs64[b + 1]));
                so.push_back(k > 1 ? rows++ : -1);
            }
        }
        B->nslices = (int64_t) sb.size();
        B->nmulti = (int64_t) mb.size();
        B->slice_len = len;
        MDP_TRY(B->slice_bin.alloc(4 * sb.size()));
        MDP_TRY(B->slice_lo.alloc(4 * sb.size()));
        MDP_TRY(B->slice_hi.alloc(4 * sb.size()));
        MDP_TRY(B->slice_out.alloc(4 * sb.size()));
        MDP_CUDA(cudaMemcpy(B->slice_bin.p, sb.data(), 4 * sb.size(), cudaMemcpyHostToDevice));
        MDP_CUDA(cudaMemcpy(B->slice_lo.p, lo.data(), 4 * lo.size(), cudaMemcpyHostToDevice));
        MDP_CUDA(cudaMemcpy(B->slice_hi.p, hi.data(), 4 * hi.size(), cudaMemcpyHostToDevice));
        MDP_CUDA(cudaMemcpy(B->slice_out.p, so.data(), 4 * so.size(), cudaMemcpyHostToDevice));
        if (!mb.empty()) {
            MDP_TRY(B->multi_bin.alloc(4 * mb.size()));
            MDP_TRY(B->multi_first.alloc(4 * mf.size()));
            MDP_TRY(B->multi_n.alloc(4 * mn.size()));
            MDP_TRY(B->partial.alloc(sizeof(double) * 3 * (size_t) bin_pix * (size_t) rows));
            MDP_CUDA(cudaMemcpy(B->multi_bin.p, mb.data(), 4 * mb.size(), cudaMemcpyHostToDevice));
            MDP_CUDA(cudaMemcpy(B->multi_first.p, mf.data(), 4 * mf.size(), cudaMemcpyHostToDevice));
            MDP_CUDA(cudaMemcpy(B->multi_n.p, mn.data(), 4 * mn.size(), cudaMemcpyHostToDevice));
        }
    }
    B->nbins = nb;
    B->bin_pix = bin_pix;
    B->valid = 1;
    return MDP_OK;
}

// x = P^T y over the slices of the bins' lists: warp k of a CTA owns slice
// PT_WARPS*blockIdx.x + k.  TY/TW: TOD and weight types (double, or float for
// the mixed solver's FP32 operator); products and sums in FP64.  U steps of 32
// rows are loaded before they are added, for memory-level parallelism.  The
// warp's sums go to the bin's map entries (a bin of one slice) or to the
// slice's row of `partial`, summed by pt_partial_sum_kernel.
template <typename TY, typename TW>
__global__ void __launch_bounds__(32 * PT_WARPS, 4) trmatvec_slices_kernel(
        const int32_t *__restrict__ off, const TW *__restrict__ w, const TY *__restrict__ y, double *__restrict__ x,
        const uint32_t *__restrict__ perm, const int32_t *__restrict__ slice_bin, const uint32_t *__restrict__ slice_lo,
        const uint32_t *__restrict__ slice_hi, const int32_t *__restrict__ slice_out, int64_t nslices,
        double *__restrict__ partial, int64_t n_map) {
    constexpr int U = 4;
    __shared__ double acc_s[PT_WARPS][3 * PT_BIN_PIX];
    const int     wid = threadIdx.x >> 5, lane = lane_id();
    const int64_t sl = (int64_t) blockIdx.x * PT_WARPS + wid;
    if (sl >= nslices) return;  // whole warps only; no CTA-wide barrier follows
    double *acc = acc_s[wid];
    for (int i = lane; i < 3 * PT_BIN_PIX; i += 32) acc[i] = 0.0;
    __syncwarp();
    const int64_t bin = slice_bin[sl];
    const int64_t s0 = slice_lo[sl], s1 = slice_hi[sl];
    const int64_t base = bin * 3 * PT_BIN_PIX;
    // the row numbers of the next U steps are loaded while the current ones are
    // gathered and added: one memory latency per U steps on the warp's path
    uint32_t tn[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
        const int64_t i = s0 + 32 * u + lane;
        tn[u] = (i < s1) ? perm[i] : 0u;
    }
    for (int64_t i0 = s0; i0 < s1; i0 += 32 * U) {
        uint32_t tc[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            tc[u] = tn[u];
            const int64_t i = i0 + 32 * (U + u) + lane;
            tn[u] = (i < s1) ? perm[i] : 0u;
        }
        int    o[U];
        double c0[U], c1[U], c2[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int64_t i = i0 + 32 * u + lane;
            o[u] = -1;
            c0[u] = c1[u] = c2[u] = 0.0;
            if (i < s1) {
                const int64_t t = tc[u];
                const double  v = (double) y[t];
                o[u] = (int) (off[t] - base);
                c0[u] = (double) w[3 * t] * v;
                c1[u] = (double) w[3 * t + 1] * v;
                c2[u] = (double) w[3 * t + 2] * v;
            }
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            // distinct pixels for certain when the step's offsets run strictly up
            // or down the lanes (a scan crossing the bin; the rows past the slice
            // end, o < 0, are the last lanes and are given keys that continue
            // either run); otherwise the lanes are grouped by pixel
            const int  ku = o[u] >= 0 ? o[u] : (1 << 20) + lane, kd = o[u] >= 0 ? o[u] : -1 - lane;
            const int  nu = __shfl_down_sync(0xffffffffu, ku, 1), nd = __shfl_down_sync(0xffffffffu, kd, 1);
            const bool up = __all_sync(0xffffffffu, lane == 31 || ku < nu);
            const bool down = __all_sync(0xffffffffu, lane == 31 || kd > nd);
            unsigned   peers = 1u << lane;
            if (!up && !down) peers = __match_any_sync(0xffffffffu, o[u]);
            const bool alone = o[u] < 0 || peers == (1u << lane);
            if (__all_sync(0xffffffffu, alone)) {
                if (o[u] >= 0) {  // distinct pixels: one add per entry
                    acc[o[u]] += c0[u];
                    acc[o[u] + 1] += c1[u];
                    acc[o[u] + 2] += c2[u];
                }
            } else {
                // rows of one pixel in this step: the lowest lane of each group sums
                // the others' products in lane order, then adds the group's sum
                // (groups hit distinct pixels, so their adds do not collide)
                const bool lead = o[u] >= 0 && (__ffs(peers) - 1) == lane;
                unsigned   rest = lead ? (peers & ~(1u << lane)) : 0u;
                double     s0 = c0[u], s1 = c1[u], s2 = c2[u];
                const int  steps = (int) __reduce_max_sync(0xffffffffu, (unsigned) __popc(rest));
                for (int k = 0; k < steps; k++) {
                    const int    src = rest ? __ffs(rest) - 1 : lane;
                    const double d0 = __shfl_sync(0xffffffffu, c0[u], src);
                    const double d1 = __shfl_sync(0xffffffffu, c1[u], src);
                    const double d2 = __shfl_sync(0xffffffffu, c2[u], src);
                    if (rest) {
                        s0 += d0;
                        s1 += d1;
                        s2 += d2;
                        rest &= rest - 1u;
                    }
                }
                if (lead) {
                    acc[o[u]] += s0;
                    acc[o[u] + 1] += s1;
                    acc[o[u] + 2] += s2;
                }
            }
            __syncwarp();
        }
    }
    const int out = slice_out[sl];
    if (out < 0) {
        const int64_t lim = min((int64_t) 3 * PT_BIN_PIX, n_map - base);
        for (int i = lane; i < lim; i += 32) x[base + i] = acc[i];
    } else {
        double *pr = partial + (int64_t) out * 3 * PT_BIN_PIX;
        for (int i = lane; i < 3 * PT_BIN_PIX; i += 32) pr[i] = acc[i];
    }
}

// map entries of the bins of several slices: their partial maps summed in slice order
__global__ void pt_partial_sum_kernel(const double *__restrict__ partial, const int32_t *__restrict__ multi_bin,
                                      const int32_t *__restrict__ multi_first, const int32_t *__restrict__ multi_n,
                                      int64_t nmulti, double *__restrict__ x, int64_t n_map) {
    constexpr int E = 3 * PT_BIN_PIX;
    for (int64_t idx = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; idx < nmulti * E;
         idx += (int64_t) gridDim.x * blockDim.x) {
        const int64_t k = idx / E, e = idx % E;
        const int64_t xi = (int64_t) multi_bin[k] * E + e;
        if (xi >= n_map) continue;
        const double *pr = partial + (int64_t) multi_first[k] * E + e;
        double        s = 0.0;
        for (int j = 0; j < multi_n[k]; j++) s += pr[(int64_t) j * E];
        x[xi] = s;
    }
}

// P^T over the slices (both kernels), FP64 or FP32 TOD and weights
template <typename TY, typename TW>
static int trmatvec_slices(mdp_context *ctx, const mdp_pointing *A, const TW *w, const TY *d_y, double *d_x) {
    const mdp_pt_bins &B = A->bins;
    if (B.nslices > 0) {
        trmatvec_slices_kernel<TY, TW><<<(unsigned) ((B.nslices + PT_WARPS - 1) / PT_WARPS), 32 * PT_WARPS, 0,
                                         ctx->stream>>>(
                A->off.as<int32_t>(), w, d_y, d_x, B.perm.as<uint32_t>(), B.slice_bin.as<int32_t>(),
                B.slice_lo.as<uint32_t>(), B.slice_hi.as<uint32_t>(), B.slice_out.as<int32_t>(), B.nslices,
                B.partial.as<double>(), A->n_map());
        MDP_CHECK_LAUNCH(ctx);
    }
    if (B.nmulti > 0) {
        pt_partial_sum_kernel<<<grid_for(B.nmulti * 3 * PT_BIN_PIX, 256, ctx->sm_count * 8), 256, 0, ctx->stream>>>(
                B.partial.as<double>(), B.multi_bin.as<int32_t>(), B.multi_first.as<int32_t>(),
                B.multi_n.as<int32_t>(), B.nmulti, d_x, A->n_map());
        MDP_CHECK_LAUNCH(ctx);
    }
    return MDP_OK;
}

__global__ void trmatvec32_kernel(const int32_t *__restrict__ off, const float *__restrict__ w,
                                  const float *__restrict__ y, double *__restrict__ x, int64_t m) {
    for (int64_t t = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; t < m; t += (int64_t) gridDim.x * blockDim.x) {
        const int32_t o = off[t];
        if (o < 0) continue;
        const double v = (double) y[t];
        atomicAdd(x + o, (double) w[3 * t] * v);
        atomicAdd(x + o + 1, (double) w[3 * t + 1] * v);
        atomicAdd(x + o + 2, (double) w[3 * t + 2] * v);
    }
}

__global__ void weights_to_float_kernel(const double *__restrict__ in, float *__restrict__ out, int64_t n) {
    for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x)
        out[i] = (float) in[i];
}

int mdp_pointing_prepare_fp32(mdp_context *ctx, mdp_pointing *A) {
    if (!A->triplet) {
        mdp_set_error("the FP32 operator needs the (I,Q,U) triplet pointing layout");
        return MDP_EUNSUPPORTED;
    }
    if (A->w32.p) return MDP_OK;
    MDP_TRY(A->w32.alloc(sizeof(float) * 3 * A->m));
    weights_to_float_kernel<<<grid_for(3 * A->m, 256, ctx->sm_count * 16), 256, 0, ctx->stream>>>(
            A->values, A->w32.as<float>(), 3 * A->m);
    MDP_CHECK_LAUNCH(ctx);
    return MDP_OK;
}

static bool use_bins(const mdp_pointing *A) { return A->triplet && A->m >= (1 << 20); }
bool mdp_pointing_binned(const mdp_pointing *A) { return use_bins(A); }
int  mdp_pointing_bins(mdp_context *ctx, mdp_pointing *A) {
    if (!A->bins.valid || A->bins.bin_pix != PT_BIN_PIX) MDP_TRY(mdp_build_bins(ctx, A, PT_BIN_PIX, &A->bins, true));
    return MDP_OK;
}

int mdp_trmatvec_launch(mdp_context *ctx, const mdp_pointing *A, const double *d_y, double *d_x) {
    if (use_bins(A)) {
        mdp_pointing *Am = const_cast<mdp_pointing *>(A);  // the bin list is a cache of the pointing
        MDP_TRY(mdp_pointing_bins(ctx, Am));
        // every map entry is written by its bin's slice or by the partial sums
        return trmatvec_slices<double, double>(ctx, A, A->values, d_y, d_x);
    }
    MDP_CUDA(cudaMemsetAsync(d_x, 0, sizeof(double) * A->n_map(), ctx->stream));
    if (A->triplet && !aligned16(A->values, d_y)) {
        trmatvec_triplet_scalar_kernel<<<grid_for(A->m, 256, ctx->sm_count * 16), 256, 0, ctx->stream>>>(
                A->off.as<int32_t>(), A->values, d_y, d_x, A->m);
    } else if (A->triplet) {
        int64_t npair = A->m >> 1;
        trmatvec_triplet_kernel<<<grid_for(npair > 0 ? npair : 1, 256, ctx->sm_count * 16), 256, 0, ctx->stream>>>(
                A->off.as<int32_t>(), A->values, d_y, d_x, A->m);
    } else {
        trmatvec_general_kernel<<<grid_for(A->m, 256, ctx->sm_count * 16), 256, 0, ctx->stream>>>(
                A->local.as<int32_t>(), A->values, d_y, d_x, A->m, A->nnz, A->trash_pix);
    }
    MDP_CHECK_LAUNCH(ctx);
    return MDP_OK;
}

extern "C" int mdp_trmatvec(mdp_context *ctx, const mdp_pointing *A, const double *d_y, double *d_x) {
    if (!ctx || !A || !d_x || !d_y) return MDP_EINVAL;
    return mdp_trmatvec_launch(ctx, A, d_y, d_x);
}

// x (FP64, n_map) = P^T y (FP32 TOD) with the FP32 weights
int mdp_trmatvec32_launch(mdp_context *ctx, mdp_pointing *A, const float *d_y, double *d_x) {
    MDP_TRY(mdp_pointing_prepare_fp32(ctx, A));
    if (use_bins(A)) {
        MDP_TRY(mdp_pointing_bins(ctx, A));
        return trmatvec_slices<float, float>(ctx, A, A->w32.as<float>(), d_y, d_x);
    }
    MDP_CUDA(cudaMemsetAsync(d_x, 0, sizeof(double) * A->n_map(), ctx->stream));
    trmatvec32_kernel<<<grid_for(A->m, 256, ctx->sm_count * 16), 256, 0, ctx->stream>>>(
            A->off.as<int32_t>(), A->w32.as<float>(), d_y, d_x, A->m);
    MDP_CHECK_LAUNCH(ctx);
    return MDP_OK;
}

// y32 = P x with FP32 weights (x FP64), when the fused block-sum kernel does not apply
__global__ void matvec32_kernel(const int32_t *__restrict__ off, const float *__restrict__ w,
                                const double *__restrict__ x, float *__restrict__ y, int64_t m) {
    for (int64_t t = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; t < m; t += (int64_t) gridDim.x * blockDim.x) {
        const int32_t o = off[t];
        y[t] = (o >= 0) ? w[3 * t] * (float) x[o] + w[3 * t + 1] * (float) x[o + 1] + w[3 * t + 2] * (float) x[o + 2]
                        : 0.0f;
    }
}

int mdp_matvec32_launch(mdp_context *ctx, mdp_pointing *A, const double *d_x, float *d_y) {
    MDP_TRY(mdp_pointing_prepare_fp32(ctx, A));
    matvec32_kernel<<<grid_for(A->m, 256, ctx->sm_count * 16), 256, 0, ctx->stream>>>(A->off.as<int32_t>(),
                                                                                     A->w32.as<float>(), d_x, d_y, A->m);
    MDP_CHECK_LAUNCH(ctx);
    return MDP_OK;
}
