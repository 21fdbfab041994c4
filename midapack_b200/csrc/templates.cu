// MTmap's template filter: set-up on the host (as in the reference) and the
// weighting of its PCG on the device.
//
// MTmap (mappraiser/src/mappraiser.c:387-800) marginalises per-block template
// amplitudes: Legendre polynomials of orders 0..npoly-1 on every sweep, the
// scan-synchronous ground signal in azimuth bins, and HWP harmonics whose cos and
// sin amplitudes are constant over delta_t seconds (algebra/src/templates/templates.c).
// Every sample carries exactly one (bin, weight) pair per template class, so the
// template matrix of a CES is stored in ELL form: n_class = npoly + ground + 2 nhwp
// pairs per sample, the bins numbered from 0 within a block in the reference's
// amplitude order (Tlist_init, templates.c:634-677).  The kernels
// B_b = pinv(w_b T_b^T T_b) (BuildKernel + InvKernel, templates.c:192-418) are built
// here on the host, as the reference builds them, with the same DGELSS rule
// (singular values <= 1e-12 s_max dropped).
#include "mdp_internal.cuh"
#include "smalldense.h"

#include <algorithm>
#include <cmath>
#include <memory>
#include <vector>

namespace {

struct Scan {
    const mdp_template_scan *s;
    std::vector<int64_t> sweep_row, sample_row;   // offsets of each CES's rows
    int n_class = 0;

    int nsw(int i) const { return s->nsweeps[i]; }
    const int32_t *sweeps(int i) const { return s->sweeps + sweep_row[i]; }
    int length(int i) const { return sweeps(i)[nsw(i)]; }
    int hwp_bins(int i) const { return (int) std::ceil(length(i) / (s->delta_t * s->fs)); }
    int nt(int i) const {
        return s->npoly * nsw(i) + s->ground * s->n_sss_bins + 2 * s->nhwp * hwp_bins(i);
    }
};

int make_scan(const mdp_template_scan *s, Scan *sc) {
    if (!s || s->nces < 1 || s->ndet < 1 || !s->nsweeps || !s->sweeps || s->npoly < 0 || s->nhwp < 0 ||
        (s->ground != 0 && s->ground != 1) || (s->ground && (s->n_sss_bins < 1 || !s->az || !s->az_min || !s->az_max)) ||
        (s->nhwp && (!s->hwp || !(s->delta_t > 0.0))) || !(s->fs > 0.0)) {
        mdp_set_error("template scan: bad argument");
        return MDP_EINVAL;
    }
    sc->s = s;
    sc->n_class = s->npoly + s->ground + 2 * s->nhwp;
    if (sc->n_class < 1) {
        mdp_set_error("template scan: no template class");
        return MDP_EINVAL;
    }
    sc->sweep_row.assign(s->nces + 1, 0);
    sc->sample_row.assign(s->nces + 1, 0);
    for (int i = 0; i < s->nces; ++i) {
        if (s->nsweeps[i] < 1) {
            mdp_set_error("template scan: CES %d has no sweep", i);
            return MDP_EINVAL;
        }
        sc->sweep_row[i + 1] = sc->sweep_row[i] + s->nsweeps[i] + 1;
        const int32_t *sw = s->sweeps + sc->sweep_row[i];
        // the reference leaves samples outside the sweeps on bin 0 of the whole list with
        // weight 0, and divides by zero on one-sample sweeps: both are rejected here
        if (sw[0] != 0) {
            mdp_set_error("template scan: CES %d: the first sweep must start at sample 0", i);
            return MDP_EINVAL;
        }
        for (int k = 0; k < s->nsweeps[i]; ++k)
            if (sw[k + 1] - sw[k] < 2) {
                mdp_set_error("template scan: CES %d: sweep %d has fewer than 2 samples", i, k);
                return MDP_EINVAL;
            }
        sc->sample_row[i + 1] = sc->sample_row[i] + sw[s->nsweeps[i]];
    }
    return MDP_OK;
}

// Legendre (templates.c:526-549): P_n on [a, b], three-term recurrence
double legendre(double x, double a, double b, int n) {
    const double t = (2 * x - a - b) / (b - a);
    double p0 = 1.0, p1 = t;
    if (n == 0) return p0;
    for (int k = 2; k <= n; ++k) {
        const double p2 = ((2 * k - 1) * t * p1 - (k - 1) * p0) / k;
        p0 = p1;
        p1 = p2;
    }
    return p1;
}

// ELL rows of CES i: bins/wghts [length(i)][n_class]
int layout_ces(const Scan &sc, int i, int32_t *bins, double *wghts) {
    const mdp_template_scan *s = sc.s;
    const int L = sc.length(i), nc = sc.n_class, ns = sc.nsw(i);
    const int32_t *sw = sc.sweeps(i);
    const double fs = s->fs;
    int c = 0;
    for (int k = 0; k < s->npoly; ++k, ++c) {   // expandpolydata
        for (int q = 0; q < ns; ++q)
            for (int t = sw[q]; t < sw[q + 1]; ++t) {
                bins[(int64_t) t * nc + c] = k * ns + q;
                wghts[(int64_t) t * nc + c] = legendre((double) t / fs, (double) sw[q] / fs,
                                                       (double) (sw[q + 1] - 1) / fs, k);
            }
    }
    int base = s->npoly * ns;
    if (s->ground) {   // bin_az + expandSSSdata
        const double *az = s->az + sc.sample_row[i];
        const double lo = s->az_min[i], width = (s->az_max[i] - s->az_min[i]) / s->n_sss_bins;
        for (int t = 0; t < L; ++t) {
            int b = (int) std::floor((az[t] - lo) / width);
            if (b > s->n_sss_bins - 1) b = s->n_sss_bins - 1;
            if (b < 0) {
                mdp_set_error("template scan: CES %d sample %d: azimuth below az_min", i, t);
                return MDP_EINVAL;
            }
            bins[(int64_t) t * nc + c] = base + b;
            wghts[(int64_t) t * nc + c] = 1.0;
        }
        ++c;
        base += s->n_sss_bins;
    }
    if (s->nhwp) {   // build_hwpss_w + expandHWPSSdata
        const double *ang = s->hwp + sc.sample_row[i];
        const int hb = sc.hwp_bins(i);
        for (int t = 0; t < L; ++t) {
            const double c1 = std::cos(ang[t]), s1 = std::sin(ang[t]);
            double ch = c1, sh = s1;
            const int chunk = (int) std::floor((double) t / (fs * s->delta_t));
            for (int h = 1; h <= s->nhwp; ++h) {
                if (h > 1) {
                    const double cn = ch * c1 - sh * s1;
                    const double sn = sh * c1 + ch * s1;
                    ch = cn;
                    sh = sn;
                }
                const int cc = c + 2 * (h - 1);
                bins[(int64_t) t * nc + cc] = base + 2 * (h - 1) * hb + chunk;
                wghts[(int64_t) t * nc + cc] = ch;
                bins[(int64_t) t * nc + cc + 1] = base + (2 * h - 1) * hb + chunk;
                wghts[(int64_t) t * nc + cc + 1] = sh;
            }
        }
    }
    return MDP_OK;
}

}  // namespace

extern "C" int mdp_template_layout(const mdp_template_scan *scan, int32_t *h_bins, double *h_wghts,
                                   int32_t *h_nt) {
    Scan sc;
    MDP_TRY(make_scan(scan, &sc));
    if (!h_bins || !h_wghts) {
        mdp_set_error("mdp_template_layout: bad argument");
        return MDP_EINVAL;
    }
    for (int i = 0; i < scan->nces; ++i) {
        MDP_TRY(layout_ces(sc, i, h_bins + sc.sample_row[i] * sc.n_class, h_wghts + sc.sample_row[i] * sc.n_class));
        if (h_nt) h_nt[i] = sc.nt(i);
    }
    return MDP_OK;
}

namespace {

// pinv(w_b T_b^T T_b) of every block, block after block into h_kinv
int kernels_impl(const Scan &sc, const double *h_w_block, double *h_kinv) {
    const mdp_template_scan *scan = sc.s;
    const int nc = sc.n_class;
    int64_t at = 0;
    std::vector<int32_t> bins;
    std::vector<double> wg, K;
    for (int i = 0; i < scan->nces; ++i) {
        const int L = sc.length(i), nt = sc.nt(i);
        bins.assign((size_t) L * nc, 0);
        wg.assign((size_t) L * nc, 0.0);
        MDP_TRY(layout_ces(sc, i, bins.data(), wg.data()));
        for (int j = 0; j < scan->ndet; ++j) {
            // BuildKernel: B[b_k][b_l] += w * w_k(t) * w_l(t) over the samples
            const double w = h_w_block[i * scan->ndet + j];
            K.assign((size_t) nt * nt, 0.0);
            for (int t = 0; t < L; ++t)
                for (int a = 0; a < nc; ++a) {
                    const double wa = w * wg[(size_t) t * nc + a];
                    const int ba = bins[(size_t) t * nc + a];
                    for (int b = 0; b < nc; ++b) K[(size_t) ba * nt + bins[(size_t) t * nc + b]] += wa * wg[(size_t) t * nc + b];
                }
            // InvKernel: DGELSS(B, I) with rcond 1e-12
            const std::vector<double> P = mdp_dense::pinv_gelss(nt, K, 1e-12);
            std::copy(P.begin(), P.end(), h_kinv + at);
            at += (int64_t) nt * nt;
        }
    }
    return MDP_OK;
}

}  // namespace

extern "C" int mdp_template_kernels(const mdp_template_scan *scan, const double *h_w_block, double *h_kinv) {
    Scan sc;
    MDP_TRY(make_scan(scan, &sc));
    if (!h_w_block || !h_kinv) {
        mdp_set_error("mdp_template_kernels: bad argument");
        return MDP_EINVAL;
    }
    return kernels_impl(sc, h_w_block, h_kinv);
}

// ====================================================================== device filter
// F x = W x - W T B T^T W x, W = diag(w_b) per block (MTmap's white N^-1, lambda = 1),
// B_b = pinv(w_b T_b^T T_b): the weighting of PCG_GLS_templates
// (mappraiser/src/pcg_true.c:301-365, 433-462).  TOD blocks are consecutive, block
// b = i*ndet + j of ces_length(i) samples; the ELL rows of CES i are shared by its
// detectors.
struct mdp_templates {
    int     nb = 0, nc = 0, max_nt = 0, max_len = 0;
    int64_t m = 0, namp = 0;
    DevBuf  bins, wg;                       // int32 / double [sum ces_length][nc]
    DevBuf  blk_off, blk_row, blk_amp, blk_kinv;   // int64 [nb]
    DevBuf  blk_len, blk_nt;                // int32 [nb]
    DevBuf  blk_w;                          // double [nb]
    DevBuf  kinv;                           // double [sum nt^2]
    DevBuf  amp, coef;                      // double [namp] work
};

namespace {

constexpr int kTplThreads = 256;
constexpr int kTplMaxNt = 6144;   // one block's amplitudes in 48 KB of shared memory

// a_b += T_b^T (w_b x_b) over a chunk of the block's samples (grid: chunks x blocks):
// a shared-memory histogram of the block's amplitudes, then one global add per amplitude
__global__ void __launch_bounds__(kTplThreads) tpl_tt_kernel(const double *x, const int32_t *bins, const double *wg,
                                                             int nc, const int64_t *blk_off, const int64_t *blk_row,
                                                             const int32_t *blk_len, const int32_t *blk_nt,
                                                             const int64_t *blk_amp, const double *blk_w,
                                                             double *amp) {
    extern __shared__ double hist[];
    const int b = blockIdx.y;
    const int nt = blk_nt[b];
    const int64_t L = blk_len[b];
    for (int k = threadIdx.x; k < nt; k += blockDim.x) hist[k] = 0.0;
    __syncthreads();
    const double w = blk_w[b];
    const double *xb = x + blk_off[b];
    const int32_t *bb = bins + blk_row[b] * nc;
    const double *wb = wg + blk_row[b] * nc;
    for (int64_t t = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; t < L; t += (int64_t) gridDim.x * blockDim.x) {
        const double v = w * xb[t];
        for (int c = 0; c < nc; ++c) {
            const int k = bb[t * nc + c];
            if ((unsigned) k < (unsigned) nt) atomicAdd(&hist[k], wb[t * nc + c] * v);
        }
    }
    __syncthreads();
    double *ab = amp + blk_amp[b];
    for (int k = threadIdx.x; k < nt; k += blockDim.x)
        if (hist[k] != 0.0) atomicAdd(&ab[k], hist[k]);
}

// c_b = B_b a_b (row-major B_b, as PCG_GLS_templates applies it): one CTA per block
__global__ void __launch_bounds__(kTplThreads) tpl_b_kernel(const double *kinv, const int64_t *blk_kinv,
                                                            const int32_t *blk_nt, const int64_t *blk_amp,
                                                            const double *amp, double *coef) {
    const int b = blockIdx.x;
    const int nt = blk_nt[b];
    const double *K = kinv + blk_kinv[b];
    const double *a = amp + blk_amp[b];
    double *c = coef + blk_amp[b];
    for (int r = threadIdx.x; r < nt; r += blockDim.x) {
        double acc = 0.0;
        for (int l = 0; l < nt; ++l) acc += K[(int64_t) r * nt + l] * a[l];
        c[r] = acc;
    }
}

// y_b = w_b x_b - w_b T_b c_b (y may be x)
__global__ void __launch_bounds__(kTplThreads) tpl_t_kernel(const double *x, const int32_t *bins, const double *wg,
                                                            int nc, const int64_t *blk_off, const int64_t *blk_row,
                                                            const int32_t *blk_len, const int32_t *blk_nt,
                                                            const int64_t *blk_amp, const double *blk_w,
                                                            const double *coef, double *y) {
    const int b = blockIdx.y;
    const int nt = blk_nt[b];
    const int64_t L = blk_len[b];
    const double w = blk_w[b];
    const int64_t off = blk_off[b];
    const int32_t *bb = bins + blk_row[b] * nc;
    const double *wb = wg + blk_row[b] * nc;
    const double *cb = coef + blk_amp[b];
    for (int64_t t = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; t < L; t += (int64_t) gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int c = 0; c < nc; ++c) {
            const int k = bb[t * nc + c];
            if ((unsigned) k < (unsigned) nt) s += wb[t * nc + c] * cb[k];
        }
        y[off + t] = w * x[off + t] - w * s;
    }
}

template <class T>
int upload(DevBuf &d, const std::vector<T> &h) {
    MDP_TRY(d.alloc(h.size() * sizeof(T)));
    if (!h.empty()) MDP_CUDA(cudaMemcpy(d.p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
    return MDP_OK;
}

}  // namespace

extern "C" int mdp_templates_create(mdp_context *ctx, const mdp_template_scan *scan, const double *h_w_block,
                                    mdp_templates **out) {
    if (!ctx || !out || !h_w_block) {
        mdp_set_error("mdp_templates_create: bad argument");
        return MDP_EINVAL;
    }
    *out = nullptr;
    Scan sc;
    MDP_TRY(make_scan(scan, &sc));
    const int nc = sc.n_class, nces = scan->nces, ndet = scan->ndet;
    auto T = new mdp_templates();
    std::unique_ptr<mdp_templates> guard(T);
    T->nb = nces * ndet;
    T->nc = nc;
    const int64_t rows = sc.sample_row[nces];
    std::vector<int32_t> bins((size_t) rows * nc);
    std::vector<double> wg((size_t) rows * nc);
    std::vector<int64_t> off(T->nb), row(T->nb), ampo(T->nb), kino(T->nb);
    std::vector<int32_t> len(T->nb), nt(T->nb);
    std::vector<double> w(h_w_block, h_w_block + T->nb);
    int64_t at = 0, na = 0, nk = 0;
    for (int i = 0; i < nces; ++i) {
        MDP_TRY(layout_ces(sc, i, bins.data() + sc.sample_row[i] * nc, wg.data() + sc.sample_row[i] * nc));
        const int nti = sc.nt(i);
        if (nti > kTplMaxNt) {
            mdp_set_error("mdp_templates_create: CES %d has %d template amplitudes per block (at most %d)", i, nti,
                          kTplMaxNt);
            return MDP_EUNSUPPORTED;
        }
        T->max_nt = std::max(T->max_nt, nti);
        T->max_len = std::max(T->max_len, sc.length(i));
        for (int j = 0; j < ndet; ++j) {
            const int b = i * ndet + j;
            off[b] = at;
            row[b] = sc.sample_row[i];
            len[b] = sc.length(i);
            nt[b] = nti;
            ampo[b] = na;
            kino[b] = nk;
            at += sc.length(i);
            na += nti;
            nk += (int64_t) nti * nti;
        }
    }
    T->m = at;
    T->namp = na;
    std::vector<double> kinv((size_t) nk);
    MDP_TRY(kernels_impl(sc, h_w_block, kinv.data()));
    MDP_TRY(upload(T->bins, bins));
    MDP_TRY(upload(T->wg, wg));
    MDP_TRY(upload(T->blk_off, off));
    MDP_TRY(upload(T->blk_row, row));
    MDP_TRY(upload(T->blk_amp, ampo));
    MDP_TRY(upload(T->blk_kinv, kino));
    MDP_TRY(upload(T->blk_len, len));
    MDP_TRY(upload(T->blk_nt, nt));
    MDP_TRY(upload(T->blk_w, w));
    MDP_TRY(upload(T->kinv, kinv));
    MDP_TRY(T->amp.alloc((size_t) na * sizeof(double)));
    MDP_TRY(T->coef.alloc((size_t) na * sizeof(double)));
    *out = guard.release();
    return MDP_OK;
}

extern "C" void mdp_templates_destroy(mdp_templates *T) { delete T; }

extern "C" int mdp_templates_samples(const mdp_templates *T, int64_t *m, int64_t *n_amplitudes) {
    if (!T) return MDP_EINVAL;
    if (m) *m = T->m;
    if (n_amplitudes) *n_amplitudes = T->namp;
    return MDP_OK;
}

extern "C" int mdp_templates_filter(mdp_context *ctx, const mdp_templates *T, const double *d_in, double *d_out) {
    if (!ctx || !T || !d_in || !d_out) {
        mdp_set_error("mdp_templates_filter: bad argument");
        return MDP_EINVAL;
    }
    double *amp = T->amp.as<double>(), *coef = T->coef.as<double>();
    MDP_CUDA(cudaMemsetAsync(amp, 0, (size_t) T->namp * sizeof(double), ctx->stream));
    const int chunks = (int) std::max<int64_t>(1, std::min<int64_t>(64, (T->max_len + 2047) / 2048));
    const dim3 grid(chunks, T->nb);
    tpl_tt_kernel<<<grid, kTplThreads, (size_t) T->max_nt * sizeof(double), ctx->stream>>>(
        d_in, T->bins.as<int32_t>(), T->wg.as<double>(), T->nc, T->blk_off.as<int64_t>(), T->blk_row.as<int64_t>(),
        T->blk_len.as<int32_t>(), T->blk_nt.as<int32_t>(), T->blk_amp.as<int64_t>(), T->blk_w.as<double>(), amp);
    MDP_CHECK_LAUNCH(ctx);
    tpl_b_kernel<<<T->nb, kTplThreads, 0, ctx->stream>>>(T->kinv.as<double>(), T->blk_kinv.as<int64_t>(),
                                                         T->blk_nt.as<int32_t>(), T->blk_amp.as<int64_t>(), amp,
                                                         coef);
    MDP_CHECK_LAUNCH(ctx);
    tpl_t_kernel<<<grid, kTplThreads, 0, ctx->stream>>>(
        d_in, T->bins.as<int32_t>(), T->wg.as<double>(), T->nc, T->blk_off.as<int64_t>(), T->blk_row.as<int64_t>(),
        T->blk_len.as<int32_t>(), T->blk_nt.as<int32_t>(), T->blk_amp.as<int64_t>(), T->blk_w.as<double>(), coef,
        d_out);
    MDP_CHECK_LAUNCH(ctx);
    return MDP_OK;
}

// MTmap's solve (PCG_GLS_templates, mappraiser/src/pcg_true.c:243-560, as MTmap calls it,
// mappraiser.c:586-680): block Jacobi from the white noise operator N (lambda = 1, the
// blocks' weights) with the rcond cut, then the PCG_GLS_true recurrences with the
// weighting W - W T B T^T W.
extern "C" int mdp_gls_solve_templates(mdp_context *ctx, mdp_pointing *A, const mdp_noise *N, const mdp_templates *T,
                                       const double *d_signal, const double *d_noise, const mdp_solve_params *params,
                                       double *d_x, int32_t *d_lstid, double *d_cond, int32_t *d_hits,
                                       double *h_res_rel, mdp_solve_info *info) {
    if (!ctx || !A || !N || !T || !d_signal || !d_noise || !params || !d_x) {
        mdp_set_error("mdp_gls_solve_templates: invalid arguments");
        return MDP_EINVAL;
    }
    if (N->lambda != 1 || N->nb != T->nb || T->m != A->m || N->nrow_end > A->m) {
        mdp_set_error("mdp_gls_solve_templates: the noise operator must be white (lambda 1) with one block per "
                      "template block, and the filter must cover the pointing's %lld rows", (long long) A->m);
        return MDP_EINVAL;
    }
    if (params->precond != 0) {
        mdp_set_error("mdp_gls_solve_templates: only the block-Jacobi preconditioner (precond 0)");
        return MDP_EUNSUPPORTED;
    }
    MDP_CUDA(cudaSetDevice(ctx->device));
    const BJState *bjp = nullptr;
    MDP_TRY(mdp_bj_cached(ctx, A, N, &bjp));
    const BJState &bj = *bjp;
    cudaStream_t st = ctx->stream;
    if (d_lstid)
        MDP_CUDA(cudaMemcpyAsync(d_lstid, A->lindices.as<int32_t>() + 3 * A->trash_pix, 4 * A->n_map(),
                                 cudaMemcpyDeviceToDevice, st));
    if (d_cond) MDP_CUDA(cudaMemcpyAsync(d_cond, bj.rcond.p, 8 * bj.npix, cudaMemcpyDeviceToDevice, st));
    if (d_hits) MDP_CUDA(cudaMemcpyAsync(d_hits, bj.hits.p, 4 * bj.npix, cudaMemcpyDeviceToDevice, st));
    MDP_TRY(mdp_pcg_run(ctx, A, N, bj.inv.as<double>(), bj.npix, d_signal, d_noise, params, d_x, h_res_rel, info,
                        nullptr, T));
    if (info) {
        info->n_cut = bj.ncut;
        info->n_map = A->n_map();
        info->outer_iterations = 0;
        info->fp64_applications = info->iterations;
    }
    return MDP_OK;
}
