// Set-up of MTmap's template-filtered solve (host side, as in the reference).
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

#include <cmath>
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

extern "C" int mdp_template_kernels(const mdp_template_scan *scan, const double *h_w_block, double *h_kinv) {
    Scan sc;
    MDP_TRY(make_scan(scan, &sc));
    if (!h_w_block || !h_kinv) {
        mdp_set_error("mdp_template_kernels: bad argument");
        return MDP_EINVAL;
    }
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
