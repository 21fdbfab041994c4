// Small dense symmetric problems solved on the host (at most 128 x 128): the
// eigen-decomposition and pseudo-inverse of the two-level preconditioners
// (precond.c:770-788, 1190-1212 call LAPACK dsyev / dgelss on the host) and
// the Cholesky / eigen factors of the ECG block orthonormalisation.
#pragma once
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <vector>

namespace mdp_dense {

// Cyclic two-sided Jacobi eigen-decomposition of the symmetric K x K matrix a
// (row-major, destroyed): eigenvalues ascending in w, eigenvectors as the
// columns of y (row-major).  Golub & Van Loan, Matrix Computations 4th ed., 8.5.
inline void jacobi_eigh(int K, std::vector<double> &a, std::vector<double> &w, std::vector<double> &y) {
    std::vector<double> v((size_t) K * K, 0.0);
    for (int i = 0; i < K; i++) v[(size_t) i * K + i] = 1.0;
    auto A = [&](int i, int j) -> double & { return a[(size_t) i * K + j]; };
    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0.0, tot = 0.0;
        for (int i = 0; i < K; i++)
            for (int j = 0; j < K; j++) {
                tot += A(i, j) * A(i, j);
                if (i != j) off += A(i, j) * A(i, j);
            }
        if (off == 0.0 || off <= DBL_EPSILON * DBL_EPSILON * tot) break;
        for (int p = 0; p < K - 1; p++)
            for (int q = p + 1; q < K; q++) {
                const double apq = A(p, q);
                if (apq == 0.0) continue;
                const double theta = (A(q, q) - A(p, p)) / (2.0 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < K; k++) {
                    const double akp = A(k, p), akq = A(k, q);
                    A(k, p) = c * akp - s * akq;
                    A(k, q) = s * akp + c * akq;
                }
                for (int k = 0; k < K; k++) {
                    const double apk = A(p, k), aqk = A(q, k);
                    A(p, k) = c * apk - s * aqk;
                    A(q, k) = s * apk + c * aqk;
                }
                for (int k = 0; k < K; k++) {
                    const double vkp = v[(size_t) k * K + p], vkq = v[(size_t) k * K + q];
                    v[(size_t) k * K + p] = c * vkp - s * vkq;
                    v[(size_t) k * K + q] = s * vkp + c * vkq;
                }
            }
    }
    std::vector<int> ord(K);
    for (int i = 0; i < K; i++) ord[i] = i;
    std::stable_sort(ord.begin(), ord.end(), [&](int x, int z) { return A(x, x) < A(z, z); });
    w.assign(K, 0.0);
    y.assign((size_t) K * K, 0.0);
    for (int j = 0; j < K; j++) {
        w[j] = A(ord[j], ord[j]);
        for (int i = 0; i < K; i++) y[(size_t) i * K + j] = v[(size_t) i * K + ord[j]];
    }
}

// Pseudo-inverse of the n x n matrix e (row-major) as DGELSS(e, I) computes
// it: the minimum-norm least-squares solution, singular values <= rcond *
// s_max treated as zero.  One-sided Jacobi SVD (Hestenes 1958; Demmel &
// Veselic, SIAM J. Matrix Anal. Appl. 13:1204, 1992) on the columns of e.
inline std::vector<double> pinv_gelss(int n, const std::vector<double> &e, double rcond) {
    std::vector<double> u(e), v((size_t) n * n, 0.0), out((size_t) n * n, 0.0), sv(n);
    auto U = [&](int i, int j) -> double & { return u[(size_t) i * n + j]; };
    auto Vm = [&](int i, int j) -> double & { return v[(size_t) i * n + j]; };
    for (int i = 0; i < n; i++) Vm(i, i) = 1.0;
    for (int sweep = 0; sweep < 100; sweep++) {
        bool rotated = false;
        for (int p = 0; p < n - 1; p++)
            for (int q = p + 1; q < n; q++) {
                double al = 0.0, be = 0.0, ga = 0.0;
                for (int k = 0; k < n; k++) {
                    al += U(k, p) * U(k, p);
                    be += U(k, q) * U(k, q);
                    ga += U(k, p) * U(k, q);
                }
                if (ga == 0.0 || std::fabs(ga) <= DBL_EPSILON * std::sqrt(al * be)) continue;
                rotated = true;
                const double zeta = (be - al) / (2.0 * ga);
                const double t = (zeta >= 0 ? 1.0 : -1.0) / (std::fabs(zeta) + std::sqrt(1.0 + zeta * zeta));
                const double c = 1.0 / std::sqrt(1.0 + t * t), s = c * t;
                for (int k = 0; k < n; k++) {
                    const double up = U(k, p), uq = U(k, q);
                    U(k, p) = c * up - s * uq;
                    U(k, q) = s * up + c * uq;
                }
                for (int k = 0; k < n; k++) {
                    const double vp = Vm(k, p), vq = Vm(k, q);
                    Vm(k, p) = c * vp - s * vq;
                    Vm(k, q) = s * vp + c * vq;
                }
            }
        if (!rotated) break;
    }
    double smax = 0.0;
    for (int j = 0; j < n; j++) {
        double nn = 0.0;
        for (int k = 0; k < n; k++) nn += U(k, j) * U(k, j);
        sv[j] = std::sqrt(nn);
        smax = std::max(smax, sv[j]);
    }
    // e = sum_j (u_j / s_j) s_j v_j^T  =>  e^+ = sum_j v_j u_j^T / s_j^2 over the kept j
    for (int j = 0; j < n; j++) {
        if (!(sv[j] > rcond * smax)) continue;
        const double s2 = sv[j] * sv[j];
        for (int r = 0; r < n; r++)
            for (int c = 0; c < n; c++) out[(size_t) r * n + c] += Vm(r, j) * U(c, j) / s2;
    }
    return out;
}

// Cholesky factor L (lower, row-major) of the symmetric positive definite
// n x n matrix g; false when a pivot is not positive.
inline bool cholesky(int n, const std::vector<double> &g, std::vector<double> &L) {
    L.assign((size_t) n * n, 0.0);
    for (int j = 0; j < n; j++) {
        double d = g[(size_t) j * n + j];
        for (int k = 0; k < j; k++) d -= L[(size_t) j * n + k] * L[(size_t) j * n + k];
        if (!(d > 0.0)) return false;
        const double ljj = std::sqrt(d);
        L[(size_t) j * n + j] = ljj;
        for (int i = j + 1; i < n; i++) {
            double s = g[(size_t) i * n + j];
            for (int k = 0; k < j; k++) s -= L[(size_t) i * n + k] * L[(size_t) j * n + k];
            L[(size_t) i * n + j] = s / ljj;
        }
    }
    return true;
}

// Inverse of the lower-triangular n x n matrix L (row-major), by forward substitution.
inline std::vector<double> lower_inverse(int n, const std::vector<double> &L) {
    std::vector<double> X((size_t) n * n, 0.0);
    for (int c = 0; c < n; c++)
        for (int i = c; i < n; i++) {
            double s = (i == c) ? 1.0 : 0.0;
            for (int k = c; k < i; k++) s -= L[(size_t) i * n + k] * X[(size_t) k * n + c];
            X[(size_t) i * n + c] = s / L[(size_t) i * n + i];
        }
    return X;
}

}  // namespace mdp_dense
