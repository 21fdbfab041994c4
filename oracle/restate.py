"""CPU restatement of the reference's GLS map-making path (numpy / scipy).

TEST INFRASTRUCTURE ONLY: imported by tests/, by the smoke check and by
bench.py's CPU-baseline leg, always as the checker, never as the thing
measured or shipped.  The product path (midapack_b200) never imports it.

Each function restates one reference routine (file:line in its docstring,
paths relative to the reference project root).  The restatement is pinned
against the reference's own compiled C (oracle/_ref, built by
oracle/build_ref.sh) in tests/test_oracle_pin.py.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


# --------------------------------------------------------------------------- pointing
@dataclass
class Pointing:
    m: int
    nnz: int
    local: np.ndarray      # int32 [m*nnz] local indices (position in lindices)
    values: np.ndarray     # f64  [m*nnz]
    lindices: np.ndarray   # int32 sorted unique global indices
    trash_pix: int

    @property
    def lcount(self) -> int:
        return int(self.lindices.size)

    @property
    def n(self) -> int:
        """Map-domain size: lcount - nnz*trash_pix (mappraiser.c:96-98)."""
        return self.lcount - self.nnz * self.trash_pix


def local_shape(gindices: np.ndarray, values: np.ndarray, m: int, nnz: int) -> Pointing:
    """MatInit -> MatLocalShape (algebra/src/mapmat/mapmat.c:54-73, 496-521).

    lindices = sorted unique global indices (counting_sort, csort.c:111-135);
    each index becomes its position in lindices (sindex/dichotomy,
    cindex.c:34-42, 102-116); trash_pix = 1 when lindices[0] < 0.
    """
    g = np.asarray(gindices, dtype=np.int32)
    lind = np.unique(g)
    local = np.searchsorted(lind, g).astype(np.int32)
    trash = 1 if lind.size and lind[0] < 0 else 0
    return Pointing(m, nnz, local, np.asarray(values, dtype=np.float64), lind.astype(np.int32), trash)


def matvec(A: Pointing, x: np.ndarray) -> np.ndarray:
    """y = P x, MatVecProd (mapmat.c:704-729), including the trash-row skip."""
    idx = A.local.reshape(A.m, A.nnz).astype(np.int64)
    val = A.values.reshape(A.m, A.nnz)
    if A.trash_pix:
        keep = idx[:, 0] != 0
        y = np.zeros(A.m)
        xi = x[np.where(keep[:, None], idx - A.nnz, 0)]
        # accumulate in the reference's j order: ((0 + v0 x0) + v1 x1) + v2 x2
        acc = np.zeros(A.m)
        for j in range(A.nnz):
            acc = acc + val[:, j] * xi[:, j]
        y[keep] = acc[keep]
        return y
    acc = np.zeros(A.m)
    for j in range(A.nnz):
        acc = acc + val[:, j] * x[idx[:, j]]
    return acc


def trmatvec(A: Pointing, y: np.ndarray) -> np.ndarray:
    """x = P^T y, TrMatVecProd (mapmat.c:819-859); single rank, so the
    ALLREDUCE of greedyreduce (mapmat.c:1008-1141) is the identity.
    np.add.at accumulates in sample order, like the reference loop."""
    idx = A.local.reshape(A.m, A.nnz).astype(np.int64)
    val = A.values.reshape(A.m, A.nnz)
    x = np.zeros(A.n)
    if A.trash_pix:
        keep = idx[:, 0] != 0
        ii = (idx[keep] - A.nnz)
        contrib = val[keep] * y[keep][:, None]
    else:
        ii = idx
        contrib = val * y[:, None]
    np.add.at(x, ii.reshape(-1), contrib.reshape(-1))
    return x


# --------------------------------------------------------------------------- Toeplitz
def block_offsets(block_sizes: np.ndarray) -> np.ndarray:
    """idv of each block (create_toeplitz.c:27-47, id0 = 0)."""
    off = np.zeros(len(block_sizes) + 1, dtype=np.int64)
    off[1:] = np.cumsum(np.asarray(block_sizes, dtype=np.int64))
    return off


def banded_toeplitz_fft(v: np.ndarray, t: np.ndarray) -> np.ndarray:
    """Exact (within a block, zero outside) symmetric banded Toeplitz product,
    computed as one linear convolution by FFT of a padded length.  The
    reference's overlap-save tiling (toeplitz.c:731-865) computes the same
    product tile by tile."""
    n = v.size
    lam = t.size
    if lam == 1:
        return v * t[0]
    h = np.concatenate([t[:0:-1], t])  # kernel, taps -(lam-1)..(lam-1)
    L = n + h.size - 1
    nfft = 1 << int(np.ceil(np.log2(L)))
    full = np.fft.irfft(np.fft.rfft(v, nfft) * np.fft.rfft(h, nfft), nfft)[:L]
    return full[lam - 1: lam - 1 + n]


def banded_toeplitz_direct(v: np.ndarray, t: np.ndarray) -> np.ndarray:
    """Same product by direct summation in long double: the exact arbiter for
    small cases (the reference's no-FFT product, toeplitz_nofft.c:104-150,
    computed here for the edges too)."""
    n = v.size
    lam = t.size
    vl = v.astype(np.longdouble)
    out = vl * np.longdouble(t[0])
    for k in range(1, min(lam, n)):
        tk = np.longdouble(t[k])
        out[k:] += tk * vl[:-k]
        out[:-k] += tk * vl[k:]
    return out.astype(np.float64)


def stbmm(V: np.ndarray, block_sizes: np.ndarray, lam: int, invtt: np.ndarray, exact: bool = False) -> np.ndarray:
    """apply_weights (pcg_true.c:578-600) -> stbmmProd (toeplitz_wizard.c:80-111):
    per block, subtract the block mean, then the banded Toeplitz product; with
    lambda == 1 only the diagonal scaling (no mean removal)."""
    out = np.array(V, dtype=np.float64, copy=True)
    off = block_offsets(block_sizes)
    for b in range(len(block_sizes)):
        s, e = off[b], off[b + 1]
        t = np.asarray(invtt[b * lam:(b + 1) * lam], dtype=np.float64)
        if lam == 1:
            out[s:e] = t[0] * out[s:e]
            continue
        seg = out[s:e]
        seg = seg - seg.sum() / (e - s)
        out[s:e] = banded_toeplitz_direct(seg, t) if exact else banded_toeplitz_fft(seg, t)
    return out


# --------------------------------------------------------------------------- block Jacobi
def local_W(A: Pointing, block_sizes: np.ndarray, lam: int, invtt: np.ndarray):
    """getlocalW (mappraiser/src/precond.c:42-161): per-pixel 3x3 blocks of
    P^T diag(N^-1) P and hit counts; diag(N^-1) = T_block[0] inside a block."""
    nnz = A.nnz
    off = block_offsets(block_sizes)
    diag = np.empty(A.m)
    for b in range(len(block_sizes)):
        diag[off[b]:off[b + 1]] = invtt[b * lam]
    if off[-1] < A.m:
        diag[off[-1]:] = 1.0
    idx = A.local.reshape(A.m, nnz).astype(np.int64)
    val = A.values.reshape(A.m, nnz)
    keep = (idx[:, 0] != 0) if A.trash_pix else np.ones(A.m, dtype=bool)
    npx = A.n // nnz
    W = np.zeros(npx * nnz * nnz)
    hits = np.zeros(npx, dtype=np.int64)
    ik = idx[keep] - nnz * A.trash_pix
    vk = val[keep]
    dk = diag[keep]
    np.add.at(hits, ik[:, 0] // nnz, 1)
    for j in range(nnz):
        for k in range(nnz):
            np.add.at(W, nnz * ik[:, j] + k, vk[:, j] * vk[:, k] * dk)
    return W.reshape(npx, nnz, nnz), hits


def bj_blocks(W: np.ndarray):
    """Per pixel: anorm = dlange('1'), LU = dgetrf, rcond = dgecon('1'); keep
    the pixel when rcond > 0.1 and invert with dgetri
    (precond.c:511-583).  Uses scipy's LAPACK, i.e. the real routines."""
    from scipy.linalg import lapack

    npx = W.shape[0]
    rcond = np.zeros(npx)
    inv = np.zeros_like(W)
    for p in range(npx):
        a = np.array(W[p], dtype=np.float64, order="F")
        anorm = np.abs(a).sum(axis=0).max()
        lu, piv, info = lapack.dgetrf(a)
        rc, info2 = lapack.dgecon(lu, anorm, norm="1")
        rcond[p] = rc
        if rc > 1e-1:
            ainv, info3 = lapack.dgetri(lu, piv)
            inv[p] = ainv
    return rcond, inv


@dataclass
class BJResult:
    A: Pointing               # pointing after the cut (re-initialised)
    signal: np.ndarray        # b with cut samples zeroed
    inv: np.ndarray           # [n/3, 3, 3] inverse blocks of kept pixels
    W: np.ndarray             # [n/3, 3, 3] blocks of kept pixels
    cond: np.ndarray          # rcond of kept pixels
    hits: np.ndarray          # hits of kept pixels
    cut: np.ndarray           # bool per pre-cut pixel


def precond_blockjacobi(A: Pointing, signal: np.ndarray, block_sizes, lam, invtt) -> BJResult:
    """precondblockjacobilike (precond.c:456-702): cut pixels with rcond <= 0.1,
    point their samples to the trash triplet (-3,-2,-1) with zero weights, zero
    their signal samples, then MatInit again on the rewritten global indices."""
    nnz = A.nnz
    W, hits = local_W(A, block_sizes, lam, invtt)
    rcond, inv = bj_blocks(W)
    cut = ~(rcond > 1e-1)
    gl = A.lindices[A.local.astype(np.int64)].astype(np.int32)  # back to global indices
    vals = A.values.copy()
    sig = np.array(signal, dtype=np.float64, copy=True)
    if cut.any():
        # The reference walks the pixel->samples linked list from
        # id_last_pix[u + trash_pix] for the u-th pixel block
        # (precond.c:521, 585-600), while MLmap indexes id_last_pix by
        # u itself (mappraiser.c:130-142).  With flagged samples present the
        # samples rewritten are therefore those of pixel u + 1; that is kept
        # here as the reference behaves (a target past the last pixel rewrites
        # nothing).
        idx = A.local.reshape(A.m, nnz).astype(np.int64)
        valid = (idx[:, 0] != 0) if A.trash_pix else np.ones(A.m, dtype=bool)
        pixrow = np.where(valid, idx[:, 0] // nnz - A.trash_pix, -1)
        npx = cut.size
        target = np.zeros(npx, dtype=bool)
        cu = np.nonzero(cut)[0] + A.trash_pix
        target[cu[cu < npx]] = True
        rows = valid & target[np.clip(pixrow, 0, None)]
        g2 = gl.reshape(A.m, nnz)
        g2[rows] = np.arange(nnz, dtype=np.int32) - nnz
        vals.reshape(A.m, nnz)[rows] = 0.0
        sig[rows] = 0.0
        gl = g2.reshape(-1)
    A2 = local_shape(gl, vals, A.m, nnz)
    if cut.any():
        A2.trash_pix = 1
    keep = ~cut
    inv_k, W_k, rc_k, h_k = inv[keep], W[keep], rcond[keep], hits[keep]
    npix2 = A2.n // nnz
    if npix2 > inv_k.shape[0]:
        # with flagged samples and the last pixel cut, the cut target lies past
        # the end: no pixel leaves the map and the reference leaves the last
        # preconditioner rows unset (uninitialised); they are zero blocks here
        pad = npix2 - inv_k.shape[0]
        inv_k = np.concatenate([inv_k, np.zeros((pad, nnz, nnz))])
        W_k = np.concatenate([W_k, np.zeros((pad, nnz, nnz))])
        rc_k = np.concatenate([rc_k, np.zeros(pad)])
        h_k = np.concatenate([h_k, np.zeros(pad, dtype=h_k.dtype)])
    return BJResult(A2, sig, inv_k, W_k, rc_k, h_k, cut)


def apply_bj(inv: np.ndarray, g: np.ndarray) -> np.ndarray:
    """apply_precond, precond = 0 (precond.c:1403-1409): MatVecProd(BJ_inv, g)."""
    gp = g.reshape(-1, 3)
    out = np.zeros_like(gp)
    for j in range(3):
        out = out + inv[:, :, j] * gp[:, j:j + 1]
    return out.reshape(-1)


# --------------------------------------------------------------------------- two-level preconditioners
EPS_2LVL = 1.0e-15  # precond.c:25


def build_Z(A: Pointing, Zn: int) -> np.ndarray:
    """build_Z (precond.c:791-938), one rank: the a-priori deflation columns.

    The rows are split into Zn equal groups (m // Zn rows each, the rest left
    out); count[g][i] counts local index i in group g and tcount[i] sums the
    groups.  Column g holds, at the I entry i = 3q of every local pixel,
    count_flat[g * group + i] / tcount[i] with count_flat the [group][lcount]
    array flattened -- the reference's index (precond.c:878), kept as it is --
    and zero at the Q and U entries; the trash entries are then dropped.
    Returns Z as [Zn][n]."""
    size = 1
    group = Zn // size if Zn > size else 1
    lc, nnz = A.lcount, A.nnz
    per = (A.m // group) * nnz
    count = np.zeros(group * lc, dtype=np.int64)
    for g in range(group):
        count[g * lc:(g + 1) * lc] = np.bincount(A.local[g * per:(g + 1) * per].astype(np.int64), minlength=lc)
    tcount = count.reshape(group, lc).sum(axis=0)
    Z = np.zeros((group * size, lc))
    i = np.arange(0, lc, nnz)
    with np.errstate(divide="ignore", invalid="ignore"):
        for g in range(group):
            Z[g, i] = count[g * group + i].astype(np.float64) / tcount[i].astype(np.float64)
    return Z[:, nnz * A.trash_pix:].copy()


def build_AZ(op, Z: np.ndarray) -> np.ndarray:
    """build_AZ (precond.c:1003-1024): AZ[i] = P^T N^-1 P Z[i]."""
    return np.stack([op(z) for z in Z])


def pinv_gelss(E: np.ndarray, rcond: float = EPS_2LVL) -> np.ndarray:
    """inverse_svd_bis (precond.c:772-788): LAPACKE_dgelss(E, I) with rcond = eps,
    the minimum-norm least-squares inverse; singular values <= rcond * s_max
    count as zero."""
    U, sv, Vt = np.linalg.svd(E)
    keep = sv > rcond * sv[0] if sv.size else sv.astype(bool)
    return (Vt[keep].T / sv[keep]) @ U[:, keep].T


def build_Em1(Z: np.ndarray, AZ: np.ndarray) -> np.ndarray:
    """build_Em1 (precond.c:951-1000), pixpond = 1: E[i][j] = sum_k Z[j][k] AZ[i][k],
    then its dgelss pseudo-inverse."""
    return pinv_gelss(AZ @ Z.T)


def lanczos_eig(op, w0: np.ndarray, K: int):
    """Lanczos_eig (precond.c:1028-1252), pixpond = 1: K Lanczos steps from
    w0 = P^T N^-1 (b + noise - P x0), the K x K tridiagonal T, its eigenvectors Y
    (dsyev) and the Ritz vectors Z = V Y, AZ = (A V) Y.

    Kept as the reference does: the first three-term update subtracts
    beta * vold with vold still zero (precond.c:1161,1196-1200), and a step
    with beta <= eps leaves its Lanczos vector column zero and v unchanged.
    The reference's last operator application (step K) only feeds entries
    that its K x K truncation drops, so it is not made here."""
    n = w0.size
    beta = float(np.sqrt(np.dot(w0, w0)))
    v = w0 / beta if beta > EPS_2LVL else np.zeros(n)
    V = np.zeros((K + 1, n))
    AV = np.zeros((K + 1, n))
    V[0] = v
    Av = op(v)
    alpha = float(np.dot(v, Av))
    AV[0] = Av
    w = Av - alpha * v
    vold = np.zeros(n)
    T = np.zeros((K + 1, K + 1))
    for i in range(K):
        beta = float(np.sqrt(np.dot(w, w)))
        if beta > EPS_2LVL:
            v = w / beta
            V[i + 1] = v
        T[i, i], T[i, i + 1], T[i + 1, i] = alpha, beta, beta
        if i == K - 1:
            break
        Av = op(v)
        alpha = float(np.dot(v, Av))
        AV[i + 1] = Av
        w = Av - alpha * v - beta * vold
        vold = v
    _, Y = np.linalg.eigh(T[:K, :K])
    return Y.T @ V[:K], Y.T @ AV[:K]


@dataclass
class TwoLevel:
    Z: np.ndarray     # [Zn][n]
    AZ: np.ndarray    # [Zn][n]
    Em1: np.ndarray   # [Zn][Zn]


def apply_2lvl(p: TwoLevel, inv: np.ndarray, g: np.ndarray) -> np.ndarray:
    """apply_precond, precond 1/2 (precond.c:1412-1423; build_Qtx, mul_ZQtx at
    :1026-1069): Qtx = Em1 Z^T g; Cg = BJ_inv (g - AZ Qtx) + Z Qtx."""
    Qtx = p.Em1 @ (p.Z @ g)
    Qg = p.Z.T @ Qtx
    AQg = g - p.AZ.T @ Qtx
    return apply_bj(inv, AQg) + Qg


# --------------------------------------------------------------------------- PCG
@dataclass
class PCGResult:
    x: np.ndarray
    iters: int
    res_rel: list
    bj: BJResult


def pcg(gindices, values, signal, noise, block_sizes, lam, invtt, tol=1e-8, maxiter=500,
        nnz: int = 3, exact_toeplitz: bool = False, precond: int = 0, z_2lvl: int = 0) -> PCGResult:
    """PCG_GLS_true (mappraiser/src/pcg_true.c:20-241), single rank (pixpond = 1):
    Polak-Ribiere PCG on (P^T N^-1 P) x = P^T N^-1 (b + noise), stop when
    sum(g^2) <= tol^2 * sum(g0^2).  precond 0: block Jacobi; 1: two-level a
    priori (build_Z); 2: two-level a posteriori (Lanczos_eig), with z_2lvl
    deflation columns (0: one per rank, pcg_true.c:52)."""
    m = len(signal)
    A = local_shape(gindices, values, m, nnz)
    bj = precond_blockjacobi(A, signal, block_sizes, lam, invtt)
    A = bj.A
    n = A.n
    x = np.zeros(n)
    N = lambda v: stbmm(v, block_sizes, lam, invtt, exact=exact_toeplitz)  # noqa: E731
    op = lambda v: trmatvec(A, N(matvec(A, v)))  # noqa: E731
    _g = bj.signal + noise - matvec(A, x)
    g = trmatvec(A, N(_g))
    Zn = z_2lvl if z_2lvl else 1
    if precond == 0:
        M = lambda r: apply_bj(bj.inv, r)  # noqa: E731
    elif precond in (1, 2):
        if precond == 1:
            Z = build_Z(A, Zn)
            AZ = build_AZ(op, Z)
        else:
            Z, AZ = lanczos_eig(op, g, Zn)
        tl = TwoLevel(Z, AZ, build_Em1(Z, AZ))
        M = lambda r: apply_2lvl(tl, bj.inv, r)  # noqa: E731
    else:
        raise ValueError(f"precond {precond}")
    Cg = M(g)
    h = Cg.copy()
    g2pix = float(np.dot(Cg, g))
    res = float(np.dot(g, g))
    res0 = res
    tol2rel = tol * tol * res
    res_rel = [1.0]
    k = 1
    if res <= tol:
        return PCGResult(x, 0, res_rel, bj)
    while k < maxiter:
        gp = g
        Ah = matvec(A, h)
        AtNm1Ah = trmatvec(A, N(Ah))
        coeff = float(np.dot(h, AtNm1Ah))
        ro = g2pix / coeff
        x = x + ro * h
        g = gp - ro * AtNm1Ah
        Cg = M(g)
        g2pixp = g2pix
        g2pix = float(np.dot(Cg, g))
        g2pix_polak = float(np.dot(Cg, g - gp))
        res = float(np.dot(g, g))
        res_rel.append(float(np.sqrt(res) / np.sqrt(res0)))
        if res <= tol2rel:
            break
        gamma = g2pix_polak / g2pixp
        h = h * gamma + Cg
        k += 1
    return PCGResult(x, k, res_rel, bj)


# --------------------------------------------------------------------------- ECG
def ecg_split(r: np.ndarray, t: int) -> np.ndarray:
    """The enlarged residual T(r): column j keeps the entries of the j-th of t
    contiguous ranges of the map's pixels (unknowns sorted by global index,
    pixel triples kept together), zero elsewhere.  Returns [t][n]."""
    n = r.size
    npix = n // 3
    col = (np.arange(n) // 3) * t // max(npix, 1)
    R = np.zeros((t, n))
    R[col, np.arange(n)] = r
    return R


def a_orthonormalize(P: np.ndarray, AP: np.ndarray, bs_red: bool, tol: float = 1e-12):
    """P <- P G^{-1/2}-like factor with G = P^T A P: the Cholesky factor
    G = L L^T gives P L^-T (bs unchanged); with bs_red a rank-revealing
    eigen-decomposition G = V diag(l) V^T keeps the directions with
    l > tol * max(l) and scales them to l^-1/2 (the block size may shrink).
    Returns (P, AP) with P^T A P = I."""
    G = P @ AP.T
    G = 0.5 * (G + G.T)
    if not bs_red:
        L = np.linalg.cholesky(G)
        Li = np.linalg.inv(L)
        return Li @ P, Li @ AP
    lam, V = np.linalg.eigh(G)
    keep = lam > tol * lam.max()
    F = V[:, keep] / np.sqrt(lam[keep])
    return F.T @ P, F.T @ AP


@dataclass
class ECGResult:
    x: np.ndarray
    iters: int
    res_rel: list
    bs: list
    bj: BJResult


def ecg(gindices, values, signal, noise, block_sizes, lam, invtt, tol=1e-8, maxiter=500, enl=4, ortho_alg=1,
        bs_red=0, nnz: int = 3) -> ECGResult:
    """ECG_GLS (mappraiser/src/ecg.c:44-175) with the enlarged conjugate
    gradient of preAlps (absent here; restated from Grigori, Moufawad & Nataf,
    SIAM J. Matrix Anal. Appl. 37:744, 2016, and Grigori & Tissot, "Reducing
    the communication and computational costs of enlarged Krylov subspaces
    conjugate gradient", Numer. Algorithms 80:1333, 2019), one rank:

      R_0 = T(r_0), P_1 = M^-1 R_0, A-orthonormalised
      k = 1, 2, ...: alpha = P^T R; X += P alpha; R -= AP alpha;
        stop when ||sum_j R_j|| < tol ||r_0|| (ecg.c:131-136);
        Orthomin (ortho_alg 1): Z = M^-1 R, P <- Z - P (AP^T Z);
        Orthodir (ortho_alg 0): Z = M^-1 AP, P <- Z - P (AP^T Z) - P_prev (AP_prev^T Z);
        AP = A P, A-orthonormalise (bs_red: rank-revealing, the block may shrink)
      x = sum_j X_j.
    M is the block-Jacobi preconditioner with the rcond cut (ecg.c:67)."""
    m = len(signal)
    A = local_shape(gindices, values, m, nnz)
    bj = precond_blockjacobi(A, signal, block_sizes, lam, invtt)
    A = bj.A
    n = A.n
    N = lambda v: stbmm(v, block_sizes, lam, invtt)  # noqa: E731
    op = lambda v: trmatvec(A, N(matvec(A, v)))  # noqa: E731
    Mi = lambda V: np.stack([apply_bj(bj.inv, v) for v in V])  # noqa: E731
    opb = lambda V: np.stack([op(v) for v in V])  # noqa: E731
    r0 = trmatvec(A, N(bj.signal + noise))
    normb = float(np.sqrt(np.dot(r0, r0)))
    R = ecg_split(r0, enl)
    X = np.zeros((enl, n))
    P = Mi(R)
    AP = opb(P)
    P, AP = a_orthonormalize(P, AP, bool(bs_red))
    Pp = APp = None
    res_rel = [1.0]
    bs = [P.shape[0]]
    it = 0
    while it < maxiter:
        alpha = P @ R.T                      # [bs][t]
        X = X + alpha.T @ P
        R = R - alpha.T @ AP
        it += 1
        r = R.sum(axis=0)
        res = float(np.sqrt(np.dot(r, r)))
        res_rel.append(res / normb)
        if res < tol * normb:
            break
        if ortho_alg == 1:
            Z = Mi(R)
            Pn = Z - (AP @ Z.T).T @ P
        else:
            Z = Mi(AP)
            Pn = Z - (AP @ Z.T).T @ P
            if Pp is not None:
                Pn = Pn - (APp @ Z.T).T @ Pp
            Pp, APp = P, AP
        P, AP = a_orthonormalize(Pn, opb(Pn), bool(bs_red))
        bs.append(P.shape[0])
    return ECGResult(X.sum(axis=0), it, res_rel, bs, bj)


def x2map_pol(x, lstid, cond, hits, npix):
    """x2map_pol (mappraiser/src/mappraiser.c:836-853)."""
    mapI = np.zeros(npix)
    mapQ = np.zeros(npix)
    mapU = np.zeros(npix)
    Cond = np.zeros(npix)
    Hits = np.zeros(npix, dtype=np.int32)
    p = (np.asarray(lstid[0::3]) // 3).astype(np.int64)
    mapI[p] = x[0::3]
    mapQ[p] = x[1::3]
    mapU[p] = x[2::3]
    Cond[p] = cond
    Hits[p] = hits
    return mapI, mapQ, mapU, Cond, Hits


# --------------------------------------------------------------------------- noise2invtt
NOISE_FIT_P0 = (-7.0, -1.0, 0.1, 1e-6)
NOISE_FIT_BOUNDS = ([-20.0, -10.0, 0.0, 0.0], [0.0, 0.0, 20.0, 1.0])


def logpsd_model(f, a, alpha, fknee, fmin):
    """logpsd_model (mappraiser/python/TOAST_interface/utils.py:488-489)."""
    return a + np.log10(1 + ((f + fmin) / fknee) ** alpha)


def inversepsd_model(f, sigma, alpha, fknee, fmin):
    """inversepsd_model (utils.py:492-493)."""
    return sigma * 1.0 / (1 + ((f + fmin) / fknee) ** alpha)


def apod_window(lam: int, apod: str = "chebwin") -> np.ndarray:
    """Apodisation window after ifftshift, first lam points (utils.py:567-582)."""
    from scipy.signal import get_window
    if apod == "gaussian":
        w = get_window(("general_gaussian", 1, 1 / 3 * lam), 2 * lam)
    elif apod == "chebwin":
        w = get_window(("chebwin", 150), 2 * lam)
    else:
        raise RuntimeError(f"Apodisation window '{apod}' is not supported.")
    return np.fft.ifftshift(w)[:lam]


def chebwin_exact(lam: int) -> np.ndarray:
    """Arbiter for the chebwin window of apod_window: the same Dolph-Chebyshev
    window (scipy.signal.windows.chebwin, 2*lam + 1 points, 150 dB, ifftshift,
    first lam) with its samples T_{2 lam}(beta cos(pi k/M)) evaluated in 30-digit
    arithmetic (mpmath), then an FP64 FFT.  scipy's own window differs from it by
    up to 5e-9 at lam = 2^14 (rounding of beta cos(pi k/M) amplified near 1)."""
    import mpmath
    mpmath.mp.dps = 30
    M = 2 * lam + 1
    beta = mpmath.cosh(mpmath.acosh(mpmath.mpf(10) ** (mpmath.mpf(150) / 20)) / (M - 1))
    p = np.empty(lam + 1)
    for k in range(lam + 1):
        x = beta * mpmath.cos(mpmath.pi * k / M)
        p[k] = float(mpmath.cosh((M - 1) * mpmath.acosh(x)) if x > 1 else mpmath.cos((M - 1) * mpmath.acos(x)))
    w = np.real(np.fft.fft(np.concatenate([p, p[1:][::-1]])))[:lam + 1]
    return w[:lam] / w.max()


def periodogram(x: np.ndarray, fsamp: float):
    """One-segment Welch periodogram of a block (utils.py:531)."""
    import scipy.signal
    return scipy.signal.welch(x, fsamp, window="hann", nperseg=x.size, detrend="linear")


def fit_cost(psd: np.ndarray, nn: int, fsamp: float, params) -> float:
    """Least-squares cost of noise2invtt's fit (utils.py:534-541) at params:
    0.5 * sum (logpsd_model(f[1:], *params) - log10 psd[1:])^2."""
    f = np.fft.rfftfreq(nn, 1.0 / fsamp)
    r = logpsd_model(f[1:], *params) - np.log10(psd[1:])
    return 0.5 * float(r @ r)


def noise2invtt(nsetod: np.ndarray, nn: int, lam: int, fsamp: float, apod: str = "chebwin", tight: bool = False):
    """noise2invtt (utils.py:500-584): Welch periodogram, curve_fit of the log PSD
    model, irfft of the inverse PSD, apodisation.  tight=True runs curve_fit to
    ftol = xtol = gtol = 1e-15 (maxfev 20000): the least-squares minimum, which the
    reference's defaults (ftol = 1e-8) approach to about 1e-5.  Returns
    (invtt, popt, psd)."""
    from scipy.optimize import curve_fit
    f, psd = periodogram(np.asarray(nsetod, dtype=np.float64), fsamp)
    kw = dict(ftol=1e-15, xtol=1e-15, gtol=1e-15, maxfev=20000) if tight else dict(maxfev=1000)
    popt, _ = curve_fit(logpsd_model, f[1:], np.log10(psd[1:]), p0=np.array(NOISE_FIT_P0),
                        bounds=NOISE_FIT_BOUNDS, **kw)
    f_full = np.fft.rfftfreq(nn, 1.0 / fsamp)
    with np.errstate(divide="ignore"):
        psdm1 = inversepsd_model(f_full, 10 ** (-popt[0]), *popt[1:])
    inv_tt = np.fft.irfft(psdm1, n=nn)
    if lam > nn // 2:
        raise RuntimeError("Bandwidth cannot be larger than timestream.")
    return np.multiply(apod_window(lam, apod), inv_tt[:lam], dtype=np.float64), popt, psd


# --------------------------------------------------------------------------- templates (MTmap)
@dataclass
class TemplateScan:
    """The scan description MTmap takes (mappraiser/src/mappraiser.c:387-391): per CES
    the sweep time stamps (nsweeps + 1 values, the last = the CES length), boresight
    azimuth and its range, HWP angle; the template set (npoly Legendre orders per sweep,
    ground = azimuth-binned scan-synchronous signal with n_sss_bins bins, nhwp HWP
    harmonics as cos/sin amplitudes constant over delta_t seconds).  Block b = i*ndet + j
    is detector j in CES i, ces_length(i) samples."""
    sweeps: list
    az: list
    az_min: np.ndarray
    az_max: np.ndarray
    hwp: list
    ndet: int
    npoly: int
    ground: int
    n_sss_bins: int
    nhwp: int
    delta_t: float
    fs: float

    @property
    def nces(self) -> int:
        return len(self.sweeps)

    def ces_length(self, i: int) -> int:
        return int(self.sweeps[i][-1])

    def hwp_bins(self, i: int) -> int:
        return int(np.ceil(self.ces_length(i) / (self.delta_t * self.fs)))

    def n_templates_block(self, i: int) -> int:
        return (self.npoly * (len(self.sweeps[i]) - 1) + self.ground * self.n_sss_bins
                + 2 * self.nhwp * self.hwp_bins(i))

    @property
    def block_sizes(self) -> np.ndarray:
        return np.array([self.ces_length(i) for i in range(self.nces) for _ in range(self.ndet)], dtype=np.int32)

    @property
    def n_templates(self) -> int:
        return sum(self.ndet * self.n_templates_block(i) for i in range(self.nces))

    @property
    def kernel_size(self) -> int:
        return sum(self.ndet * self.n_templates_block(i) ** 2 for i in range(self.nces))


def legendre(x: np.ndarray, a: float, b: float, n: int) -> np.ndarray:
    """Legendre (algebra/src/templates/templates.c:526-549): P_n on [a, b] by the
    three-term recurrence."""
    t = (2 * x - a - b) / (b - a)
    p0, p1 = np.ones_like(t), t
    if n == 0:
        return p0
    for k in range(2, n + 1):
        p0, p1 = p1, ((2 * k - 1) * t * p1 - (k - 1) * p0) / k
    return p1


def template_basis(sc: TemplateScan, i: int) -> np.ndarray:
    """Dense template matrix of CES i, [ces_length, n_templates_block] in the
    reference's amplitude order (Tlist_init, templates.c:634-677): Legendre order k
    on sweep s (expandpolydata), then the azimuth bins (bin_az, expandSSSdata), then
    per HWP harmonic h its cos and its sin over delta_t chunks (build_hwpss_w,
    expandHWPSSdata)."""
    L = sc.ces_length(i)
    sw = np.asarray(sc.sweeps[i])
    nsw = len(sw) - 1
    Phi = np.zeros((L, sc.n_templates_block(i)))
    j = np.arange(L)
    for k in range(sc.npoly):
        for s in range(nsw):
            r = np.arange(sw[s], sw[s + 1])
            Phi[r, k * nsw + s] = legendre(r / sc.fs, sw[s] / sc.fs, (sw[s + 1] - 1) / sc.fs, k)
    col = sc.npoly * nsw
    if sc.ground:
        az = np.asarray(sc.az[i])
        width = (sc.az_max[i] - sc.az_min[i]) / sc.n_sss_bins
        b = np.minimum(sc.n_sss_bins - 1, np.floor((az - sc.az_min[i]) / width).astype(np.int64))
        Phi[j, col + b] = 1.0
        col += sc.n_sss_bins
    if sc.nhwp:
        hb = sc.hwp_bins(i)
        c1, s1 = np.cos(sc.hwp[i]), np.sin(sc.hwp[i])
        ch, sh = c1.copy(), s1.copy()
        b = np.floor(j / (sc.fs * sc.delta_t)).astype(np.int64)
        for h in range(1, sc.nhwp + 1):
            if h > 1:
                ch, sh = ch * c1 - sh * s1, sh * c1 + ch * s1
            Phi[j, col + 2 * (h - 1) * hb + b] = ch
            Phi[j, col + (2 * h - 1) * hb + b] = sh
    return Phi


def templates_ops(sc: TemplateScan, w_block, d, tau):
    """TrTVecProd, TVecProd (templates.c:28-190) and the pseudo-inverted kernels
    w_b T_b^T T_b (BuildKernel, InvKernel with rcond 1e-12: templates.c:192-418),
    blocks one after the other.  Returns (T^T d, T tau, kernels, pseudo-inverses)."""
    amp, tod, kern, kinv = np.zeros(sc.n_templates), np.zeros(len(d)), [], []
    at = ta = 0
    for i in range(sc.nces):
        Phi = template_basis(sc, i)
        L, nt = Phi.shape
        for jd in range(sc.ndet):
            amp[ta:ta + nt] = Phi.T @ d[at:at + L]
            tod[at:at + L] = Phi @ tau[ta:ta + nt]
            K = w_block[i * sc.ndet + jd] * (Phi.T @ Phi)
            kern.append(K.ravel())
            kinv.append(np.linalg.pinv(K, rcond=1e-12).ravel())
            at += L
            ta += nt
    return amp, tod, np.concatenate(kern), np.concatenate(kinv)


def pcg_templates(gindices, values, signal, noise, sc: TemplateScan, invtt, tol=1e-8, maxiter=500, nnz: int = 3,
                  kinv=None):
    """PCG_GLS_templates (mappraiser/src/pcg_true.c:243-560) as MTmap runs it
    (mappraiser.c:586-680): white noise per block (invtt[b], MTmap's lambda = 1), the
    weighting F v = N^-1 v - N^-1 T B T^T N^-1 v with B_b = pinv(invtt[b] T_b^T T_b), block
    Jacobi from N^-1 alone, the PCG_GLS_true recurrences and stop test.  kinv: the B_b
    to use instead (block after block, row-major), e.g. another implementation's."""
    m = len(signal)
    bs = sc.block_sizes
    A = local_shape(gindices, values, m, nnz)
    bj = precond_blockjacobi(A, signal, bs, 1, invtt)
    A = bj.A
    n = A.n
    blocks = []
    at = ka = 0
    for i in range(sc.nces):
        Phi = template_basis(sc, i)
        nt = Phi.shape[1]
        for jd in range(sc.ndet):
            b = i * sc.ndet + jd
            if kinv is None:
                B = np.linalg.pinv(invtt[b] * (Phi.T @ Phi), rcond=1e-12)
            else:
                B = np.asarray(kinv[ka:ka + nt * nt]).reshape(nt, nt)
            blocks.append((at, at + Phi.shape[0], invtt[b], Phi, B))
            at += Phi.shape[0]
            ka += nt * nt

    def F(v):
        out = np.empty_like(v)
        for s, e, w, Phi, B in blocks:
            u = w * v[s:e]
            out[s:e] = u - w * (Phi @ (B @ (Phi.T @ u)))
        return out

    x = np.zeros(n)
    g = trmatvec(A, F(bj.signal + noise - matvec(A, x)))
    Cg = apply_bj(bj.inv, g)
    h = Cg.copy()
    g2pix = float(np.dot(Cg, g))
    res = float(np.dot(g, g))
    res0 = res
    tol2rel = tol * tol * res
    res_rel = [1.0]
    k = 1
    if res <= tol:
        return PCGResult(x, 0, res_rel, bj)
    while k < maxiter:
        gp = g
        AtFAh = trmatvec(A, F(matvec(A, h)))
        ro = g2pix / float(np.dot(h, AtFAh))
        x = x + ro * h
        g = gp - ro * AtFAh
        Cg = apply_bj(bj.inv, g)
        g2pixp = g2pix
        g2pix = float(np.dot(Cg, g))
        g2pix_polak = float(np.dot(Cg, g - gp))
        res = float(np.dot(g, g))
        res_rel.append(float(np.sqrt(res) / np.sqrt(res0)))
        if res <= tol2rel:
            break
        h = h * (g2pix_polak / g2pixp) + Cg
        k += 1
    return PCGResult(x, k, res_rel, bj)
