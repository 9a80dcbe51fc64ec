"""TEST INFRASTRUCTURE ONLY -- the CPU oracle of the SketchySVD sketch path.

An FP64 restatement of the reference's algorithm (jeremy-myers/skema), used
only by tests/, the smoke check and the CPU baseline of the benchmark to
check and time the CUDA library. The product never imports this module.

What it follows (reference file:line):
  maps        src/Skema_DimRedux.hpp:98-128 (Gauss: uniform on +-maxval),
              :191-268 (SparseSign); orientation src/Skema_SketchySVD.cpp:30-95
              and SketchySPD :769-775. Entry values come from Philox4x32-10
              (oracle/skema_oracle.c); the reference's Kokkos XorShift64
              stream is not reproducible without Kokkos, so map VALUES are
              pinned by the Philox known-answer vectors, not by the reference.
  update      src/Skema_SketchySVD.cpp:256-268 (dense, Gauss), :271-293
              (dense, SparseSign), :296-316 (CRS, Gauss), :319-335 (CRS,
              SparseSign); the window loop :120-246; axpy :667-716
              (Y = nu*Y + eta*y, called as axpy(nu, X, eta, x)).
  approx      initial_approx :338-566 and low_rank_approx :569-664 with the
              same LAPACK routines: dgeqrf+dorgqr (scipy qr 'economic'),
              dgels on T1/T2, dgesvd.
  kernel      GaussRBF::compute src/Skema_Kernel.cpp:6-81 (explicit
              differences, unit diagonal).
Pinned against: the reference's own known-answer fixtures
(test/data/*_svals.txt, stored in tests/golden/kat_fixtures.npz) end to end,
and the Random123 Philox known-answer vectors for the generator.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess

import numpy as np
import scipy.linalg as sla
import scipy.sparse as sp

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libskema_oracle.so")

_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        src = os.path.join(HERE, "skema_oracle.c")
        if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
            build()
        L = C.CDLL(LIB_PATH)
        P, I64, I32, D = C.c_void_p, C.c_int64, C.c_int, C.c_double
        L.oracle_philox4x32_10.argtypes = [P, P, P]
        L.oracle_gauss_maxval.argtypes = [I64, I64]
        L.oracle_gauss_maxval.restype = D
        L.oracle_gauss_map.argtypes = [C.c_uint32, I64, I64, P]
        L.oracle_zeta.argtypes = [I64]
        L.oracle_zeta.restype = I32
        L.oracle_sparse_sign_map.argtypes = [C.c_uint32, I64, I64, P, P]
        L.oracle_csr_sparse_sign_window.argtypes = [I64, I64, I64, I64, P, P, P, I64, I64,
                                                    P, P, I32, P, P, I32, P, P, I32, P, P, I32,
                                                    P, P, P]
        L.oracle_csr_sparse_sign_y.argtypes = [I64, P, P, P, I64, P, P, I32, P]
        L.oracle_rbf_window.argtypes = [P, I64, I64, I64, D, I64, I64, P]
        L.oracle_num_threads.restype = I32
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data


def philox4x32_10(ctr, key):
    c = np.array(ctr, dtype=np.uint32)
    k = np.array(key, dtype=np.uint32)
    o = np.zeros(4, dtype=np.uint32)
    lib().oracle_philox4x32_10(_p(c), _p(k), _p(o))
    return [int(x) for x in o]


# ----------------------------------------------------------------- maps ----
def gauss_map(seed: int, nrow: int, ncol: int) -> np.ndarray:
    """Stored nrow x ncol Gauss map (FP64), entries uniform on +-maxval."""
    out = np.empty((ncol, nrow), dtype=np.float64)  # column-major fill
    lib().oracle_gauss_map(seed & 0xFFFFFFFF, nrow, ncol, _p(out))
    return out.T


def sparse_sign_map(seed: int, nrow: int, ncol: int):
    """(indices int32 nrow x zeta, values float64 nrow x zeta), rows sorted."""
    z = lib().oracle_zeta(ncol)
    idx = np.empty((nrow, z), dtype=np.int32)
    val = np.empty((nrow, z), dtype=np.float64)
    lib().oracle_sparse_sign_map(seed & 0xFFFFFFFF, nrow, ncol, _p(idx), _p(val))
    return idx, val


def sparse_to_dense(idx, val, ncol) -> np.ndarray:
    """Dense nrow x ncol from zeta entries per row (duplicates summed)."""
    nrow, z = idx.shape
    out = np.zeros((nrow, ncol))
    np.add.at(out, (np.repeat(np.arange(nrow), z), idx.ravel()), val.ravel())
    return out


def sparse_to_csr(idx, val, ncol) -> sp.csr_matrix:
    nrow, z = idx.shape
    return sp.csr_matrix((val.ravel(), idx.ravel().astype(np.int64), np.arange(0, nrow * z + 1, z)),
                         shape=(nrow, ncol))


class Map:
    """One DimRedux map: stored shape, orientation and values."""

    def __init__(self, kind: int, nrow: int, ncol: int, seed: int, transposed: bool, ref_flag: bool):
        self.kind, self.nrow, self.ncol, self.seed = kind, nrow, ncol, seed
        self.transposed = transposed      # logical = stored^T
        self.init_transposed = ref_flag   # the reference ctor's flag
        self._dense = None
        if kind == 0:
            self._dense = gauss_map(seed, nrow, ncol)
            self.idx = self.val = None
        else:
            self.idx, self.val = sparse_sign_map(seed, nrow, ncol)

    @property
    def dense(self) -> np.ndarray:
        """Stored map as a dense FP64 matrix (built on first use)."""
        if self._dense is None:
            self._dense = sparse_to_dense(self.idx, self.val, self.ncol)
        return self._dense

    @property
    def logical(self) -> np.ndarray:
        return self.dense.T if self.transposed else self.dense


def resolve(m, n, rank, sketch_range=1, sketch_core=1):
    """range/core defaults (src/Skema_SketchySVD.cpp:20-24)."""
    k = 4 * rank + 1 if sketch_range < rank else sketch_range
    s = 2 * k + 1 if sketch_core < rank else sketch_core
    return k, s


def make_maps(m, n, k, s, kind, issparse, seeds=(0, 1, 2, 3), spd=False):
    """Orientation rules of src/Skema_SketchySVD.cpp:30-95 (and :769-775)."""
    if spd:
        return {"omega": Map(kind, n, k, seeds[0], True, False)}
    gs = issparse and kind == 0
    ot = bool(issparse)
    return {
        "upsilon": Map(kind, m if gs else k, k if gs else m, seeds[0], gs, gs),
        "omega": Map(kind, n if ot else k, k if ot else n, seeds[1], ot, ot),
        "phi": Map(kind, m if gs else s, s if gs else m, seeds[2], gs, gs),
        "psi": Map(kind, n if ot else s, s if ot else n, seeds[3], ot, ot),
    }


# ------------------------------------------------------------- updates -----
def update_dense(maps, Aw, r0):
    """x, y, z for one dense window (update(dense, *), :256-293), using the
    reference association z = (Phi(:, idx) A_w) Psi^T."""
    w = Aw.shape[0]
    U = maps["upsilon"].logical[:, r0:r0 + w]
    O = maps["omega"].logical
    F = maps["phi"].logical[:, r0:r0 + w]
    P = maps["psi"].logical
    x = U @ Aw
    y = Aw @ O.T
    wmat = F @ Aw
    z = wmat @ P.T
    return x, y, z


def update_csr_gauss(maps, Aw: sp.csr_matrix, r0):
    """update(crs, Gauss) (:296-316): all maps stored transposed."""
    w = Aw.shape[0]
    Ut = maps["upsilon"].dense[r0:r0 + w, :]  # m x k rows
    x = (Aw.T @ Ut).T
    y = Aw @ maps["omega"].dense
    wt = Aw.T @ maps["phi"].dense[r0:r0 + w, :]
    z = np.asarray(wt).T @ maps["psi"].dense
    return np.asarray(x), np.asarray(y), np.asarray(z)


def update_csr_ssign(maps, Aw: sp.csr_matrix, r0, m, n, k, s):
    """update(crs, SparseSign) (:319-335) through the C Gustavson restatement."""
    w = Aw.shape[0]
    rowptr = np.ascontiguousarray(Aw.indptr, dtype=np.int64)
    col = np.ascontiguousarray(Aw.indices, dtype=np.int32)
    val = np.ascontiguousarray(Aw.data, dtype=np.float64)
    x = np.empty((k, n))
    y = np.empty((w, k))
    z = np.empty((s, s))
    U, O, F, P = maps["upsilon"], maps["omega"], maps["phi"], maps["psi"]
    lib().oracle_csr_sparse_sign_window(
        m, n, r0, w, _p(rowptr), _p(col), _p(val), k, s,
        _p(U.idx), _p(U.val), U.idx.shape[1], _p(O.idx), _p(O.val), O.idx.shape[1],
        _p(F.idx), _p(F.val), F.idx.shape[1], _p(P.idx), _p(P.val), P.idx.shape[1],
        _p(x), _p(y), _p(z))
    return x, y, z


def rbf_window(X, gamma, r0, w):
    """K(r0:r0+w, :) with explicit differences and unit diagonal (FP64)."""
    X = np.asfortranarray(np.asarray(X, dtype=np.float64))
    N, d = X.shape
    out = np.empty((w, N))
    lib().oracle_rbf_window(_p(X), N, N, d, float(gamma), r0, w, _p(out))
    return out


def rbf_kernel(X, gamma):
    return rbf_window(X, gamma, 0, X.shape[0])


class OracleSketch:
    """SketchySVD restated in FP64 (three-sketch) or SketchySPD (Y only)."""

    def __init__(self, m, n, rank, window, kind=0, issparse=False, sketch_range=1, sketch_core=1,
                 eta=1.0, nu=1.0, seeds=(0, 1, 2, 3), spd=False, kernel_gamma=None):
        self.m, self.n, self.rank, self.window = m, n, rank, window
        self.kind, self.issparse, self.eta, self.nu = kind, issparse, eta, nu
        self.k, self.s = resolve(m, n, rank, sketch_range, sketch_core)
        self.spd = spd
        self.kernel_gamma = kernel_gamma
        self.maps = make_maps(m, n, self.k, self.s, kind, issparse, seeds, spd)
        self.reset()

    def reset(self):
        self.X = np.zeros((self.k, self.n))
        self.Y = np.zeros((self.m, self.k))
        self.Z = np.zeros((self.s, self.s))

    def _window_rows(self, A, r0, w):
        if self.kernel_gamma is not None:
            return rbf_window(A, self.kernel_gamma, r0, w)
        if self.issparse:
            return A[r0:r0 + w]
        return np.asarray(A[r0:r0 + w], dtype=np.float64)

    def update_rows(self, A, row0=0, nrows=None):
        """Windows of `window` rows over [row0, row0+nrows) (:167-233)."""
        nrows = (self.m - row0) if nrows is None else nrows
        for off in range(0, nrows, self.window):
            w = min(self.window, nrows - off)
            r0 = row0 + off
            Aw = self._window_rows(A, r0, w)
            if self.spd:
                O = self.maps["omega"]
                y = Aw @ O.dense
                self.Y[r0:r0 + w] = self.nu * self.Y[r0:r0 + w] + self.eta * np.asarray(y)
                continue
            if self.issparse and self.kind == 0:
                x, y, z = update_csr_gauss(self.maps, Aw, r0)
            elif self.issparse:
                x, y, z = update_csr_ssign(self.maps, Aw, r0, self.m, self.n, self.k, self.s)
            else:
                x, y, z = update_dense(self.maps, Aw, r0)
            self.X = self.nu * self.X + self.eta * x
            self.Z = self.nu * self.Z + self.eta * z
            self.Y[r0:r0 + w] = self.nu * self.Y[r0:r0 + w] + self.eta * y

    def linear_update(self, A):
        self.reset()
        self.update_rows(A, 0, self.m)

    def linear_update_traced(self, A):
        """linear_update with sketch_compute_svals_iters
        (src/Skema_SketchySVD.cpp:164-216): the top-rank singular values of
        the fixed-rank approximation after every window, keyed "0", "1", ...
        The approximation here leaves Y intact (the reference's QR overwrites
        it, App. A Q6, which this restatement does not repeat)."""
        self.reset()
        traces = {}
        for w, r0 in enumerate(range(0, self.m, self.window)):
            self.update_rows(A, r0, min(self.window, self.m - r0))
            traces[str(w)] = {"svals": [float(x) for x in self.low_rank_approx()[1]]}
        return traces

    # --------------------------------------------------------- approx ----
    def initial_approx(self):
        """(Q, C, P) of src/Skema_SketchySVD.cpp:338-566."""
        k = self.k
        P = sla.qr(self.X.T, mode="economic")[0]          # dgeqrf + dorgqr
        Q = sla.qr(self.Y.copy(), mode="economic")[0]
        U1 = self.maps["phi"].logical @ Q
        U2 = self.maps["psi"].logical @ P
        U1, T1 = sla.qr(U1, mode="economic")
        U2, T2 = sla.qr(U2, mode="economic")
        Z2 = (U1.T @ self.Z) @ U2
        Z2 = _dgels(T1, Z2)                                 # Z2 = T1 \ Z2
        Z2t = _dgels(T2, Z2.T.copy())                       # W^T = Z2 / T2'
        C = Z2t.T
        assert C.shape == (k, k)
        return Q, C, P

    def spd_low_rank_approx(self, nystrom=False):
        """(U, S) of SketchySPD::low_rank_approx (src/Skema_SketchySVD.cpp:
        935-1151), FP64, from the Y sketch and the stored Omega (n x k).
        nystrom=False follows the reference's steps as they run:
          nu = ||Y||_2; eta = eps * ||Y||_2 (the reference takes this second
          norm of a buffer dgesvd has already overwritten, :964-965, so its
          value depends on the LAPACK build; it enters only at the level of
          eps); Y_eta = Y + eta Omega (Gauss axpy), or for SparseSign each
          stored entry of Omega multiplies its Y entry by eta * sign
          (SparseSignDimRedux::axpy, src/Skema_DimRedux_SparseSign.cpp:
          113-123, `*=`); B = Omega^T Y_eta; R^T R = (B + B^T) / 2 (dpotrf
          'U'); E = Y R^{-1} from the unshifted Y (:1094-1103); U S V^T =
          svd(E); S_j <- max(0, S_j^2 - nu) (:1145-1147).
        nystrom=True is the fixed-rank Nystrom approximation the reference's
        comments describe (Tropp, Yurtsever, Udell and Cevher, 2017): the
        shift eta = eps ||Y||_2 is added as Y_eta = Y + eta Omega for both
        map kinds, E = Y_eta R^{-1}, and S_j <- max(0, S_j^2 - eta). Its eps
        is the FP32 machine epsilon, the precision the library holds Y in
        (the reference holds Y in FP64 and uses the FP64 epsilon); the
        reference's steps keep the FP64 epsilon."""
        import scipy.linalg as sla

        Y = np.asarray(self.Y, dtype=np.float64)
        om = self.maps["omega"]
        Om = np.asarray(om.dense, dtype=np.float64)
        nu = np.linalg.svd(Y, compute_uv=False)[0]
        eta = float(np.finfo(np.float32 if nystrom else np.float64).eps) * nu
        Ye = Y.copy()
        if not nystrom and om.kind == 1:
            for i in range(om.nrow):
                for cidx, v in zip(om.idx[i], om.val[i]):
                    Ye[i, cidx] *= eta * v
        else:
            Ye += eta * Om
        B = Om.T @ Ye
        R = sla.cholesky(0.5 * (B + B.T), lower=False)
        E = sla.solve_triangular(R, (Ye if nystrom else Y).T, trans="T", lower=False).T
        U, S, _ = np.linalg.svd(E, full_matrices=False)
        r = self.rank
        sub = eta if nystrom else nu
        return U[:, :r], np.maximum(0.0, S[:r] ** 2 - sub)

    def low_rank_approx(self):
        """(U, S, V) of src/Skema_SketchySVD.cpp:569-664 (dgesvd)."""
        Q, C, P = self.initial_approx()
        Uc, S, Vt = sla.svd(C, full_matrices=False, lapack_driver="gesvd")
        r = self.rank
        return (Q @ Uc)[:, :r], S[:r], (P @ Vt.T)[:, :r]


def residuals(A, U, S, V, window=None):
    """Residual norms of src/Skema_Residuals.hpp:160-217 (two-sided, with
    map_A_by_window :58-110): per column j,
    ||[(A^T U - V S)(:, j); (A V - U S)(:, j)]||_2, A^T U accumulated window
    by window as the reference does. A: dense (m x n) FP64 array or scipy CSR.
    U None: the SketchySPD form ||(A V - V S)(:, j)||_2 (:112-158)."""
    m = A.shape[0]
    w = m if window is None else window
    S = np.asarray(S, dtype=np.float64)
    AV = np.zeros((m, V.shape[1]))
    AtU = np.zeros((A.shape[1], V.shape[1])) if U is not None else None
    for r0 in range(0, m, w):
        Aw = A[r0:r0 + w]
        AV[r0:r0 + w] = Aw @ V
        if U is not None:
            AtU += Aw.T @ U[r0:r0 + w]
    if U is None:
        return np.linalg.norm(AV - V * S, axis=0)
    d1 = AtU - V * S
    d2 = AV - U * S
    return np.sqrt((d1 ** 2).sum(0) + (d2 ** 2).sum(0))


def _dgels(A, B):
    """LAPACK dgels on a square A (the reference's linalg::ls)."""
    from scipy.linalg import lapack

    lqr, x, info = lapack.dgels(np.asfortranarray(A), np.asfortranarray(B))[:3]
    if info != 0:
        raise RuntimeError(f"dgels info={info}")
    return x[: A.shape[1]]


# ------------------------------------------------- RBF sketch and VJP ------
def rbf_fwd64(X, gamma, Omega):
    """Y = K Omega^T in FP64 (Omega: k x N)."""
    return rbf_kernel(X, gamma) @ Omega.T


def rbf_vjp64(X, gamma, Omega, Ybar):
    """Exact FP64 gradient of <Ybar, K Omega^T> w.r.t. gamma and X, with the
    unit diagonal contributing nothing."""
    X = np.asarray(X, dtype=np.float64)
    K = rbf_kernel(X, gamma)
    N = X.shape[0]
    D2 = np.empty((N, N))
    for i0 in range(0, N, 64):  # explicit differences, 64 rows at a time
        D2[i0:i0 + 64] = ((X[i0:i0 + 64, None, :] - X[None, :, :]) ** 2).sum(-1)
    M = Ybar @ Omega
    E = M * K
    np.fill_diagonal(E, 0.0)
    dgamma = -(E * D2).sum()
    S = E + E.T
    dX = -2.0 * gamma * (S.sum(1)[:, None] * X - S @ X)
    return dX, dgamma


# ---------------------------------------------------- synthetic inputs ------
def mixture_points(N, d, seed, components=8):
    """Gaussian mixture: means ~ N(0, 4I), unit covariance, equal weights."""
    rng = np.random.default_rng(seed)
    means = rng.normal(0.0, 2.0, size=(components, d))
    lab = rng.integers(0, components, size=N)
    return (means[lab] + rng.normal(size=(N, d))).astype(np.float32)


def median_gamma(X, sample=1000, seed=0):
    """gamma = 1 / (2 * median squared pairwise distance of a subsample)."""
    rng = np.random.default_rng(seed)
    S = X[rng.choice(X.shape[0], size=min(sample, X.shape[0]), replace=False)].astype(np.float64)
    D2 = ((S[:, None, :] - S[None, :, :]) ** 2).sum(-1)
    iu = np.triu_indices(S.shape[0], 1)
    return 1.0 / (2.0 * float(np.median(D2[iu])))


def num_threads() -> int:
    return int(lib().oracle_num_threads())
