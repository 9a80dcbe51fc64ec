"""CPU tests of the oracle: it must be pinned before it can check the CUDA path.

Pins: the Random123 known-answer vectors of Philox4x32-10 (the generator
both the oracle and the library use), and the reference's own fixtures
(test/data/*_svals.txt) reproduced end to end by the oracle's SketchySVD.
"""
import os

import numpy as np
import pytest
import scipy.sparse as sp

from conftest import rel_fro

# Random123 kat_vectors, philox4x32_10: (ctr, key) -> out
PHILOX_KAT = [
    ([0, 0, 0, 0], [0, 0], [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]),
    ([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2, [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]),
    ([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0],
     [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]),
]


@pytest.mark.parametrize("ctr,key,out", PHILOX_KAT)
def test_philox_kat(oracle, ctr, key, out):
    assert oracle.philox4x32_10(ctr, key) == out


def test_gauss_map_distribution(oracle):
    M = oracle.gauss_map(7, 64, 500)
    maxval = np.sqrt(2 * np.log(64 * 500))
    assert M.shape == (64, 500)
    assert np.all(np.abs(M) <= maxval)
    # uniform on [-maxval, maxval]: mean 0, variance maxval^2/3
    assert abs(M.mean()) < 0.05 * maxval
    assert abs(M.var() / (maxval**2 / 3) - 1) < 0.05
    # deterministic and seed-dependent
    assert np.array_equal(M, oracle.gauss_map(7, 64, 500))
    assert not np.array_equal(M, oracle.gauss_map(8, 64, 500))


@pytest.mark.parametrize("ncol", [1, 2, 5, 8, 81, 100000])
def test_sparse_sign_map_structure(oracle, ncol):
    idx, val = oracle.sparse_sign_map(3, 2000, ncol)
    zeta = max(2, min(ncol, 8))
    assert idx.shape == (2000, zeta)
    assert np.all(idx >= 0) and np.all(idx < ncol)
    assert np.all(np.diff(idx, axis=1) >= 0)  # sorted, duplicates allowed
    assert set(np.unique(val)) <= {-1.0, 1.0}
    assert abs((val > 0).mean() - 0.5) < 0.03


def test_sparse_sign_duplicates_summed(oracle):
    idx, val = oracle.sparse_sign_map(1, 5000, 3)
    D = oracle.sparse_to_dense(idx, val, 3)
    for r in range(50):
        expect = np.zeros(3)
        for t in range(idx.shape[1]):
            expect[idx[r, t]] += val[r, t]
        assert np.array_equal(D[r], expect)


def _rect_csr(kat):
    return sp.csr_matrix((kat["rect_csr_val"], kat["rect_csr_col"], kat["rect_csr_rowptr"]),
                         shape=tuple(kat["rect_csr_shape"]))


@pytest.mark.parametrize("kind", [0, 1])
@pytest.mark.parametrize("window", [1, 5, 32])
def test_oracle_rect_kat_dense(oracle, kat, kind, window):
    o = oracle.OracleSketch(32, 14, 10, window=window, kind=kind, sketch_range=12, sketch_core=25)
    o.linear_update(kat["rect_dense"])
    U, S, V = o.low_rank_approx()
    assert np.max(np.abs(S - kat["rect_svals"][:10])) / S[0] < 1e-12
    assert np.allclose(U.T @ U, np.eye(10), atol=1e-12)
    assert np.abs(U @ np.diag(S) @ V.T - kat["rect_dense"]).max() < 1e-12


@pytest.mark.parametrize("kind", [0, 1])
def test_oracle_rect_kat_csr(oracle, kat, kind):
    o = oracle.OracleSketch(32, 14, 10, window=7, kind=kind, issparse=True, sketch_range=12,
                            sketch_core=25)
    o.linear_update(_rect_csr(kat))
    U, S, V = o.low_rank_approx()
    assert np.max(np.abs(S - kat["rect_svals"][:10])) / S[0] < 1e-12


def test_oracle_sym_kat(oracle, kat):
    for kind in (0, 1):
        o = oracle.OracleSketch(27, 27, 10, window=4, kind=kind, sketch_range=27, sketch_core=27)
        o.linear_update(kat["sym_dense"])
        _, S, _ = o.low_rank_approx()
        assert np.max(np.abs(S - kat["sym_svals"][:10])) / S[0] < 1e-9


def test_oracle_kernel_kat(oracle, kat):
    # gamma = 1.0 is the kernel_gamma default the fixture was made with
    o = oracle.OracleSketch(25, 25, 5, window=6, kind=0, sketch_range=21, sketch_core=25,
                            kernel_gamma=1.0)
    o.linear_update(kat["kernel_points"])
    _, S, _ = o.low_rank_approx()
    assert np.max(np.abs(S - kat["kernel_svals"][:5])) / S[0] < 1e-6
    K = oracle.rbf_kernel(kat["kernel_points"], 1.0)
    assert np.allclose(np.diag(K), 1.0)
    assert np.max(np.abs(np.linalg.svd(K, compute_uv=False) - kat["kernel_svals"])) < 1e-12


def test_oracle_eta_nu_semantics(oracle):
    """X = nu*X + eta*x per window (src/Skema_SketchySVD.cpp:187-189)."""
    rng = np.random.default_rng(0)
    A = rng.normal(size=(40, 12))
    o = oracle.OracleSketch(40, 12, 2, window=10, kind=0, eta=0.5, nu=0.9)
    o.linear_update(A)
    ref = oracle.OracleSketch(40, 12, 2, window=10, kind=0)
    X = np.zeros_like(ref.X)
    for w in range(4):
        x, y, z = oracle.update_dense(ref.maps, A[10 * w:10 * w + 10], 10 * w)
        X = 0.9 * X + 0.5 * x
    assert rel_fro(o.X, X) < 1e-14


def test_oracle_csr_matches_dense(oracle):
    """CRS x SparseSign via the C Gustavson restatement equals the dense algebra."""
    rng = np.random.default_rng(1)
    A = sp.random(300, 120, density=0.05, random_state=2, format="csr")
    o = oracle.OracleSketch(300, 120, 3, window=64, kind=1, issparse=True)
    o.linear_update(A)
    X = o.maps["upsilon"].logical @ A.toarray()
    Y = A.toarray() @ o.maps["omega"].logical.T
    Z = o.maps["phi"].logical @ A.toarray() @ o.maps["psi"].logical.T
    assert rel_fro(o.X, X) < 1e-13
    assert rel_fro(o.Y, Y) < 1e-13
    assert rel_fro(o.Z, Z) < 1e-13


def test_oracle_vjp_matches_finite_differences(oracle):
    """The FP64 gradient formula of the RBF sketch against central FD."""
    rng = np.random.default_rng(5)
    X = oracle.mixture_points(60, 3, seed=1).astype(np.float64)
    Om = rng.normal(size=(7, 60))
    Yb = rng.normal(size=(60, 7))
    g = 0.3

    def L(Xv, gv):
        return float((Yb * oracle.rbf_fwd64(Xv, gv, Om)).sum())

    dX, dg = oracle.rbf_vjp64(X, g, Om, Yb)
    h = 1e-3 * g
    fd = (L(X, g + h) - L(X, g - h)) / (2 * h)
    assert abs(fd - dg) / abs(dg) < 1e-5
    V = rng.normal(size=X.shape)
    hx = 1e-3
    fdx = (L(X + hx * V, g) - L(X - hx * V, g)) / (2 * hx)
    assert abs(fdx - (dX * V).sum()) / abs(fdx) < 1e-5


def test_residuals_restatement_pins():
    """Skema::residuals (src/Skema_Residuals.hpp:58-217) restated: exact
    singular triplets give zero, the windowed A^T U sum equals the one-shot
    product, CSR equals dense, and the SPD form is ||A V - V S||."""
    import scipy.sparse as sp

    from oracle import sketchy_oracle as O

    rng = np.random.default_rng(3)
    A = rng.normal(size=(90, 40))
    U, S, Vt = np.linalg.svd(A, full_matrices=False)
    r = 6
    assert np.max(O.residuals(A, U[:, :r], S[:r], Vt[:r].T, window=7)) < 1e-12 * S[0]
    Up = np.linalg.qr(rng.normal(size=(90, r)))[0]
    Vp = np.linalg.qr(rng.normal(size=(40, r)))[0]
    Sp = np.sort(rng.uniform(1, 2, size=r))[::-1]
    one = O.residuals(A, Up, Sp, Vp)
    win = O.residuals(A, Up, Sp, Vp, window=16)
    assert np.allclose(one, win, rtol=1e-13)
    direct = np.sqrt(((A.T @ Up - Vp * Sp) ** 2).sum(0) + ((A @ Vp - Up * Sp) ** 2).sum(0))
    assert np.allclose(one, direct, rtol=1e-13)
    Asp = sp.random(90, 40, density=0.1, random_state=1, format="csr")
    assert np.allclose(O.residuals(Asp, Up, Sp, Vp, window=32), O.residuals(Asp.toarray(), Up, Sp, Vp), rtol=1e-13)
    B = A[:40] @ A[:40].T
    assert np.allclose(O.residuals(B, None, Sp, Vp), np.linalg.norm(B @ Vp - Vp * Sp, axis=0), rtol=1e-13)


def test_spd_approx_restatement_pins():
    """SketchySPD::low_rank_approx (src/Skema_SketchySVD.cpp:935-1151)
    restated. The Nystrom form recovers the reference's kernel fixture
    (25 points, gamma = 1) exactly with a full-range sketch and to ~3e-5 with
    k = 21; the reference's own steps subtract ||Y||_2 from the squared
    singular values, which leaves nothing of this spectrum, and its
    SparseSign shift (`*=` in SparseSignDimRedux::axpy) leaves (B + B^T) / 2
    indefinite here."""
    from oracle import sketchy_oracle as O

    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "kat_fixtures.npz"))
    X = d["kernel_points"].astype(np.float64)
    sv = d["kernel_svals"]
    N = X.shape[0]
    for k, tol in ((25, 1e-12), (21, 5e-5)):
        for kind in (0, 1):
            o = O.OracleSketch(N, N, 5, N, kind=kind, sketch_range=k, spd=True, kernel_gamma=1.0)
            o.linear_update(X)
            U, S = o.spd_low_rank_approx(nystrom=True)
            assert np.max(np.abs(S - sv[:5]) / sv[:5]) < tol, (k, kind, S)
            assert np.allclose(U.T @ U, np.eye(5), atol=1e-10)
    o = O.OracleSketch(N, N, 5, N, kind=0, sketch_range=25, spd=True, kernel_gamma=1.0)
    o.linear_update(X)
    assert np.all(o.spd_low_rank_approx(nystrom=False)[1] == 0.0)
    o = O.OracleSketch(N, N, 5, N, kind=1, sketch_range=25, spd=True, kernel_gamma=1.0)
    o.linear_update(X)
    with pytest.raises(np.linalg.LinAlgError):
        o.spd_low_rank_approx(nystrom=False)
