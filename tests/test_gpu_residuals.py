"""GPU tests of the residual pass (skema_residuals_*), the second stream of
A behind SketchySVD::compute_residuals (src/Skema_SketchySVD.cpp:719-727,
src/Skema_Residuals.hpp:58-217).

The pass is FP64 on FP32 input values, so it is compared with the oracle's
restatement of Skema::residuals on the same U, S, V (those of the library's
own low_rank_approx) and the same input values at 1e-9 relative. Cases:
dense row- and column-major host input, a device input streamed in two
blocks, CSR, the Gauss RBF kernel input, and exact singular triplets, whose
residuals are zero up to round-off.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from test_gpu_sketch import alg, csr_input, dense_input

pytestmark = pytest.mark.gpu

TOL = 1e-9


@pytest.fixture(scope="module")
def sk(lib_built):
    import skema_b200

    return skema_b200


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("layout", ["C", "F"])
def test_residuals_dense_against_oracle(sk, oracle, layout):
    m, n = 1500, 700
    A = dense_input(m, n, seed=3).astype(np.float32)
    A = np.asfortranarray(A) if layout == "F" else np.ascontiguousarray(A)
    a = alg(sk, m, n, 8, 128, 0)
    with sk.SketchySVD(a) as s:
        s.linear_update(A)
        U, S, V = s.low_rank_approx()
        got = s.compute_residuals(A)
    ref = oracle.residuals(A.astype(np.float64), U, S, V, window=128)
    assert got.shape == (8,)
    assert rel(got, ref) < TOL, (got, ref)
    assert (got > 0).all()


def test_residuals_device_blocks_and_exact_triplets(sk, oracle):
    import torch

    m, n = 1024, 512
    A = dense_input(m, n, seed=4).astype(np.float32)
    a = alg(sk, m, n, 6, 200, 0)
    Ad = torch.from_numpy(A).cuda()
    # exact singular triplets of the FP32 matrix (FP64 SVD): residuals ~ 0
    Uf, Sf, Vt = np.linalg.svd(A.astype(np.float64), full_matrices=False)
    with sk.SketchySVD(a) as s:
        exact = s.residuals(None, Uf[:, :6], Sf[:6], Vt[:6].T, row_blocks=[(0, Ad[:600]), (600, Ad[600:])])
        s.linear_update(Ad)
        U, S, V = s.low_rank_approx()
        got = s.residuals(None, U, S, V, row_blocks=[(600, Ad[600:]), (0, Ad[:600])])
    assert np.max(exact) < 1e-9 * Sf[0], exact
    ref = oracle.residuals(A.astype(np.float64), U, S, V)
    assert rel(got, ref) < TOL, (got, ref)


def test_residuals_csr_against_oracle(sk, oracle):
    m, n = 3000, 900
    A = csr_input(m, n, nnz_row=9, seed=6)
    a = alg(sk, m, n, 5, 700, 1, issparse=True)
    with sk.SketchySVD(a) as s:
        s.linear_update(A)
        U, S, V = s.low_rank_approx()
        got = s.compute_residuals(A)
    A64 = sp.csr_matrix(A, dtype=np.float64)
    ref = oracle.residuals(A64, U, S, V)
    assert rel(got, ref) < TOL, (got, ref)


def test_residuals_rbf_against_oracle(sk, oracle):
    N, d = 600, 4
    P = oracle.mixture_points(N, d, seed=2)
    g = oracle.median_gamma(P)
    a = alg(sk, N, N, 5, 128, 0, kernel_func=1, kernel_gamma=g, force_three_sketch=True)
    with sk.SketchySVD(a) as s:
        s.linear_update(P)
        U, S, V = s.low_rank_approx()
        got = s.compute_residuals(P)
    K = oracle.rbf_kernel(P.astype(np.float64), g)
    ref = oracle.residuals(K, U, S, V)
    # K is formed in FP32 on the device (explicit differences, expf): the
    # residuals see that rounding, about 1e-7 of the entries
    print("rbf residuals", got, ref)
    assert rel(got, ref) < 1e-4, (got, ref)


def test_residuals_need_an_open_pass(sk):
    from skema_b200 import _lib as L

    a = alg(sk, 100, 50, 2, 50, 0)
    with sk.SketchySVD(a) as s:
        out = np.empty(2)
        assert s.lib.skema_residuals_finish(s.h, out.ctypes.data, L.MEM_HOST) == L.ESTATE
        A = np.zeros((100, 50), np.float32)
        assert s.lib.skema_residuals_update_dense(s.h, A.ctypes.data, 50, L.ROW_MAJOR, 0, 100, L.MEM_HOST) == L.ESTATE


def test_residuals_from_the_kept_factors(sk, oracle):
    # skema_set_keep_factors: the last approximation's U, S, V stay on the
    # device, and a pass opened with NULL factors equals one given them from
    # the host; explicit factors replace the kept ones; keeping off drops them
    import skema_b200._lib as L

    rng = np.random.default_rng(12)
    m, n = 3000, 400
    A = ((rng.standard_normal((m, 12)) @ rng.standard_normal((12, n))) + 0.01 * rng.standard_normal((m, n))
         ).astype(np.float32)
    a = sk.AlgParams(matrix_m=m, matrix_n=n, rank=8, window=512, dim_redux=0)
    with sk.SketchySVD(a) as s:
        s.update_rows(A)
        U, S, V = s.low_rank_approx()
        kept = s.residuals(A, None, None, None)
        host = s.residuals(A, U, S, V)
        assert np.max(np.abs(kept - host) / np.abs(host)) < 1e-12
        with pytest.raises(sk.SkemaError) as e:  # replaced by the explicit factors
            s.residuals(A, None, None, None)
        assert e.value.status == L.ESTATE
        assert np.max(np.abs(s.compute_residuals(A) - host) / np.abs(host)) < 1e-12  # falls back to U, S, V
        s.low_rank_approx()
        assert np.max(np.abs(s.residuals(A, None, None, None) - host) / np.abs(host)) < 1e-12
        assert s.lib.skema_set_keep_factors(s.h, 0) == L.OK
        with pytest.raises(sk.SkemaError):
            s.residuals(A, None, None, None)
    b = sk.AlgParams(matrix_m=n, matrix_n=n, rank=5, window=128, dim_redux=0, issymmetric=True)
    P = (rng.standard_normal((n, 20)) @ rng.standard_normal((20, n)) / n).astype(np.float64)
    P = (P @ P.T).astype(np.float32)
    with sk.SketchySPD(b) as s:
        s.update_rows(P)
        Us, Ss = s.low_rank_approx()
        kept = s.residuals(P, None, None, None)
        host = s.residuals(P, None, Ss, Us)
        assert np.max(np.abs(kept - host) / np.maximum(np.abs(host), 1e-300)) < 1e-12
