"""GPU tests of the SketchySPD fixed-rank approximation
(SketchySPD::low_rank_approx, src/Skema_SketchySVD.cpp:935-1151) through the
C ABI, in both forms (params.spd_approx).

The device approximation is FP64. To isolate it from the FP32 sketch, the
oracle restatement runs on the device's own Y sketch and the device's map
values (exported), and eigenvalues are compared at 1e-9 of the largest,
eigenvectors up to sign. End to end, the Nystrom form recovers the
reference's kernel fixture (25 points, gamma = 1, full range) to the FP32
rounding of the sketch. The reference's own steps fail the Cholesky with a
SparseSign map on that fixture, as the oracle does: the library reports
SKEMA_ENOTPD.
"""
import os

import numpy as np
import pytest

from test_gpu_sketch import alg, dense_input, oracle_for

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sk(lib_built):
    import skema_b200

    return skema_b200


def spd_params(sk, n, rank, window, kind, mode, k, **kw):
    a = alg(sk, n, n, rank, window, kind, issymmetric=True, sketch_range=k, **kw)
    a.spd_approx = mode
    return a


def oracle_on_device_sketch(oracle, s, a, gamma=None):
    o = oracle_for(oracle, a, spd=True, gamma=gamma)
    o.Y = s.get_sketch(1).astype(np.float64)  # Y
    if a.dim_redux == 0:
        o.maps["omega"]._dense = np.asarray(s.map_export(1)[0], dtype=np.float64)
    return o


def check(U, S, Uo, So):
    assert np.isfinite(U).all() and np.isfinite(S).all()
    scale = max(abs(So[0]), 1e-300)
    assert np.max(np.abs(S - So)) / scale < 1e-9, (S, So)
    d = np.abs(np.sum(U * Uo, axis=0))  # |cos| per column, eigenvectors up to sign
    big = So > 1e-6 * scale
    assert np.all(d[big] > 1 - 1e-7), d


@pytest.mark.parametrize("kind", [0, 1])
@pytest.mark.parametrize("mode", ["nystrom", "reference-steps"])
def test_spd_dense_against_oracle_on_device_sketch(sk, oracle, kind, mode):
    from skema_b200 import _lib as L

    n = 600
    B = dense_input(n, n, seed=8)
    A = (B @ B.T / n).astype(np.float32)  # symmetric positive semidefinite
    md = L.SPD_NYSTROM if mode == "nystrom" else L.SPD_REFERENCE_STEPS
    a = spd_params(sk, n, 6, 150, kind, md, 40)
    with sk.SketchySPD(a) as s:
        s.linear_update(A)
        o = oracle_on_device_sketch(oracle, s, a)
        try:
            Uo, So = o.spd_low_rank_approx(nystrom=(mode == "nystrom"))
        except np.linalg.LinAlgError:
            with pytest.raises(sk.SkemaError) as e:
                s.low_rank_approx()
            assert e.value.status == L.ENOTPD
            return
        U, S = s.low_rank_approx()
    check(U, S, Uo, So)


def test_spd_kernel_fixture_nystrom_and_residuals(sk, oracle):
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "kat_fixtures.npz"))
    X = d["kernel_points"].astype(np.float32)
    sv = d["kernel_svals"]
    N = X.shape[0]
    a = spd_params(sk, N, 5, 10, 0, 0, 25, kernel_func=1, kernel_gamma=1.0)
    with sk.SketchySPD(a) as s:
        s.linear_update(X)
        U, S = s.low_rank_approx()
        o = oracle_on_device_sketch(oracle, s, a, gamma=1.0)
        Uo, So = o.spd_low_rank_approx(nystrom=True)
        rn = s.compute_residuals(X)
    check(U, S, Uo, So)
    # end to end: FP32 sketch of an exactly recoverable spectrum
    assert np.max(np.abs(S - sv[:5]) / sv[:5]) < 1e-4, (S, sv[:5])
    K = oracle.rbf_kernel(X.astype(np.float64), 1.0)
    ref = oracle.residuals(K, None, S, U)
    assert np.max(np.abs(rn - ref)) <= 1e-5 * sv[0] + 1e-9, (rn, ref)


def test_spd_reference_steps_sparse_sign_not_pd(sk, oracle):
    from skema_b200 import _lib as L

    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "kat_fixtures.npz"))
    X = d["kernel_points"].astype(np.float32)
    N = X.shape[0]
    a = spd_params(sk, N, 5, 10, 1, L.SPD_REFERENCE_STEPS, 25, kernel_func=1, kernel_gamma=1.0)
    with sk.SketchySPD(a) as s:
        s.linear_update(X)
        with pytest.raises(sk.SkemaError) as e:
            s.low_rank_approx()
        assert e.value.status == L.ENOTPD
