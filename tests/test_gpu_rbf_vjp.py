"""GPU tests of the RBF-kernel sketch forward/VJP pair through the C ABI.

Forward against the FP64 oracle; VJP against the FP64 reference gradient
and against central finite differences of the FP64 forward (h = 1e-3
relative), the adjoint bar being 1e-4 relative.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup(lib_built, oracle):
    import torch

    N, d, k = 500, 6, 17
    X = oracle.mixture_points(N, d, seed=1)
    gamma = oracle.median_gamma(X)
    rng = np.random.default_rng(5)
    Om = rng.uniform(-1, 1, size=(k, N)).astype(np.float32)
    Yb = rng.normal(size=(N, k)).astype(np.float32)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    return dict(N=N, d=d, k=k, X=X, gamma=gamma, Om=Om, Yb=Yb, dev=dev)


def test_rbf_fwd(setup, oracle):
    import skema_b200 as sk

    s = setup
    Y = sk.rbf_sketch_fwd(s["dev"](s["X"]), s["gamma"], s["dev"](s["Om"])).cpu().numpy()
    Y64 = oracle.rbf_fwd64(s["X"].astype(np.float64), s["gamma"], s["Om"].astype(np.float64))
    assert np.linalg.norm(Y - Y64) / np.linalg.norm(Y64) < 1e-5


def test_rbf_vjp_vs_fp64_gradient(setup, oracle):
    import skema_b200 as sk

    s = setup
    dX, dg = sk.rbf_sketch_vjp(s["dev"](s["X"]), s["gamma"], s["dev"](s["Om"]), s["dev"](s["Yb"]))
    dX = dX.cpu().numpy()
    dX64, dg64 = oracle.rbf_vjp64(s["X"].astype(np.float64), s["gamma"], s["Om"].astype(np.float64),
                                  s["Yb"].astype(np.float64))
    assert abs(dg - dg64) / abs(dg64) < 1e-4
    assert np.linalg.norm(dX - dX64) / np.linalg.norm(dX64) < 1e-4


def test_rbf_vjp_vs_finite_differences(setup, oracle):
    """L = ||Y||_F^2 with Ybar = 2Y; FD of the FP64 forward, h = 1e-3 relative."""
    import skema_b200 as sk

    s = setup
    X64 = s["X"].astype(np.float64)
    Om64 = s["Om"].astype(np.float64)
    g = s["gamma"]
    L = lambda Xv, gv: float((oracle.rbf_fwd64(Xv, gv, Om64) ** 2).sum())
    Y = sk.rbf_sketch_fwd(s["dev"](s["X"]), g, s["dev"](s["Om"]))
    dX, dg = sk.rbf_sketch_vjp(s["dev"](s["X"]), g, s["dev"](s["Om"]), 2.0 * Y)
    dX = dX.cpu().numpy().astype(np.float64)
    h = 1e-3 * g
    fd_g = (L(X64, g + h) - L(X64, g - h)) / (2 * h)
    assert abs(dg - fd_g) / abs(fd_g) < 1e-4
    rng = np.random.default_rng(11)
    V = rng.normal(size=X64.shape)
    hx = 1e-3 * np.linalg.norm(X64) / np.linalg.norm(V)
    fd_x = (L(X64 + hx * V, g) - L(X64 - hx * V, g)) / (2 * hx)
    assert abs((dX * V).sum() - fd_x) / abs(fd_x) < 1e-4
    for _ in range(8):  # single coordinates
        i, f = rng.integers(0, s["N"]), rng.integers(0, s["d"])
        E = np.zeros_like(X64)
        hh = 1e-3 * max(abs(X64[i, f]), 1.0)
        E[i, f] = hh
        fd = (L(X64 + E, g) - L(X64 - E, g)) / (2 * hh)
        assert abs(dX[i, f] - fd) <= 1e-4 * np.abs(dX).max() + 1e-4 * abs(fd)
