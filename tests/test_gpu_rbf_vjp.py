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


# BF16 tensor-core form of the pair (BF16 context, d <= 64, k <= 192): kernel
# tiles from BF16-rounded points via the Gram expansion, M = Ybar Omega and
# E X from BF16 operands, FP32 accumulation. Bars against the FP64 oracle:
# Y and dL/dX 1e-2 and 3e-2 relative (Frobenius). dL/dgamma = -sum E d^2 is
# a sum of terms of both signs whose total can be far smaller than the
# terms (condition sum|E d^2| / |dL/dgamma| reaches 2e4 on the 64-point
# case), so its bar is normwise: |error| <= 2e-3 sum|E d^2| against FP64,
# and <= 1e-4 sum|E d^2| against the same sum from BF16-rounded operands.
BF16_CASES = [
    (500, 6, 17, 1),     # one 64-column slice of Ybar / Omega
    (700, 64, 129, 2),   # the benchmark's d and k on a small N; three slices
    (777, 33, 192, 3),   # k at the limit, ragged N and d
    (130, 1, 64, 4),     # d = 1, k one full slice
    (64, 8, 5, 5),       # a single key block
]


@pytest.mark.parametrize("N,d,k,seed", BF16_CASES)
def test_rbf_pair_bf16_against_fp64(lib_built, oracle, N, d, k, seed):
    import torch

    import skema_b200 as sk
    from skema_b200 import _lib as L

    X = oracle.mixture_points(N, d, seed=seed)
    g = oracle.median_gamma(X)
    rng = np.random.default_rng(seed)
    Om = rng.uniform(-1, 1, size=(k, N)).astype(np.float32)
    Yb = rng.normal(size=(N, k)).astype(np.float32)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    Y = sk.rbf_sketch_fwd(dev(X), g, dev(Om), precision=L.PREC_BF16).cpu().numpy()
    dX, dg = sk.rbf_sketch_vjp(dev(X), g, dev(Om), dev(Yb), precision=L.PREC_BF16)
    dX = dX.cpu().numpy()
    X64, Om64 = X.astype(np.float64), Om.astype(np.float64)
    Y64 = oracle.rbf_fwd64(X64, g, Om64)
    dX64, dg64 = oracle.rbf_vjp64(X64, g, Om64, Yb.astype(np.float64))
    ey = np.linalg.norm(Y - Y64) / np.linalg.norm(Y64)
    ex = np.linalg.norm(dX - dX64) / np.linalg.norm(dX64)
    # the dgamma sum from BF16-rounded points and Ybar / Omega, FP64 arithmetic
    bf = lambda a: torch.from_numpy(np.asarray(a, np.float32)).bfloat16().double().numpy()
    Xb = bf(X)
    n2 = (Xb ** 2).sum(1)
    D2b = np.maximum(n2[:, None] + n2[None, :] - 2.0 * Xb @ Xb.T, 0.0)
    Eb = (bf(Yb) @ bf(Om)) * np.exp(-g * D2b)
    np.fill_diagonal(Eb, 0.0)
    dgb = -(Eb * D2b).sum()
    scale = np.abs(Eb * D2b).sum()
    eg, egb = abs(dg - dg64) / scale, abs(dg - dgb) / scale
    print(f"bf16 pair N={N} d={d} k={k}: Y {ey:.2e} dX {ex:.2e} dgamma {eg:.2e} (vs BF16 operands {egb:.2e})")
    assert np.isfinite(Y).all() and np.isfinite(dX).all() and np.isfinite(dg)
    assert ey < 1e-2 and ex < 3e-2, (ey, ex)
    assert eg < 2e-3 and egb < 1e-4, (eg, egb)


@pytest.mark.parametrize("d,k", [(65, 17), (6, 193)])
def test_rbf_pair_bf16_context_outside_the_tensor_core_shapes(lib_built, oracle, d, k):
    """Shapes past d = 64 or k = 192 take the FP32 form in a BF16 context."""
    import torch

    import skema_b200 as sk
    from skema_b200 import _lib as L

    N = 300
    X = oracle.mixture_points(N, d, seed=7)
    g = oracle.median_gamma(X)
    Om = np.random.default_rng(7).uniform(-1, 1, size=(k, N)).astype(np.float32)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    Y = sk.rbf_sketch_fwd(dev(X), g, dev(Om), precision=L.PREC_BF16).cpu().numpy()
    Y64 = oracle.rbf_fwd64(X.astype(np.float64), g, Om.astype(np.float64))
    assert np.linalg.norm(Y - Y64) / np.linalg.norm(Y64) < 1e-5


def test_rbf_vjp_at_the_adjoint_workload_dimensions(lib_built, oracle):
    """The adjoint workload's d = 64 and k = 129 on a 3,000-point subsample
    of the same mixture recipe (seed 1), FP32 form: the VJP against central
    finite differences of the FP64 forward (h = 1e-3 relative) along a seeded
    direction and in gamma, and against the FP64 gradient; bar 1e-4. The
    cotangent is a seeded N(0, 1) matrix plus 2 Y (L = ||Y||_F^2 + <G, Y>)."""
    import torch

    import skema_b200 as sk

    N, d, k = 3000, 64, 129
    X = oracle.mixture_points(N, d, seed=1)
    g = oracle.median_gamma(X)
    rng = np.random.default_rng(5)
    Om = rng.uniform(-1, 1, size=(k, N)).astype(np.float32)
    G = rng.normal(size=(N, k)).astype(np.float32)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    X64, Om64 = X.astype(np.float64), Om.astype(np.float64)
    Y = sk.rbf_sketch_fwd(dev(X), g, dev(Om))
    Yb = (2.0 * Y + dev(G)).contiguous()
    dX, dg = sk.rbf_sketch_vjp(dev(X), g, dev(Om), Yb)
    dX = dX.cpu().numpy().astype(np.float64)
    Yb64 = Yb.cpu().numpy().astype(np.float64)
    f = lambda Xv, gv: float((Yb64 * oracle.rbf_fwd64(Xv, gv, Om64)).sum())
    dX64, dg64 = oracle.rbf_vjp64(X64, g, Om64, Yb64)
    assert np.linalg.norm(dX - dX64) / np.linalg.norm(dX64) < 1e-4
    assert abs(dg - dg64) / abs(dg64) < 1e-4
    h = 1e-3 * g
    fd_g = (f(X64, g + h) - f(X64, g - h)) / (2 * h)
    assert abs(dg - fd_g) / abs(fd_g) < 1e-4, (dg, fd_g)
    V = np.random.default_rng(11).normal(size=X64.shape)
    hx = 1e-3 * np.linalg.norm(X64) / np.linalg.norm(V)
    fd_x = (f(X64 + hx * V, g) - f(X64 - hx * V, g)) / (2 * hx)
    assert abs((dX * V).sum() - fd_x) / abs(fd_x) < 1e-4, ((dX * V).sum(), fd_x)
