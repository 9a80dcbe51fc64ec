"""GPU test of skema_rbf_sketch_fwd_noalloc, the allocation-free entry point.

Some callers cannot let a library call cudaMalloc: a host framework that
owns all device memory through its own pool or cap, or a latency-critical
loop where cudaMalloc's device-wide synchronisation would stall other
streams. For them the RBF sketch forward pass has a variant whose scratch is
a static array compiled into the library. This file checks, through the C
ABI, on two calls in a row (the array keeps the previous call's contents,
which must not leak into the next result):
  - that it agrees with the FP64 oracle (oracle.rbf_fwd64) to the FP32 bar,
    and with the regular entry point in an FP32 context;
  - that it computes in FP32 in a BF16 context too;
  - that the device's free memory is the same before and after the calls on
    a warmed context (the first call looks the array's address up, and the
    library image with the array may be loaded then);
  - that it refuses inputs larger than the array.
It is named to be collected last.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-5  # FP32 result vs FP64 oracle / FP32 entry point, relative Frobenius


def _rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("precision", [0, 1])
def test_rbf_fwd_noalloc_matches_oracle_and_regular_entry_point(lib_built, oracle, precision):
    import torch

    from skema_b200 import _lib as L
    from skema_b200.sketchy import _ctx_for_standalone

    ctx = _ctx_for_standalone(0, precision=precision)
    lib = L.load()
    try:
        cases = [(3000, 7, 33, 1), (2500, 4, 20, 2)]
        data = []
        for N, d, k, seed in cases:
            X = oracle.mixture_points(N, d, seed=seed)
            gamma = oracle.median_gamma(X)
            Om = np.random.default_rng(seed).uniform(-1, 1, size=(k, N)).astype(np.float32)
            Xd, Od = torch.from_numpy(X).cuda(), torch.from_numpy(Om).cuda()
            Yd = torch.full((N, k), float("nan"), dtype=torch.float32, device="cuda")
            data.append((N, d, k, X, gamma, Om, Xd, Od, Yd))
        torch.cuda.synchronize()  # the inputs' copies are complete before the library's stream reads them
        # warm-up call: the array's address is looked up on first use
        N, d, k, X, gamma, Om, Xd, Od, Yd = data[0]
        assert lib.skema_rbf_sketch_fwd_noalloc(ctx.h, Xd.data_ptr(), N, d, gamma, Od.data_ptr(), k,
                                                Yd.data_ptr()) == L.OK
        ctx.synchronize()
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        results = []
        for N, d, k, X, gamma, Om, Xd, Od, Yd in data:
            Yd.fill_(float("nan"))
            torch.cuda.synchronize()
            st = lib.skema_rbf_sketch_fwd_noalloc(ctx.h, Xd.data_ptr(), N, d, gamma, Od.data_ptr(), k,
                                                  Yd.data_ptr())
            assert st == L.OK, lib.skema_last_error(ctx.h)
            ctx.synchronize()
            results.append(Yd.cpu().numpy())
        free1 = torch.cuda.mem_get_info()[0]
        assert free1 == free0, (free0, free1)
        for (N, d, k, X, gamma, Om, Xd, Od, Yd), got in zip(data, results):
            assert np.isfinite(got).all()
            ref64 = oracle.rbf_fwd64(X, gamma, Om.astype(np.float64))
            assert _rel(got, ref64) < TOL, _rel(got, ref64)
            if precision == 0:
                Yr = torch.empty((N, k), dtype=torch.float32, device="cuda")
                assert lib.skema_rbf_sketch_fwd(ctx.h, Xd.data_ptr(), N, d, gamma, Od.data_ptr(), k,
                                                Yr.data_ptr()) == L.OK
                ctx.synchronize()
                assert _rel(got, Yr.cpu().numpy()) < TOL
    finally:
        ctx.close()


def test_rbf_fwd_noalloc_rejects_inputs_beyond_the_scratch(lib_built):
    import torch

    from skema_b200 import _lib as L
    from skema_b200.sketchy import _ctx_for_standalone

    ctx = _ctx_for_standalone(0)
    lib = L.load()
    try:
        N, d, k = (1 << 22) + 1, 1, 1
        X = torch.zeros((N, d), dtype=torch.float32, device="cuda")
        Om = torch.zeros((k, N), dtype=torch.float32, device="cuda")
        Y = torch.zeros((N, k), dtype=torch.float32, device="cuda")
        st = lib.skema_rbf_sketch_fwd_noalloc(ctx.h, X.data_ptr(), N, d, 1.0, Om.data_ptr(), k, Y.data_ptr())
        assert st == L.EINVAL
        assert b"npts exceeds the no-alloc scratch" in lib.skema_last_error(ctx.h)
    finally:
        ctx.close()
