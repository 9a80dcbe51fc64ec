"""GPU test of skema_rbf_sketch_fwd_noalloc, the allocation-free entry point.

Some callers cannot let a library call cudaMalloc: a host framework that
owns all device memory through its own pool or cap, or a latency-critical
loop where cudaMalloc's device-wide synchronisation would stall other
streams. For them the RBF sketch forward pass has a variant whose scratch is
a static array compiled into the library. This file checks, through the C
ABI, that it returns what the regular entry point returns, on two calls in
a row (the array keeps the previous call's contents, which must not leak
into the next result), and that it refuses inputs larger than the array.
It is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_rbf_fwd_noalloc_matches_regular_entry_point(lib_built, oracle):
    import torch

    import skema_b200 as sk
    from skema_b200 import _lib as L
    from skema_b200.sketchy import _ctx_for_standalone

    ctx = _ctx_for_standalone(0)
    lib = L.load()
    try:
        for call, (N, d, k, seed) in enumerate([(3000, 7, 33, 1), (2500, 4, 20, 2)]):
            X = oracle.mixture_points(N, d, seed=seed)
            gamma = oracle.median_gamma(X)
            rng = np.random.default_rng(seed)
            Om = rng.uniform(-1, 1, size=(k, N)).astype(np.float32)
            Xd = torch.from_numpy(X).cuda()
            Od = torch.from_numpy(Om).cuda()
            Y_ref = torch.empty((N, k), dtype=torch.float32, device="cuda")
            Y_new = torch.full((N, k), float("nan"), dtype=torch.float32, device="cuda")
            assert lib.skema_rbf_sketch_fwd(ctx.h, Xd.data_ptr(), N, d, gamma, Od.data_ptr(), k,
                                            Y_ref.data_ptr()) == L.OK
            st = lib.skema_rbf_sketch_fwd_noalloc(ctx.h, Xd.data_ptr(), N, d, gamma, Od.data_ptr(), k,
                                                  Y_new.data_ptr())
            assert st == L.OK, lib.skema_last_error(ctx.h)
            ctx.synchronize()
            a, b = Y_new.cpu().numpy(), Y_ref.cpu().numpy()
            assert np.isfinite(a).all()
            assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-5, call
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
