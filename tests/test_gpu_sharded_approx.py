"""GPU tests of skema_low_rank_approx_rows: the fixed-rank approximation of
a sketch sharded by row blocks, its row reductions summed through the
caller's all-reduce.

One GPU stands in for the ranks: each rank is a context in its own host
thread, holding its block of Y and the summed X and Z, and the all-reduce
is a host-side sum across the threads (a barrier with a time limit; the
kernels of the contexts never wait for one another). The result is held to
the one-context approximation of the same sketches (Y stacked from the
blocks): the blocks' rows of U, and S and V, to FP64 summation order.
"""
import threading

import numpy as np
import pytest
import scipy.sparse as sp

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sk(lib_built):
    import skema_b200

    return skema_b200


class ThreadSum:
    """allreduce(ptr, count) for n threads of one process."""

    def __init__(self, n):
        self.n = n
        self.bar = threading.Barrier(n)
        self.parts = [None] * n
        self.total = None
        self.calls = [0] * n

    def for_rank(self, r):
        import torch

        from skema_b200.distributed import _DeviceBuffer

        def allreduce(ptr, count):
            t = torch.as_tensor(_DeviceBuffer(ptr, count), device="cuda")
            self.parts[r] = t.cpu().numpy().copy()
            self.calls[r] += 1
            self.bar.wait(timeout=120)
            if r == 0:
                self.total = np.sum(np.stack(self.parts), axis=0)
            self.bar.wait(timeout=120)
            t.copy_(torch.from_numpy(self.total).cuda())
            torch.cuda.synchronize()
            self.bar.wait(timeout=120)

        return allreduce


def sharded_run(sk, a, A, world, window):
    from skema_b200.distributed import shard_rows, windows_after

    m = a.matrix_m
    ctxs, blocks = [], []
    for r in range(world):
        row0, nrows = shard_rows(m, world, r, window)
        c = sk.SketchySVD(a)
        if nrows:
            c.update_rows(A[row0:row0 + nrows], row0)
        ctxs.append(c)
        blocks.append((row0, nrows))
    # X and Z summed over the ranks, each partial weighted by nu^(windows after it)
    nu = a.sketch_nu
    X = sum(np.asarray(c.get_sketch(0), np.float64) * nu ** windows_after(m, world, r, window)
            for r, c in enumerate(ctxs))
    Z = sum(np.asarray(c.get_sketch(2), np.float64) * nu ** windows_after(m, world, r, window)
            for r, c in enumerate(ctxs))
    Y = sum(np.asarray(c.get_sketch(1), np.float64) for c in ctxs)  # disjoint rows
    for c in ctxs:
        c.set_sketch(0, X.astype(np.float32))
        c.set_sketch(2, Z.astype(np.float32))
    ts = ThreadSum(world)
    out = [None] * world
    errs = []

    def run(r):
        try:
            out[r] = ctxs[r].low_rank_approx_rows(blocks[r][0], blocks[r][1], ts.for_rank(r))
        except BaseException as e:
            errs.append(e)
            ts.bar.abort()

    th = [threading.Thread(target=run, args=(r,)) for r in range(world)]
    for t in th:
        t.start()
    for t in th:
        t.join(timeout=300)
    assert not errs, errs
    assert ts.calls == [3] * world
    # the one-context approximation of the same sketches
    with sk.SketchySVD(a) as s:
        s.set_sketch(0, X.astype(np.float32))
        s.set_sketch(1, Y.astype(np.float32))
        s.set_sketch(2, Z.astype(np.float32))
        U0, S0, V0 = s.low_rank_approx()
    for c in ctxs:
        c.close()
    U = np.concatenate([out[r][0] for r in range(world)], axis=0)
    return (U, out[0][1], out[0][2]), (U0, S0, V0), out


def check(res, ref, out):
    (U, S, V), (U0, S0, V0) = res, ref
    assert np.max(np.abs(S - S0)) <= 1e-10 * S0[0]
    for o in out:  # every rank has the same S and V
        assert np.max(np.abs(o[1] - S)) <= 1e-10 * S0[0]
        assert np.max(np.abs(o[2] - V)) <= 1e-8
    assert np.max(np.abs(U - U0)) <= 1e-8 * max(1.0, np.abs(U0).max())
    assert np.max(np.abs(V - V0)) <= 1e-8 * max(1.0, np.abs(V0).max())


@pytest.mark.parametrize("kind", [0, 1])
@pytest.mark.parametrize("world", [2, 4])
def test_sharded_csr_approx_matches_one_context(sk, kind, world):
    # 6000 rows in windows of 700: four ranks leave the last one no rows
    rng = np.random.default_rng(kind)
    m, n = 6000, 1500
    A = sp.random(m, n, density=0.006, format="csr", random_state=kind, dtype=np.float64)
    A.data = rng.standard_normal(A.nnz).astype(np.float32).astype(np.float64)
    P = rng.standard_normal((m, 15)) @ rng.standard_normal((15, n)) * 0.05
    A = sp.csr_matrix(A + sp.csr_matrix(np.where(np.abs(P) > 0.08, P, 0.0)))
    a = sk.AlgParams(matrix_m=m, matrix_n=n, rank=12, window=700, dim_redux=kind, issparse=True,
                     sketch_nu=0.95)
    check(*sharded_run(sk, a, A, world, 700))


def test_sharded_dense_approx_matches_one_context(sk):
    rng = np.random.default_rng(7)
    m, n = 3000, 500
    A = (rng.standard_normal((m, 40)) * np.logspace(0, -2, 40)) @ rng.standard_normal((40, n))
    A = (A + 1e-3 * rng.standard_normal((m, n))).astype(np.float32)
    a = sk.AlgParams(matrix_m=m, matrix_n=n, rank=10, window=512, dim_redux=0)
    check(*sharded_run(sk, a, A, 3, 512))


def test_sharded_approx_reports_a_failed_allreduce(sk):
    from skema_b200 import SkemaError

    m, n = 800, 300
    A = np.random.default_rng(3).standard_normal((m, n)).astype(np.float32)
    a = sk.AlgParams(matrix_m=m, matrix_n=n, rank=5, window=128, dim_redux=0)

    def broken(ptr, count):
        raise RuntimeError("peer gone")

    with sk.SketchySVD(a) as s:
        s.update_rows(A)
        with pytest.raises(SkemaError) as ei:
            s.low_rank_approx_rows(0, m, broken)
        assert ei.value.status == 9  # SKEMA_ECOLLECTIVE
        U, S, V = s.low_rank_approx()  # the context stays usable
        assert np.all(np.isfinite(S))


def test_torch_distributed_callback_on_one_rank(sk):
    # the torch.distributed binding (NCCL all_reduce on the library's device
    # buffers) in a one-rank group: the sharded call over all rows equals
    # the single-context approximation
    import os
    import socket

    import torch.distributed as dist

    from skema_b200 import distributed

    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    os.environ["MASTER_PORT"] = str(port)
    rng = np.random.default_rng(5)
    m, n = 2000, 600
    A = (rng.standard_normal((m, 20)) @ rng.standard_normal((20, n))).astype(np.float32)
    a = sk.AlgParams(matrix_m=m, matrix_n=n, rank=8, window=256, dim_redux=0)
    dist.init_process_group("nccl", rank=0, world_size=1)
    try:
        with sk.SketchySVD(a) as s:
            s.update_rows(A)
            U0, S0, V0 = s.low_rank_approx()
            U, S, V = distributed.low_rank_approx_sharded(s, m, 256)
        assert np.max(np.abs(S - S0)) <= 1e-12 * S0[0]
        assert np.max(np.abs(U - U0)) <= 1e-9 and np.max(np.abs(V - V0)) <= 1e-9
    finally:
        dist.destroy_process_group()
