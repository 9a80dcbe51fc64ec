"""Multi-process sketch update on CPU: two gloo ranks, each sketching its own
row block with the oracle, then the weighted all-reduce of X and Z from
skema_b200.distributed; rank 0 checks the result against one process
sketching the whole matrix (the reference's sequential window loop). The
GPU path runs the same host logic with the CUDA library per rank and NCCL.
"""
import os
import socket

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, cfg, out_path):
    import torch
    import torch.distributed as dist

    from oracle import sketchy_oracle as O
    from skema_b200 import distributed as D

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        m, n, rank_r, w, nu, eta = cfg
        rng = np.random.default_rng(5)
        A = rng.standard_normal((m, n))
        o = O.OracleSketch(m, n, rank_r, w, kind=0, eta=eta, nu=nu)
        o.reset()
        row0, nrows = D.shard_rows(m, world, rank, w)
        if nrows:
            o.update_rows(A, row0, nrows)
        X = torch.from_numpy(o.X.copy())
        Z = torch.from_numpy(o.Z.copy())
        Y = torch.from_numpy(o.Y.copy())
        D.reduce_partial_sketches(X, Z, m, w, nu)
        dist.all_reduce(Y)  # rows are disjoint: the sum assembles Y
        if rank == 0:
            ref = O.OracleSketch(m, n, rank_r, w, kind=0, eta=eta, nu=nu)
            ref.linear_update(A)
            errs = [np.linalg.norm(a.numpy() - b) / np.linalg.norm(b) for a, b in ((X, ref.X), (Y, ref.Y), (Z, ref.Z))]
            np.save(out_path, np.array(errs))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,cfg", [
    (2, (300, 40, 3, 25, 1.0, 1.0)),
    (2, (310, 40, 3, 25, 0.85, 1.3)),   # nu != 1: the partials are weighted before the sum
    (3, (301, 32, 2, 50, 0.9, 0.7)),    # uneven blocks, the last one short
])
def test_gloo_row_block_sharding_matches_one_process(tmp_path, world, cfg):
    import torch.multiprocessing as mp

    out = str(tmp_path / "errs.npy")
    mp.start_processes(_worker, args=(world, _free_port(), cfg, out), nprocs=world, join=True, start_method="spawn")
    errs = np.load(out)
    assert (errs < 1e-12).all(), errs


def test_shard_rows_cover_and_align():
    from skema_b200.distributed import shard_rows, windows_after

    for m, world, w in [(1000, 4, 64), (7, 3, 2), (5, 8, 1), (1_000_000, 8, 10_000)]:
        blocks = [shard_rows(m, world, r, w) for r in range(world)]
        assert sum(nr for _, nr in blocks) == m
        pos = 0
        for r, (r0, nr) in enumerate(blocks):
            assert r0 == pos or nr == 0
            assert r0 % w == 0 or nr == 0
            pos = r0 + nr if nr else pos
        assert windows_after(m, world, world - 1, w) == 0
