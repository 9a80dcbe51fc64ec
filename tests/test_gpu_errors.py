"""GPU tests of the error statuses that need a device.

SKEMA_ETIMEOUT: every wait of the tensor-core kernels is bounded. A context
whose wait limit is set to 1 ns makes the first wait that does not pass at
once run out; the kernel then stops issuing, lets what it has in flight land,
frees its tensor memory and returns, and the next synchronising call reports
the time-out. The context stays usable: with the default limit restored, a
reset and a new update match the oracle. Nothing here hangs or faults the
device: the waits end by themselves.

SKEMA_ENOMEM: a map too large for the device fails skema_create, and a
context whose workspace is capped fails the update that would grow it, then
works again once the cap is lifted.
"""
import numpy as np
import pytest

from conftest import rel_fro

pytestmark = pytest.mark.gpu

BF16_TOL = 6e-3  # BF16 sketch vs FP64 oracle, relative Frobenius
FP32_TOL = 1e-5


@pytest.fixture(scope="module")
def sk(lib_built):
    import skema_b200

    return skema_b200


def _dense(m, n, seed):
    rng = np.random.default_rng(seed)
    return rng.normal(size=(m, n)).astype(np.float32)


def _oracle(oracle, a, A):
    o = oracle.OracleSketch(a.matrix_m, a.matrix_n, a.rank, a.window, kind=a.dim_redux, issparse=a.issparse)
    o.linear_update(A.astype(np.float64))
    return o


def _check(s, o, tol):
    X, Y, Z = s.get_sketches()
    for got, ref in ((X, o.X), (Y, o.Y), (Z, o.Z)):
        assert rel_fro(got, ref) < tol, rel_fro(got, ref)


def test_wait_limit_runs_out_then_context_recovers(sk, oracle):
    import torch

    from skema_b200 import _lib as L

    m, n = 4096, 2048
    A = _dense(m, n, 3)
    a = sk.AlgParams(matrix_m=m, matrix_n=n, rank=8, window=1024, precision=L.PREC_BF16)
    o = _oracle(oracle, a, A)
    Ad = torch.from_numpy(A).cuda()
    with sk.SketchySVD(a) as s:
        assert s.lib.skema_set_wait_limit(s.h, 1) == L.OK
        with pytest.raises(sk.SkemaError) as e:
            s.linear_update(Ad)
            s.synchronize()
        assert e.value.status == L.ETIMEOUT, e.value
        assert b"gave up waiting" in s.lib.skema_last_error(s.h)
        # the status word was cleared when it was reported
        assert s.lib.skema_synchronize(s.h) == L.OK
        assert s.lib.skema_set_wait_limit(s.h, 0) == L.OK
        s.linear_update(Ad)
        s.synchronize()
        _check(s, o, BF16_TOL)


def test_enomem_when_a_map_does_not_fit(sk):
    from skema_b200 import _lib as L

    # Upsilon alone would be 21 x 2^38 FP32 values (23 TB)
    a = sk.AlgParams(matrix_m=1 << 38, matrix_n=64, rank=5, window=4096)
    with pytest.raises(sk.SkemaError) as e:
        sk.SketchySVD(a)
    assert e.value.status == L.ENOMEM, e.value


@pytest.mark.parametrize("device_input", [True, False])
def test_enomem_from_the_workspace_cap(sk, oracle, device_input):
    import torch

    from skema_b200 import _lib as L

    m, n = 3000, 700
    A = _dense(m, n, 5)
    a = sk.AlgParams(matrix_m=m, matrix_n=n, rank=6, window=700)
    o = _oracle(oracle, a, A)
    inp = torch.from_numpy(A).cuda() if device_input else A
    with sk.SketchySVD(a) as s:
        assert s.lib.skema_set_workspace_limit(s.h, -1) == L.EINVAL
        assert s.lib.skema_set_workspace_limit(s.h, 4096) == L.OK
        with pytest.raises(sk.SkemaError) as e:
            s.linear_update(inp)
            s.synchronize()
        assert e.value.status == L.ENOMEM, e.value
        assert b"skema_set_workspace_limit" in s.lib.skema_last_error(s.h)
        assert s.lib.skema_set_workspace_limit(s.h, 0) == L.OK
        s.linear_update(inp)
        s.synchronize()
        _check(s, o, FP32_TOL)
