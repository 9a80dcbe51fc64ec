"""GPU parity tests of the BF16 tensor-core form of the dense Gauss sketch.

The context holds its maps on the BF16 grid (every value rounded to BF16,
also in the FP32 copies the approximation uses), so the oracle takes the
same maps. The input window is rounded to BF16 (8-bit significand, unit
roundoff 2^-9) and every product accumulates in FP32, so the sketches are
compared with the FP64 oracle on the same inputs and maps at a relative
Frobenius tolerance of 6e-3: about three times the error of one rounding of
each operand of a sum of random-signed terms. Z sees two roundings (T is
kept in BF16 between its two products) and gets 1e-2.

Shapes cover: windows whose first row is and is not a multiple of 8 (the
Upsilon / Phi window slices are TMA operands in place or copied), row- and
column-major host input, device input, split-K (the rank-50 shape: k = 201,
s = 403, 24 output tiles per product) with eta / nu and two update calls,
and the Gauss RBF kernel input.
"""
import numpy as np
import pytest

from conftest import rel_fro
from test_gpu_sketch import alg, dense_input, oracle_for

pytestmark = pytest.mark.gpu

TOL_XY = 6e-3
TOL_Z = 1e-2


@pytest.fixture(scope="module")
def sk(lib_built):
    import skema_b200

    return skema_b200


def bf16(a, sk):
    a.precision = sk._lib.PREC_BF16
    return a


def bf16_grid(maps):
    """The BF16 context's version of the oracle maps (dict name -> Map): the
    FP64 values rounded to FP32, then to BF16 (round to nearest even)."""
    import torch

    for mp in maps.values():
        mp._dense = torch.from_numpy(np.asarray(mp.dense)).float().bfloat16().double().numpy()


def oracle_bf16(oracle, a, **kw):
    o = oracle_for(oracle, a, **kw)
    bf16_grid(o.maps)
    return o


def test_bf16_maps_on_the_bf16_grid(sk, oracle):
    m, n = 600, 300
    a = bf16(alg(sk, m, n, 5, 100, 0), sk)
    o = oracle_bf16(oracle, a)
    with sk.SketchySVD(a) as s:
        for which, name in ((sk._lib.UPSILON, "upsilon"), (sk._lib.OMEGA, "omega"), (sk._lib.PHI, "phi"),
                            (sk._lib.PSI, "psi")):
            got = s.map_export(which)[0]
            assert np.array_equal(got, o.maps[name].dense), name


def check(s, o, tag=""):
    X, Y, Z = s.get_sketches()
    ex, ey, ez = rel_fro(X, o.X), rel_fro(Y, o.Y), rel_fro(Z, o.Z)
    assert np.isfinite(X).all() and np.isfinite(Y).all() and np.isfinite(Z).all(), tag
    assert ey < TOL_XY, (tag, "Y", ey)
    assert ex < TOL_XY, (tag, "X", ex)
    assert ez < TOL_Z, (tag, "Z", ez)
    return ex, ey, ez


@pytest.mark.parametrize("layout", ["C", "F"])
def test_dense_bf16_parity(sk, oracle, layout):
    m, n = 2000, 1000
    A = dense_input(m, n).astype(np.float32)
    A = np.asfortranarray(A) if layout == "F" else np.ascontiguousarray(A)
    a = bf16(alg(sk, m, n, 10, 100, 0), sk)  # windows start at 100, 200, ...: both alignments
    o = oracle_bf16(oracle, a)
    o.linear_update(A.astype(np.float64))
    with sk.SketchySVD(a) as s:
        s.linear_update(A)
        check(s, o, layout)


def test_dense_bf16_split_k_eta_nu_two_calls(sk, oracle):
    import torch

    m, n = 4096, 3000
    A = dense_input(m, n, seed=11).astype(np.float32)
    a = bf16(alg(sk, m, n, 50, 2048, 0, sketch_eta=1.25, sketch_nu=0.8), sk)
    o = oracle_bf16(oracle, a)
    o.linear_update(A.astype(np.float64))
    At = torch.from_numpy(A).cuda()
    with sk.SketchySVD(a) as s:
        assert (s.range, s.core) == (201, 403)
        s.update_rows(At[:2048], 0)
        s.update_rows(At[2048:], 2048)
        check(s, o, "split-k")


@pytest.mark.parametrize("layout", ["C", "F"])
@pytest.mark.parametrize("n", [333, 336])
def test_dense_bf16_ragged_window(sk, oracle, layout, n):
    # 129-row windows, the last one 3 rows. Strides that are not a multiple
    # of 4 elements (n = 333 row-major, 129 / 3 column-major) take the
    # separate conversion pass; the others are read as FP32 by the X^T product.
    m = 777
    A = dense_input(m, n, seed=5).astype(np.float32)
    A = np.asfortranarray(A) if layout == "F" else np.ascontiguousarray(A)
    a = bf16(alg(sk, m, n, 7, 129, 0, sketch_nu=0.5), sk)
    o = oracle_bf16(oracle, a)
    o.linear_update(A.astype(np.float64))
    with sk.SketchySVD(a) as s:
        s.linear_update(A)
        check(s, o, "ragged")


def test_dense_bf16_device_column_major_offsets(sk, oracle):
    # a column-major device matrix (ld = m): windows start at rows 0, 96, 192
    # (16-byte aligned: FP32 read by TMA) and the last window is ragged
    import torch

    m, n = 252, 512
    A = dense_input(m, n, seed=12).astype(np.float32)
    a = bf16(alg(sk, m, n, 5, 96, 0, sketch_eta=0.5), sk)
    o = oracle_bf16(oracle, a)
    o.linear_update(A.astype(np.float64))
    At = torch.from_numpy(np.asfortranarray(A)).cuda().t().contiguous().t()
    assert At.stride() == (1, m)
    with sk.SketchySVD(a) as s:
        s.linear_update(At)
        check(s, o, "device-F")


def test_rbf_bf16_parity(sk, oracle):
    N, d = 700, 5
    P = oracle.mixture_points(N, d, seed=1)
    gamma = oracle.median_gamma(P)
    a = bf16(alg(sk, N, N, 6, 128, 0, kernel_func=1, kernel_gamma=gamma, force_three_sketch=True), sk)
    o = oracle_bf16(oracle, a, gamma=gamma)
    o.linear_update(P.astype(np.float64))
    with sk.SketchySVD(a) as s:
        s.linear_update(P)
        check(s, o, "rbf")


@pytest.mark.parametrize("N,d,rank,window,eta,nu", [
    (3000, 64, 20, 1024, 1.0, 1.0),     # one d-subtile; k + s = 244, one output chunk
    (2600, 100, 20, 999, 0.75, 0.9),    # two d-subtiles, unaligned windows (map slices copied)
    (2048, 32, 70, 512, 1.0, 1.0),      # k = 281, s = 563: three row-pass chunks, wide X chunk
])
def test_rbf_bf16_tensor_core_parity(sk, oracle, N, d, rank, window, eta, nu):
    # the kernel is never stored: both passes regenerate its tiles from the
    # BF16 points (Gram on the tensor cores, exp in registers)
    P = oracle.mixture_points(N, d, seed=3)
    gamma = oracle.median_gamma(P)
    a = bf16(alg(sk, N, N, rank, window, 0, kernel_func=1, kernel_gamma=gamma, force_three_sketch=True,
                 sketch_eta=eta, sketch_nu=nu), sk)
    o = oracle_bf16(oracle, a, gamma=gamma)
    o.linear_update(P.astype(np.float64))
    with sk.SketchySVD(a) as s:
        s.linear_update(P)
        check(s, o, f"rbf-tc N={N} d={d}")


@pytest.mark.parametrize("nu", [0.8, -0.5])
def test_rbf_bf16_blocks_and_dirty_rows(sk, oracle, nu):
    # several calls over row blocks, one of them repeated (its Y rows get the
    # nu term); nu > 0 folds each call's windows into one pass with weights,
    # nu <= 0 takes them one window at a time
    N, d = 2000, 48
    P = oracle.mixture_points(N, d, seed=7)
    gamma = oracle.median_gamma(P)
    a = bf16(alg(sk, N, N, 10, 300, 0, kernel_func=1, kernel_gamma=gamma, force_three_sketch=True,
                 sketch_eta=1.1, sketch_nu=nu), sk)
    o = oracle_bf16(oracle, a, gamma=gamma)
    o.reset()
    calls = [(0, 1000), (1000, 1000), (400, 600)]
    for r0, nr in calls:
        o.update_rows(P.astype(np.float64), r0, nr)
    with sk.SketchySVD(a) as s:
        s.reset()
        for r0, nr in calls:
            s.update_rows(P, r0, nr)
        check(s, o, f"rbf blocks nu={nu}")


def test_bf16_low_rank_approx(sk, oracle):
    m, n = 2000, 1000
    A = dense_input(m, n).astype(np.float32)
    a32 = alg(sk, m, n, 10, 256, 0)
    with sk.SketchySVD(a32) as s:
        s.linear_update(A)
        _, S32, _ = s.low_rank_approx()
    with sk.SketchySVD(bf16(alg(sk, m, n, 10, 256, 0), sk)) as s:
        s.linear_update(A)
        U, S, V = s.low_rank_approx()
    assert np.max(np.abs(S - S32)) / S32[0] < 1e-2
    assert np.allclose(U.T @ U, np.eye(10), atol=1e-8)
    assert np.allclose(V.T @ V, np.eye(10), atol=1e-8)


def test_bf16_map_import_refreshes_copies(sk, oracle):
    m, n = 512, 256
    A = dense_input(m, n, seed=8).astype(np.float32)
    a = bf16(alg(sk, m, n, 4, 128, 0), sk)
    with sk.SketchySVD(a) as s:
        v, ix = s.map_export(1)  # Omega~
        s.map_import(1, -v, ix)
        s.linear_update(A)
        Y = s.get_sketch(1)
    with sk.SketchySVD(bf16(alg(sk, m, n, 4, 128, 0), sk)) as s:
        s.linear_update(A)
        Y0 = s.get_sketch(1)
    assert rel_fro(Y, -Y0) < 1e-6


# ---------------------------------------------------------------- FP8 form --
# The FP8 context holds its Gauss maps on the E4M3 grid scaled by one power of
# two (2^floor(log2(448 / max maxval))), so the oracle takes the same maps:
# the FP64 oracle maps rounded to FP32, scaled, rounded to E4M3 (round to
# nearest even) and scaled back -- the map test checks that bit for bit. The
# window is scaled by a power of two from its amax and rounded to E4M3 for
# the [Y | T] product; X^T stays on the BF16 path. Bars (relative Frobenius
# against the FP64 oracle with the same maps): X 6e-3 (BF16), Y and Z 4e-2
# (one E4M3 rounding of every window entry: relative spacing 2^-3, so up to
# 2^-4 per entry and about 2.5e-2 in the mean square).
TOL_X8 = 6e-3
TOL_YZ8 = 4e-2


def fp8(a, sk):
    a.precision = sk._lib.PREC_FP8
    return a


def e4m3_grid(maps):
    """The FP8 context's version of the oracle maps (dict name -> Map)."""
    import math

    import torch

    mx = max(math.sqrt(2.0 * math.log(mp.nrow * mp.ncol)) for mp in maps.values())
    r = np.float32(448.0) / np.float32(mx)
    e = int((np.frombuffer(np.float32(r).tobytes(), np.uint32)[0] >> 23) & 0xFF) - 127
    sm = 2.0 ** e
    for mp in maps.values():
        f32 = torch.from_numpy(np.asarray(mp.dense)).float()
        q = (f32 * sm).to(torch.float8_e4m3fn).float() / sm
        mp._dense = q.double().numpy()
    return sm


def test_fp8_maps_on_the_e4m3_grid(sk, oracle):
    m, n = 600, 300
    a = fp8(alg(sk, m, n, 5, 100, 0), sk)
    o = oracle_for(oracle, a)
    e4m3_grid(o.maps)
    with sk.SketchySVD(a) as s:
        for which, name in ((sk._lib.UPSILON, "upsilon"), (sk._lib.OMEGA, "omega"), (sk._lib.PHI, "phi"),
                            (sk._lib.PSI, "psi")):
            got = s.map_export(which)[0]
            assert np.array_equal(got, o.maps[name].dense), name


def check8(s, o, tag=""):
    X, Y, Z = s.get_sketches()
    ex, ey, ez = rel_fro(X, o.X), rel_fro(Y, o.Y), rel_fro(Z, o.Z)
    print(f"fp8 {tag}: X {ex:.2e} Y {ey:.2e} Z {ez:.2e}")
    assert np.isfinite(X).all() and np.isfinite(Y).all() and np.isfinite(Z).all(), tag
    assert ex < TOL_X8, (tag, "X", ex)
    assert ey < TOL_YZ8, (tag, "Y", ey)
    assert ez < TOL_YZ8, (tag, "Z", ez)


@pytest.mark.parametrize("layout", ["C", "F"])
def test_dense_fp8_parity(sk, oracle, layout):
    m, n = 2000, 1000
    A = dense_input(m, n).astype(np.float32)
    A = np.asfortranarray(A) if layout == "F" else np.ascontiguousarray(A)
    a = fp8(alg(sk, m, n, 10, 100, 0), sk)
    o = oracle_for(oracle, a)
    e4m3_grid(o.maps)
    o.linear_update(A.astype(np.float64))
    with sk.SketchySVD(a) as s:
        s.linear_update(A)
        check8(s, o, layout)


def test_dense_fp8_split_k_eta_nu_two_calls(sk, oracle):
    import torch

    m, n = 4096, 3000
    A = dense_input(m, n, seed=11).astype(np.float32)
    a = fp8(alg(sk, m, n, 50, 2048, 0, sketch_eta=1.25, sketch_nu=0.8), sk)
    o = oracle_for(oracle, a)
    e4m3_grid(o.maps)
    o.linear_update(A.astype(np.float64))
    At = torch.from_numpy(A).cuda()
    with sk.SketchySVD(a) as s:
        s.update_rows(At[:2048], 0)
        s.update_rows(At[2048:], 2048)
        check8(s, o, "split-k")


@pytest.mark.parametrize("n", [333, 336])
def test_dense_fp8_ragged_window(sk, oracle, n):
    # n = 333 row-major: the separate BF16 conversion and its amax pass
    m = 777
    A = np.ascontiguousarray(dense_input(m, n, seed=5).astype(np.float32))
    a = fp8(alg(sk, m, n, 7, 129, 0, sketch_nu=0.5), sk)
    o = oracle_for(oracle, a)
    e4m3_grid(o.maps)
    o.linear_update(A.astype(np.float64))
    with sk.SketchySVD(a) as s:
        s.linear_update(A)
        check8(s, o, f"ragged n={n}")


def test_dense_fp8_window_scale_tracks_amax(sk, oracle):
    # two windows whose magnitudes differ by 2^20: each gets its own scale,
    # so the small one keeps its relative accuracy
    m, n = 256, 512
    A = dense_input(m, n, seed=9).astype(np.float32)
    A[128:] *= 2.0 ** -20
    a = fp8(alg(sk, m, n, 5, 128, 0), sk)
    o = oracle_for(oracle, a)
    e4m3_grid(o.maps)
    o.linear_update(A.astype(np.float64))
    with sk.SketchySVD(a) as s:
        s.linear_update(A)
        Y = s.get_sketch(sk._lib.SKETCH_Y)
    for r0 in (0, 128):
        e = rel_fro(Y[r0:r0 + 128], o.Y[r0:r0 + 128])
        print(f"fp8 window at {r0}: Y {e:.2e}")
        assert e < TOL_YZ8, (r0, e)


@pytest.mark.parametrize("prec", ["bf16", "fp8"])
@pytest.mark.parametrize("window", [500, 512])
def test_dense_tc_many_windows_one_call_nu(sk, oracle, prec, window):
    # a device input of six windows (the last ragged) in one call. Windows of
    # 512 rows (64-row blocks) form one group: X^T per window, one [Y | T]
    # product and one Z^T product for the group, T weighted nu^(G-1-w);
    # windows of 500 rows take the per-window path
    import torch

    m, n = 2900, 700
    A = dense_input(m, n, seed=21).astype(np.float32)
    a = alg(sk, m, n, 8, window, 0, sketch_eta=1.25, sketch_nu=0.8)
    a = bf16(a, sk) if prec == "bf16" else fp8(a, sk)
    o = oracle_for(oracle, a)
    if prec == "fp8":
        e4m3_grid(o.maps)
    o.linear_update(A.astype(np.float64))
    with sk.SketchySVD(a) as s:
        s.linear_update(torch.from_numpy(A).cuda())
        if prec == "bf16":
            check(s, o, "six windows")
        else:
            check8(s, o, "six windows")


@pytest.mark.parametrize("prec", ["bf16", "fp8"])
@pytest.mark.parametrize("sms,windows", [(40, 1), (74, 2)])
def test_dense_tc_two_stream_pipeline(sk, oracle, monkeypatch, prec, sms, windows):
    # X^T on its own share of the SMs (context stream) beside [Y | T] and Z
    # of the previous group (side stream), two window-copy buffers in turn:
    # seven 256-row windows give four to seven groups, so each buffer is
    # refilled while the other one's group is still being read; two calls,
    # the second over rows the first wrote (its Y rows get the nu term)
    import torch

    monkeypatch.setenv("SKEMA_DENSE_PIPE_SMS", str(sms))
    monkeypatch.setenv("SKEMA_DENSE_PIPE_WINDOWS", str(windows))
    m, n = 1800, 600
    A = dense_input(m, n, seed=33).astype(np.float32)
    a = alg(sk, m, n, 8, 256, 0, sketch_eta=0.75, sketch_nu=0.9)
    a = bf16(a, sk) if prec == "bf16" else fp8(a, sk)
    o = oracle_for(oracle, a)
    if prec == "fp8":
        e4m3_grid(o.maps)
    o.linear_update(A.astype(np.float64))
    o.update_rows(A[:1024].astype(np.float64), 0, 1024)
    with sk.SketchySVD(a) as s:
        At = torch.from_numpy(A).cuda()
        s.linear_update(At)
        s.update_rows(At[:1024], 0)
        if prec == "bf16":
            check(s, o, f"pipeline {sms} SMs, {windows} windows per group")
        else:
            check8(s, o, f"pipeline {sms} SMs, {windows} windows per group")
