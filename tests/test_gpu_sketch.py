"""GPU parity tests: the CUDA library through the C ABI against the oracle.

Bars: map indices/signs and Gauss entries bit-exact; FP32 sketches X, Y, Z
within 1e-5 relative Frobenius error of the FP64 oracle on the same inputs
and maps; singular values of the fixed-rank approximation against the
reference's own fixtures.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from conftest import rel_fro

pytestmark = pytest.mark.gpu

TOL = 1e-5  # FP32 sketch vs FP64 oracle, relative Frobenius


@pytest.fixture(scope="module")
def sk(lib_built):
    import skema_b200

    return skema_b200


def dense_input(m, n, seed=0, noise=1e-4):
    """U diag(s) V^T + noise with s_i = 10^(-0.1 i) (the small dense recipe)."""
    rng = np.random.default_rng(seed)
    p = min(m, n, 64)
    U = np.linalg.qr(rng.normal(size=(m, p)))[0]
    V = np.linalg.qr(rng.normal(size=(n, p)))[0]
    s = 10.0 ** (-0.1 * np.arange(p))
    return (U * s) @ V.T + noise * rng.normal(size=(m, n))


def csr_input(m, n, nnz_row=10, seed=2, empty_every=0):
    rng = np.random.default_rng(seed)
    rows = np.repeat(np.arange(m), nnz_row)
    cols = rng.integers(0, n, size=m * nnz_row)
    vals = rng.normal(size=m * nnz_row)
    A = sp.csr_matrix((vals, (rows, cols)), shape=(m, n))  # duplicates summed
    A.sum_duplicates()
    if empty_every:
        A = A.tolil()
        for i in range(0, m, empty_every):
            A.rows[i] = []
            A.data[i] = []
        A = A.tocsr()
    A.data = A.data.astype(np.float32).astype(np.float64)
    return A


def alg(sk, m, n, rank, window, kind, issparse=False, **kw):
    a = sk.AlgParams(matrix_m=m, matrix_n=n, rank=rank, window=window, dim_redux=kind, issparse=issparse)
    for key, v in kw.items():
        setattr(a, key, v)
    return a


def oracle_for(oracle, a, spd=False, gamma=None):
    return oracle.OracleSketch(a.matrix_m, a.matrix_n, a.rank, a.window, kind=a.dim_redux,
                               issparse=a.issparse, sketch_range=a.sketch_range, sketch_core=a.sketch_core,
                               eta=a.sketch_eta, nu=a.sketch_nu, seeds=tuple(a.seeds), spd=spd,
                               kernel_gamma=gamma)


def check_sketches(s, o):
    X, Y, Z = s.get_sketches()
    assert rel_fro(Y, o.Y) < TOL, rel_fro(Y, o.Y)
    assert rel_fro(X, o.X) < TOL, rel_fro(X, o.X)
    assert rel_fro(Z, o.Z) < TOL, rel_fro(Z, o.Z)


# ------------------------------------------------------------------ maps ----
@pytest.mark.parametrize("kind", [0, 1])
@pytest.mark.parametrize("issparse", [False, True])
def test_maps_bitexact(sk, oracle, kind, issparse):
    a = alg(sk, 700, 300, 4, 50, kind, issparse)
    o = oracle_for(oracle, a)
    with sk.SketchySVD(a) as s:
        for which, name in enumerate(["upsilon", "omega", "phi", "psi"]):
            om = o.maps[name]
            nr, nc, z, tr = s.map_info(which)
            assert (nr, nc, tr) == (om.nrow, om.ncol, om.init_transposed)
            vals, idx = s.map_export(which)
            if kind == 0:
                assert z == 0
                assert np.array_equal(vals, om.dense.astype(np.float32).astype(np.float64))
            else:
                assert np.array_equal(idx, om.idx)
                assert np.array_equal(vals, om.val)


def test_map_import_roundtrip(sk, oracle):
    a = alg(sk, 300, 200, 3, 50, 1, True)
    with sk.SketchySVD(a) as s:
        v, ix = s.map_export(1)
        ix2 = np.sort((ix + 1) % ix.max(), axis=1)
        s.map_import(1, -v, ix2)
        v3, ix3 = s.map_export(1)
        assert np.array_equal(ix3, ix2) and np.array_equal(v3, -v)
        with pytest.raises(sk.SkemaError):
            s.map_import(1, v * 0.5, ix)  # sparse-sign values must be +-1


# ------------------------------------------------------------ dense FP32 ----
@pytest.mark.parametrize("kind", [0, 1])
@pytest.mark.parametrize("layout", ["C", "F"])
def test_dense_fp32_parity(sk, oracle, kind, layout):
    m, n = 2000, 1000
    A = dense_input(m, n).astype(np.float32)
    A = np.asfortranarray(A) if layout == "F" else np.ascontiguousarray(A)
    a = alg(sk, m, n, 10, 100, kind)  # k = 41, s = 83 (config 1 shape)
    o = oracle_for(oracle, a)
    o.linear_update(A.astype(np.float64))
    with sk.SketchySVD(a) as s:
        assert (s.range, s.core) == (41, 83)
        s.linear_update(A)
        check_sketches(s, o)


def test_dense_device_input_partial_window_eta_nu(sk, oracle):
    import torch

    m, n = 1234, 333
    A = dense_input(m, n, seed=3).astype(np.float32)
    a = alg(sk, m, n, 6, 200, 0, sketch_eta=0.75, sketch_nu=0.9)
    o = oracle_for(oracle, a)
    o.linear_update(A.astype(np.float64))
    At = torch.from_numpy(A).cuda()
    with sk.SketchySVD(a) as s:
        s.linear_update(At)
        check_sketches(s, o)
        # column-major view of the same data
        s.linear_update(At.t().contiguous().t())
        check_sketches(s, o)


def test_dense_streaming_blocks_equal_one_shot(sk, oracle):
    m, n = 1200, 256
    A = dense_input(m, n, seed=4).astype(np.float32)
    a = alg(sk, m, n, 5, 100, 0)
    with sk.SketchySVD(a) as s:
        s.linear_update(A)
        X1, Y1, Z1 = s.get_sketches()
        s.reset()
        s.update_rows(A[:500], 0)
        s.update_rows(A[500:], 500)
        s.update_rows(A[:0], 0)  # empty call is a no-op
        X2, Y2, Z2 = s.get_sketches()
    assert rel_fro(X2, X1) < 1e-6 and rel_fro(Y2, Y1) < 1e-6 and rel_fro(Z2, Z1) < 1e-6


def test_single_shot_window_equals_m(sk, oracle):
    m, n = 300, 120
    A = dense_input(m, n, seed=6).astype(np.float32)
    a = alg(sk, m, n, 4, m, 0)
    o = oracle_for(oracle, a)
    o.linear_update(A.astype(np.float64))
    with sk.SketchySVD(a) as s:
        s.linear_update(A)
        check_sketches(s, o)


# ------------------------------------------------------------------- CSR ----
@pytest.mark.parametrize("kind", [1, 0])
def test_csr_parity(sk, oracle, kind):
    m, n = 20500, 5000
    A = csr_input(m, n, empty_every=97)
    a = alg(sk, m, n, 20, 1000, kind, issparse=True)  # k = 81, s = 163
    o = oracle_for(oracle, a)
    o.linear_update(A)
    with sk.SketchySVD(a) as s:
        s.linear_update(A)
        check_sketches(s, o)


def test_csr_device_input_and_eta_nu(sk, oracle):
    import torch

    m, n = 8000, 3000
    A = csr_input(m, n, nnz_row=7, seed=9)
    a = alg(sk, m, n, 8, 999, 1, issparse=True, sketch_eta=1.5, sketch_nu=0.5)
    o = oracle_for(oracle, a)
    o.linear_update(A)
    rp = torch.from_numpy(A.indptr.astype(np.int64)).cuda()
    cl = torch.from_numpy(A.indices.astype(np.int32)).cuda()
    vl = torch.from_numpy(A.data.astype(np.float32)).cuda()
    with sk.SketchySVD(a) as s:
        s.linear_update((rp, cl, vl))
        check_sketches(s, o)


@pytest.mark.parametrize("m", [1000, 1001])
def test_csr_blocks_dirty_rows_and_offsets(sk, oracle, m):
    # Both write-outs of the Y kernel: 16-byte (full 32-row tiles, first row
    # and m multiples of 4) and per-lane (any other start row, odd m, a
    # clipped tile), on clean rows and on rows updated again with the nu term.
    n = 700
    A = csr_input(m, n, nnz_row=9, seed=13)
    a = alg(sk, m, n, 5, 100, 1, issparse=True, sketch_eta=0.75, sketch_nu=0.9)
    o = oracle_for(oracle, a)
    o.reset()
    # (500, 3): a 3-row tile clipped at row 503, whose rows must stay
    # untouched until the (503, ...) call writes them
    calls = [(0, 500), (500, 3), (503, m - 503), (0, 500), (200, 300)]
    for r0, nr in calls:
        o.update_rows(A, r0, nr)
    with sk.SketchySVD(a) as s:
        s.reset()
        for r0, nr in calls:
            s.update_rows(A[r0:r0 + nr], r0)
        check_sketches(s, o)


def test_csr_duplicate_columns_are_summed(sk, oracle):
    m, n = 64, 40
    rowptr = np.arange(0, 3 * m + 1, 3, dtype=np.int64)
    col = np.tile(np.array([5, 5, 17], dtype=np.int32), m)
    val = np.tile(np.array([1.0, 2.0, -1.0], dtype=np.float32), m)
    a = alg(sk, m, n, 2, 16, 1, issparse=True)
    # copies: scipy aliases the index arrays and sum_duplicates() compacts them in place
    merged = sp.csr_matrix((val.astype(np.float64), col.copy(), rowptr.copy()), shape=(m, n))
    merged.sum_duplicates()
    o = oracle_for(oracle, a)
    o.linear_update(merged)
    with sk.SketchySVD(a) as s:
        s.linear_update((rowptr, col, val))
        check_sketches(s, o)


@pytest.mark.parametrize("issparse", [True, False])
def test_reset_then_read_or_update(sk, oracle, issparse):
    # A reset leaves X and Z to be zeroed by the next call: a read-back sees
    # zeros, and an update after the reset equals one on a fresh context
    # (the CSR update zeroes them on its side stream beside the Y kernel).
    m, n = 2000, 600
    A = csr_input(m, n, nnz_row=8, seed=4) if issparse else dense_input(m, n, seed=4)
    a = alg(sk, m, n, 6, 500, 1, issparse=issparse, sketch_nu=0.8)
    o = oracle_for(oracle, a)
    o.linear_update(A)
    with sk.SketchySVD(a) as s:
        s.update_rows(A, 0, None)
        s.update_rows(A, 0, None)
        s.reset()
        for sketch in s.get_sketches():
            assert not np.any(sketch)
        s.update_rows(A, 0, None)
        s.reset()
        s.update_rows(A, 0, None)
        check_sketches(s, o)


# name: (kind, issparse, precision, spd, window, row blocks, bar)
OVERLAP_CASES = {
    "csr-ssign": (1, True, 0, False, 40, [(0, 100), (50, 100)], TOL),
    "csr-gauss": (0, True, 0, False, 40, [(0, 100), (50, 100)], TOL),
    "dense-gauss": (0, False, 0, False, 40, [(0, 100), (50, 100)], TOL),
    "dense-ssign": (1, False, 0, False, 40, [(0, 100), (50, 100)], TOL),
    "dense-bf16-window": (0, False, 1, False, 40, [(0, 100), (50, 100)], 6e-3),
    "dense-bf16-group": (0, False, 1, False, 64, [(0, 256), (128, 256)], 6e-3),
    "spd-gauss": (0, False, 0, True, 40, [(0, 100), (50, 100)], TOL),
    "spd-ssign": (1, False, 0, True, 40, [(0, 100), (50, 100)], TOL),
}


@pytest.mark.parametrize("case", sorted(OVERLAP_CASES))
def test_reset_then_overlapping_row_blocks(sk, oracle, case):
    # After a reset, Y rows that no update has written since are zero, also
    # where a block overlaps rows written before: reset, update [0, 100),
    # then [50, 150). Rows [100, 150) start from zero, not from what Y held
    # before the reset; rows [50, 100) get nu * Y + eta * y twice.
    import torch

    kind, issparse, prec, spd, W, blocks, bar = OVERLAP_CASES[case]
    m, n = (400, 400) if spd else (600, 300)
    A = csr_input(m, n, nnz_row=7, seed=11) if issparse else dense_input(m, n, seed=11)
    a = alg(sk, m, n, 5, W, kind, issparse, sketch_nu=0.5, sketch_eta=2.0, precision=prec)
    if spd:
        A = 0.5 * (A + A.T)
        a.issymmetric = True
    o = oracle_for(oracle, a, spd=spd)
    cls = sk.SketchySPD if spd else sk.SketchySVD

    def block(r0, nr):
        if issparse:
            return A[r0:r0 + nr]
        return torch.from_numpy(np.ascontiguousarray(A[r0:r0 + nr], dtype=np.float32)).cuda()

    with cls(a) as s:
        s.update_rows(block(0, m), 0, m)  # Y holds data from before the reset
        s.update_rows(block(0, m), 0, m)
        s.reset()
        for r0, nr in blocks:
            s.update_rows(block(r0, nr), r0, nr)
            o.update_rows(A, r0, nr)
        if spd:
            Y = s.get_sketches()
            assert rel_fro(Y, o.Y) < bar, rel_fro(Y, o.Y)
        else:
            X, Y, Z = s.get_sketches()
            for got, ref in ((X, o.X), (Y, o.Y), (Z, o.Z)):
                assert rel_fro(got, ref) < bar, rel_fro(got, ref)
        end = blocks[-1][0] + blocks[-1][1]
        assert not np.any(np.asarray(Y)[end:])


def test_csr_sparse_sign_top_bin(sk, oracle):
    # k = 256: bin 255, whose 16-bit offset 255 * 128 = 32640 sits just under
    # the sign bit, is used on the GPU.
    m, n = 3000, 700
    A = csr_input(m, n, nnz_row=9, seed=256)
    a = alg(sk, m, n, 20, 1000, 1, issparse=True, sketch_range=256, sketch_nu=0.9)
    o = oracle_for(oracle, a)
    o.linear_update(A)
    assert o.k == 256 and np.any(o.maps["omega"].idx == 255)
    with sk.SketchySVD(a) as s:
        assert s.range == 256
        s.linear_update(A)
        check_sketches(s, o)


@pytest.mark.parametrize("rank", [32, 40, 63])
def test_csr_sparse_sign_wide_range(sk, oracle, rank):
    # k = 4 r + 1 = 129, 161, 253: the 16-bit offset form with bins above 127
    m, n = 5000, 1500
    A = csr_input(m, n, nnz_row=9, seed=rank, empty_every=41)
    a = alg(sk, m, n, rank, 1200, 1, issparse=True, sketch_nu=0.9)
    o = oracle_for(oracle, a)
    o.linear_update(A)
    with sk.SketchySVD(a) as s:
        assert s.range == 4 * rank + 1
        s.linear_update(A)
        check_sketches(s, o)


def test_csr_update_on_caller_stream(sk, oracle):
    # The CSR update forks its X / Z work onto a side stream and joins it
    # back before returning; on a caller's stream the sketches read back in
    # that stream's order must be complete.
    import torch

    m, n = 6000, 2000
    A = csr_input(m, n, nnz_row=9, seed=17)
    a = alg(sk, m, n, 8, 1500, 1, issparse=True, sketch_nu=0.7)
    o = oracle_for(oracle, a)
    o.linear_update(A)
    rp = torch.from_numpy(A.indptr.astype(np.int64)).cuda()
    cl = torch.from_numpy(A.indices.astype(np.int32)).cuda()
    vl = torch.from_numpy(A.data.astype(np.float32)).cuda()
    st = torch.cuda.Stream()
    with sk.SketchySVD(a) as s, torch.cuda.stream(st):
        s.set_stream(st.cuda_stream)
        for _ in range(3):
            s.reset()
            s.update_rows((rp, cl, vl), 0, m)
        X = torch.empty((s.range, n), dtype=torch.float32, device="cuda")
        s.get_sketch(0, X)
        Xh = X.cpu().numpy()
        s.set_stream(None)
        check_sketches(s, o)
    assert rel_fro(Xh, o.X) < TOL


def test_csr_long_rows_and_tail(sk, oracle):
    # rows of 900 nonzeros among rows of 0-5, two empty 32-row tiles, and a
    # nonzero count that is not a multiple of 4
    rng = np.random.default_rng(31)
    m, n = 2600, 2000
    counts = np.where(np.arange(m) % 97 == 0, 900, rng.integers(0, 6, size=m))
    counts[64:128] = 0  # two empty 32-row tiles
    rows = np.repeat(np.arange(m), counts)
    cols = np.concatenate([rng.choice(n, size=c, replace=False) for c in counts])
    A = sp.csr_matrix((rng.normal(size=rows.size), (rows, cols)), shape=(m, n))
    A.data = A.data.astype(np.float32).astype(np.float64)
    if A.nnz % 4 == 0:
        A = A[:-1]
        m -= 1
    assert A.nnz % 4 != 0
    a = alg(sk, m, n, 20, 700, 1, issparse=True)
    o = oracle_for(oracle, a)
    o.linear_update(A)
    with sk.SketchySVD(a) as s:
        s.linear_update(A)
        check_sketches(s, o)


def test_csr_unaligned_device_arrays(sk, oracle):
    # col / val device arrays that do not start on 16 bytes
    import torch

    m, n = 4000, 1300
    A = csr_input(m, n, nnz_row=11, seed=23, empty_every=13)
    a = alg(sk, m, n, 20, 900, 1, issparse=True, sketch_nu=0.75)
    o = oracle_for(oracle, a)
    o.linear_update(A)
    rp = torch.from_numpy(A.indptr.astype(np.int64)).cuda()
    cl = torch.from_numpy(np.concatenate([[0], A.indices]).astype(np.int32)).cuda()[1:]
    vl = torch.from_numpy(np.concatenate([[0.0], A.data]).astype(np.float32)).cuda()[1:]
    assert cl.data_ptr() % 16 != 0 and vl.data_ptr() % 16 != 0
    with sk.SketchySVD(a) as s:
        s.linear_update((rp, cl, vl))
        check_sketches(s, o)


def test_csr_imported_map_unsorted_duplicate_bins(sk):
    # The zeta = 8, k <= 128 kernel takes the map in a 16-bit offset form
    # sorted by bin with repeated bins flagged; an imported map may list its
    # rows unsorted with repeats anywhere.
    m, n = 3000, 900
    A = csr_input(m, n, nnz_row=11, seed=21)
    a = alg(sk, m, n, 20, m, 1, issparse=True)  # k = 81, zeta = 8
    rng = np.random.default_rng(5)
    with sk.SketchySVD(a) as s:
        _, ix = s.map_export(1)
        assert ix.shape == (n, 8)
        ix2 = rng.integers(0, 81, size=ix.shape).astype(np.int32)
        ix2[::3, 1] = ix2[::3, 0]  # adjacent repeat
        ix2[::5, 7] = ix2[::5, 2]  # repeat far apart
        ix2[::7, 3:6] = ix2[::7, 6:7]  # four of one bin
        v2 = np.where(rng.random(ix.shape) < 0.5, -1.0, 1.0)
        s.map_import(1, v2, ix2)
        s.linear_update(A)
        Y = s.get_sketches()[1]
    OmT = np.zeros((n, 81))
    np.add.at(OmT, (np.repeat(np.arange(n), 8), ix2.ravel()), v2.ravel())
    assert rel_fro(Y, A @ OmT) < 1e-6


# ------------------------------------------------------------- SketchySPD ----
@pytest.mark.parametrize("kind", [0, 1])
@pytest.mark.parametrize("issparse", [False, True])
def test_spd_update(sk, oracle, kind, issparse):
    m = 900
    B = dense_input(m, m, seed=7)
    B = (B + B.T).astype(np.float32)
    A = sp.csr_matrix(np.where(np.abs(B) > 2e-3, B, 0).astype(np.float64)) if issparse else B
    a = alg(sk, m, m, 5, 128, kind, issparse=issparse, issymmetric=True)
    o = oracle_for(oracle, a, spd=True)
    o.linear_update(A if issparse else A.astype(np.float64))
    with sk.SketchySPD(a) as s:
        assert s.spd
        s.linear_update(A)
        Y = s.get_sketches()
    assert rel_fro(Y, o.Y) < TOL


# ------------------------------------------------------------------- RBF ----
@pytest.mark.parametrize("kind", [0, 1])
def test_rbf_update_parity(sk, oracle, kind):
    N, d = 700, 5
    P = oracle.mixture_points(N, d, seed=1)
    gamma = oracle.median_gamma(P)
    a = alg(sk, N, N, 6, 128, kind, kernel_func=1, kernel_gamma=gamma, force_three_sketch=True)
    o = oracle_for(oracle, a, gamma=gamma)
    o.linear_update(P.astype(np.float64))
    with sk.SketchySVD(a) as s:
        s.linear_update(P)
        check_sketches(s, o)


# -------------------------------------------------------- approximation ----
@pytest.mark.parametrize("kind", [0, 1])
def test_kat_rect(sk, kat, kind):
    a = alg(sk, 32, 14, 10, 5, kind, sketch_range=12, sketch_core=25)
    with sk.SketchySVD(a) as s:
        s.linear_update(kat["rect_dense"].astype(np.float32))
        U, S, V = s.low_rank_approx()
    assert np.max(np.abs(S - kat["rect_svals"][:10])) / S[0] < 1e-5
    assert np.allclose(U.T @ U, np.eye(10), atol=1e-8)
    assert np.allclose(V.T @ V, np.eye(10), atol=1e-8)


def test_kat_rect_csr(sk, kat):
    A = sp.csr_matrix((kat["rect_csr_val"], kat["rect_csr_col"], kat["rect_csr_rowptr"]),
                      shape=tuple(kat["rect_csr_shape"]))
    for kind in (0, 1):
        a = alg(sk, 32, 14, 10, 7, kind, issparse=True, sketch_range=12, sketch_core=25)
        with sk.SketchySVD(a) as s:
            s.linear_update(A)
            _, S, _ = s.low_rank_approx()
        assert np.max(np.abs(S - kat["rect_svals"][:10])) / S[0] < 1e-5


def test_kat_symmetric(sk, kat):
    a = alg(sk, 27, 27, 10, 4, 0, sketch_range=27, sketch_core=27)
    with sk.SketchySVD(a) as s:
        s.linear_update(kat["sym_dense"].astype(np.float32))
        _, S, _ = s.low_rank_approx()
    assert np.max(np.abs(S - kat["sym_svals"][:10])) / S[0] < 1e-5


def test_kat_kernel(sk, kat):
    a = alg(sk, 25, 25, 5, 6, 0, sketch_range=21, sketch_core=25, kernel_func=1, kernel_gamma=1.0,
            force_three_sketch=True)
    with sk.SketchySVD(a) as s:
        s.linear_update(kat["kernel_points"].astype(np.float32))
        _, S, _ = s.low_rank_approx()
    assert np.max(np.abs(S - kat["kernel_svals"][:5])) / S[0] < 1e-5


@pytest.mark.parametrize("rank", [10, 50])
def test_low_rank_approx_vs_oracle(sk, oracle, rank):
    # rank 10: k = 41, the single-CTA shared-memory Jacobi and the tensor-core
    # tall products; rank 50: k = 201, s = 403, the block Jacobi (A and V do
    # not fit one CTA) and the general FP64 products for k > 128
    m, n = 2000, 1000
    A = dense_input(m, n).astype(np.float32)
    a = alg(sk, m, n, rank, 100, 0)
    o = oracle_for(oracle, a)
    with sk.SketchySVD(a) as s:
        s.linear_update(A)
        X, Y, Z = s.get_sketches()
        U, S, V = s.low_rank_approx()
    # the oracle's approximation from the GPU's own sketches and the same
    # FP32-rounded Phi, Psi (the maps the sketches were formed with) isolates
    # the FP64 solver: CholeskyQR2 + Jacobi vs Householder + dgesvd
    o.X, o.Y, o.Z = X.astype(np.float64), Y.astype(np.float64), Z.astype(np.float64)
    for name in ("phi", "psi"):
        o.maps[name]._dense = o.maps[name].dense.astype(np.float32).astype(np.float64)
    Uo, So, Vo = o.low_rank_approx()
    assert np.max(np.abs(S - So) / So[0]) < 1e-11
    # singular vectors agree up to sign
    assert np.allclose(np.abs(np.sum(U * Uo, axis=0)), 1.0, atol=1e-6)
    assert np.allclose(np.abs(np.sum(V * Vo, axis=0)), 1.0, atol=1e-6)


# ------------------------------------------------------------- errors ------
def test_error_paths(sk):
    a = alg(sk, 100, 50, 3, 10, 0)
    with sk.SketchySVD(a) as s:
        with pytest.raises(sk.SkemaError) as e:
            s.update_rows(np.zeros((10, 50), np.float32), 95)  # rows past m
        assert e.value.status == sk._lib.EINVAL
        rp, cl, vl = np.array([0, 1], np.int64), np.array([0], np.int32), np.ones(1, np.float32)
        st = s.lib.skema_linear_update_csr(s.h, rp.ctypes.data, cl.ctypes.data, vl.ctypes.data, 0, 1,
                                           sk._lib.MEM_HOST)
        assert st == sk._lib.ESTATE  # a dense context refuses a CSR update
        Xs = np.arange(s.range * 50, dtype=np.float32).reshape(s.range, 50)
        s.set_sketch(0, Xs)
        assert np.array_equal(s.get_sketch(0), Xs)
