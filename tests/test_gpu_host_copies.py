"""GPU tests of the host-memory paths of the C ABI that the end-to-end step
uses.

skema_get_sketch into host memory in the other layout than the sketch is
stored in (Y is column-major, X and Z row-major) transposes on the device
and copies out in chunks of about 8 M values through two staging slots, the
transpose of one chunk beside the copy of the one before. The results must
equal the same sketch fetched in its stored layout, bit for bit, also when
there are several chunks in either direction.

skema_linear_update_csr from host memory checks the row map on the host
while its copies run; a decreasing row map is still rejected with
SKEMA_EINVAL, launches nothing, and leaves the context usable.
"""

import numpy as np
import pytest
import scipy.sparse as sp

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sk(lib_built):
    import skema_b200

    return skema_b200


def _csr(m, n, nnz_row, seed):
    rng = np.random.default_rng(seed)
    rows = np.repeat(np.arange(m), nnz_row)
    cols = rng.integers(0, n, size=m * nnz_row)
    A = sp.csr_matrix((rng.normal(size=m * nnz_row), (rows, cols)), shape=(m, n))
    A.sum_duplicates()
    A.sort_indices()
    return A


def _fetch(s, which, layout):
    import skema_b200._lib as L

    rows, cols = s._sketch_shape(which)
    if layout == L.ROW_MAJOR:
        out = np.empty((rows, cols), dtype=np.float32)
        s._check(s.lib.skema_get_sketch(s.h, which, out.ctypes.data, cols, L.ROW_MAJOR, L.MEM_HOST))
        return out
    out = np.empty((cols, rows), dtype=np.float32)  # column-major rows x cols
    s._check(s.lib.skema_get_sketch(s.h, which, out.ctypes.data, rows, L.COL_MAJOR, L.MEM_HOST))
    return out.T


@pytest.mark.parametrize("m,n", [(300_000, 600), (1_000, 200_000)])
def test_transposed_host_fetch_equals_stored_layout(sk, m, n):
    # (300,000 x 81) Y: 3 chunks of rows in row-major; (81 x 200,000) X: 2
    # chunks of columns in column-major
    A = _csr(m, n, 4, seed=m % 97)
    a = sk.AlgParams(matrix_m=m, matrix_n=n, rank=20, window=min(m, 50_000), dim_redux=1, issparse=True)
    with sk.SketchySVD(a) as s:
        s.update_rows(A)
        for which in range(3):
            r = _fetch(s, which, 1)
            c = _fetch(s, which, 0)
            assert r.shape == c.shape
            assert np.array_equal(r, c), which
            assert np.any(r)


def test_host_csr_with_a_decreasing_row_map_is_rejected(sk):
    import skema_b200._lib as L

    m, n = 2_000, 300
    A = _csr(m, n, 5, seed=4)
    a = sk.AlgParams(matrix_m=m, matrix_n=n, rank=5, window=500, dim_redux=1, issparse=True)
    rp = np.ascontiguousarray(A.indptr, dtype=np.int64)
    col = np.ascontiguousarray(A.indices, dtype=np.int32)
    val = np.ascontiguousarray(A.data, dtype=np.float32)
    bad = rp.copy()
    bad[700] = bad[701] + 1  # one decreasing step inside the map; the ends are unchanged
    with sk.SketchySVD(a) as s, sk.SketchySVD(a) as ref:
        st = s.lib.skema_linear_update_csr(s.h, bad.ctypes.data, col.ctypes.data, val.ctypes.data, 0, m, L.MEM_HOST)
        assert st == L.EINVAL
        assert b"decreasing" in s.lib.skema_last_error(s.h)
        s.update_rows(A)
        ref.update_rows(A)
        for x, y in zip(s.get_sketches(), ref.get_sketches()):
            assert np.array_equal(np.asarray(x), np.asarray(y)) or \
                np.linalg.norm(np.asarray(x, np.float64) - y) <= 1e-6 * np.linalg.norm(y)


def test_transposed_host_fetch_with_a_wide_range(sk):
    # k = 4 r + 1 = 257 > 256: the chunks take the general tiled transpose
    rng = np.random.default_rng(9)
    m, n = 3000, 700
    A = rng.standard_normal((m, n)).astype(np.float32)
    a = sk.AlgParams(matrix_m=m, matrix_n=n, rank=64, window=1000, dim_redux=0)
    with sk.SketchySVD(a) as s:
        assert s.range == 257
        s.update_rows(A)
        for which in range(3):
            r = _fetch(s, which, 1)
            c = _fetch(s, which, 0)
            assert np.array_equal(r, c), which
