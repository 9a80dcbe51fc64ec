"""GPU tests of skema_update_from_file: matrix files streamed into the
sketches equal the same rows passed as arrays.

A binary CRS file is read one window at a time through two pinned buffers;
its FP64 values are rounded to FP32 on the host, so values that are FP32
numbers give the array path's Y exactly (its rows are summed in a fixed
order); X and Z are sums of atomic partial terms, whose order varies from
run to run, so they are held to 1e-6 relative Frobenius error.
MatrixMarket files are read whole first and then take the same update as
the arrays.
"""
import numpy as np
import pytest
import scipy.sparse as sp

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sk(lib_built):
    import skema_b200

    return skema_b200


def csr_fp32_values(m, n, nnz_row, seed):
    rng = np.random.default_rng(seed)
    rows = np.repeat(np.arange(m), nnz_row)
    cols = rng.integers(0, n, size=m * nnz_row)
    A = sp.csr_matrix((rng.normal(size=m * nnz_row), (rows, cols)), shape=(m, n))
    A.sum_duplicates()
    A = A.tolil()
    for i in range(0, m, 13):  # empty rows
        A.rows[i] = []
        A.data[i] = []
    A = A.tocsr()
    A.data = A.data.astype(np.float32).astype(np.float64)
    return A


def alg(sk, m, n, window, kind, issparse, **kw):
    a = sk.AlgParams(matrix_m=m, matrix_n=n, rank=10, window=window, dim_redux=kind, issparse=issparse)
    for key, v in kw.items():
        setattr(a, key, v)
    return a


def sketches(s):
    return [np.array(x, copy=True) for x in s.get_sketches()]


def same(s1, s2, y_exact=True):
    (x1, y1, z1), (x2, y2, z2) = sketches(s1), sketches(s2)
    if y_exact:
        assert np.array_equal(y1, y2)
    for a, b in ((x1, x2), (y1, y2), (z1, z2)):
        assert np.linalg.norm(a - b) <= 1e-6 * max(np.linalg.norm(b), 1e-30)


@pytest.mark.parametrize("kind", [0, 1])
def test_bin_file_streams_like_the_arrays(sk, tmp_path, kind):
    m, n = 5000, 1200
    A = csr_fp32_values(m, n, 9, seed=kind + 3)
    path = str(tmp_path / "a.bin")
    sk.write_matrix(A, path)
    a = alg(sk, m, n, 700, kind, True, sketch_eta=1.25, sketch_nu=0.9)
    with sk.SketchySVD(a) as s1, sk.SketchySVD(a) as s2:
        s1.update_rows(A)
        s2.update_from_file(path)
        same(s1, s2)
        # a row block of the file, starting inside a window
        s1.reset()
        s2.reset()
        s1.update_rows(A[1234:4000], 1234)
        s2.update_from_file(path, 1234, 4000 - 1234)
        same(s1, s2)


def test_mtx_files_stream_like_the_arrays(sk, tmp_path):
    m, n = 900, 400
    A = csr_fp32_values(m, n, 6, seed=11)
    path = str(tmp_path / "a.mtx")
    sk.write_matrix(A, path)
    a = alg(sk, m, n, 128, 1, True)
    with sk.SketchySVD(a) as s1, sk.SketchySVD(a) as s2:
        s1.update_rows(A)
        s2.update_from_file(path)
        same(s1, s2)
    # a dense MatrixMarket array file for a dense context
    rng = np.random.default_rng(2)
    D = rng.normal(size=(300, 70)).astype(np.float32)
    dpath = str(tmp_path / "d.mtx")
    with open(dpath, "w") as f:
        f.write("%%MatrixMarket matrix array real general\n300 70\n")
        for v in D.T.ravel():  # column-major values
            f.write(f"{float(v):.9g}\n")
    b = alg(sk, 300, 70, 64, 0, False)
    with sk.SketchySVD(b) as s1, sk.SketchySVD(b) as s2:
        s1.update_rows(np.asfortranarray(D))
        s2.update_from_file(dpath)
        same(s1, s2, y_exact=False)


def test_file_stream_errors(sk, tmp_path):
    from skema_b200 import SkemaError

    A = csr_fp32_values(200, 50, 4, seed=1)
    path = str(tmp_path / "a.bin")
    sk.write_matrix(A, path)
    with sk.SketchySVD(alg(sk, 100, 50, 32, 1, True)) as s:  # fewer rows than the file
        with pytest.raises(SkemaError):
            s.update_from_file(path)
        s.update_from_file(path, 0, 100)  # the first 100 rows fit
    with sk.SketchySVD(alg(sk, 200, 40, 32, 1, True)) as s:  # a column outside A
        if A[:, 40:].nnz:
            with pytest.raises(SkemaError):
                s.update_from_file(path)
    with sk.SketchySVD(alg(sk, 200, 50, 32, 0, False)) as s:  # a dense context
        with pytest.raises(SkemaError):
            s.update_from_file(path)
