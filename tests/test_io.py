"""CPU tests of the matrix-file readers and writer (skema_read_crs,
skema_read_dense, skema_write_crs; Skema::read_matrix / write_matrix,
src/Skema_IO.cpp:8-104) through the C ABI. No GPU is needed.

Pins: the reference's own test files, where present in this checkout, read
to the committed fixture arrays (tests/golden/kat_fixtures.npz, made from
those files); files written from the fixture arrays in each format read
back to the same arrays; the format rules (symmetric expansion, pattern
values, duplicates summed, the dense .bin rejection) on small hand files.
"""
import os

import numpy as np
import pytest
import scipy.sparse as sp

from conftest import ROOT

GOLD = os.path.join(ROOT, "tests", "golden", "kat_fixtures.npz")
# A checkout of the reference, named by SKEMA_REFERENCE; the test that reads
# its files is skipped when the variable is unset.
_REF = os.environ.get("SKEMA_REFERENCE", "")
REF_DATA = os.path.join(_REF, "test", "data") if _REF else ""


@pytest.fixture(scope="module")
def sk(lib_built):
    import skema_b200

    return skema_b200


def golden():
    return np.load(GOLD)


def csr_of(d, stem):
    return sp.csr_matrix((d[stem + "_val"], d[stem + "_col"], d[stem + "_rowptr"]), shape=tuple(d[stem + "_shape"]))


@pytest.mark.skipif(not REF_DATA or not os.path.isdir(REF_DATA), reason="SKEMA_REFERENCE does not name a reference checkout")
def test_reference_files_read_to_the_fixtures(sk):
    d = golden()
    R = sk.read_matrix(os.path.join(REF_DATA, "rectangular_sparse.mtx"))
    assert (R != csr_of(d, "rect_csr")).nnz == 0 and R.shape == (32, 14)
    assert np.allclose(R.toarray(), d["rect_dense"], rtol=0, atol=1e-14)
    S = sk.read_matrix(os.path.join(REF_DATA, "symmetric_sparse.mtx"))
    assert S.nnz == 279 and (S != S.T).nnz == 0
    assert (S != csr_of(d, "sym_csr")).nnz == 0
    B = sk.read_matrix(os.path.join(REF_DATA, "symmetric_sparse.bin"))
    assert B.shape == (27, 27) and (B != S).nnz == 0
    assert np.array_equal(B.indptr, d["sym_bin_rowptr"])


def test_round_trip_through_both_formats(sk, tmp_path):
    d = golden()
    for stem in ("rect_csr", "sym_csr"):
        A = csr_of(d, stem)
        for ext in (".mtx", ".bin"):
            if ext == ".bin" and A.shape[0] != A.shape[1]:
                continue  # the binary layout carries no column count
            p = str(tmp_path / (stem + ext))
            sk.write_matrix(A, p)
            B = sk.read_matrix(p)
            assert B.shape == A.shape and np.array_equal(B.indptr, A.indptr)
            assert np.array_equal(B.indices, A.indices) and np.array_equal(B.data, A.data)


def test_dense_array_file(sk, tmp_path):
    d = golden()
    A = d["rect_dense"]
    p = tmp_path / "a.mtx"
    with open(p, "w") as f:
        f.write("%%MatrixMarket matrix array real general\n% a comment\n")
        f.write(f"{A.shape[0]} {A.shape[1]}\n")
        for x in A.T.ravel():  # column-major
            f.write(f"{x:.17g}\n")
    B = sk.read_matrix(str(p))
    assert B.shape == A.shape and np.array_equal(B, A)
    with pytest.raises(sk.SkemaError):
        sk.read_matrix(str(p), sparse=True)  # an array file is not a CRS input


def test_coordinate_rules(sk, tmp_path):
    p = tmp_path / "s.mtx"
    p.write_text("%%MatrixMarket matrix coordinate pattern symmetric\n3 3 3\n1 1\n3 1\n3 2\n")
    A = sk.read_matrix(str(p)).toarray()
    assert np.array_equal(A, [[1, 0, 1], [0, 0, 1], [1, 1, 0]])
    p.write_text("%%MatrixMarket matrix coordinate real skew-symmetric\n2 2 1\n2 1 4.5\n")
    assert np.array_equal(sk.read_matrix(str(p)).toarray(), [[0, -4.5], [4.5, 0]])
    p.write_text("%%MatrixMarket matrix coordinate real general\n2 3 3\n1 3 1.5\n1 3 2.0\n2 1 -1\n")
    B = sk.read_matrix(str(p))
    assert B.nnz == 2 and B[0, 2] == 3.5 and B[1, 0] == -1.0  # duplicates summed
    p.write_text("%%MatrixMarket matrix coordinate real general\n2 2 1\n3 1 1.0\n")
    with pytest.raises(sk.SkemaError):
        sk.read_matrix(str(p))  # entry outside the matrix
    q = tmp_path / "d.bin"
    q.write_bytes(b"\0" * 16)
    with pytest.raises(sk.SkemaError) as e:
        sk.read_matrix(str(q), sparse=False)
    assert "binary" in str(e.value)


# ------------------------------------------------- row blocks of a .bin file --
def _csr_with_empty_rows(m, n, seed):
    rng = np.random.default_rng(seed)
    A = sp.random(m, n, density=0.03, format="csr", random_state=seed, dtype=np.float64)
    A.data = rng.standard_normal(A.nnz)
    A = A.tolil()
    for i in range(0, m, 7):
        A.rows[i] = []
        A.data[i] = []
    return A.tocsr()


@pytest.mark.parametrize("r0,nr", [(0, 300), (0, 1), (17, 50), (299, 1), (123, 0), (250, -1), (0, -1)])
def test_read_crs_rows_blocks_match_the_whole_file(sk, tmp_path, r0, nr):
    # rows of a binary CRS file read from their offsets equal the same rows
    # of the whole-file read (the file's rows are sorted, so file order is
    # sorted order here); the layout has no column count, so the block is
    # as wide as the file has rows unless a column is larger
    A = _csr_with_empty_rows(300, 120, seed=4)
    path = str(tmp_path / "a.bin")
    sk.write_matrix(A, path)
    whole = sk.read_matrix(path)
    B = sk.read_crs_rows(path, r0, nr)
    end = 300 if nr < 0 else r0 + nr
    assert B.shape == (end - r0, 300)
    assert np.array_equal(B.indptr, whole[r0:end].indptr)
    assert np.array_equal(B.indices, whole[r0:end].indices)
    assert np.array_equal(B.data, whole[r0:end].data)
    assert (B[:, :120] != A[r0:end]).nnz == 0


def test_read_crs_rows_rejects_bad_ranges_and_files(sk, tmp_path):
    from skema_b200 import SkemaError

    A = _csr_with_empty_rows(40, 40, seed=5)
    path = str(tmp_path / "a.bin")
    sk.write_matrix(A, path)
    for r0, nr in [(-1, 3), (39, 2), (41, -1)]:
        with pytest.raises(SkemaError):
            sk.read_crs_rows(path, r0, nr)
    raw = open(path, "rb").read()
    short = str(tmp_path / "short.bin")
    with open(short, "wb") as f:
        f.write(raw[:-8])  # one value missing
    with pytest.raises(SkemaError):
        sk.read_crs_rows(short, 0, 5)
    with pytest.raises(SkemaError):
        sk.read_crs_rows(str(tmp_path / "missing.bin"), 0, 1)
