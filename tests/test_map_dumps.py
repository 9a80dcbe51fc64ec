"""CPU tests of the reader for the reference's map dumps (--debug-file:
src/Skema_DimRedux.hpp:124-127, 264-267, written by Impl::write,
src/Skema_Common.hpp:175-190): a Gauss map as nrow lines of "%.16f "
values, a SparseSign map as a MatrixMarket coordinate file with its zeta
entries per row as stored (repeats kept)."""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def sk(lib_built):
    import skema_b200

    return skema_b200


def write_gauss_dump(path, M):
    with open(path, "w") as f:
        for row in M:
            f.write("".join("%.16f " % v for v in row))
            f.write("\n")


def write_sparse_dump(path, nrow, ncol, idx, val):
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n")
        f.write(f"{nrow} {ncol} {idx.size}\n")
        for r in range(nrow):
            for c, v in zip(idx[r], val[r]):
                f.write(f"{r + 1} {c + 1} {v:.1f}\n")


def test_gauss_dump_round_trip(sk, tmp_path):
    rng = np.random.default_rng(0)
    M = rng.uniform(-3, 3, size=(7, 40))
    p = str(tmp_path / "run_Omega.txt")
    write_gauss_dump(p, M)
    vals, idx = sk.read_reference_map_dump(p, 7, 40)
    assert idx is None
    assert np.max(np.abs(vals - M)) < 1e-15  # 16 decimals
    with pytest.raises(ValueError):
        sk.read_reference_map_dump(p, 40, 7)


def test_sparse_dump_keeps_rows_and_repeats(sk, tmp_path):
    rng = np.random.default_rng(1)
    nrow, ncol, zeta = 30, 9, 8
    idx = rng.integers(0, ncol, size=(nrow, zeta)).astype(np.int32)
    idx[::4, 1] = idx[::4, 0]  # a repeated column in a row, as sampling with replacement gives
    val = np.where(rng.random((nrow, zeta)) < 0.5, -1.0, 1.0)
    p = str(tmp_path / "run_Phi.mtx")
    write_sparse_dump(p, nrow, ncol, idx, val)
    v2, i2 = sk.read_reference_map_dump(p, nrow, ncol)
    assert np.array_equal(i2, idx) and np.array_equal(v2, val)
    # entries listed out of row order come back grouped by row, file order kept within a row
    lines = open(p).read().splitlines()
    body = lines[2:]
    rng.shuffle(body)
    perm = str(tmp_path / "perm_Phi.mtx")
    with open(perm, "w") as f:
        f.write("\n".join(lines[:2] + body) + "\n")
    v3, i3 = sk.read_reference_map_dump(perm, nrow, ncol)
    for r in range(nrow):
        assert sorted(zip(i3[r], v3[r])) == sorted(zip(idx[r], val[r]))
    # an uneven row is rejected
    with open(perm, "w") as f:
        f.write("\n".join(lines[:2] + lines[2:-1]) + "\n")
    with pytest.raises(ValueError):
        sk.read_reference_map_dump(perm, nrow, ncol)


def test_library_writers_use_the_reference_formats(sk, tmp_path):
    from skema_b200.sketchy import write_dense_text, write_reference_map_dump

    rng = np.random.default_rng(2)
    # Gauss: byte for byte the "%.16f " lines of Impl::write
    M = rng.uniform(-3, 3, size=(5, 11))
    write_reference_map_dump(str(tmp_path / "a_Omega.txt"), M)
    write_gauss_dump(str(tmp_path / "b_Omega.txt"), M)
    assert open(tmp_path / "a_Omega.txt").read() == open(tmp_path / "b_Omega.txt").read()
    # a vector: one "%.16f" value per line
    v = rng.standard_normal(6)
    write_dense_text(str(tmp_path / "run_S.txt"), v)
    assert open(tmp_path / "run_S.txt").read() == "".join("%.16f\n" % x for x in v)
    # SparseSign: a coordinate file that reads back exactly, repeats kept
    nrow, ncol, zeta = 13, 7, 8
    idx = rng.integers(0, ncol, size=(nrow, zeta)).astype(np.int32)
    idx[::3, 2] = idx[::3, 1]
    val = np.where(rng.random((nrow, zeta)) < 0.5, -1.0, 1.0)
    p = str(tmp_path / "run_Psi.mtx")
    write_reference_map_dump(p, val, idx, ncol)
    lines = open(p).read().splitlines()
    assert lines[0] == "%%MatrixMarket matrix coordinate real general"
    assert lines[1] == f"{nrow} {ncol} {nrow * zeta}"
    v2, i2 = sk.read_reference_map_dump(p, nrow, ncol)
    assert np.array_equal(i2, idx) and np.array_equal(v2, val)
