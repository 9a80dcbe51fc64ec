"""GPU test: maps imported from dumps in the reference's --debug-file
formats reproduce the exporting context's maps and sketches (dense Gauss
and CSR SparseSign three-sketch contexts)."""
import numpy as np
import pytest
import scipy.sparse as sp

from test_map_dumps import write_gauss_dump, write_sparse_dump

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sk(lib_built):
    import skema_b200

    return skema_b200


def dump_all(s, stem):
    from skema_b200.sketchy import MAP_LABELS

    for which, label in MAP_LABELS.items():
        nr, nc, z, _ = s.map_info(which)
        vals, idx = s.map_export(which)
        if z == 0:
            write_gauss_dump(f"{stem}_{label}.txt", vals)
        else:
            write_sparse_dump(f"{stem}_{label}.mtx", nr, nc, idx, vals)


@pytest.mark.parametrize("kind,sparse", [(0, False), (1, True)])
def test_maps_from_reference_dumps(sk, tmp_path, kind, sparse):
    rng = np.random.default_rng(kind)
    m, n = 1500, 400
    if sparse:
        A = sp.random(m, n, density=0.02, format="csr", random_state=kind, dtype=np.float64)
        A.data = rng.standard_normal(A.nnz).astype(np.float32).astype(np.float64)
    else:
        A = rng.standard_normal((m, n)).astype(np.float32)
    a = sk.AlgParams(matrix_m=m, matrix_n=n, rank=6, window=300, dim_redux=kind, issparse=sparse)
    b = sk.AlgParams(matrix_m=m, matrix_n=n, rank=6, window=300, dim_redux=kind, issparse=sparse,
                     seeds=[11, 12, 13, 14])
    stem = str(tmp_path / "run")
    with sk.SketchySVD(a) as s1, sk.SketchySVD(b) as s2:
        dump_all(s1, stem)
        s2.map_import_reference_dumps(stem)
        for which in range(4):
            v1, i1 = s1.map_export(which)
            v2, i2 = s2.map_export(which)
            if i1 is None:
                # the text dump has 16 decimals; the maps are FP32 values
                assert np.max(np.abs(v2 - v1)) <= 1e-7 * np.max(np.abs(v1))
            else:
                assert np.array_equal(i1, i2) and np.array_equal(v1, v2)
        s1.update_rows(A)
        s2.update_rows(A)
        for x, y in zip(s1.get_sketches(), s2.get_sketches()):
            assert np.linalg.norm(np.asarray(x, np.float64) - y) <= 1e-6 * np.linalg.norm(y)


@pytest.mark.parametrize("kind,sparse", [(0, False), (1, True)])
def test_debug_file_dumps(sk, tmp_path, monkeypatch, kind, sparse):
    # AlgParams.debug_filename: maps at construction, the sketches after
    # every window and at the end, U / S / V from sketchysvd, all as
    # <stem>_<name> in the working directory
    monkeypatch.chdir(tmp_path)
    rng = np.random.default_rng(kind + 5)
    m, n, w = 1200, 300, 500
    if sparse:
        A = sp.random(m, n, density=0.03, format="csr", random_state=kind, dtype=np.float64)
        A.data = rng.standard_normal(A.nnz).astype(np.float32).astype(np.float64)
    else:
        A = rng.standard_normal((m, n)).astype(np.float32)
    a = sk.AlgParams(matrix_m=m, matrix_n=n, rank=5, window=w, dim_redux=kind, issparse=sparse,
                     debug_filename="out/run.json")
    with sk.SketchySVD(a) as s:
        ext = ".mtx" if kind == 1 else ".txt"
        for label in ("Upsilon", "Omega", "Phi", "Psi"):
            assert (tmp_path / f"run_{label}{ext}").exists()
        s.linear_update(A)
        final = s.get_sketches()
        for name, x in zip("XYZ", final):
            for win in range(3):
                assert (tmp_path / f"run_{name}.txt.{win}").exists()
            d = np.loadtxt(tmp_path / f"run_{name}.txt", ndmin=2)
            assert np.array_equal(d.astype(np.float32), x)  # 16 decimals of FP32 values
            assert np.array_equal(np.loadtxt(tmp_path / f"run_{name}.txt.2", ndmin=2), d)
        # after the first window only its rows of Y are set
        y0 = np.loadtxt(tmp_path / "run_Y.txt.0", ndmin=2)
        assert np.array_equal(y0[:w].astype(np.float32), final[1][:w]) and not np.any(y0[w:])
    # the dumped maps reproduce the sketches in a context with other seeds
    b = sk.AlgParams(matrix_m=m, matrix_n=n, rank=5, window=w, dim_redux=kind, issparse=sparse,
                     seeds=[21, 22, 23, 24])
    with sk.SketchySVD(b) as s2:
        s2.map_import_reference_dumps("run")
        s2.linear_update(A)
        for x, y in zip(final, s2.get_sketches()):
            assert np.linalg.norm(np.asarray(x, np.float64) - y) <= 1e-6 * np.linalg.norm(x)
    U, S, V = sk.sketchysvd(A, a)
    assert np.max(np.abs(np.loadtxt(tmp_path / "run_S.txt") - S)) < 1e-15 * max(1.0, S[0])
    assert np.loadtxt(tmp_path / "run_U.txt", ndmin=2).shape == U.shape
    assert np.max(np.abs(np.loadtxt(tmp_path / "run_V.txt", ndmin=2) - V)) < 1e-15


def test_debug_file_dumps_spd(sk, tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    rng = np.random.default_rng(3)
    n = 400
    B = rng.standard_normal((n, 30))
    A = (B @ B.T / n).astype(np.float32)
    a = sk.AlgParams(matrix_m=n, matrix_n=n, rank=4, window=150, dim_redux=0, issymmetric=True,
                     debug_filename="spd.txt")
    with sk.SketchySPD(a) as s:
        assert (tmp_path / "spd_Omega.txt").exists() and not (tmp_path / "spd_Phi.txt").exists()
        s.linear_update(A)
        assert np.array_equal(np.loadtxt(tmp_path / "spd_Y.txt", ndmin=2).astype(np.float32), s.get_sketch(1))
        assert not (tmp_path / "spd_Y.txt.0").exists()
    # one window of all rows writes no sketch dump, as the reference returns first
    c = sk.AlgParams(matrix_m=n, matrix_n=n, rank=4, window=n, dim_redux=0, debug_filename="one.txt")
    with sk.SketchySVD(c) as s:
        s.linear_update(A)
        assert (tmp_path / "one_Omega.txt").exists() and not (tmp_path / "one_X.txt").exists()
