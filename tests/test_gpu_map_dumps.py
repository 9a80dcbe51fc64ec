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
