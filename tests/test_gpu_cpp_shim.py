"""GPU tests of the C++ drop-in layer (include/skema.hpp).

The reference-style driver (tests/cpp/sketch_driver.cpp) reads the
reference's own known-answer matrices (tests/golden/kat_fixtures.npz,
written back to MatrixMarket / binary CRS files here) and runs
Skema::sketchysvd end to end; the singular values it saves with
--history-file must match the fixtures' exact ones to the FP32 bar. The
DimRedux check (tests/cpp/dimredux_check.cpp) compares every lmap / rmap
form with explicit FP64 products of the exported maps.
"""
import json
import os
import subprocess

import numpy as np
import pytest
import scipy.sparse as sp

pytestmark = pytest.mark.gpu

BAR = 1e-5  # top-r singular values, relative to sigma_1, FP32 sketches


def write_array_mtx(path, A):
    A = np.asarray(A, dtype=np.float64)
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix array real general\n")
        f.write(f"{A.shape[0]} {A.shape[1]}\n")
        for v in A.T.ravel():
            f.write(f"{v:.17g}\n")


def run_driver(exe, cwd, args):
    res = subprocess.run([exe] + args + ["--solver", "sketch", "--history-file", "hist.json"], cwd=cwd,
                         capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stdout + res.stderr
    with open(os.path.join(cwd, "hist.json")) as f:
        return json.load(f)


def test_driver_dense_rect(cpp_bins, kat, tmp_path):
    write_array_mtx(tmp_path / "rect.mtx", kat["rect_dense"])
    for model in ("gauss", "sparse-sign"):
        h = run_driver(cpp_bins["sketch_driver"], tmp_path, ["--input", "rect.mtx", "--rank", "10", "--window", "5",
                                                              "--range", "12", "--core", "25", "--model", model])
        S = np.array(h["svals"])
        assert np.max(np.abs(S - kat["rect_svals"][:10])) / S[0] < BAR, (model, S)
        assert len(h["rnrms"]) == 10 and np.all(np.isfinite(h["rnrms"]))
        assert set(h) == {"rnrms", "svals", "timings", "traces"}
        # the reference's timing keys (src/Skema_SketchySVD.cpp:101-116), from the device stage timers
        t = h["timings"]
        assert set(t["update"]) == {"upsilon", "omega", "phi", "psi", "window", "daxpy"}
        assert set(t["approx"]) == {"phi", "psi", "dgeqrf", "dgemm", "dgels", "dgesvd"}
        assert t["approx"]["dgesvd"] > 0 and t["approx"]["dgeqrf"] > 0


def test_driver_sparse_rect(cpp_bins, kat, tmp_path):
    import skema_b200 as sk

    A = sp.csr_matrix((kat["rect_csr_val"], kat["rect_csr_col"], kat["rect_csr_rowptr"]),
                      shape=tuple(kat["rect_csr_shape"]))
    sk.write_matrix(A, str(tmp_path / "rect.bin"))
    for model in ("gauss", "sparse-sign"):
        h = run_driver(cpp_bins["sketch_driver"], tmp_path, ["--input", "rect.bin", "--sparse", "--rank", "10",
                                                              "--window", "7", "--range", "12", "--core", "25",
                                                              "--model", model])
        S = np.array(h["svals"])
        assert np.max(np.abs(S - kat["rect_svals"][:10])) / S[0] < BAR, (model, S)


def test_driver_kernel_points(cpp_bins, kat, tmp_path):
    write_array_mtx(tmp_path / "points.mtx", kat["kernel_points"])
    h = run_driver(cpp_bins["sketch_driver"], tmp_path, ["--input", "points.mtx", "--kernel", "gaussrbf", "--gamma",
                                                          "1", "--force-three-sketch", "--rank", "5", "--window", "6",
                                                          "--range", "21", "--core", "25"])
    S = np.array(h["svals"])
    assert np.max(np.abs(S - kat["kernel_svals"][:5])) / S[0] < BAR, S


def test_driver_traces_per_window(cpp_bins, kat, tmp_path):
    # windows of 12 rows: after the first window Y already has rank 12 = range
    write_array_mtx(tmp_path / "rect.mtx", kat["rect_dense"])
    h = run_driver(cpp_bins["sketch_driver"], tmp_path, ["--input", "rect.mtx", "--rank", "10", "--window", "12",
                                                          "--range", "12", "--core", "25",
                                                          "--sketch-compute-svals-iters"])
    assert sorted(h["traces"], key=int) == ["0", "1", "2"]
    last = np.array(h["traces"]["2"]["svals"])
    assert np.max(np.abs(last - np.array(h["svals"]))) / last[0] < 1e-12


def test_dimredux_products(cpp_bins):
    res = subprocess.run([cpp_bins["dimredux_check"]], capture_output=True, text=True, timeout=300)
    print(res.stdout)
    assert res.returncode == 0, res.stdout + res.stderr


@pytest.mark.parametrize("model,kind", [("gauss", 0), ("sparse-sign", 1)])
def test_driver_debug_file_dumps(cpp_bins, kat, tmp_path, model, kind):
    # --debug-file: the maps at construction, the sketches after each of the
    # seven 5-row windows and at the end, and U / S / V, as <stem>_<name> in
    # the working directory; the map dumps equal the Python mirror's maps
    # for the same parameters
    import skema_b200 as sk

    write_array_mtx(tmp_path / "rect.mtx", kat["rect_dense"])
    h = run_driver(cpp_bins["sketch_driver"], tmp_path, ["--input", "rect.mtx", "--rank", "10", "--window", "5",
                                                          "--range", "12", "--core", "25", "--model", model,
                                                          "--debug-file", "out/dbg.json"])
    for name in "XYZ":
        for w in range(7):
            assert (tmp_path / f"dbg_{name}.txt.{w}").exists()
        assert np.array_equal(np.loadtxt(tmp_path / f"dbg_{name}.txt.6", ndmin=2),
                              np.loadtxt(tmp_path / f"dbg_{name}.txt", ndmin=2))
    assert not (tmp_path / "dbg_X.txt.7").exists()
    S = np.loadtxt(tmp_path / "dbg_S.txt")
    assert np.max(np.abs(S - np.array(h["svals"]))) <= 1e-15 * S[0]
    assert np.loadtxt(tmp_path / "dbg_U.txt", ndmin=2).shape == (32, 10)
    assert np.loadtxt(tmp_path / "dbg_V.txt", ndmin=2).shape == (14, 10)
    a = sk.AlgParams(matrix_m=32, matrix_n=14, rank=10, window=5, sketch_range=12, sketch_core=25, dim_redux=kind)
    with sk.SketchySVD(a) as s:
        for which, label in sk.sketchy.MAP_LABELS.items():
            nr, nc, z, _ = s.map_info(which)
            vals, idx = sk.read_reference_map_dump(str(tmp_path / f"dbg_{label}{'.mtx' if z else '.txt'}"), nr, nc)
            v0, i0 = s.map_export(which)
            if z:
                assert np.array_equal(idx, i0) and np.array_equal(vals, v0)
            else:
                assert np.max(np.abs(vals - v0)) <= 1e-15 * max(1.0, np.abs(v0).max())
        # the final Y dump is the sketch of the same input through the mirror
        s.linear_update(np.asarray(kat["rect_dense"], dtype=np.float32))
        y = np.loadtxt(tmp_path / "dbg_Y.txt", ndmin=2)
        assert np.max(np.abs(y - s.get_sketch(1))) <= 1e-5 * np.abs(y).max()
