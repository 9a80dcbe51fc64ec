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
