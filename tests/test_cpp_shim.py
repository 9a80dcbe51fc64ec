"""CPU tests of the C++ drop-in layer (include/skema.hpp).

A driver with the reference's call pattern (driver/main.cpp:42-210:
build_arg_list, parse_filepath, AlgParams::parse, read_matrix, main_driver,
Skema::sketchysvd) and a check of the DimRedux lmap / rmap products compile
against the header with g++ -Wall -Wextra -Werror and link the CUDA library.
AlgParams::parse consumes the same flags with the same results as the Python
mirror. No GPU is needed: the programs that touch the device run in
tests/test_gpu_cpp_shim.py.
"""
import os
import subprocess

import pytest

from conftest import ROOT


def test_header_compiles_standalone():
    res = subprocess.run(["g++", "-std=c++17", "-Wall", "-Wextra", "-Werror", "-fsyntax-only", "-x", "c++",
                          os.path.join(ROOT, "include", "skema.hpp")], capture_output=True, text=True)
    assert res.returncode == 0, res.stderr


def test_programs_compile_and_link(cpp_bins):
    for path in cpp_bins.values():
        assert os.access(path, os.X_OK)


def test_driver_help_needs_no_device(cpp_bins):
    res = subprocess.run([cpp_bins["sketch_driver"], "--help"], capture_output=True, text=True, timeout=60)
    assert res.returncode == 0 and "Sketch options" in res.stdout


def _cpp_parse(exe, args):
    out = subprocess.run([exe] + args, capture_output=True, text=True, timeout=60).stdout
    if out.startswith("error "):
        return "error"
    f = {}
    for line in out.splitlines():
        key, _, rest = line.partition(" ")
        f[key] = rest
    return f


def _py_parse(args):
    import skema_b200 as sk

    a = sk.AlgParams()
    left = list(args)
    try:
        a.parse(left)
    except RuntimeError:
        return "error"
    b = lambda v: str(int(bool(v)))
    g = lambda v: f"{v:g}"
    return {"matrix_m": str(a.matrix_m), "matrix_n": str(a.matrix_n), "rank": str(a.rank), "window": str(a.window),
            "sketch_range": str(a.sketch_range), "sketch_core": str(a.sketch_core), "sketch_eta": g(a.sketch_eta),
            "sketch_nu": g(a.sketch_nu), "dim_redux": str(a.dim_redux), "kernel_func": str(a.kernel_func),
            "kernel_gamma": g(a.kernel_gamma), "solver": str(a.solver), "issparse": b(a.issparse),
            "issymmetric": b(a.issymmetric), "force_three_sketch": b(a.force_three_sketch),
            "precision": str(a.precision), "spd_approx": str(a.spd_approx),
            "seeds": " ".join(str(s) for s in a.seeds), "unused": " ".join(left)}


ARGS = [
    [],
    ["--rank", "5", "--window", "100", "--model", "sparse-sign", "--seeds", "[4,5,6,7]"],
    ["--sparse", "--symmetric", "--force-three-sketch", "--range", "41", "--core", "83", "--eta", "0.5",
     "--nu", "2"],
    ["--kernel", "gaussrbf", "--gamma", "0.25", "--precision", "bf16", "--spd-approx", "reference-steps",
     "--solver", "sketch", "leftover", "--m", "300", "--n", "200"],
    ["rank", "7", "window", "3"],                    # bare flag names are accepted
    ["--rank", "0"],                                 # below the range: error
    ["--model", "hadamard"],                         # not one of the names: error
    ["--seeds", "1,2"],                              # not of the form [..]: error
    ["--window", "12abc", "--eta", "1e-3"],          # strtol prefix
]


@pytest.mark.parametrize("args", ARGS, ids=[" ".join(a) or "defaults" for a in ARGS])
def test_algparams_parse_matches_the_python_mirror(cpp_bins, args):
    assert _cpp_parse(cpp_bins["parse_params"], args) == _py_parse(args)
