"""CPU tests of the C-ABI boundary and the host-side mirror of AlgParams."""
import ctypes as C
import os
import re
import subprocess

import pytest

from conftest import HAS_GPU, ROOT

HEADER = os.path.join(ROOT, "include", "skema_c.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(skema_[a-z_0-9]+)\s*\(", src)))


def test_header_compiles_as_c():
    res = subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-fsyntax-only", "-x", "c", HEADER],
                         capture_output=True, text=True)
    assert res.returncode == 0, res.stderr


def test_library_exports_every_declared_symbol(lib_built):
    out = subprocess.run(["nm", "-D", "--defined-only", lib_built], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (skema_\w+)", out))
    missing = [f for f in declared_functions() if f not in exported]
    assert not missing, missing
    lib = C.CDLL(lib_built)
    for f in declared_functions():
        assert getattr(lib, f) is not None


def test_python_binding_covers_header(lib_built):
    from skema_b200 import _lib

    assert sorted(_lib.SIGNATURES) == declared_functions()


def test_build_targets_sm100a_only():
    from skema_b200 import build

    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
    assert all(f.endswith(".cu") for f in build.sources())


def test_params_defaults_match_algparams(lib_built):
    from skema_b200 import _lib

    p = _lib.default_params()
    # src/Skema_AlgParams.cpp:10-57 and :275-278
    assert (p.rank, p.sketch_range, p.sketch_core, p.window) == (1, 1, 1, 1)
    assert list(p.seeds) == [0, 1, 2, 3]
    assert p.sketch_eta == 1.0 and p.sketch_nu == 1.0
    assert p.kernel_gamma == 1.0
    assert p.dim_redux == _lib.MAP_GAUSS and p.kernel_func == _lib.KERNEL_NONE


@pytest.mark.skipif(HAS_GPU, reason="checks the no-device error path")
def test_create_without_device_fails_loudly(lib_built):
    import skema_b200 as sk

    with pytest.raises(sk.SkemaError) as e:
        sk.SketchySVD(sk.AlgParams(matrix_m=10, matrix_n=8, rank=2))
    assert e.value.status in (sk._lib.ENOKERNEL, sk._lib.ECUDA)


def test_create_rejects_bad_params(lib_built):
    from skema_b200 import _lib

    lib = _lib.load()
    p = _lib.default_params()
    h = C.c_void_p()
    assert lib.skema_create(C.byref(p), C.byref(h)) == _lib.EINVAL  # m = n = 0
    assert b"matrix_m" in lib.skema_last_error(None)
    p.matrix_m, p.matrix_n = 10, 10
    p.window = 0
    assert lib.skema_create(C.byref(p), C.byref(h)) == _lib.EINVAL
    p.window = 1
    p.kernel_func, p.issparse = _lib.KERNEL_GAUSSRBF, 1
    assert lib.skema_create(C.byref(p), C.byref(h)) == _lib.EUNSUPPORTED
    assert lib.skema_reset(None) == _lib.EINVAL


def test_algparams_parse_matches_reference_flags():
    from skema_b200.sketchy import AlgParams

    args = ["--solver", "sketch", "--model", "sparse-sign", "--rank", "20", "--range", "81",
            "--core", "163", "--window", "10000", "--seeds", "[5,6,7,8]", "--eta", "0.5",
            "--nu", "2", "--kernel", "gaussrbf", "--gamma", "0.25", "--force-three-sketch",
            "--sparse", "--precision", "bf16", "--leftover"]
    a = AlgParams()
    a.parse(args)
    assert args == ["--leftover"]  # consumed flags are erased (AlgParams::parse)
    assert (a.solver, a.dim_redux, a.rank, a.sketch_range, a.sketch_core, a.window) == (1, 1, 20, 81, 163, 10000)
    assert a.seeds == [5, 6, 7, 8] and a.sketch_eta == 0.5 and a.sketch_nu == 2.0
    assert a.kernel_func == 1 and a.kernel_gamma == 0.25 and a.force_three_sketch and a.issparse
    assert a.precision == 1
    b = AlgParams()
    b.parse(["rank", "3", "window", "inf"])  # '--' may be omitted; inf -> INT_MAX
    assert b.rank == 3 and b.window == 2**31 - 1


def test_algparams_parse_errors():
    from skema_b200.sketchy import AlgParams

    with pytest.raises(RuntimeError):
        AlgParams().parse(["--rank", "0"])  # below min 1
    with pytest.raises(RuntimeError):
        AlgParams().parse(["--model", "gaussian"])
    with pytest.raises(RuntimeError):
        AlgParams().parse(["--seeds", "1,2"])
    with pytest.raises(RuntimeError):
        AlgParams().parse(["--window", "abc"])


def test_spd_approx_flag():
    from skema_b200 import _lib as L
    from skema_b200.sketchy import AlgParams

    a = AlgParams()
    assert a.spd_approx == L.SPD_NYSTROM and L.default_params().spd_approx == L.SPD_NYSTROM
    args = ["--spd-approx", "reference-steps"]
    a.parse(args)
    assert a.spd_approx == L.SPD_REFERENCE_STEPS and a.to_c().spd_approx == L.SPD_REFERENCE_STEPS
