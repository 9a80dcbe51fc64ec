import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden", "kat_fixtures.npz")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running")


def _has_gpu() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


HAS_GPU = _has_gpu()


def pytest_collection_modifyitems(config, items):
    if HAS_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def kat():
    return dict(np.load(GOLDEN))


@pytest.fixture(scope="session")
def lib_built():
    """Build the CUDA library (no-op when up to date) and return its path."""
    from skema_b200 import build

    return build.build()


@pytest.fixture(scope="session")
def oracle():
    from oracle import sketchy_oracle

    sketchy_oracle.lib()
    return sketchy_oracle


def rel_fro(a, b) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


CPP_PROGRAMS = ("sketch_driver", "dimredux_check", "parse_params")


@pytest.fixture(scope="session")
def cpp_bins(lib_built, tmp_path_factory):
    """The C++ programs under tests/cpp, compiled with g++ against
    include/skema.hpp and linked with the CUDA library (name -> path)."""
    import subprocess

    out = tmp_path_factory.mktemp("cpp")
    libdir = os.path.join(ROOT, "skema_b200")
    bins = {}
    for name in CPP_PROGRAMS:
        exe = str(out / name)
        cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I" + os.path.join(ROOT, "include"),
               os.path.join(ROOT, "tests", "cpp", name + ".cpp"), "-L" + libdir, "-lskema_b200",
               "-Wl,-rpath," + libdir, "-o", exe]
        res = subprocess.run(cmd, capture_output=True, text=True)
        assert res.returncode == 0, res.stderr
        bins[name] = exe
    return bins
