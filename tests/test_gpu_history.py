"""GPU test of the per-window singular-value traces
(--sketch-compute-svals-iters, src/Skema_SketchySVD.cpp:164-216) and of the
history file that carries them (save_history, :730-755).

After every window the fixed-rank approximation runs on the sketches so far;
the traces are compared with the oracle's after each window at the 1e-5 bar
of the FP32 sketches (relative to the largest value). The library's
approximation leaves Y intact, so later windows are not corrupted as in the
reference (its QR runs in place on Y).
"""
import json

import numpy as np
import pytest

from test_gpu_sketch import alg, dense_input, oracle_for

pytestmark = pytest.mark.gpu


def test_svals_traces_and_history(lib_built, oracle, tmp_path):
    import skema_b200 as sk

    m, n = 600, 300
    A = dense_input(m, n, seed=4).astype(np.float32)
    a = alg(sk, m, n, 5, 100, 0, sketch_range=21, sketch_core=43)
    a.sketch_compute_svals_iters = True
    o = oracle_for(oracle, a)
    ref = o.linear_update_traced(A.astype(np.float64))
    with sk.SketchySVD(a) as s:
        s.linear_update(A)
        assert sorted(s.traces, key=int) == [str(w) for w in range(6)]
        for w, t in ref.items():
            got = np.asarray(s.traces[w]["svals"])
            exp = np.asarray(t["svals"])
            assert np.max(np.abs(got - exp)) / exp[0] < 1e-5, (w, got, exp)
        s.low_rank_approx()
        s.compute_residuals(A)
        p = tmp_path / "hist.json"
        s.save_history(str(p))
    h = json.loads(p.read_text())
    assert set(h["traces"]) == {str(w) for w in range(6)}
    assert np.allclose(h["traces"]["5"]["svals"], h["svals"], rtol=1e-12)
    assert len(h["rnrms"]) == 5
