"""CPU tests of host-side pieces of the reference-facing mirror in
skema_b200/sketchy.py that need no device: the save_history JSON writer."""
def test_write_history_layout(tmp_path):
    """save_history's JSON (src/Skema_SketchySVD.cpp:730-755): keys, the
    reference's timing map and a 4-space indent."""
    import json

    from skema_b200.sketchy import write_history

    p = tmp_path / "hist.json"
    text = write_history(str(p), [3.0, 2.0, 1.0], [0.1, 0.2, 0.3], {"omega": 1.5})
    d = json.loads(p.read_text())
    assert set(d) == {"timings", "traces", "svals", "rnrms"}
    assert d["svals"] == [3.0, 2.0, 1.0] and d["rnrms"] == [0.1, 0.2, 0.3]
    assert set(d["timings"]) == {"init", "update", "approx"}
    assert set(d["timings"]["update"]) == {"upsilon", "omega", "phi", "psi", "window", "daxpy"}
    assert d["timings"]["update"]["omega"] == 1.5
    assert set(d["timings"]["approx"]) == {"phi", "psi", "dgeqrf", "dgemm", "dgels", "dgesvd"}
    assert text.splitlines()[1].startswith("    \"")
    assert write_history(None, [1.0], [0.0]) == json.dumps(json.loads(write_history(None, [1.0], [0.0])), indent=4)
    # keys in sorted order at every level, as the reference's JSON object prints them
    assert list(json.loads(text)) == ["rnrms", "svals", "timings", "traces"]
    assert list(json.loads(text)["timings"]) == ["approx", "init", "update"]
    assert list(json.loads(text)["timings"]["update"]) == sorted(d["timings"]["update"])
    t = json.loads(write_history(None, [2.0], [0.0], None, {"0": {"svals": [2.5]}, "1": {"svals": [2.0]}}))
    assert t["traces"] == {"0": {"svals": [2.5]}, "1": {"svals": [2.0]}}
