"""Host-side pieces of the benchmark (no GPU): the request mix of the batched
and serving workloads, the comparison count, and the latency/throughput
summary of an open-loop run."""
from __future__ import annotations

import numpy as np

import bench
from irisb200.batched import Request
from irisb200.serving import Completion


def test_request_mix_proportions():
    z = np.zeros((3, 16, 1), np.uint16)
    planted = {0: (5, 0), 10: (77, 3)}
    reqs = bench.request_mix(4000, z, z, planted, 1000, seed=1, p_append=0.01)
    kinds = [r.kind for r in reqs]
    n_app = kinds.count("append")
    n_re = kinds.count("reauth")
    n_u = kinds.count("uniqueness")
    assert 20 <= n_app <= 70
    assert 0.15 < n_re / (n_re + n_u) < 0.25
    rots = [r.n_rot for r in reqs if r.kind != "append"]
    assert set(rots) == {1, 16, 31}
    mir = np.mean([r.mirrored for r in reqs if r.kind != "append"])
    assert 0.45 < mir < 0.55
    for i, r in enumerate(reqs):
        if r.kind == "reauth":
            assert 0 <= r.target < 1000
            if i % 16 in planted:
                assert r.target == planted[i % 16][0]
    # seeded: the same seed gives the same mix
    again = bench.request_mix(4000, z, z, planted, 1000, seed=1, p_append=0.01)
    assert [(r.kind, r.n_rot, r.mirrored, r.target) for r in again] == \
        [(r.kind, r.n_rot, r.mirrored, r.target) for r in reqs]


def test_comparisons_and_latency_summary():
    u = Request(code=None, mask=None, n_rot=16, mirrored=True)
    r = Request(code=None, mask=None, kind="reauth", target=3)
    a = Request(code=None, mask=None, kind="append")
    assert bench.comparisons_of(u, 1000) == 2000
    assert bench.comparisons_of(r, 1000) == 1
    reqs = [u, r, a, u]
    comps = [Completion(0, 10.0, 10.1, None), Completion(1, 10.0, 10.3, None), Completion(2, 10.0, 10.0, None),
             Completion(3, 10.5, 11.0, None)]
    st = bench._latency_stats(comps, reqs, 10.0, [1000, 1000, 1001, 1001])
    assert st["completed"] == 4
    assert abs(st["p50_ms"] - 300.0) < 1e-6 and abs(st["max_ms"] - 500.0) < 1e-6
    assert abs(st["comparisons_per_s"] - (2000 + 1 + 2002) / 1.0) < 1e-6


def test_measured_peaks_parsing(tmp_path, monkeypatch):
    """MEASURED_PEAKS.json figures are read as numbers or {"value": n};
    absent or malformed figures come back as None."""
    import json
    import bench
    monkeypatch.setattr(bench, "ROOT", str(tmp_path))
    assert bench.measured_peaks()["present"] is False
    (tmp_path / "MEASURED_PEAKS.json").write_text(json.dumps(
        {"hbm_gbs": 6540.5, "bf16_tflops": {"value": 1590}, "bf16_tflops_sustained": "n/a"}))
    mp = bench.measured_peaks()
    assert mp == {"hbm_gbs": 6540.5, "bf16_tflops": 1590.0, "bf16_tflops_sustained": None, "present": True}
    (tmp_path / "MEASURED_PEAKS.json").write_text("{not json")
    assert bench.measured_peaks()["hbm_gbs"] is None


def test_percentiles_and_threshold_roofline(tmp_path, monkeypatch):
    """Latency percentiles are nearest-rank (p99 of 200 samples is the 198th
    value, not the maximum); the threshold roofline takes its instructions per
    word from the profile counters file and its ceiling from the SM count and
    the sampled clock."""
    import json
    assert bench.pct(list(range(1, 201)), 99) == 198
    assert bench.pct(list(range(1, 101)), 50) == 50
    assert bench.pct([7.0], 99) == 7.0
    monkeypatch.setattr(bench, "ROOT", str(tmp_path))
    rf = bench.threshold_roofline(10.0, 1000, 148, 1500.0, [(0, 1)])
    assert rf["achieved"] is None and rf["frac"] is None
    assert rf["peak"] == 148 * 4 * 32 * 1500.0e6
    assert abs(rf["words_per_s"] - 1000 / 0.01) < 1e-6
    (tmp_path / "profiles").mkdir()
    (tmp_path / "profiles" / "threshold_bitmap_counters.json").write_text(
        json.dumps({"inst_per_word": 20000.0, "source": "test"}))
    rf = bench.threshold_roofline(10.0, 1000, 148, 1500.0, [(0, 1)])
    assert abs(rf["achieved"] - 20000.0 * 1000 / 0.01) < 1e-3
    assert abs(rf["frac"] - rf["achieved"] / rf["peak"]) < 1e-12
    assert "binding_pipe" not in rf
    (tmp_path / "profiles" / "threshold_bitmap_counters.json").write_text(
        json.dumps({"inst_per_word": 20000.0, "source": "test", "alu_pipe_pct": 87.5, "issue_active_pct": 71.0}))
    rf = bench.threshold_roofline(10.0, 1000, 148, 1500.0, [(0, 1)])
    assert rf["binding_pipe"]["pipe"] == "alu" and abs(rf["binding_pipe"]["frac"] - 0.875) < 1e-12


def test_cpu_mpc_simulation_matches_plaintext():
    """The secondary CPU leg runs the whole 3-party protocol (masked dot
    shares, threshold circuit, open, rotation OR) on the oracle and must equal
    the plaintext predicate on its sample; query 0 is planted at entry 0."""
    out = bench.cpu_mpc_simulation(n_query=2, n_db=48, n_entries=40, min_seconds=0.0)
    assert out["equal_to_plaintext"]
    assert out["matches"] >= 1
    assert out["value"] > 0 and out["kind"] == "port"
