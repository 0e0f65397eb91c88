"""Host-side logic of bench.py, on the CPU: the measured-traffic record is
used only for the solver sources it was captured from, the CPU baseline's
step window, the core count, and the roofline byte counts."""
import json
import os
import sys

import pytest

from conftest import ROOT

sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_traffic_record_matches_only_current_sources(tmp_path, monkeypatch):
    key = bench.solver_source_key()
    assert len(key) == 16 and int(key, 16) >= 0
    rec = {"kernel": "k_dfsph_solve(density)", "workload": "double_dam_break_dfsph_1m", "source_key": key,
           "dram_bytes_per_pass": 2.0e8}
    stale = dict(rec, source_key="0" * 16, dram_bytes_per_pass=9.9e9)
    path = tmp_path / "traffic.json"
    path.write_text(json.dumps({"records": [stale, rec]}))
    monkeypatch.setattr(bench, "TRAFFIC_RECORDS", str(path))
    assert bench.traffic_record("k_dfsph_solve(density)", "double_dam_break_dfsph_1m") == rec
    assert bench.traffic_record("k_dfsph_solve(density)", "dam_break_dfsph_125k") is None
    path.write_text(json.dumps({"records": [stale]}))
    assert bench.traffic_record("k_dfsph_solve(density)", "double_dam_break_dfsph_1m") is None
    monkeypatch.setattr(bench, "TRAFFIC_RECORDS", str(tmp_path / "missing.json"))
    assert bench.traffic_record("k_dfsph_solve(density)", "double_dam_break_dfsph_1m") is None


def test_committed_traffic_record_is_well_formed():
    """Every committed record names its kernel, workload, source key, bytes
    per pass and the capture command."""
    if not os.path.exists(bench.TRAFFIC_RECORDS):
        pytest.skip("no traffic record committed")
    with open(bench.TRAFFIC_RECORDS) as f:
        recs = json.load(f)["records"]
    assert recs
    for r in recs:
        assert {"kernel", "workload", "source_key", "dram_bytes_per_pass", "command"} <= set(r)
        assert r["dram_bytes_per_pass"] > 0 and len(r["source_key"]) == 16


def test_reference_window_follows_the_gpu_window_when_short():
    assert bench.reference_window(20, 5) == (20, 5)       # the driver's window: same steps
    assert bench.reference_window(35, 5) == (35, 5)
    assert bench.reference_window(300, 5) == (20, 5)      # long windows: a bounded sample
    assert bench.reference_window(100, 200) == (20, 5)


def test_physical_cores_and_baseline_entry():
    n = bench.physical_cores()
    assert 1 <= n <= (os.cpu_count() or 1)
    res = {"particle_steps_per_s": 1.5e6, "threads": 8, "steps": 20, "warmup": 5, "mean_iterations": 2.0,
           "mean_iterations_v": 1.0}
    e = bench.cpu_baseline_entry(res, None, "the same scene")
    assert e["value"] == 1.5e6 and e["cores"] == 8 and e["kind"] == "reference"
    assert "20 timed steps after 5 warm-up steps" in e["sample"]
    e = bench.cpu_baseline_entry(None, "reference build missing", "x")
    assert e["value"] is None and e["sample"] == "reference build missing"


def test_roofline_byte_counts():
    # density solver launch: predict 36 + warm start 76 + its x 84 + positions 36 per fluid particle,
    # plus 16 B per boundary particle with a fluid neighbour per neighbour pass (2 + 2 its)
    assert bench.bytes_per_launch("density_solve", 1000, 10, 2) == 1000 * (36 + 76 + 2 * 84 + 36) + 16 * 10 * 6
    assert bench.bytes_per_launch("divergence_solve", 1000, 10, 1) == 1000 * (76 + 84) + 16 * 10 * 4
    ns = bench.neighbor_search_roofline(1000, 30000, {"sort": {"ms": 0.5}, "lists": {"ms": 1.5}}, 10, 6500.0,
                                        "measured")
    assert ns["algorithmic_bytes_per_step"] == 1000 * 72 + 4 * 30000
    assert abs(ns["achieved"] - (1000 * 72 + 4 * 30000) / 0.2e-3 / 1e9) < 1e-9
    assert abs(ns["frac"] - ns["achieved"] / 6500.0) < 1e-12


def test_reference_arm_prints_one_line(tmp_path):
    """`bench.py --impl reference` runs the reference's OpenMP build on the
    host (no GPU needed) and prints the contract's JSON line."""
    import subprocess

    if not os.path.exists(bench.REF_BIN):
        pytest.skip("reference build missing (make -C oracle)")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload",
                        "dam_break_wcsph_8k", "--steps", "3", "--warmup", "1"], capture_output=True, text=True,
                       timeout=600, cwd=str(tmp_path))
    assert r.returncode == 0, r.stderr[-500:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "particle-steps/s" and d["value"] > 0
    assert d["steps"] == 3 and d["warmup"] == 1 and d["higher_is_better"] is True
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["h2d_bytes_per_step"] == 0
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] >= 1
    assert d["config"]["fluid_particles"] == 8000


def test_pair_evaluation_count():
    """Neighbour passes of a DFSPH step: density + alpha + divergence error,
    forces, the density solver's warm start (2) and 2 per iteration, the
    divergence solver's warm-start correction and 2 per iteration (its
    warm-start residual comes from the density pass); normals with surface
    tension."""
    import bench
    prof = {"density_solve": {"ms": 10.0}}
    r = bench.pair_evaluations(1000, 2.0, 1.0, prof, 20, 30.0)
    assert r["passes_per_step"] == 2 + 6 + 3
    assert r["per_step"] == 11000
    assert abs(r["per_s"] - 11000 * 20 / 0.030) < 1e-6
    assert abs(r["density_solver_per_s"] - 1000 * 6 * 20 / 0.010) < 1e-6
    assert bench.pair_evaluations(1000, 2.0, 1.0, prof, 20, 30.0, surface_tension=True)["passes_per_step"] == 12
