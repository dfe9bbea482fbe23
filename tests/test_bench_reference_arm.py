"""`bench.py --impl reference` (the reference's CPU algorithm, timed on the
host cores over the whole workload every step) keeps the benchmark line's
contract and describes the same workload as the GPU arm; it needs no GPU,
so it runs here on a tiny grid. Under torchrun only rank 0 works and prints."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CMD = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--grid", "6,3,4", "--steps", "2",
       "--warmup", "1"]


def _run(env_extra):
    env = dict(os.environ, **env_extra)
    return subprocess.run(CMD, capture_output=True, text=True, timeout=600, cwd=ROOT, env=env)


def test_reference_line_contract():
    import bench

    r = _run({"RANK": "0", "WORLD_SIZE": "1"})
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == bench.METRIC and d["unit"] == bench.UNIT
    assert d["value"] > 0 and d["higher_is_better"] is True and d["steps"] == 2 and d["warmup"] == 1
    assert d["config"]["tets"] == 6 * 3 * 4 * 6 and d["config"]["workload"] == "wr90_dielectric"
    wl = bench.make_workload("wr90_dielectric", grid="6,3,4")
    m = wl.field.mesh
    nnz = 4 * m.n_edges + 52 * m.n_tris + 168 * m.n_tets
    assert d["config"] == json.loads(json.dumps(bench.arm_config(wl, nnz)))  # the GPU arm's config dict
    assert abs(d["ms_per_step"] * 1e-3 * d["value"] - d["config"]["tets"]) <= 1e-6 * d["config"]["tets"]
    assert "whole" in d["cpu_baseline"]["sample"]
    cb = d["cpu_baseline"]
    assert set(cb) >= {"value", "unit", "cores", "kind", "sample"} and cb["kind"] == "port"
    assert cb["value"] == d["value"] and cb["cores"] >= 1
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_other_ranks_exit_without_work():
    r = _run({"RANK": "1", "WORLD_SIZE": "2"})
    assert r.returncode == 0, r.stderr[-2000:]
    assert not [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
