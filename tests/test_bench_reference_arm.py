"""bench.py on the CPU: the reference arm (the CPU implementation of the path
-- the oracle, the reference being an unbuildable Fortran program -- timed on
the host, printed as one JSON line with the contract's keys and the same
workload as the GPU arm), and the multi-rank launch (`--gpus N` starts N
ranks itself; a dry run sets up a gloo process group and prints the line's
layout without touching a GPU)."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_contract_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "3", "--n", "96"], capture_output=True, text=True, cwd=ROOT, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.strip().startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == "zone-updates/s" and d["unit"] == "zone-updates/s"
    assert d["value"] > 0 and d["higher_is_better"] is True and d["n_gpus"] == 1
    assert d["steps"] == 1 and d["warmup"] >= 3 and "workload" in d["config"]
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    # the GPU arm's workload name, so the two lines describe the same config
    assert d["config"]["workload"] == "blast3d_96^3_weno_hlld_ct_rk3_cfl0.4"
    assert "96x96x64" in cb["sample"]


def test_reference_arm_sample_shrinks_with_the_step_count():
    """Every step is timed, each on a thinner slab, so long runs stay short."""
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "200",
                        "--warmup", "3", "--n", "24"], capture_output=True, text=True, cwd=ROOT, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    d = json.loads([ln for ln in r.stdout.splitlines() if ln.strip().startswith("{")][0])
    assert d["steps"] == 200 and "24x24x32" in d["cpu_baseline"]["sample"]


def test_gpus_n_spawns_n_ranks_dry_run():
    env = dict(os.environ)
    env.pop("WORLD_SIZE", None)
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--dry-run"],
                       capture_output=True, text=True, cwd=ROOT, timeout=300, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.strip().startswith("{")]
    assert len(lines) == 1  # rank 0 alone prints
    d = json.loads(lines[0])
    assert d["n_gpus"] == 2 and d["ranks"] == {"world_size": 2, "backend": "gloo"}
    assert d["scaling"] == "strong" and d["config"]["parallelism"].startswith("z-slabs x 2")
    # replicas stay available behind a flag
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--dry-run", "--replicas"],
                       capture_output=True, text=True, cwd=ROOT, timeout=300, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    d = json.loads([ln for ln in r.stdout.splitlines() if ln.strip().startswith("{")][0])
    assert d["n_gpus"] == 2 and d["scaling"] == "weak" and d["config"]["parallelism"] == "replicas"
