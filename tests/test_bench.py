"""bench.py's reference arm (the reference's own CPU renderer on the host cores) keeps the JSON-line
contract, and under several ranks only rank 0 works and prints -- all on the CPU."""
import json
import os
import subprocess
import sys

from conftest import ROOT

BENCH = os.path.join(ROOT, "bench.py")


def run_reference_arm(rank, world):
    env = dict(os.environ, RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    return subprocess.run([sys.executable, BENCH, "--impl", "reference", "--steps", "1", "--warmup", "3"],
                          capture_output=True, text=True, env=env, timeout=600)


def test_reference_arm_prints_one_contract_line():
    r = run_reference_arm(0, 1)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.strip()]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == "Gaussians/s fwd" and d["unit"] == "Gaussians/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 1 and d["warmup"] == 3 and d["n_gpus"] == 1
    assert d["scaling"] == "weak" and d["vs_baseline"] is None and d["dtype"] == "fp32"
    assert "740k" in d["config"]["workload"] and d["config"]["gaussians"] == 740000
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["unit"] == d["unit"] and cb["cores"] >= 1
    assert cb["kind"] in ("reference", "port") and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert "reference_gpu" in d  # timed on a GPU box, else the reason it is not
    # the arm runs the reference alone: the library under test is never mapped in its process
    assert d["repo_libraries_loaded"] is not None
    assert not [p for p in d["repo_libraries_loaded"] if p.startswith("aniso_b200")], d["repo_libraries_loaded"]


def test_reference_arm_other_ranks_exit_without_work():
    r = run_reference_arm(1, 2)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""
