"""CPU checks of bench.py's reference arm (the oracle timed on the host):
the JSON line keeps the bench contract, and under several ranks only rank 0
works and prints."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(env_extra):
    env = dict(os.environ)
    env.update(env_extra)
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0",
                        "--n", "32"], cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return [ln for ln in r.stdout.splitlines() if ln.startswith("{")]


def test_reference_arm_line():
    lines = _run({})
    assert len(lines) == 1
    line = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["impl"] == "reference" and line["higher_is_better"] is False and line["n_gpus"] == 1
    assert line["value"] > 0 and line["e2e"]["value"] == line["value"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    cb = line["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["value"] == line["value"] and cb["sample"]
    assert line["solve"]["pcg_iterations"] > 0
    # the same configuration dict as the GPU arm's headline (the metric's plain Poisson case)
    sys.path.insert(0, ROOT)
    import bench

    class A:
        n = 32

    assert line["config"] == bench.poisson_config(A)
    assert "Poisson" in line["config"]["workload"] and line["config"]["rel_tol"] == 1e-7


def test_reference_arm_ranks():
    """Under torchrun only rank 0 times and prints; the others exit 0."""
    assert _run({"RANK": "1", "LOCAL_RANK": "1", "WORLD_SIZE": "2"}) == []
    lines = _run({"RANK": "0", "LOCAL_RANK": "0", "WORLD_SIZE": "2"})
    assert len(lines) == 1 and json.loads(lines[0])["n_gpus"] == 2
