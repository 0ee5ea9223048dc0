"""bench.py's reference arm on the CPU: the JSON line it prints for rank 0,
and no work and no output on the other ranks of a multi-rank launch."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(env_extra):
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                           "--steps", "1", "--warmup", "3"], capture_output=True, text=True,
                          env=env, cwd=ROOT, timeout=600)


def test_reference_arm_prints_one_contract_line():
    r = _run({"WORLD_SIZE": "1", "RANK": "0"})
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    out = json.loads(lines[0])
    assert out["impl"] == "reference"
    assert out["metric"] == "particle-timesteps/s" and out["higher_is_better"] is True
    assert out["value"] > 0 and out["n_gpus"] == 1
    assert out["config"]["workload"].startswith("capsule")
    cb = out["cpu_baseline"]
    assert cb["kind"] == "port" and cb["value"] == out["value"] and cb["cores"] >= 1
    assert out["e2e"] == {"value": out["value"], "unit": out["unit"], "h2d_bytes_per_step": 0,
                          "d2h_bytes_per_step": 0}
    legacy = out.get("legacy_dsmc_cpu")
    if legacy is not None and "value" in legacy:
        assert legacy["label"] == "reference dsmc_cpu (2-D legacy)" and legacy["cores"] == 1


def test_reference_arm_other_ranks_do_no_work():
    r = _run({"WORLD_SIZE": "2", "RANK": "1"})
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""
