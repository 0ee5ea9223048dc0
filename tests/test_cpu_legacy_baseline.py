"""The reference's legacy 2-D CPU solver as a timed baseline (CPU only).

oracle/_ref/dsmc_cpu_legacy links the reference's src/dsmc_cpu.cpp,
src/mtwister.cpp and src/genmtrand.c unchanged; bench.py reports its
particle-timesteps/s as "reference dsmc_cpu (2-D legacy)".  These tests check
the driver's contract: a fixed problem size, a fixed step count, a
deterministic result for a seed, and a clear error for a parameter file that
is too short.
"""
import json
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "oracle", "_ref", "dsmc_cpu_legacy")
DAT = os.path.join(ROOT, "oracle", "_ref", "MersenneTwister.dat")

needs_driver = pytest.mark.skipif(not (os.path.isfile(EXE) and os.path.isfile(DAT)),
                                  reason="oracle/_ref/dsmc_cpu_legacy not built (make -C oracle ref)")


def _run(*args, dat=DAT):
    return subprocess.run([EXE, dat, *map(str, args)], capture_output=True, text=True, timeout=120)


@needs_driver
def test_legacy_driver_runs_fixed_steps_deterministically():
    outs = []
    for _ in range(2):
        r = _run(10, 60, 20, 999)
        assert r.returncode == 0, r.stderr
        outs.append(json.loads(r.stdout.strip().splitlines()[-1]))
    a, b = outs
    # the compile-time 30 x 18 grid of the reference (include/dsmc.h:45-46)
    assert a["cells"] == 540 and a["particles"] == 5400
    assert a["steps"] == 20 and a["value"] > 0
    assert a["checksum"] == b["checksum"]
    # another seed gives another state
    c = json.loads(_run(10, 60, 20, 1000).stdout.strip().splitlines()[-1])
    assert c["checksum"] != a["checksum"]


@needs_driver
def test_legacy_driver_rejects_short_parameter_file(tmp_path):
    short = tmp_path / "short.dat"
    short.write_bytes(open(DAT, "rb").read(1000))
    r = _run(10, 1, 1, 999, dat=str(short))
    assert r.returncode == 1
    assert "cannot convert" in r.stderr


def test_bench_reports_legacy_baseline_or_nothing():
    import sys
    sys.path.insert(0, ROOT)
    import bench
    res = bench.legacy_cpu_sample(budget_s=0.5, particles_per_cell=10)
    if not (os.path.isfile(EXE) and os.path.isfile(DAT)):
        assert res is None
        return
    assert res["label"] == "reference dsmc_cpu (2-D legacy)"
    assert res["cores"] == 1 and res["value"] > 0
    assert "5400 particles" in res["sample"]
