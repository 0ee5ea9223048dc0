"""The C++ layer (include/dsmc_solver.hpp) through the dsmc_bench driver, the
reference's main with its flags: errors surface as std::runtime_error, as
checkCUDAErrorAndThrow does in the reference, and the driver exits 1 with the
message instead of crashing."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "cudadsmc_b200", "dsmc_bench")

pytestmark = pytest.mark.skipif(not os.path.isfile(EXE), reason="dsmc_bench not built")


def _run(args, cwd):
    return subprocess.run([EXE, *args], capture_output=True, text=True, cwd=cwd, timeout=120)


def _config(tmp_path):
    (tmp_path / "gases.xml").write_text(
        "<gases>\n<gas name=\"argon\"><mass>6.63e-26</mass><diam>4.17e-10</diam><temp>273</temp>"
        "</gas>\n</gases>\n")
    (tmp_path / "cfg.xml").write_text(
        "<config><grid><min>0 0 0</min><max>0.2 0.2 0.2</max><dim>8 8 8</dim></grid>"
        "<density>1e20</density><fnum>1.5e13</fnum><temp>300</temp><streamvel>0 0 0</streamvel>"
        "<periodic>n</periodic><gas file=\"gases.xml\">argon</gas></config>\n")
    return "cfg.xml"


def test_mt_flag_is_taken_by_the_driver(tmp_path):
    """-mt reaches the driver (the settings parser alone rejects it); without
    a GPU the run stops at Init, before the twister file is read."""
    import torch
    cfg = _config(tmp_path)
    r = _run(["-f", cfg, "-mt", "-mt-file", "missing.dat", "-steps", "1"], tmp_path)
    assert r.returncode == 1
    assert "readFromCmdLine" not in r.stderr
    if torch.cuda.is_available():
        assert "UseTwisters (twister file)" in r.stderr
    else:
        assert "Exception: Init: CUDA error" in r.stderr


def test_missing_config_is_an_io_error(tmp_path):
    r = _run(["-f", str(tmp_path / "missing.xml")], tmp_path)
    assert r.returncode == 1
    assert "cannot read" in r.stderr


def test_run_without_a_gpu_fails_cleanly_or_runs_with_one(tmp_path):
    import torch
    cfg = _config(tmp_path)
    r = _run(["-f", cfg, "-benchmark", "-steps", "2", "-stats", "stats.txt"], tmp_path)
    if torch.cuda.is_available():
        assert r.returncode == 0, r.stderr
        assert "Benchmark is done" in r.stdout and (tmp_path / "stats.txt").exists()
    else:
        assert r.returncode == 1
        assert "Exception: Init: CUDA error" in r.stderr
