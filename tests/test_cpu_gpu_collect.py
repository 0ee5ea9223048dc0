"""The GPU tests collect on a machine without a GPU, and every argument of
every GPU test resolves to a fixture or a parameter, so a broken test fails
here and not at setup on the GPU box."""
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_gpu_tests_collect_with_resolved_arguments():
    env = dict(os.environ, DSMC_CHECK_FIXTURES="1")
    r = subprocess.run([sys.executable, "-m", "pytest", "tests", "-m", "gpu", "--collect-only", "-q",
                        "-p", "no:cacheprovider"], cwd=ROOT, env=env, capture_output=True, text=True,
                       timeout=300)
    out = r.stdout + r.stderr
    assert r.returncode == 0, out[-4000:]
    n = sum(1 for line in r.stdout.splitlines() if "::" in line)
    assert n >= 60, out[-2000:]
