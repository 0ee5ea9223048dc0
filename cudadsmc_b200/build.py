"""In-tree build of the sm_100a library (libdsmc_b200.so) and dsmc_bench."""
import os
import subprocess

_HERE = os.path.dirname(os.path.abspath(__file__))


def build(verbose=False):
    out = subprocess.run(["make", "-C", os.path.join(_HERE, "csrc"), "-j8"],
                         capture_output=not verbose, text=True)
    if out.returncode != 0:
        raise RuntimeError("building libdsmc_b200.so failed:\n" + (out.stdout or "") + (out.stderr or ""))
    return os.path.join(_HERE, "libdsmc_b200.so")
