"""In-tree build of the engine for B200 (sm_100a).

``build()`` runs ``make`` in csrc/, producing ``libbw_b200.so`` next to this
file and the drop-in executables under ``bin/``.  nvcc cross-compiles for
sm_100a without a GPU.
"""
import os
import subprocess
from pathlib import Path

PKG = Path(__file__).resolve().parent


def build(jobs=None, verbose=False):
    jobs = jobs or max(1, os.cpu_count() or 1)
    cmd = ["make", "-C", str(PKG / "csrc"), f"-j{jobs}"]
    if not verbose:
        cmd.insert(1, "-s")
    subprocess.run(cmd, check=True)
    return PKG / "libbw_b200.so"


if __name__ == "__main__":
    print(build(verbose=True))
