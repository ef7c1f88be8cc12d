"""In-tree build of the engine for B200 (sm_100a).

``build()`` runs ``make`` in csrc/, producing ``libbw_b200.so`` next to this
file and the drop-in executables under ``bin/``.  nvcc cross-compiles for
sm_100a without a GPU.
"""
import os
import subprocess
from pathlib import Path

PKG = Path(__file__).resolve().parent


DATA = PKG / "_data"   # paper instances staged from a reference checkout (not committed)


def stage_paper_instances(src_dir):
    """Copy the reference's shipped paper instances (g20..g30 JSON) next to the
    package, where the paper-mode bench workloads read them."""
    import shutil
    DATA.mkdir(exist_ok=True)
    for f in sorted(Path(src_dir).glob("g[0-9][0-9].json")):
        shutil.copyfile(f, DATA / f.name)
    return DATA


def build(jobs=None, verbose=False):
    jobs = jobs or max(1, os.cpu_count() or 1)
    cmd = ["make", "-C", str(PKG / "csrc"), f"-j{jobs}"]
    if not verbose:
        cmd.insert(1, "-s")
    subprocess.run(cmd, check=True)
    return PKG / "libbw_b200.so"


if __name__ == "__main__":
    print(build(verbose=True))
