"""Build step for libexcfv: nvcc for sm_100a, in-tree (exciting_b200/libexcfv.so)."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")


def build_library(jobs: int = 8, verbose: bool = False) -> str:
    """Compile every CUDA source for sm_100a and link libexcfv.so (make -C csrc)."""
    cmd = ["make", "-C", CSRC, f"-j{jobs}"]
    res = subprocess.run(cmd, capture_output=not verbose, text=True)
    if res.returncode != 0:
        out = (res.stdout or "") + (res.stderr or "")
        raise RuntimeError(f"libexcfv build failed:\n{out[-4000:]}")
    path = os.path.join(HERE, "libexcfv.so")
    if not os.path.exists(path):
        raise RuntimeError("libexcfv build produced no library")
    return path


if __name__ == "__main__":
    print(build_library(verbose="-v" in sys.argv))
