"""Build libfmcuda.so in-tree (nvcc, sm_100a) with the Makefile in ../csrc."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "csrc")


def build(jobs: int = 3, verbose: bool = False) -> str:
    cmd = ["make", "-C", CSRC, f"-j{jobs}"]
    res = subprocess.run(cmd, capture_output=not verbose, text=True)
    if res.returncode != 0:
        sys.stderr.write((res.stdout or "") + (res.stderr or ""))
        raise RuntimeError("libfmcuda build failed")
    return os.path.join(HERE, "libfmcuda.so")


if __name__ == "__main__":
    print(build(verbose=True))
