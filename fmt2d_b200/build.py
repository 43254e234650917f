"""Build the native library for sm_100a (nvcc cross-compiles without a GPU)."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def build(jobs: int = 8) -> str:
    subprocess.run(["make", "-s", "-j", str(jobs), "-C", os.path.join(HERE, "csrc")], check=True)
    return os.path.join(HERE, "_lib", "libfmt2d_b200.so")


if __name__ == "__main__":
    print(build())
