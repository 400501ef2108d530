"""Builds libmdb200.so in-tree (md_simulation_cuda_b200/libmdb200.so) for sm_100a."""
from __future__ import annotations

import os
import subprocess

_HERE = os.path.dirname(os.path.abspath(__file__))


def build(jobs: int = 8) -> str:
    subprocess.run(["make", "-C", os.path.join(_HERE, "csrc"), f"-j{jobs}"], check=True,
                   stdout=subprocess.DEVNULL)
    return os.path.join(_HERE, "libmdb200.so")


if __name__ == "__main__":
    print(build())
