"""Build step for libzkb200.so (nvcc, sm_100a) — used by __graft_entry__.build()."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def build(jobs: int = 8) -> str:
    subprocess.check_call(["make", "-s", "-j", str(jobs), "-C", HERE])
    return os.path.join(HERE, "libzkb200.so")


if __name__ == "__main__":
    print(build())
