"""Build recipe: compiles libgpuga_b200.so and the gpuga CLI for sm_100a in-tree.

    python -m gpuga_b200.build
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def build(jobs: int | None = None) -> str:
    jobs = jobs or max(1, min(8, os.cpu_count() or 1))
    subprocess.run(["make", "-s", "-C", HERE, f"-j{jobs}"], check=True)
    return os.path.join(HERE, "_build", "libgpuga_b200.so")


if __name__ == "__main__":
    print(build(int(sys.argv[1]) if len(sys.argv) > 1 else None))
