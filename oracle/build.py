"""Compile the C oracle (test infrastructure) into oracle/liboracle.so.

    python -m oracle.build [--force]

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs load
this library; the product (solarsystemsimulator_b200) never does.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
FLAGS = ["-O2", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off", "-fno-fast-math",
         "-std=c11"]


def build(force: bool = False) -> str:
    srcs = sorted(glob.glob(os.path.join(HERE, "*.c")))
    if (not force and os.path.exists(LIB)
            and all(os.path.getmtime(s) <= os.path.getmtime(LIB) for s in srcs)):
        return LIB
    cmd = ["gcc", *FLAGS, "-o", LIB + ".tmp", *srcs, "-lm"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("gcc failed building the oracle")
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
