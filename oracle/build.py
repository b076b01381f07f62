"""Build recipe for the oracle (test infrastructure only): compiles
oracle/oracle.c with gcc into oracle/_build/liboracle.so.

The reference (QuasiStrided.jl) is Julia, so there is no reference source
that gcc could compile into an oracle/_ref library; the oracle is this C
restatement alone.
"""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_build")
LIB = os.path.join(OUT, "liboracle.so")


def build() -> str:
    os.makedirs(OUT, exist_ok=True)
    src = os.path.join(HERE, "oracle.c")
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(src):
        return LIB
    cmd = ["gcc", "-O3", "-mavx2", "-mfma", "-fopenmp", "-fPIC", "-shared", "-std=gnu11",
           "-o", LIB, src, "-lquadmath", "-lm"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{res.stdout}\n{res.stderr}")
    return LIB


if __name__ == "__main__":
    print(build())
