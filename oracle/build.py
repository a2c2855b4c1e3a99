"""Build recipe of the CPU oracle (test infrastructure only).

Compiles ``hs_oracle.cpp`` with g++ into ``oracle/_build/libhsoracle.so``.
The reference itself (MolSpin, C++17 + Armadillo 12.8.4) cannot be compiled
in this environment -- Armadillo's headers and libraries are absent and every
file on the HSGeneral path includes <armadillo> -- so there is no
``oracle/_ref`` build; the oracle is pinned by the reference's known-answer
tests instead (tests/test_oracle_pins.py).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_build")
LIB = os.path.join(OUT, "libhsoracle.so")
SRC = os.path.join(HERE, "hs_oracle.cpp")


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OUT, exist_ok=True)
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-pthread", SRC, "-o", LIB]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
