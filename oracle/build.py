"""Build recipe for the CPU oracle (test infrastructure only).

Compiles ``oracle/keq_oracle.c`` into ``oracle/liboracle.so`` with gcc.
No -ffast-math and -ffp-contract=off, so the restated sequential kernels keep
the reference CPU extensions' rounding (plain -O3 x86-64, no FMA).
"""
from __future__ import annotations

import os
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "keq_oracle.c"
LIB = HERE / "liboracle.so"


def build(force: bool = False) -> Path:
    if LIB.exists() and not force and LIB.stat().st_mtime >= SRC.stat().st_mtime:
        return LIB
    cmd = [
        os.environ.get("KEQ_ORACLE_CC", "gcc"), "-O2", "-ffp-contract=off", "-fno-fast-math", "-fopenmp",
        "-fPIC", "-shared", "-Wall", str(SRC), "-o", str(LIB), "-lm",
    ]
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force=True))
