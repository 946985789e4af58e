"""Build the oracle (test infrastructure only): ``oracle/liboracle.so``.

The oracle is the CPU restatement of the reference's step in ``zoracle.cpp``.
It is compiled with ``-ffp-contract=off`` (no fused multiply-add, as in the
reference's x86-64 build without ``-march``) so that its floating point
matches the reference operation for operation.
"""
from __future__ import annotations

import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "liboracle.so"
SRC = HERE / "zoracle.cpp"
INCS = [HERE / "zoracle_mm.inc", HERE / "zoracle_tr.inc"]  # multi-material step, transport; included


def build(force: bool = False, verbose: bool = False) -> Path:
    if force or not OUT.exists() or OUT.stat().st_mtime < max(p.stat().st_mtime for p in [SRC, *INCS]):
        cxx = shutil.which("g++") or "g++"
        cmd = [cxx, "-O2", "-std=c++17", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared",
               "-pthread", "-o", str(OUT), str(SRC)]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(OUT)
