"""Builds the CPU oracle (test infrastructure only) as oracle/libbeams_oracle.so.

g++ -O2 -fopenmp -ffp-contract=off: float expressions keep the reference's
roundings (no FMA contraction), OpenMP parallelises over rays.
"""
from __future__ import annotations

import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "beams_oracle.cpp"
HDR = HERE / "beams_oracle.h"
LIB = HERE / "libbeams_oracle.so"


def build(verbose: bool = False, force: bool = False) -> Path:
    if not force and LIB.exists() and LIB.stat().st_mtime >= max(SRC.stat().st_mtime, HDR.stat().st_mtime,
                                                                    Path(__file__).stat().st_mtime):
        return LIB
    cmd = ["g++", "-O2", "-std=c++17", "-fopenmp", "-ffp-contract=off", "-fPIC", "-shared",
           str(SRC), "-o", str(LIB)]
    if verbose:
        print(" ".join(cmd))
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        sys.stderr.write(p.stdout + p.stderr)
        raise RuntimeError("oracle build failed")
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, force="-f" in sys.argv))
