"""Builds libbeams_b200.so (CUDA, sm_100a) in-tree.

Every .cu in csrc/ is compiled to its own object and linked into
pilot_b200/lib/libbeams_b200.so. Flags:
  -gencode arch=compute_100a,code=sm_100a   B200 only, no PTX fallback
  -fmad=false                               keeps a*b+c as two roundings, as the
                                            reference's float32 arithmetic does;
                                            kernels request fusion with fmaf()
  -Xcompiler -ffp-contract=off              same rule for host-side parameter setup
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "lib" / "libbeams_b200.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CFLAGS = ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "--expt-relaxed-constexpr",
          "-Xcompiler", "-fPIC,-ffp-contract=off,-O2", "-I", str(PKG.parent / "include")]


def _newer(out: Path, deps) -> bool:
    if not out.exists():
        return False
    t = out.stat().st_mtime
    return all(Path(d).stat().st_mtime <= t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(str(c) for c in cmd), flush=True)
    p = subprocess.run([str(c) for c in cmd], capture_output=True, text=True)
    if p.returncode != 0:
        sys.stderr.write(p.stdout + p.stderr)
        raise RuntimeError(f"command failed ({p.returncode}): {cmd[0]} ... {cmd[-1]}")
    if verbose and (p.stdout or p.stderr):
        sys.stderr.write(p.stdout + p.stderr)
    return p


def build(verbose: bool = False, force: bool = False, extra_flags=None) -> Path:
    BUILD.mkdir(exist_ok=True)
    LIB.parent.mkdir(exist_ok=True)
    headers = sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + sorted((PKG.parent / "include").glob("*.h"))
    sources = sorted(CSRC.glob("*.cu"))
    flags = CFLAGS + list(extra_flags or [])

    def compile_one(src: Path) -> Path:
        obj = BUILD / (src.stem + ".o")
        if force or not _newer(obj, [src, *headers, Path(__file__)]):
            _run([NVCC, *ARCH, *flags, "-c", src, "-o", obj], verbose)
        return obj

    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(compile_one, sources))
    if force or not _newer(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-o", LIB, *objs], verbose)
    # the driver executable (host C++ over the C ABI)
    drv = PKG / "driver" / "beams_run.cpp"
    exe = PKG / "bin" / "beams_run"
    if drv.exists() and (force or not _newer(exe, [drv, LIB, *headers])):
        exe.parent.mkdir(exist_ok=True)
        _run([os.environ.get("CXX", "g++"), "-O2", "-std=c++17", "-I", PKG.parent / "include", drv, "-o", exe,
              "-L", LIB.parent, "-lbeams_b200", "-Wl,-rpath,$ORIGIN/../lib"], verbose)
    return LIB


def ptxas_report(src_name: str) -> str:
    """Registers / spills / shared memory of one kernel file (-Xptxas -v)."""
    src = CSRC / src_name
    p = subprocess.run([NVCC, *ARCH, *CFLAGS, "-Xptxas", "-v", "-c", str(src), "-o", os.devnull],
                       capture_output=True, text=True)
    return p.stdout + p.stderr


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
