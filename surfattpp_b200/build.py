"""Build recipe for libsurfatt_gpu.so (sm_100a), in-tree.

Each translation unit gets the flags its arithmetic contract needs:
  eik64.cu   -fmad=false: FP64 parity path, every operation rounds as written
  noalloc.cu -fmad=false: its geometry and metric planes round as the plan's
  eik32.cu   fast FP32 division/sqrt, FTZ: the FP32 sweep path
  surfker*.cu -fmad=false: surfdisp96 / sregn96 operation for operation
  postproc.cu -fmad=false: PDE smoothing rounds as the reference's FP64
  multigrid.cu -fmad=false: multigrid smoothing, likewise
  others     default IEEE flags
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
LIB = os.path.join(HERE, "libsurfatt_gpu.so")
BUILD = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I", CSRC, "-I", INCLUDE]
UNITS = {
    "eik64.cu": ["-fmad=false"],
    "eik32.cu": ["-prec-div=false", "-prec-sqrt=false", "-ftz=true"],
    "surfker.cu": ["-fmad=false"],
    "surfker_group.cu": ["-fmad=false"],
    "util.cu": [],
    "capi.cu": ["-Xcompiler", "-ffp-contract=off"],
    "noalloc.cu": ["-fmad=false"],
    "postproc.cu": ["-fmad=false"],
    "multigrid.cu": ["-fmad=false", "-Xcompiler", "-ffp-contract=off"],
    "optimize.cu": ["-fmad=false"],
    "topo.cu": ["-fmad=false"],
    "srcrec.cpp": ["-Xcompiler", "-ffp-contract=off"],
}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(out: str, deps: list[str]) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False, defines: list[str] | None = None,
          out: str | None = None, build_dir: str | None = None) -> str:
    """Compile every unit and link the library.  ``defines`` (``NAME=VALUE``
    strings), ``out`` and ``build_dir`` build a variant next to the default."""
    lib = out or LIB
    bdir = build_dir or BUILD
    dflags = [f"-D{d}" for d in (defines or [])]
    os.makedirs(bdir, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(INCLUDE, "surfatt_gpu.h"))
    objs = []
    for unit, flags in UNITS.items():
        src = os.path.join(CSRC, unit)
        if not os.path.exists(src):
            continue
        obj = os.path.join(bdir, unit.rsplit(".", 1)[0] + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            cmd = [nvcc()] + ARCH + COMMON + dflags + flags + ["-c", src, "-o", obj]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
                print(" ".join(cmd), file=sys.stderr)
            subprocess.run(cmd, check=True)
    if force or _stale(lib, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", lib] + objs + ["-lcudart"]
        subprocess.run(cmd, check=True)
    return lib


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(LIB)
