"""Build libawfl.so (the C-ABI library of include/awfl.h) for sm_100a with nvcc.

Translation units and their numerics flags:
  awfl_capi.cu  host code: -ffp-contract=off (init-time tables/background bit-identical
                to the reference CPU build)
  awfl_fp64.cu  FP64 kernels: --fmad=false (no contracted multiply-add, like the
                reference CPU build)
  awfl_fp32.cu  FP32 precision form: contraction, approximate division/sqrt, flush-to-zero
  awfl_noalloc.cu  allocation-free CFL variant: --fmad=false (same arithmetic as awfl_cfl)
  awfl_adjoint.cu  tangent-linear sweep: --fmad=false (its value part replays the FP64 path)
  awfl_adjrev.cu   adjoint reverse sweeps: --fmad=true (a derivative, not a replay)
  awfl_ens32.cu    ensemble persistent sweeps, FP32 form: the awfl_fp32.cu flags
  awfl_ens64.cu    ensemble persistent sweeps, FP64 path: --fmad=false
  awfl_ensemble.cu ensemble host side: work lists, CUDA graph, autotuner (host code only)
  awfl_netcdf.cu   netCDF output file writer (host code only)
  awfl_tracers.cu  tracer transport of the FP64 path: --fmad=false
  awfl_tracers32.cu  tracer transport of the FP32 form: the FP32 form's flags

The library lands in-tree at awflcloud_b200/lib/libawfl.so so that it travels with the
source tree. ``python -m awflcloud_b200.build [--force]``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
ROOT = os.path.dirname(HERE)
LIBDIR = os.path.join(HERE, "lib")
OBJDIR = os.path.join(HERE, "_build")
LIB = os.path.join(LIBDIR, "libawfl.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off",
          "-I" + SRC, "-I" + os.path.join(ROOT, "include")]
UNITS = {
    "awfl_capi.cu": ["--fmad=false"],
    "awfl_fp64.cu": ["--fmad=false"],
    "awfl_fp32.cu": ["--fmad=true", "-prec-div=false", "-prec-sqrt=false", "-ftz=true"],
    "awfl_noalloc.cu": ["--fmad=false"],
    "awfl_adjoint.cu": ["--fmad=false"],
    "awfl_adjrev.cu": ["--fmad=true"],
    "awfl_ens32.cu": ["--fmad=true", "-prec-div=false", "-prec-sqrt=false", "-ftz=true"],
    "awfl_ens64.cu": ["--fmad=false"],
    "awfl_ensemble.cu": [],
    "awfl_netcdf.cu": [],
    "awfl_tracers.cu": ["--fmad=false"],
    "awfl_tracers32.cu": ["--fmad=true", "-prec-div=false", "-prec-sqrt=false", "-ftz=true"],
}


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _deps(unit: str):
    hdrs = [os.path.join(SRC, f) for f in os.listdir(SRC) if f.endswith((".h", ".cuh"))]
    hdrs.append(os.path.join(ROOT, "include", "awfl.h"))
    return [os.path.join(SRC, unit)] + hdrs


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(OBJDIR, exist_ok=True)
    objs, cmds = [], []
    for unit, flags in UNITS.items():
        src = os.path.join(SRC, unit)
        if not os.path.exists(src):
            continue
        obj = os.path.join(OBJDIR, unit.replace(".cu", ".o"))
        objs.append(obj)
        if force or _stale(obj, _deps(unit)):
            cmd = [nvcc()] + ARCH + COMMON + flags + ["-c", src, "-o", obj]
            if ptxas_info:
                cmd += ["-Xptxas", "-v"]
            cmds.append(cmd)
    # the translation units are independent: compile them concurrently
    from concurrent.futures import ThreadPoolExecutor
    jobs = max(1, min(len(cmds), os.cpu_count() or 1))

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        return subprocess.run(cmd, capture_output=True, text=True)

    with ThreadPoolExecutor(max_workers=jobs) as ex:
        results = list(ex.map(run, cmds))
    for cmd, r in zip(cmds, results):
        if r.stdout or r.stderr:
            sys.stdout.write(r.stdout + r.stderr)
        if r.returncode != 0:
            raise subprocess.CalledProcessError(r.returncode, cmd)
    rebuilt = bool(cmds)
    if rebuilt or force or _stale(LIB, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_info="-v" in sys.argv)
