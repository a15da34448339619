"""Build libseisfem_b200.so in-tree for sm_100a (nvcc, no JIT cache).

``python -m seisfem_b200.build`` (or ``build()``) compiles every CUDA source
with ``-gencode arch=compute_100a,code=sm_100a``.  The assembly unit is
compiled with ``-fmad=false`` so that FP64 element matrices keep the
reference's exact operation order; the step kernels use contraction freely
(the FP64 step kernel spells its arithmetic with round-to-nearest
intrinsics instead).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libseisfem_b200.so")
BUILD = os.path.join(HERE, "_build")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2"]
UNITS = {
    "sfg_assemble.cu": ["-fmad=false"],
    "sfg_step.cu": [],
    "sfg_step32.cu": [],
    "sfg_api.cu": [],
    "sfg_seams.cu": ["-fmad=false"],
    "sfg_noalloc.cu": ["-fmad=false"],
    "sfg_fno.cu": [],
    "sfg_dict.cu": [],
    "sfg_locate.cu": ["-fmad=false"],
    "sfg_acoustic.cu": ["-fmad=false"],
}
C_UNITS = ["elastic_wave_dropin.c", "acoustic_dropin.c"]


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _cc() -> str:
    return "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else (shutil.which("gcc") or "cc")


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ...")
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr)
    return r


def _stale(obj, srcs):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(s) > t for s in srcs)


def build(verbose: bool = False, ptxas_info: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers += [os.path.join(HERE, "..", "include", f) for f in ("seisfem_b200.h", "seisfem_fno.h", "seisfem_acoustic.h")]
    objs = []
    for unit, extra in UNITS.items():
        src = os.path.join(CSRC, unit)
        obj = os.path.join(BUILD, unit.replace(".cu", ".o"))
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            cmd = [nvcc, *ARCH, *NVFLAGS, *extra, "-c", src, "-o", obj]
            if ptxas_info:
                cmd += ["-Xptxas", "-v"]
            _run(cmd, verbose or ptxas_info)
    for unit in C_UNITS:
        csrc = os.path.join(CSRC, unit)
        cobj = os.path.join(BUILD, unit.replace(".c", ".o"))
        objs.append(cobj)
        if force or _stale(cobj, [csrc] + headers):
            _run([_cc(), "-O2", "-fPIC", "-std=gnu11", "-Wall", "-c", csrc, "-o", cobj], verbose)
    if force or _stale(OUT, objs):
        _run([nvcc, *ARCH, "-shared", "-o", OUT, *objs, "-cudart", "static"], verbose)
    return OUT


if __name__ == "__main__":
    build(verbose=True, ptxas_info="--ptxas" in sys.argv, force="--force" in sys.argv)
