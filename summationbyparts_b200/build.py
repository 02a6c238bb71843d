"""Build the sbp_b200 CUDA library in-tree for sm_100a.

    python -m summationbyparts_b200.build [--force]

Every translation unit in csrc/ is compiled with nvcc for sm_100a (in parallel) and linked,
with a static CUDA runtime, into summationbyparts_b200/_lib/libsbp_b200.so.  Units whose
f64 results must match the reference's rounding are compiled with -fmad=false; the
compensated-f32 stage kernels use fast single-precision division and square root.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libsbp_b200.so")
ROOT = os.path.dirname(HERE)

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
          "-I" + CSRC, "-I" + os.path.join(ROOT, "include"), "--expt-relaxed-constexpr"]
EXACT = ["-fmad=false"]
FAST32 = ["-use_fast_math"]

UNITS = {
    "capi.cu": EXACT,
    "system.cu": EXACT,
    "system_kernels.cu": EXACT,
    "op_apply.cu": EXACT,
    "metrics_noalloc.cu": EXACT,
    "cnn.cu": [],
    "interp.cu": EXACT,
    "stage_f64_u4.cu": EXACT,
    "stage_f64_u9.cu": EXACT,
    "stage_f64_sbp.cu": EXACT,
    "stage_f32_u4.cu": FAST32,
    "stage_f32_u9.cu": FAST32,
    "stage_f32_sbp.cu": FAST32,
    "stage_f64_x49a.cu": EXACT,
    "stage_f64_x49b.cu": EXACT,
    "stage_f64_xsa.cu": EXACT,
    "stage_f64_xsb.cu": EXACT,
    "stage_f32_x49.cu": FAST32,
    "stage_f32_xs.cu": FAST32,
}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newest_dep_mtime() -> float:
    t = 0.0
    for d in (CSRC, os.path.join(ROOT, "include")):
        for f in os.listdir(d):
            t = max(t, os.path.getmtime(os.path.join(d, f)))
    return t


def _compile(unit: str, flags: list[str], force: bool) -> str:
    src = os.path.join(CSRC, unit)
    obj = os.path.join(OBJ, unit.replace(".cu", ".o"))
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= _newest_dep_mtime():
        return obj
    cmd = [nvcc()] + ARCH + COMMON + flags + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {unit}:\n{r.stdout}\n{r.stderr}")
    return obj


def build(force: bool = False, verbose: bool = True) -> str:
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= _newest_dep_mtime():
        return LIB
    jobs = min(len(UNITS), max(2, os.cpu_count() or 2))
    with cf.ThreadPoolExecutor(jobs) as ex:
        objs = list(ex.map(lambda kv: _compile(kv[0], kv[1], force), UNITS.items()))
    cmd = [nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    if verbose:
        print(f"built {LIB}")
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv)
