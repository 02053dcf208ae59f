"""Build the in-tree CUDA library ``ibis_b200/_lib/libibis_b200.so`` for sm_100a.

Each translation unit is compiled by ``nvcc`` directly (no JIT cache, so the
library travels with the source tree); the build is skipped when the sources
have not changed since the last one.  Run ``python -m ibis_b200.build``.
"""
from __future__ import annotations

import concurrent.futures as cf
import hashlib
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libibis_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", os.path.join(REPO, "include")]

# FP32 kernels: fast single-precision math (MUFU exp/log/pow, approximate
# division and square root, denormals flushed) and FP32 saturation terms inside
# the FP64 canopy solve.  Their error against the float64 kernels is measured by
# tests/test_gpu_precision.py.
F32_FLAGS = ["-use_fast_math", "-DIBIS_FAST_SAT=1"]

# translation unit -> extra flags
UNITS = {
    "ibis_step_f32.cu": F32_FLAGS,
    "ibis_f32_inst_a.cu": F32_FLAGS,
    "ibis_f32_inst_b.cu": F32_FLAGS,
    "ibis_f32_inst_c.cu": F32_FLAGS,
    "ibis_f32_inst_d.cu": F32_FLAGS,
    "ibis_f32_inst_e.cu": F32_FLAGS,
    "ibis_x3_inst_a.cu": F32_FLAGS,
    "ibis_x3_inst_b.cu": F32_FLAGS,
    "ibis_x3_inst_c.cu": F32_FLAGS,
    "ibis_x3_inst_d.cu": F32_FLAGS,
    "ibis_x3_inst_e.cu": F32_FLAGS,
    "ibis_ensemble_f32.cu": F32_FLAGS,
    "ibis_ens_inst_a.cu": F32_FLAGS,
    "ibis_ens_inst_b.cu": F32_FLAGS,
    "ibis_ens_inst_c.cu": F32_FLAGS,
    "ibis_ens_inst_d.cu": F32_FLAGS,
    "ibis_ens_inst_e.cu": F32_FLAGS,
    "ibis_ens_inst_f.cu": F32_FLAGS,
    "ibis_ens_x3_inst_a.cu": F32_FLAGS,
    "ibis_ens_x3_inst_b.cu": F32_FLAGS,
    "ibis_ens_x3_inst_c.cu": F32_FLAGS,
    "ibis_ens_x3_inst_d.cu": F32_FLAGS,
    "ibis_ens_x3_inst_e.cu": F32_FLAGS,
    "ibis_ens_x3_inst_f.cu": F32_FLAGS,
    "ibis_diurnal_f32.cu": ["-use_fast_math"],
    "ibis_step_f64.cu": ["--fmad=false"],
    "ibis_daily.cu": ["--fmad=false"],
    "ibis_month.cu": ["--fmad=false"],
    "ibis_wetland.cu": ["--fmad=false"],
}


def _nvcc():
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(exe):
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build ibis_b200")
    return exe


def _sources():
    files = sorted(f for f in os.listdir(CSRC) if f.endswith((".cu", ".cuh")))
    files = [os.path.join(CSRC, f) for f in files]
    files += [os.path.join(REPO, "include", f) for f in sorted(os.listdir(os.path.join(REPO, "include")))]
    files.append(os.path.abspath(__file__))
    return files


def _digest():
    h = hashlib.sha256()
    for f in _sources():
        with open(f, "rb") as fh:
            h.update(os.path.basename(f).encode())
            h.update(fh.read())
    return h.hexdigest()


def _compile(unit, flags, verbose):
    src = os.path.join(CSRC, unit)
    obj = os.path.join(OUT_DIR, unit.replace(".cu", ".o"))
    cmd = [_nvcc()] + ARCH + COMMON + flags + ["-c", src, "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {unit}:\n{r.stderr}")
    return obj, r.stderr


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    stamp = os.path.join(OUT_DIR, "build.sha256")
    dig = _digest()
    if not force and os.path.exists(LIB) and os.path.exists(stamp):
        with open(stamp) as f:
            if f.read().strip() == dig:
                return LIB
    units = [(u, fl) for u, fl in UNITS.items() if os.path.exists(os.path.join(CSRC, u))]
    with cf.ThreadPoolExecutor(max_workers=len(units)) as ex:
        results = list(ex.map(lambda a: _compile(a[0], a[1], verbose), units))
    objs = [o for o, _ in results]
    if verbose:
        for _, log in results:
            sys.stderr.write(log)
    tmp = LIB + ".tmp"
    cmd = [_nvcc()] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stderr}")
    os.replace(tmp, LIB)
    for o in objs:
        os.remove(o)
    with open(stamp, "w") as f:
        f.write(dig)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
