"""Build the periodfind_b200 shared libraries in-tree with nvcc for sm_100a.

    python -m periodfind_b200.build            # incremental
    python -m periodfind_b200.build --force    # rebuild everything

Output (next to this file): libpfb200.so, the C ABI of include/pf.h and its
kernels.

Per-translation-unit flags carry the two arithmetic semantics:
    kern_cudasem.cu  -use_fast_math   (the reference's CUDA build flags)
    kern_cpusem.cu   IEEE, no FTZ, no multiply-add contraction
"""

from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
OBJ = os.path.join(HERE, "_build")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", f"-I{INCLUDE}", f"-I{CSRC}"]

UNITS = {
    "kern_cudasem.cu": ["-use_fast_math"],
    "kern_cpusem.cu": ["-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false"],
    "pf_prep.cu": ["-fmad=false"],
    "pf_peaks.cu": [],
    "pf_api.cu": ["-Xcompiler", "-ffp-contract=off"],  # host float32 arithmetic as numpy
    "pf_noalloc.cu": [],
    "pf_lsgrad.cu": [],
    "pf_stats.cu": ["-fmad=false"],  # numpy's float32 arithmetic, one rounding per operation
}

LIB = os.path.join(HERE, "libpfb200.so")


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _mtime(p: str) -> float:
    return os.path.getmtime(p) if os.path.exists(p) else -1.0


def _dep_mtime() -> float:
    """Newest header any unit may include (every .h/.cuh/.inc in csrc/)."""
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)
            if f.endswith((".h", ".cuh", ".inc"))] + [os.path.join(INCLUDE, "pf.h")]
    return max(_mtime(d) for d in deps)


def _compile(src: str, flags: list[str], force: bool) -> str:
    obj = os.path.join(OBJ, os.path.splitext(src)[0] + ".o")
    path = os.path.join(CSRC, src)
    if not force and _mtime(obj) > max(_mtime(path), _dep_mtime()):
        return obj
    cmd = [nvcc()] + COMMON + ARCH + flags + ["-c", path, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj


def build(force: bool = False, verbose: bool = True) -> str:
    os.makedirs(OBJ, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=len(UNITS)) as ex:
        futs = {ex.submit(_compile, s, f, force): s for s, f in UNITS.items()}
        objs = [f.result() for f in futs]
    if force or _mtime(LIB) < max(_mtime(o) for o in objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + sorted(objs) + ["-lpthread"]
        subprocess.run(cmd, check=True)
    if verbose:
        print(f"built {LIB}")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    try:
        build(force=a.force)
    except RuntimeError as e:
        print(e, file=sys.stderr)
        sys.exit(1)
