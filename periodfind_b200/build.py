"""Build the periodfind_b200 shared libraries in-tree with nvcc for sm_100a.

    python -m periodfind_b200.build            # incremental
    python -m periodfind_b200.build --force    # rebuild everything

Outputs:
    libpfb200.so            (next to this file) the C ABI of include/pf.h and
                            its kernels
    dropin/periodfind/*.so  the Cython modules ce, aov, ls, fpw, bls that take
                            the place of periodfind's own .pyx modules inside
                            the periodfind package, calling libpfb200.so
    _host.*.so           (next to this file) curve lengths and data
                            addresses of numpy array lists for the ctypes path

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
DROPIN = os.path.join(HERE, "dropin")
DROPIN_OUT = os.path.join(DROPIN, "periodfind")
DROPIN_MODULES = ("ce", "aov", "ls", "fpw", "bls")


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
    build_dropin(force)
    build_host(force)
    if verbose:
        print(f"built {LIB}")
    return LIB


def _dropin_one(name: str, force: bool) -> str:
    """Cython -> C -> one extension module, linked to libpfb200.so (found at
    run time two directories up, through the rpath)."""
    import sysconfig

    import numpy as np

    pyx = os.path.join(DROPIN, name + ".pyx")
    so = os.path.join(DROPIN_OUT, name + sysconfig.get_config_var("EXT_SUFFIX"))
    deps = [pyx, os.path.join(DROPIN, "_common.pxi"), os.path.join(DROPIN, "pf_abi.pxd"),
            os.path.join(INCLUDE, "pf.h"), LIB]
    if not force and _mtime(so) > max(_mtime(d) for d in deps):
        return so
    c_src = os.path.join(OBJ, f"dropin_{name}.c")
    r = subprocess.run([sys.executable, "-m", "cython", "-3", "--module-name", f"periodfind.{name}",
                        "-I", DROPIN, "-o", c_src, pyx],
                       capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"cython failed for {name}.pyx:\n{r.stdout}\n{r.stderr}")
    cmd = ["gcc", "-O2", "-shared", "-fPIC", "-DNPY_NO_DEPRECATED_API=NPY_1_7_API_VERSION",
           f"-I{sysconfig.get_paths()['include']}", f"-I{np.get_include()}", f"-I{INCLUDE}",
           c_src, "-o", so, f"-L{HERE}", "-lpfb200", "-Wl,-rpath,$ORIGIN/../.."]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"gcc failed for {name}:\n{r.stdout}\n{r.stderr}")
    return so


def build_host(force: bool = False) -> str:
    """Cython -> C -> periodfind_b200/_host (numpy C API only)."""
    import sysconfig

    import numpy as np

    pyx = os.path.join(HERE, "_host.pyx")
    so = os.path.join(HERE, "_host" + sysconfig.get_config_var("EXT_SUFFIX"))
    if not force and _mtime(so) > _mtime(pyx):
        return so
    os.makedirs(OBJ, exist_ok=True)
    c_src = os.path.join(OBJ, "hostptr.c")
    r = subprocess.run([sys.executable, "-m", "cython", "-3", "--module-name",
                        "periodfind_b200._host", "-o", c_src, pyx],
                       capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"cython failed for _host.pyx:\n{r.stdout}\n{r.stderr}")
    cmd = ["gcc", "-O2", "-shared", "-fPIC", "-DNPY_NO_DEPRECATED_API=NPY_1_7_API_VERSION",
           f"-I{sysconfig.get_paths()['include']}", f"-I{np.get_include()}", c_src, "-o", so]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"gcc failed for _host:\n{r.stdout}\n{r.stderr}")
    return so


def build_dropin(force: bool = False) -> list[str]:
    os.makedirs(DROPIN_OUT, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=len(DROPIN_MODULES)) as ex:
        return list(ex.map(lambda n: _dropin_one(n, force), DROPIN_MODULES))


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    try:
        build(force=a.force)
    except RuntimeError as e:
        print(e, file=sys.stderr)
        sys.exit(1)
