"""A `periodfind` package assembled in a temporary directory around the
drop-in Cython modules (periodfind_b200/dropin/periodfind/{ce,aov,ls,fpw,
bls}), as an installation puts them in place of periodfind's own .pyx
modules.  Test infrastructure only.

The rest of the package is either
  - "reference": the reference's own periodfind/__init__.py and _utils.py,
    compiled from its sources by oracle/Makefile (target `ref`) into
    oracle/_ref/periodfind -- its device factory, Statistics, Periodogram
    and input preparation; or
  - "own": this project's result classes and input preparation, for
    machines where the reference was never compiled.
Both get a gpu/__init__.py re-exporting the five classes (the reference's
own also re-exports MatchedFilter, MultiHarmonicFourier and
ViterbiNarrowband, whose modules stay the reference's).
"""

import glob
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DROPIN = os.path.join(ROOT, "periodfind_b200", "dropin", "periodfind")
REF_PKG = os.path.join(ROOT, "oracle", "_ref", "periodfind")
MODULES = {"ConditionalEntropy": "ce", "AOV": "aov", "LombScargle": "ls", "FPW": "fpw",
           "BoxLeastSquares": "bls"}

_OWN_INIT = '''"""periodfind's package namespace over periodfind_b200's result classes."""
from periodfind_b200.results import Periodogram, Statistics


def _gpu_class(name, kwargs):
    kwargs.pop("device", None)
    from periodfind import gpu
    return getattr(gpu, name)(**kwargs)


def ConditionalEntropy(**kwargs):
    return _gpu_class("ConditionalEntropy", kwargs)


def AOV(**kwargs):
    return _gpu_class("AOV", kwargs)


def LombScargle(**kwargs):
    return _gpu_class("LombScargle", kwargs)


def FPW(**kwargs):
    return _gpu_class("FPW", kwargs)


def BoxLeastSquares(**kwargs):
    return _gpu_class("BoxLeastSquares", kwargs)
'''

_OWN_UTILS = "from periodfind_b200._utils import ensure_float32, prepare_magnitudes, validate_inputs\n"


def available(source):
    if not all(glob.glob(os.path.join(DROPIN, m + ".*.so")) for m in MODULES.values()):
        return False
    if source == "reference":
        return bool(glob.glob(os.path.join(REF_PKG, "__init__.*.so")))
    return True


def assemble(tmp, source):
    """Build <tmp>/periodfind; returns the directory to put on sys.path."""
    pkg = os.path.join(str(tmp), "periodfind")
    os.makedirs(os.path.join(pkg, "gpu"))
    for so in glob.glob(os.path.join(DROPIN, "*.so")):
        os.symlink(so, os.path.join(pkg, os.path.basename(so)))
    if source == "reference":
        for so in glob.glob(os.path.join(REF_PKG, "*.so")):
            os.symlink(so, os.path.join(pkg, os.path.basename(so)))
    else:
        with open(os.path.join(pkg, "__init__.py"), "w") as f:
            f.write(_OWN_INIT)
        with open(os.path.join(pkg, "_utils.py"), "w") as f:
            f.write(_OWN_UTILS)
    with open(os.path.join(pkg, "gpu", "__init__.py"), "w") as f:
        for cls, mod in MODULES.items():
            f.write(f"from periodfind.{mod} import {cls}\n")
    return str(tmp)


def run(path, code, timeout=600):
    """Run `code` in a fresh interpreter with the assembled package and the
    repository importable; returns the CompletedProcess."""
    env = dict(os.environ)
    env["PYTHONPATH"] = os.pathsep.join([path, ROOT] + [p for p in [env.get("PYTHONPATH")] if p])
    # The modules link libpfb200.so; an installation puts it on the loader's
    # path (their in-tree rpath does not reach it through the symlinks).
    lib_dir = os.path.join(ROOT, "periodfind_b200")
    env["LD_LIBRARY_PATH"] = os.pathsep.join(
        [lib_dir] + [p for p in [env.get("LD_LIBRARY_PATH")] if p])
    return subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                          env=env, timeout=timeout, cwd=ROOT)
