"""The drop-in Cython modules inside a periodfind package, without a GPU:
the reference's own factory (periodfind/__init__.py:81-160, compiled from
its sources) resolves periodfind.X(device='gpu') to this project's classes,
the reference's argument checks fire first, and with no CUDA device the
call fails with the library's message instead of exiting the process
(periodfind/cuda/errchk.cuh:16-29 exits)."""

import pytest

from tests import dropin_pkg

SCRIPT = r'''
import numpy as np
import periodfind

t = np.linspace(0, 10, 50).astype(np.float32)
m = np.sin(t).astype(np.float32)
P = np.linspace(1, 3, 20).astype(np.float32)
D = np.zeros(1, np.float32)
for name, mod in %(modules)r.items():
    obj = getattr(periodfind, name)(device="gpu")
    assert type(obj).__module__ == "periodfind." + mod, type(obj).__module__
    assert type(obj).__name__ == name
    # The reference's checks, before any device work.
    try:
        obj.calc([t], [m, m], P, D)
    except ValueError as e:
        assert "same number of light curves" in str(e)
    else:
        raise AssertionError("mismatched lists accepted")
    try:
        obj.calc([t.astype(np.float64)], [m], P, D)
    except TypeError as e:
        assert "expected float32" in str(e)
    else:
        raise AssertionError("float64 times accepted")
    try:
        obj.calc([t], [m], P.astype(np.float64), D)
    except ValueError as e:
        assert "Buffer dtype mismatch" in str(e)
    else:
        raise AssertionError("float64 periods accepted")
    # No GPU here: the library reports it.
    try:
        obj.calc([t], [m], P, D)
    except RuntimeError as e:
        assert "periodfind_b200 error" in str(e), str(e)
    else:
        print("calc ran (a GPU is present)")
print("ok")
'''


@pytest.mark.parametrize("source", ["reference", "own"])
def test_dropin_modules_in_package(tmp_path, source):
    if not dropin_pkg.available(source):
        pytest.skip(f"drop-in modules or the {source} package modules are not built")
    path = dropin_pkg.assemble(tmp_path, source)
    r = dropin_pkg.run(path, SCRIPT % {"modules": dropin_pkg.MODULES})
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().endswith("ok")
