"""periodfind_b200.results against the reference's own Statistics and
Periodogram (periodfind/__init__.py:253-546, compiled from its sources into
oracle/_ref/periodfind): the same picks, order, values, summary statistics,
significance and repr on random periodograms with ties, one and several
period derivatives, n = 1 and n > 1, both directions.  Runs in a fresh
interpreter (the compiled package is named periodfind)."""

import glob
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")

SCRIPT = r'''
import numpy as np
import periodfind as R
from periodfind_b200 import results as O

rng = np.random.default_rng(3)
checked = 0
for shape in ((50, 1), (40, 3), (7, 2), (200, 1)):
    params = [np.linspace(1, 2, shape[0]).astype(np.float32),
              np.linspace(0, 1e-5, shape[1]).astype(np.float32)]
    for ties in (False, True):
        data = rng.random(shape).astype(np.float32)
        if ties:
            data = np.round(data * 8) / 8
        for use_max in (False, True):
            for n in (1, 3, 5):
                for sig in ("stdmean", "madmedian"):
                    a = R.Statistics.statistics_from_data(data, params, use_max, n=n,
                                                          significance_type=sig)
                    b = O.Statistics.statistics_from_data(data, params, use_max, n=n,
                                                          significance_type=sig)
                    a = a if n > 1 else [a]
                    b = b if n > 1 else [b]
                    for x, y in zip(a, b):
                        assert x.params == y.params and x.value == y.value
                        assert (x.mean, x.std, x.median, x.mad) == (y.mean, y.std, y.median,
                                                                   y.mad)
                        assert x.significance == y.significance
                        assert repr(x) == repr(y)
                    pa = R.Periodogram(data, params, use_max)
                    pb = O.Periodogram(data, params, use_max)
                    assert pa.mean is None and pb.mean is None and repr(pa) == repr(pb)
                    ra, rb = pa.best_params(n, sig), pb.best_params(n, sig)
                    ra = ra if n > 1 else [ra]
                    rb = rb if n > 1 else [rb]
                    assert [(x.params, x.value) for x in ra] == [(y.params, y.value) for y in rb]
                    assert (pa.mean, pa.std, pa.median, pa.mad) == (pb.mean, pb.std, pb.median,
                                                                    pb.mad)
                    checked += 1
s = O.Statistics([1.0, 0.0], 2.0, 0.0, 1.0, 0.0, 1.0, "other")
try:
    s.significance
except NotImplementedError as e:
    assert "Statistic other not implemented" == str(e)
print("ok", checked)
'''


def test_results_match_reference_classes():
    if not glob.glob(os.path.join(REF, "periodfind", "__init__.*.so")):
        pytest.skip("the reference's package modules are not built (make -C oracle ref)")
    env = dict(os.environ)
    env["PYTHONPATH"] = os.pathsep.join([REF, ROOT])
    r = subprocess.run([sys.executable, "-c", SCRIPT], capture_output=True, text=True, env=env,
                       cwd=ROOT, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("ok")
