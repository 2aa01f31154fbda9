"""The drop-in Cython modules on the GPU, inside a periodfind package
(the reference's own package modules compiled from its sources, or this
project's): periodfind.X(device='gpu').calc(...) through the package's
factory returns the package's own Periodogram / Statistics, with values
equal bit for bit to periodfind_b200's ctypes path on the same data, its
'stats' equal to the package's Statistics.statistics_from_data on those
periodograms and its 'peaks' to the oracle's peak finder on them.  Where
the reference's CUDA build is present, CE and LS are also held to it with
the bounds of the other reference-parity tests (CE rtol 1e-5; LS 1e-4 of
each curve's largest power).  Each case runs in a fresh interpreter."""

import pytest

from tests import dropin_pkg

pytestmark = pytest.mark.gpu

SCRIPT = r'''
import numpy as np
import periodfind
import lightcurves as lc
from periodfind_b200 import gpu as G
from oracle import oracle as O

rng = np.random.default_rng(5)
ts, ms = [], []
for n in (3, 40, 300, 1000, 2049, 57):
    t = lc.uniform_times(rng, n, 300.0)
    ts.append(t)
    ms.append(lc.noisy(rng, lc.sinusoid(t, float(rng.uniform(1, 5)), amp=0.3, offset=15.0), 0.05))
es = [rng.uniform(0.02, 0.2, len(t)).astype(np.float32) for t in ts]
P = np.linspace(0.5, 8.0, 333).astype(np.float32)
D = np.array([0.0, 1e-5], np.float32)
cases = [("ConditionalEntropy", {"n_phase": 10, "n_mag": 10}, G.ConditionalEntropy(10, 10), False),
         ("AOV", {"n_phase": 15}, G.AOV(15), True),
         ("LombScargle", {}, G.LombScargle(), True),
         ("FPW", {"n_bins": 10}, G.FPW(10), True),
         ("BoxLeastSquares", {"n_bins": 20, "qmin": 0.05, "qmax": 0.3},
          G.BoxLeastSquares(20, 0.05, 0.3), True)]
for name, kw, mine, use_max in cases:
    obj = getattr(periodfind, name)(device="gpu", **kw)
    assert type(obj).__module__.startswith("periodfind."), type(obj).__module__
    extra = {"errs": es} if name in ("FPW", "BoxLeastSquares") else {}
    pg = obj.calc(ts, ms, P, D, output="periodogram", **extra)
    assert all(type(p) is periodfind.Periodogram for p in pg)
    want = mine.calc(ts, ms, P, D, output="periodogram", **extra)
    for a, b in zip(pg, want):
        np.testing.assert_array_equal(a.data, b.data, err_msg=name)
    st = obj.calc(ts, ms, P, D, output="stats", n_stats=3, **extra)
    for s, p in zip(st, pg):
        assert all(type(x) is periodfind.Statistics for x in s)
        ref = periodfind.Statistics.statistics_from_data(p.data, [P, D], use_max, n=3)
        # (NaN-safe: a curve shorter than the bins has NaN cells.)
        same = lambda a, b: np.array_equal(np.asarray(a, np.float64), np.asarray(b, np.float64),
                                           equal_nan=True)
        assert same([x.value for x in s], [x.value for x in ref]), name
        assert same([x.params for x in s], [x.params for x in ref]), name
        assert same([s[0].mean, s[0].std, s[0].median, s[0].mad],
                    [ref[0].mean, ref[0].std, ref[0].median, ref[0].mad]), name
    pk = obj.calc(ts, ms, P, D, output="peaks", n_peaks=5, min_distance=2, **extra)
    idx, val = O.find_top_peaks_batched(np.stack([p.data for p in pg]), 5, 2, use_max)
    for c, lst in enumerate(pk):
        k = int(np.sum(idx[c] >= 0))
        assert len(lst) == k, name
        for j, s in enumerate(lst):
            assert type(s) is periodfind.Statistics
            assert s.params == [float(P[idx[c, j] // 2]), float(D[idx[c, j] % 2])]
            assert same([s.value], [val[c, j]])
    got = np.stack([p.data for p in pg])
    if name == "ConditionalEntropy" and O.ref_available():
        msn = [lc.normalize(m) for m in ms]
        ref = O.ref_cuda("ce", ts, msn, P, D, n_phase=10, n_mag=10)
        np.testing.assert_allclose(got, ref, rtol=1e-5, atol=1e-7)
    if name == "LombScargle" and O.ref_available():
        msc = [lc.center(m) for m in ms]
        ref = O.ref_cuda("ls", ts, msc, P, D)
        scale = np.abs(ref).max(axis=(1, 2), keepdims=True)
        assert np.all(np.abs(got - ref) <= 1e-4 * scale + 1e-4 * np.abs(ref))
    print(name, "ok")
print("ok")
'''


@pytest.mark.parametrize("source", ["reference", "own"])
def test_dropin_calc_on_gpu(tmp_path, source):
    if not dropin_pkg.available(source):
        pytest.skip(f"drop-in modules or the {source} package modules are not built")
    path = dropin_pkg.assemble(tmp_path, source)
    r = dropin_pkg.run(path, SCRIPT)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().endswith("ok"), r.stdout
