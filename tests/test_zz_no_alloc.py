"""The allocation-free LS peaks entry point (pf_ls_peaks_dev_noalloc).

Some callers cannot call cudaMalloc where they need periodogram peaks: their
device memory belongs to another allocator's pool, or they sit on a path
that cannot absorb cudaMalloc's implicit synchronisation, or they work to a
fixed memory budget.  This entry point keeps all of its scratch in one
device array inside the library.  These tests call it through the C ABI and
check it against the allocating entry points (pf_ls_dev + pf_find_peaks_dev)
on two calls in a row -- the second call reuses the array the first left
behind -- and check that an oversized batch is refused with a message.

The file sorts last so that, if it fails, a run stopping at the first failure
has already run every other test; it also passes on its own.
"""

import ctypes

import numpy as np
import pytest

import lightcurves as lc

pytestmark = pytest.mark.gpu


def _batch(seed, lengths, n_per, pdts):
    rng = np.random.default_rng(seed)
    ts, ms = [], []
    for n in lengths:
        t = lc.uniform_times(rng, n, 500.0)
        ts.append(t)
        ms.append(lc.center(lc.noisy(rng, lc.sinusoid(t, float(rng.uniform(0.5, 8))), 0.05)))
    periods = np.linspace(0.3, 12.0, n_per, dtype=np.float32)
    return ts, ms, periods, np.array(pdts, np.float32)


def _run_both(torch, nat, ts, ms, periods, pdts, n_peaks, min_distance, mode):
    dev = "cuda"
    off = np.zeros(len(ts) + 1, np.int64)
    np.cumsum([len(t) for t in ts], out=off[1:])
    d_t = torch.from_numpy(np.concatenate(ts)).to(dev)
    d_m = torch.from_numpy(np.concatenate(ms)).to(dev)
    d_p = torch.from_numpy(periods).to(dev)
    d_d = torch.from_numpy(pdts).to(dev)
    n, cells = len(ts), len(periods) * len(pdts)
    stream = torch.cuda.current_stream().cuda_stream

    # Allocating path: periodogram, then the peak search.
    ctx = nat.default_context(0)
    pg = torch.empty((n, cells), dtype=torch.float32, device=dev)
    ref_idx = torch.full((n, n_peaks), -7, dtype=torch.int64, device=dev)
    ref_val = torch.full((n, n_peaks), -7.0, dtype=torch.float32, device=dev)
    with ctx.lock:
        ctx.check(ctx.lib.pf_ls_dev(ctx.handle, d_t.data_ptr(), d_m.data_ptr(), off.ctypes.data,
                                    n, d_p.data_ptr(), len(periods), d_d.data_ptr(), len(pdts),
                                    mode, pg.data_ptr(), stream))
        ctx.check(ctx.lib.pf_find_peaks_dev(ctx.handle, pg.data_ptr(), n, cells, n_peaks,
                                            min_distance, 1, ref_idx.data_ptr(),
                                            ref_val.data_ptr(), stream))

    # Allocation-free path.
    idx = torch.full((n, n_peaks), -9, dtype=torch.int64, device=dev)
    val = torch.full((n, n_peaks), -9.0, dtype=torch.float32, device=dev)
    err = ctypes.create_string_buffer(512)
    rc = ctx.lib.pf_ls_peaks_dev_noalloc(d_t.data_ptr(), d_m.data_ptr(), off.ctypes.data, n,
                                         d_p.data_ptr(), len(periods), d_d.data_ptr(), len(pdts),
                                         n_peaks, min_distance, mode, idx.data_ptr(),
                                         val.data_ptr(), stream, err, len(err))
    assert rc == 0, err.value.decode()
    torch.cuda.current_stream().synchronize()
    return ref_idx.cpu().numpy(), ref_val.cpu().numpy(), idx.cpu().numpy(), val.cpu().numpy()


def test_noalloc_matches_allocating_path_two_calls():
    torch = pytest.importorskip("torch")
    from periodfind_b200 import _native as nat

    calls = [
        # (seed, curve lengths, periods, pdts, n_peaks, min_distance, mode)
        (1, (700, 37, 2048, 5), 3000, (0.0, 1e-5), 32, 1, nat.PF_MODE_CHOSEN),
        (2, (1500, 900, 64), 1200, (0.0,), 16, 4, nat.PF_MODE_PLAIN),
    ]
    for seed, lengths, n_per, pdts, n_peaks, md, mode in calls:
        ts, ms, periods, pd = _batch(seed, lengths, n_per, pdts)
        ri, rv, ni, nv = _run_both(torch, nat, ts, ms, periods, pd, n_peaks, md, mode)
        # Same kernels on the same inputs: identical peaks (index and value).
        np.testing.assert_array_equal(ni, ri)
        np.testing.assert_array_equal(nv, rv)
        assert (ni[:, 0] >= 0).all()


def test_noalloc_allocates_nothing():
    """After a first call, further calls with other batch layouts leave the
    device's free memory exactly as it was: the entry point allocates
    nothing (the inputs and outputs are made before the measurement)."""
    torch = pytest.importorskip("torch")
    from periodfind_b200 import _native as nat

    lib = nat.load()
    batches = []
    for seed, lengths, n_per in ((3, (300, 50, 1200), 800), (4, (2000, 10, 700, 90), 1500)):
        ts, ms, periods, pd = _batch(seed, lengths, n_per, (0.0,))
        off = np.zeros(len(ts) + 1, np.int64)
        np.cumsum([len(t) for t in ts], out=off[1:])
        batches.append((torch.from_numpy(np.concatenate(ts)).cuda(),
                        torch.from_numpy(np.concatenate(ms)).cuda(), off,
                        torch.from_numpy(periods).cuda(), torch.from_numpy(pd).cuda(),
                        torch.empty((len(ts), 8), dtype=torch.int64, device="cuda"),
                        torch.empty((len(ts), 8), dtype=torch.float32, device="cuda")))
    err = ctypes.create_string_buffer(512)

    def call(b):
        d_t, d_m, off, d_p, d_d, idx, val = b
        rc = lib.pf_ls_peaks_dev_noalloc(d_t.data_ptr(), d_m.data_ptr(), off.ctypes.data,
                                         len(off) - 1, d_p.data_ptr(), d_p.numel(),
                                         d_d.data_ptr(), d_d.numel(), 8, 1, nat.PF_MODE_CHOSEN,
                                         idx.data_ptr(), val.data_ptr(), None, err, len(err))
        assert rc == 0, err.value.decode()
        torch.cuda.synchronize()

    call(batches[0])  # first call on the device: its one-time set-up
    free0, _ = torch.cuda.mem_get_info()
    call(batches[1])
    call(batches[0])
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_noalloc_rejects_batch_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    from periodfind_b200 import _native as nat

    lib = nat.load()
    n, n_per = 64, 200000  # periodograms alone need 64 * 200000 * 4 B = 51 MB > 32 MiB
    off = np.arange(n + 1, dtype=np.int64) * 16
    d_t = torch.zeros(n * 16, dtype=torch.float32, device="cuda")
    d_p = torch.ones(n_per, dtype=torch.float32, device="cuda")
    d_d = torch.zeros(1, dtype=torch.float32, device="cuda")
    idx = torch.empty((n, 4), dtype=torch.int64, device="cuda")
    val = torch.empty((n, 4), dtype=torch.float32, device="cuda")
    err = ctypes.create_string_buffer(512)
    rc = lib.pf_ls_peaks_dev_noalloc(d_t.data_ptr(), d_t.data_ptr(), off.ctypes.data, n,
                                     d_p.data_ptr(), n_per, d_d.data_ptr(), 1, 4, 1,
                                     nat.PF_MODE_CHOSEN, idx.data_ptr(), val.data_ptr(), None,
                                     err, len(err))
    assert rc == nat.PF_EINVAL
    assert b"scratch" in err.value
