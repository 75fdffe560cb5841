"""b2c_exclusive_scan_noalloc (the scan with library-owned scratch) against b2c_exclusive_scan
with caller scratch, on two calls in a row; and its size limit.  Collected last on purpose: it
must pass after every other test has used the library, as well as alone."""
import ctypes

import numpy as np
import pytest

from conftest import cuda_ok

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_ok(), reason="needs a CUDA device")]


def _scan_pair(me, x):
    import torch
    L = me._lib.load()
    dev = torch.device("cuda")
    n = len(x)
    inp = torch.from_numpy(x).to(dev)
    out_ref = torch.zeros(max(n, 1), dtype=torch.int32, device=dev)
    out_na = torch.full((max(n, 1),), -7, dtype=torch.int32, device=dev)
    scratch = torch.zeros(max(int(L.b2c_scan_scratch_ints(n)), 1), dtype=torch.int32, device=dev)
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    me._lib.check(L.b2c_exclusive_scan(p(inp), p(out_ref), n, p(scratch), s), "b2c_exclusive_scan")
    me._lib.check(L.b2c_exclusive_scan_noalloc(p(inp), p(out_na), n, s), "b2c_exclusive_scan_noalloc")
    torch.cuda.synchronize()
    return out_ref[:n].cpu().numpy(), out_na[:n].cpu().numpy()


def test_noalloc_scan_matches_scan_on_two_calls(me):
    rng = np.random.default_rng(11)
    for n in (5_000_003, 3_000):  # a multi-level scan, then a small one reusing the same scratch
        x = rng.integers(0, 50, n).astype(np.int32)
        ref, na = _scan_pair(me, x)
        np.testing.assert_array_equal(na, ref)
        np.testing.assert_array_equal(na, (np.cumsum(x) - x).astype(np.int32))


def test_noalloc_scan_rejects_too_large_n(me):
    import torch
    L = me._lib.load()
    nmax = int(L.b2c_scan_noalloc_max_n())
    assert nmax == 1 << 24
    dummy = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = L.b2c_exclusive_scan_noalloc(ctypes.c_void_p(dummy.data_ptr()), ctypes.c_void_p(dummy.data_ptr()),
                                      nmax + 1, None)
    assert rc == 1
    assert b"exceeds the maximum" in L.b2c_last_error()


def test_noalloc_setup_call_takes_null_arrays(me):
    """n = 0 with null arrays is the set-up call (it only looks up the scratch address); a
    negative n or null arrays with n > 0 are bad arguments."""
    L = me._lib.load()
    assert L.b2c_exclusive_scan_noalloc(None, None, 0, None) == 0
    assert L.b2c_exclusive_scan_noalloc(None, None, -1, None) == 1
    assert L.b2c_exclusive_scan_noalloc(None, None, 5, None) == 1
    x = np.arange(100, dtype=np.int32)
    ref, na = _scan_pair(me, x)
    np.testing.assert_array_equal(na, ref)
