"""Argument checks of the batched-ADMM and island-partition entry points, which run on the host
before any device work (no GPU needed): bad sizes, missing arrays and inconsistent flags return
B2C_EARG with a message."""
import ctypes

import pytest


def test_admm_solve_rejects_bad_arguments(me):
    L = me._lib.load()
    A, P = me._lib.Admm, me._lib.AdmmParams
    assert L.b2c_admm_solve(None, None, None) == 1
    dummy = ctypes.c_void_p(16)  # never dereferenced: every call below fails its checks first
    good = dict(flags=me._lib.ADMM_FORWARD, n_iter=10, cg_iters=4, refresh_every=4, tol=1e-8, chunk=0, desax=1,
                rho_mode=3, jacobi_sweeps=10, alpha_eta=0.0, dt=0.01, jdir=0, n_calls=0, grad_cg=10, do_mu=1)

    def call(nc=4, nv=18, **over):
        a = A(8, nc, nv, *([dummy.value] * 8), None, None, None, None, None, None, None, None, None)
        p = P(**dict(good, **over))
        return L.b2c_admm_solve(ctypes.byref(a), ctypes.byref(p), None)

    assert call(nc=9) == 1 and b"out of range" in L.b2c_last_error()
    assert call(nv=33) == 1
    assert call(nc=0) == 1
    assert call(flags=me._lib.ADMM_FORWARD | me._lib.ADMM_GRAD_GIVEN) == 1
    assert call(flags=0) == 1
    assert call(jdir=18) == 1
    assert call(n_calls=7) == 1
    assert call(rho_mode=5) == 1
    # the gradient needs its output arrays
    assert call(flags=me._lib.ADMM_FORWARD | me._lib.ADMM_GRADIENT) == 1
    assert b"NULL" in L.b2c_last_error()
    assert L.b2c_admm_smem_bytes(4, 18) > 0 and L.b2c_admm_smem_bytes(9, 18) == -1


def test_island_partition_rejects_bad_arguments(me):
    L = me._lib.load()
    info = ctypes.c_void_p(16)
    assert L.b2c_island_partition(None, None, None, None, -1, 4, info, None, None, None, info, None) == 1
    assert L.b2c_island_partition(None, None, None, None, 3, 4, info, None, None, None, info, None) == 1
    assert L.b2c_island_partition(None, None, None, None, 0, 4, None, None, None, None, info, None) == 1
    assert b"bad argument" in L.b2c_last_error()
    assert L.b2c_island_work_ints(10, 20) > 10 + 20 and L.b2c_island_work_ints(-1, 3) == -1
