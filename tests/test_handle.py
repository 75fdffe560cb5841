"""The engine handle's host side without a GPU: the body arrays it builds equal the Python box
engine's bit for bit, and configuration, body and argument errors come back as statuses."""
import ctypes

import numpy as np
import pytest


def _setup(L, centers, dims, dens, kin):
    n = len(centers)
    c, d, r = (np.ascontiguousarray(a, np.float64) for a in (centers, dims, dens))
    k = np.ascontiguousarray(kin, np.int32)
    xc4, invM = np.zeros((n, 4), np.float32), np.zeros(n, np.float32)
    IbInv, M = np.zeros((n, 12), np.float32), np.zeros(n)
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    rc = L.b2c_box_body_setup(n, p(c), p(d), p(r), p(k), p(xc4), p(invM), p(IbInv), p(M))
    return rc, xc4, invM, IbInv, M


def test_body_setup_equals_python_box_arrays(me):
    from motion_engine_b200.boxes import box_body_arrays
    L = me._lib.load()
    rng = np.random.default_rng(11)
    n = 500
    centers = rng.uniform(-10, 10, (n, 3))
    dims = rng.uniform(0.05, 1.5, (n, 3))
    dens = rng.uniform(100.0, 8000.0, n)
    kin = (rng.random(n) < 0.1).astype(np.int32)
    rc, xc4, invM, IbInv, M = _setup(L, centers, dims, dens, kin)
    assert rc == 0
    A = box_body_arrays(centers, 0.5 * dims, dens, kin)
    bits = lambda a: np.ascontiguousarray(a).view(np.uint32 if a.dtype == np.float32 else np.uint64)
    np.testing.assert_array_equal(bits(xc4[:, :3].copy()), bits(A["xc"]))
    np.testing.assert_array_equal(bits(invM), bits(A["invM"]))
    np.testing.assert_array_equal(bits(IbInv.reshape(n, 3, 4)[:, :, :3].copy()), bits(A["IbInv"]))
    np.testing.assert_array_equal(bits(M), bits(A["M"]))
    assert np.all(xc4[:, 3] == 0) and np.all(IbInv.reshape(n, 3, 4)[:, :, 3] == 0)


def test_body_setup_rejects_degenerate_boxes(me):
    L = me._lib.load()
    rc = _setup(L, [[0, 0, 0]], [[0.3, 0.3, 0.2]], [0.0], [0])[0]
    assert rc == 1 and b"degenerate" in L.b2c_last_error()


def test_config_defaults_and_bad_configs(me):
    L = me._lib.load()
    c = me._lib.Config()
    L.b2c_config_init(ctypes.byref(c))
    assert (c.kind, c.vit, c.pit, c.mu, tuple(c.dims), c.margin) == (1, 16, 10, 0.5, (0.3, 0.3, 0.2), 2e-3)
    assert (c.flags, c.color_cap, c.cand_per_body, c.barrier_timeout_ns, c.graph) == (111, 512, 16, 10 ** 9, 1)
    h = ctypes.c_void_p()
    for field, bad in (("kind", 7), ("vit", -1), ("mu", float("nan")), ("color_cap", 0), ("cand_per_body", 0),
                       ("flags", 64)):
        b = me._lib.Config()
        L.b2c_config_init(ctypes.byref(b))
        setattr(b, field, bad)
        assert L.b2c_create(ctypes.byref(b), ctypes.byref(h)) == 1, field
        assert not h.value
        if field == "kind":
            assert b"kind" in L.b2c_last_error()
    b = me._lib.Config()
    L.b2c_config_init(ctypes.byref(b))
    b.flags |= me._lib.COLOR_ISLANDS
    assert L.b2c_create(ctypes.byref(b), ctypes.byref(h)) == 1 and not h.value
    assert b"ISLANDS" in L.b2c_last_error()
    assert L.b2c_create(ctypes.byref(c), None) == 1


def test_handle_bodies_without_gpu(me):
    """Creating a handle and adding bodies does no device work; range errors are statuses."""
    e = me.HandleBoxEngine(dims=(0.4, 0.3, 0.2), mu=0.6)
    idx = e.add_boxes([[0, 0, 0.1], [1, 0, 0.1], [2, 0, 0.1]], mu=[0.3, 0.4, 0.5])
    assert list(idx) == [0, 1, 2] and e.N == 3
    assert e.add_body([3, 0, 0.1]) == 3 and e.add_box([4, 0, 0.1], dims=(0.2, 0.2, 0.2), scene=2) == 4
    assert e.header()["built"] == 0 and e.header()["bodies"] == 5
    L = e.L
    with pytest.raises(ValueError, match="out of range"):
        e._call(L.b2c_set_body_mu(e._h, 4, 2, np.ones(2).ctypes.data_as(ctypes.c_void_p)), "b2c_set_body_mu")
    with pytest.raises(ValueError, match="non-finite|non-positive"):
        e.add_box([np.nan, 0, 0])
    with pytest.raises(ValueError, match="non-finite|non-positive"):
        e.add_box([0, 0, 0], dims=(0.0, 1.0, 1.0))
    with pytest.raises(ValueError):
        e.set_kinematic(17, [0, 0, 0])
    assert e.N == 5
    e.set_kinematic(1, [1.0, 0.0, 0.5])  # before the build: host lists only
    e.close()
    assert e._h.value is None
    assert L.b2c_body_count(None) == -1
    h = ctypes.c_void_p()
    assert L.b2c_destroy(ctypes.byref(h)) == 0 and L.b2c_destroy(None) == 1
