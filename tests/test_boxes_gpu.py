"""Box engine on the GPU: the float64 SAT narrowphase against the oracle (bitwise) and against
the reference's own golden contacts, and the whole box substep (broadphase, narrowphase,
colouring, ColorCache pair solve, warm store, integration) against the oracle's box step."""
import ctypes
import importlib
import os

import numpy as np
import pytest

from conftest import cuda_ok

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_ok(), reason="needs a CUDA device")]

DT = 1 / 240
TOL = 1e-10


@pytest.fixture(scope="module")
def sat():
    return dict(np.load(os.path.join(os.path.dirname(__file__), "golden", "sat_golden.npz")))


def _narrow(me, half, x, q, bhalf=None, bx=None, bq=None, margin=2e-3):
    import torch
    L = me._lib.load()
    n = len(half)
    dev = torch.device("cuda")
    f4 = lambda a: torch.from_numpy(np.ascontiguousarray(np.pad(np.asarray(a, np.float32),
                                                                ((0, 0), (0, 4 - np.shape(a)[1]))))).to(dev)
    A = [f4(half), f4(x), f4(q)]
    B = [f4(bhalf), f4(bx), f4(bq)] if bhalf is not None else [None, None, None]
    pts = torch.zeros((n, 8, 4), dtype=torch.float64, device=dev)
    nrm = torch.zeros((n, 4), dtype=torch.float64, device=dev)
    fid = torch.zeros((n, 8), dtype=torch.int32, device=dev)
    cnt = torch.zeros(n, dtype=torch.int32, device=dev)
    p = lambda t: ctypes.c_void_p(t.data_ptr()) if t is not None else None
    rc = L.b2c_box_narrowphase_test(n, *[p(t) for t in A], *[p(t) for t in B], ctypes.c_float(margin), p(pts), p(nrm),
                                    p(fid), p(cnt), None)
    me._lib.check(rc, "b2c_box_narrowphase_test")
    torch.cuda.synchronize()
    return pts.cpu().numpy(), nrm.cpu().numpy(), fid.cpu().numpy(), cnt.cpu().numpy()


def test_box_plane_narrowphase(me, oracle_mod, sat):
    O = oracle_mod
    m32 = float(np.float32(sat["margin"]))
    pts, _, fid, cnt = _narrow(me, sat["G_half"], sat["G_x"], sat["G_q"], margin=float(sat["margin"]))
    for k in range(len(cnt)):
        p, g, f = O.box_plane(sat["G_half"][k], sat["G_x"][k], sat["G_q"][k], m32)
        assert cnt[k] == len(g)
        np.testing.assert_array_equal(fid[k, :cnt[k]], f)
        np.testing.assert_array_equal(pts[k, :cnt[k], :3], p)  # bitwise: same float64 expressions
        np.testing.assert_array_equal(pts[k, :cnt[k], 3], g)
        sel = sat["bp_box"] == k
        np.testing.assert_array_equal(f, sat["bp_f"][sel])
        np.testing.assert_allclose(p, sat["bp_p"][sel], rtol=0, atol=TOL)


def test_box_box_narrowphase(me, oracle_mod, sat):
    O = oracle_mod
    m32 = float(np.float32(sat["margin"]))
    pts, nrm, fid, cnt = _narrow(me, sat["A_half"], sat["A_x"], sat["A_q"], sat["B_half"], sat["B_x"], sat["B_q"],
                                 margin=float(sat["margin"]))
    for k in range(len(cnt)):
        p, n, g, f = O.box_box(sat["A_half"][k], sat["A_x"][k], sat["A_q"][k], sat["B_half"][k], sat["B_x"][k],
                               sat["B_q"][k], m32)
        assert cnt[k] == len(g), k
        if not len(g):
            continue
        np.testing.assert_array_equal(fid[k, :cnt[k]], f)
        np.testing.assert_array_equal(pts[k, :cnt[k], :3], p)
        np.testing.assert_array_equal(pts[k, :cnt[k], 3], g)
        np.testing.assert_array_equal(nrm[k, :3], n)
        sel = sat["bb_pair"] == k
        np.testing.assert_array_equal(f, sat["bb_f"][sel])
        np.testing.assert_allclose(g, sat["bb_g"][sel], rtol=0, atol=TOL)


def _pile(n=300, box=(6.0, 6.0, 5.0)):
    sc = importlib.import_module("motion_engine_b200.scenes")
    return sc.random_boxes(n=n, box=box)


def _fill(e, S):
    for c, d, m, de in zip(S["centers"], S["dims"], S["mu"], S["density"]):
        e.add_box(c, dims=d, density=de, mu=m)
    return e


def _state(e):
    s = e.get_state()
    return s.xc, s.Rm, s.vc, s.om


@pytest.mark.parametrize("row_form", [True, False])
def test_box_engine_matches_oracle(me, oracle_mod, row_form):
    S = _pile()
    g = _fill(me.BoxContactEngine(mu=0.5, vit=16, pit=10, row_form=row_form), S)
    o = _fill(oracle_mod.BoxOracle(mu=0.5, vit=16, pit=10, flags=111 if row_form else 47), S)
    for step in range(240):
        g.step(DT, 2)
        o.step(DT, 2)
        if step % 20 == 19 or step < 3:
            h, st = g.check_errors(), o.stats()
            assert (h["n_contacts"], h["n_pairs"], h["n_colors"]) == (st["n_contacts"], st["n_pairs"], st["n_colors"]), \
                (step, h, st)
            for a, b, name in zip(_state(g), _state(o), ("xc", "Rm", "vc", "om")):
                np.testing.assert_array_equal(a, b, err_msg=f"{name} at step {step}")
    assert g.color_cache_hits == o.stats()["hits"] and g.color_cache_misses == o.stats()["misses"]
    np.testing.assert_array_equal(g.contact_forces(), o.contact_forces())


def test_box_engine_repeatable_and_launch_forms(me):
    S = _pile(200, box=(5.0, 5.0, 4.0))
    runs = []
    for blocks, graph in ((0, True), (0, True), (1, True), (-8, False), (5, True)):
        e = _fill(me.BoxContactEngine(mu=0.5, vit=16, pit=10, solve_blocks=blocks), S)
        e.graph = graph
        for _ in range(150):
            e.step(DT, 2)
        e.check_errors()
        runs.append(_state(e))
    for r in runs[1:]:
        for a, b in zip(runs[0], r):
            np.testing.assert_array_equal(a, b)


def test_box_engine_rests(me):
    """Four boxes stacked on the ground come to rest: supports carry the weight above them."""
    e = me.BoxContactEngine(mu=0.6, vit=16, pit=10)
    z = 0.0
    for k, h in enumerate((0.4, 0.3, 0.35, 0.2)):
        e.add_box([0.01 * k, -0.01 * k, z + h / 2 + 1e-3], dims=(0.5, 0.45, h), density=1000.0)
        z += h + 1e-3
    for _ in range(480):
        e.step(DT, 2)
    xc, _, vc, _ = _state(e)
    assert np.abs(vc).max() < 1e-2
    f = e.contact_forces()
    M = e._M
    np.testing.assert_allclose(f[:, 2], M * 9.81, rtol=0.05)


def test_colouring_beyond_register_pairs(me, oracle_mod):
    """More pairs than the colouring keeps in registers (4 per thread of a 16 x 1024-thread
    cluster, 65 536): the rest take its scratch path.  Three layers of 105 x 105 cubes with a
    1.6 mm face gap (inside the 2 mm contact margin; edge and corner neighbours are not) give
    about 98 000 pairs from the first step; colours, counts and states equal the oracle's."""
    n, layers, edge, gap = 105, 3, 0.25, 1.6e-3
    pitch = edge + gap
    g = me.BoxContactEngine(mu=0.5, vit=8, pit=4)
    o = oracle_mod.BoxOracle(mu=0.5, vit=8, pit=4)
    for k in range(layers):
        for j in range(n):
            for i in range(n):
                c = ((i - n / 2) * pitch, (j - n / 2) * pitch, 0.5 * edge + gap / 2 + k * pitch)
                g.add_box(c, dims=(edge, edge, edge), density=1000.0, mu=0.5)
                o.add_box(c, dims=(edge, edge, edge), density=1000.0, mu=0.5)
    for _ in range(2):
        g.step(1 / 240, 1)
        o.step(1 / 240, 1)
    h, st = g.check_errors(), o.stats()
    assert h["n_pairs"] > 65536, h
    assert (h["n_contacts"], h["n_pairs"], h["n_colors"]) == (st["n_contacts"], st["n_pairs"], st["n_colors"])
    sg, so = g.get_state(), o.get_state()
    for name in ("xc", "Rm", "vc", "om"):
        np.testing.assert_array_equal(getattr(sg, name), getattr(so, name), err_msg=name)


def test_packed_state_round_trip(me):
    """get_state_packed / set_state_packed move the whole body state in one copy each way: a run
    that downloads and re-uploads its state every step stays bytewise equal to one that does
    not, and the packed planes are the positions, quaternions and velocities get_state reads."""
    import torch
    S = _pile(200, box=(5.0, 5.0, 4.0))
    a = _fill(me.BoxContactEngine(mu=0.5, vit=16, pit=10), S)
    b = _fill(me.BoxContactEngine(mu=0.5, vit=16, pit=10), S)
    host = torch.empty((4, len(S["centers"]), 4), dtype=torch.float32, pin_memory=True)
    for _ in range(60):
        a.step(DT, 2)
        b.get_state_packed(host)
        b.set_state_packed(host)
        b.step(DT, 2)
    torch.cuda.synchronize()
    for x, y in zip(_state(a), _state(b)):
        np.testing.assert_array_equal(x, y)
    p = b.get_state_packed().numpy()
    st = b.get_state()
    np.testing.assert_array_equal(p[0, :, :3], st.xc)
    np.testing.assert_array_equal(p[2, :, :3], st.vc)
    np.testing.assert_array_equal(p[3, :, :3], st.om)
