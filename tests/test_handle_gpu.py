"""The engine handle on the GPU: the same bits as the Python box engine over the same bodies
(state, counters, contact forces, kinematic updates), a checkpoint that resumes bit for bit,
the packed state round trip, and device error bits reported as a status."""
import importlib

import numpy as np
import pytest

from conftest import cuda_ok

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_ok(), reason="needs a CUDA device")]

DT = 1 / 240


def _scene(n=300):
    sc = importlib.import_module("motion_engine_b200.scenes")
    return sc.random_boxes(n=n, box=(5.0, 5.0, 4.0))


def _pair(me, S, **kw):
    """A Python box engine and a handle over the same boxes."""
    p = me.BoxContactEngine(mu=0.5, vit=16, pit=10, **kw)
    for c, d, m, de in zip(S["centers"], S["dims"], S["mu"], S["density"]):
        p.add_box(c, dims=d, density=de, mu=m)
    h = me.HandleBoxEngine(mu=0.5, vit=16, pit=10, **kw)
    h.add_boxes(S["centers"], dims=S["dims"], density=S["density"], mu=S["mu"])
    return p, h


def _packed_py(p):
    return p.get_state_packed().numpy()


def test_handle_equals_python_engine(me):
    S = _scene()
    p, h = _pair(me, S)
    for step in range(150):
        p.step(DT, 2)
        h.step(DT, 2)
        if step % 25 == 24 or step < 2:
            assert _packed_py(p).tobytes() == h.get_state_packed().tobytes(), step
            hp, hh = p.check_errors(), h.header()
            for k in ("n_raw", "n_kept", "n_pairs", "n_colors", "cache_hit", "error", "rounds"):
                assert hp[k] == hh[k], (step, k)
    assert (p.color_cache_hits, p.color_cache_misses) == (h.color_cache_hits, h.color_cache_misses)
    assert h.n_graph_captures == 1 and h.header()["kernels_per_step"] > 0
    np.testing.assert_array_equal(p.contact_forces(), h.contact_forces())
    sp, sh = p.get_state(), h.get_state()
    for name in ("xc", "Rm", "vc", "om"):
        np.testing.assert_array_equal(getattr(sp, name), getattr(sh, name), err_msg=name)


def test_handle_kinematic_update_and_eager_form(me):
    S = _scene(200)
    p, h = _pair(me, S)
    h2 = me.HandleBoxEngine(mu=0.5, vit=16, pit=10, graph=False, solve_blocks=-8)
    h2.add_boxes(S["centers"], dims=S["dims"], density=S["density"], mu=S["mu"])
    for step in range(80):
        if step == 30:
            for e in (p, h, h2):
                e.set_kinematic(5, [0.2, -0.1, 0.3])
        for e in (p, h, h2):
            e.step(DT, 2)
    a = _packed_py(p).tobytes()
    assert a == h.get_state_packed().tobytes() and a == h2.get_state_packed().tobytes()
    f = h.contact_forces()
    assert np.all(f[5] == 0)
    np.testing.assert_array_equal(p.contact_forces(), f)


def test_checkpoint_resumes_bit_for_bit(me):
    S = _scene(250)
    a = me.HandleBoxEngine(mu=0.5, vit=16, pit=10)
    a.add_boxes(S["centers"], dims=S["dims"], density=S["density"], mu=S["mu"])
    for _ in range(90):
        a.step(DT, 2)
    a.set_kinematic(3, [0.0, 0.0, 0.4])
    a.step(DT, 2)
    blob = a.state_save()
    for _ in range(60):
        a.step(DT, 2)
    b = me.HandleBoxEngine(mu=0.5, vit=16, pit=10)
    b.add_boxes(S["centers"], dims=S["dims"], density=S["density"], mu=S["mu"])
    b.state_load(blob)
    for _ in range(60):
        b.step(DT, 2)
    assert a.get_state_packed().tobytes() == b.get_state_packed().tobytes()
    ha, hb = a.header(), b.header()
    assert (ha["color_cache_hits"], ha["color_cache_misses"]) == (hb["color_cache_hits"], hb["color_cache_misses"])
    np.testing.assert_array_equal(a.contact_forces(), b.contact_forces())
    c = me.HandleBoxEngine(mu=0.5)
    c.add_boxes(S["centers"][:10], dims=S["dims"][:10])
    with pytest.raises(ValueError, match="does not match"):
        c.state_load(blob)


def test_load_undoes_a_later_kinematic_update(me):
    """A blob saved while body i was dynamic, loaded after b2c_set_kinematic made it kinematic:
    the body is dynamic again on the device and on the host, so the next steps and the contact
    forces (its own row included, with its mass from the build) equal those of a handle that
    never touched it.  Body i is the lowest box, which rests on the ground."""
    S = _scene(200)
    a = me.HandleBoxEngine(mu=0.5, vit=16, pit=10)
    a.add_boxes(S["centers"], dims=S["dims"], density=S["density"], mu=S["mu"])
    b = me.HandleBoxEngine(mu=0.5, vit=16, pit=10)
    b.add_boxes(S["centers"], dims=S["dims"], density=S["density"], mu=S["mu"])
    for _ in range(120):
        a.step(DT, 2)
        b.step(DT, 2)
    i = int(np.argmin(a.get_state().xc[:, 2]))
    blob = a.state_save()
    a.set_kinematic(i, [0.0, 0.0, 3.0])
    a.step(DT, 2)
    assert np.all(a.contact_forces()[i] == 0)
    a.state_load(blob)
    for _ in range(20):
        a.step(DT, 2)
        b.step(DT, 2)
    assert a.get_state_packed().tobytes() == b.get_state_packed().tobytes()
    fa, fb = a.contact_forces(), b.contact_forces()
    np.testing.assert_array_equal(fa, fb)
    assert np.any(fb[i] != 0), "the lowest box rests on the ground and carries a contact force"


def test_packed_state_round_trip_through_the_handle(me):
    S = _scene(150)
    a = me.HandleBoxEngine()
    a.add_boxes(S["centers"], dims=S["dims"], density=S["density"], mu=S["mu"])
    b = me.HandleBoxEngine()
    b.add_boxes(S["centers"], dims=S["dims"], density=S["density"], mu=S["mu"])
    for _ in range(40):
        a.step(DT, 2)
        b.set_state_packed(b.get_state_packed())
        b.step(DT, 2)
    assert a.get_state_packed().tobytes() == b.get_state_packed().tobytes()


def test_colour_cap_error_is_a_status(me):
    """Three boxes stacked 1 mm apart (inside the 2 mm margin): the middle one has two pairs, so
    the pair graph needs two colours.  With a cap of 1 the first step sets the colour-cap bit;
    the next step returns the capacity status (RuntimeError here) and clears it."""
    h = me.HandleBoxEngine(color_cap=1)
    h.add_boxes([[0, 0, 0.101], [0, 0, 0.302], [0, 0, 0.503]], dims=[(0.5, 0.5, 0.2)] * 3)
    h.step(DT, 1)
    assert h.header()["error"] != 0
    with pytest.raises(RuntimeError, match="colour cap"):
        h.step(DT, 1)
    assert h.header()["error"] == 0


def test_handle_scenes_equal_batched_engine(me):
    """Scenes on a handle (b2c_set_body_scene) give BatchedBoxEngine's bits."""
    sc = importlib.import_module("motion_engine_b200.scenes")
    scenes = sc.batched_scenes(n_scenes=12, nmin=6, nmax=200, seed_n=7)
    g = me.BatchedBoxEngine(scenes, mu=0.55, vit=16, pit=10)
    h = me.HandleBoxEngine(mu=0.55, vit=16, pit=10, cand_per_body=12)
    for k, s in enumerate(scenes):
        h.add_boxes(s["centers"], dims=s["dims"], density=s["density"], mu=s["mu"],
                    kin=s.get("kin", np.zeros(len(s["centers"]), bool)), scene=k)
    for _ in range(100):
        g.step(DT, 2)
        h.step(DT, 2)
    assert g.get_state_packed().numpy().tobytes() == h.get_state_packed().tobytes()
    hg, hh = g.check_errors(), h.header()
    assert (hg["n_pairs"], hg["n_colors"]) == (hh["n_pairs"], hh["n_colors"])
