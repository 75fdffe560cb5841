"""The exact-cone box world on the device (BoxWorldB200) against the reference's own BoxWorld.

The golden trajectory (tests/golden/world_golden.npz, tests/golden/make_world_golden.py) is the
reference's BoxWorld (ncp_gpu.py:1237-1413) -- its SAT contacts, build_scene and integration --
with its contact solve driven to convergence by the reference's float64 CPU solver.  Here the
device world runs the same scene with its NCP sweeps also driven towards convergence (2000
sweeps per substep on at most a few dozen contacts), so the two may differ only by the solvers'
residuals and float64 rounding:
  * until the first box lands on another (step 54: a face on a face, four coplanar contacts whose
    impulses the contact problem leaves undetermined -- two converged solvers may pick different
    ones, and the bounce that follows amplifies the difference), every body agrees to the bounds
    below and the contact counts are equal at every step: falls, edge and face contacts with the
    ground, a sliding box;
  * the stack of three boxes (face-on-face contacts from the start, apart from the others)
    agrees over all 90 steps.
"""
import os

import numpy as np
import pytest

from conftest import ROOT, cuda_ok

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_ok(), reason="needs a CUDA device")]


def _golden():
    return np.load(os.path.join(ROOT, "tests", "golden", "world_golden.npz"))


def _world(me, g, **kw):
    from importlib import import_module
    W = import_module("motion_engine_b200.world")
    w = W.BoxWorldB200(dt=1.0 / 240.0, mu=0.5, iters=kw.pop("iters", 2000), **kw)
    for i in range(len(g["half"])):
        w.add(g["half"][i], float(g["mass"][i]), g["x0"][i], v=g["v0"][i], q=g["q0"][i])
    return w


FIRST_LANDING = 54  # the first step whose substep has a box come down on another box
STACK = (0, 1, 2)


def test_world_follows_the_reference_box_world(me):
    g = _golden()
    w = _world(me, g)
    early = {k: 0.0 for k in ("x", "q", "v", "w")}
    stack = {k: 0.0 for k in ("x", "q", "v", "w")}
    for t in range(len(g["contacts"])):
        w.step()
        if t < FIRST_LANDING:
            assert w.n_contacts == int(g["contacts"][t]), (t, w.n_contacts, int(g["contacts"][t]))
        x, q, v, om = w.get_state()
        for k, a in (("x", x), ("q", q), ("v", v), ("w", om)):
            d = np.abs(a - g[k][t])
            if t < FIRST_LANDING:
                early[k] = max(early[k], float(d.max()))
            stack[k] = max(stack[k], float(d[list(STACK)].max()))
    print("box world vs reference: largest |d| before the first landing", early, "; the stack over 90 steps", stack)
    for worst in (early, stack):  # measured: about 1e-11 (x, q), 1e-10 (v), 5e-10 (w)
        assert worst["x"] < 1e-9 and worst["q"] < 1e-9
        assert worst["v"] < 1e-8 and worst["w"] < 1e-8


def test_world_scenes_are_independent(me):
    """Three copies of the scene as three scenes of one world, all overlapping in space: each
    copy moves as the scene alone (scene ids keep their contacts apart).  The copies' contacts
    sit in other colours than the lone scene's, so the sweeps run in another order: both are
    driven to convergence (2000 sweeps) before the states are compared."""
    g = _golden()
    alone = _world(me, g)
    from importlib import import_module
    W = import_module("motion_engine_b200.world")
    many = W.BoxWorldB200(dt=1.0 / 240.0, mu=0.5, iters=2000)
    n = len(g["half"])
    for k in range(3):
        for i in range(n):
            many.add(g["half"][i], float(g["mass"][i]), g["x0"][i], v=g["v0"][i], q=g["q0"][i], scene=k)
    for _ in range(40):
        alone.step()
        many.step()
    xa = alone.get_state()[0]
    xm = many.get_state()[0]
    assert many.n_contacts == 3 * alone.n_contacts
    for k in range(3):
        assert np.abs(xm[k * n:(k + 1) * n] - xa).max() < 1e-9
