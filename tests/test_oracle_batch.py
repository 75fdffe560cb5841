"""The oracle's box step on a batch of scenes: each scene's slice equals the scene stepped
alone, bytewise (scene ids keep scenes apart; the colouring priority is scene-local)."""
import importlib

import numpy as np

import __graft_entry__ as ge
from oracle import oracle as O


def _scenes(k=4):
    ge.load_package()
    sc = importlib.import_module("motion_engine_b200.scenes")
    return sc.batched_scenes(n_scenes=k, nmin=6, nmax=60, seed_n=9)


def _fill(o, s, scene=0):
    for c, d, de, m in zip(s["centers"], s["dims"], s["density"], s["mu"]):
        o.add_box(c, dims=d, density=de, mu=m, scene=scene)


def test_batch_slices_equal_scenes_alone():
    scenes = _scenes()
    batch = O.BoxOracle(mu=0.55, vit=8, pit=5)
    for k, s in enumerate(scenes):
        _fill(batch, s, scene=k)
    alone = []
    for s in scenes:
        o = O.BoxOracle(mu=0.55, vit=8, pit=5)
        _fill(o, s)
        alone.append(o)
    for _ in range(60):
        batch.step(1 / 240, 2)
        for o in alone:
            o.step(1 / 240, 2)
    xb, qb, vb, wb = batch.body_state()
    start = 0
    for o in alone:
        x, q, v, w = o.body_state()
        n = len(x)
        for a, b in ((xb, x), (qb, q), (vb, v), (wb, w)):
            np.testing.assert_array_equal(a[start:start + n], b)
        start += n
    assert batch.stats()["n_colors"] == max(o.stats()["n_colors"] for o in alone)
