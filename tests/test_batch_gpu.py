"""Batched box engine on the GPU: bitwise against the oracle's batch, each scene's slice bytewise
the scene advanced alone on the GPU, and the autotuner's launch forms leave results unchanged."""
import importlib

import numpy as np
import pytest

from conftest import cuda_ok

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_ok(), reason="needs a CUDA device")]

DT = 1 / 240


def _scenes(k, nmax, seed=9):
    sc = importlib.import_module("motion_engine_b200.scenes")
    return sc.batched_scenes(n_scenes=k, nmin=6, nmax=nmax, seed_n=seed)


def _state(e):
    s = e.get_state()
    return s.xc, s.Rm, s.vc, s.om


def test_batch_matches_oracle_batch(me, oracle_mod):
    scenes = _scenes(6, 80)
    g = me.BatchedBoxEngine(scenes, mu=0.55, vit=8, pit=5)
    o = oracle_mod.BoxOracle(mu=0.55, vit=8, pit=5)
    for k, s in enumerate(scenes):
        for c, d, de, m in zip(s["centers"], s["dims"], s["density"], s["mu"]):
            o.add_box(c, dims=d, density=de, mu=m, scene=k)
    for step in range(100):
        g.step(DT, 2)
        o.step(DT, 2)
    h, st = g.check_errors(), o.stats()
    assert (h["n_contacts"], h["n_pairs"], h["n_colors"]) == (st["n_contacts"], st["n_pairs"], st["n_colors"])
    for a, b in zip(_state(g), _state(o)):
        np.testing.assert_array_equal(a, b)


def test_batch_slice_equals_scene_alone(me):
    scenes = _scenes(16, 300, seed=4)
    g = me.BatchedBoxEngine(scenes, mu=0.55, vit=16, pit=10)
    alone = []
    for s in scenes:
        e = me.BoxContactEngine(mu=0.55, vit=16, pit=10, cand_per_body=12)
        for c, d, de, m in zip(s["centers"], s["dims"], s["density"], s["mu"]):
            e.add_box(c, dims=d, density=de, mu=m)
        alone.append(e)
    for _ in range(120):
        g.step(DT, 2)
        for e in alone:
            e.step(DT, 2)
    g.check_errors()
    for k, e in enumerate(alone):
        e.check_errors()
        sb = g.scene_state(k)
        for a, b in zip((sb.xc, sb.Rm, sb.vc, sb.om), _state(e)):
            np.testing.assert_array_equal(a, b)


def test_autotune_keeps_results(me):
    scenes = _scenes(24, 400, seed=2)
    a = me.BatchedBoxEngine(scenes, mu=0.55, vit=16, pit=10)
    b = me.BatchedBoxEngine(scenes, mu=0.55, vit=16, pit=10)
    for _ in range(20):
        a.step(DT, 2)
        b.step(DT, 2)
    best, times = me.autotune(a, DT, 2, steps=1)
    assert best in times and len(times) == 5 and me._lib.SOLVE_SCENES in times
    for _ in range(sum(1 + 1 for _ in times)):  # the tuner advanced a by 2 steps per candidate
        b.step(DT, 2)
    for _ in range(10):
        a.step(DT, 2)
        b.step(DT, 2)
    for x, y in zip(_state(a), _state(b)):
        np.testing.assert_array_equal(x, y)


def test_scene_schedule_same_bits(me):
    """One CTA per scene (the scene schedule) gives the bits of the grid and cluster forms: the
    scenes share no bodies and each keeps its colour order."""
    scenes = _scenes(24, 400, seed=11)
    runs = []
    for form in (148, -16, me._lib.SOLVE_SCENES):
        g = me.BatchedBoxEngine(scenes, mu=0.55, vit=16, pit=10)
        g.set_solve_blocks(form)
        for _ in range(120):
            g.step(DT, 2)
        g.check_errors()
        runs.append(g.get_state_packed().numpy().tobytes())
    assert runs[0] == runs[1] == runs[2]
    alone = me.BoxContactEngine(mu=0.55, vit=16, pit=10, cand_per_body=12)
    with pytest.raises(ValueError, match="scene schedule"):
        for c, d, de, m in zip(scenes[0]["centers"], scenes[0]["dims"], scenes[0]["density"], scenes[0]["mu"]):
            alone.add_box(c, dims=d, density=de, mu=m)
        alone.step(DT, 2)
        alone.set_solve_blocks(me._lib.SOLVE_SCENES)
