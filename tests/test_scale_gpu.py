"""Parity at the sizes the bench runs, on the GPU.

* The reference's own 10 000-body ColorCache receipt (reports/innovation_color_cache_profile_v2.npz,
  tests/golden/cc10k_golden.npz): ColorCacheContactEngine(dims=(0.3, 0.3, 0.2), mu=0.5, vit=40,
  pit=20) on lattice(10000), 10 + 30 steps (probes/innovation_color_cache_profile_v2.py:18-35).
  The GPU equals the oracle bit for bit; against the receipt, the positions, the selected
  contacts (keys, bodies, points, normals, depths) and the position impulses are bitwise, and the
  velocity impulses, velocities and forces are within the bounds stated below.
* The box engine on the bench's workloads, in lockstep with the oracle: the 10 000-box drop
  (boxes10k) for its 300 set-up steps and 20 more, the first steps of the 100 000-cube stress
  lattice, and the first steps of the 512-scene batch.  Bitwise state and counters.
"""
import hashlib
import importlib

import numpy as np
import pytest

from cc10k import check_cc10k
from conftest import DIMS, DT, cuda_ok, lattice
from fp64 import compare, resolve_from_store

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_ok(), reason="needs a CUDA device")]


def test_color_cache_lattice10k_against_reference_receipt(me, oracle_mod):
    e = me.ColorCacheContactEngine(dims=DIMS, mu=0.5, vit=40, pit=20)
    o = oracle_mod.ColoredOracle(mode="color_cache", dims=DIMS, mu=0.5, vit=40, pit=20)
    for c in lattice(10000):
        e.add_body(c)
        o.add_body(c)
    for _ in range(40):
        e.step(DT, 1)
        o.step(DT, 1)
    se, so = e.get_state(), o.get_state()
    ke, ko = e.kept_contacts(), o.kept_contacts()
    for name in ("xc", "Rm", "vc", "om"):
        assert getattr(se, name).tobytes() == getattr(so, name).tobytes(), f"GPU vs oracle: {name}"
    for k in ko:
        assert ke[k].tobytes() == ko[k].tobytes(), f"GPU vs oracle: kept {k}"
    np.testing.assert_array_equal(e.contact_forces(), o.contact_forces())
    assert (e.color_cache_hits, e.color_cache_misses) == (35, 2)  # the receipt's cache counts
    check_cc10k(se, e.contact_forces(), ke)


def test_island_solve_lattice10k_against_reference_receipt(me):
    """The island engine on the same receipt run: the island kernel takes the solve (5 041
    columns of one or two boxes: islands of at most two pairs), the result is the ColorCache engine's bit for bit and within the
    receipt's bounds (the reference's island engine gives its ColorCache bits, its probe's
    exact_reference gate)."""
    isl = me.IslandSolveContactEngine(dims=DIMS, mu=0.5, vit=40, pit=20)
    cc = me.ColorCacheContactEngine(dims=DIMS, mu=0.5, vit=40, pit=20)
    for c in lattice(10000):
        isl.add_body(c)
        cc.add_body(c)
    for _ in range(40):
        isl.step(DT, 1)
        cc.step(DT, 1)
    assert isl.island_solve_active and isl.island_count == 5041 and isl.max_island_pairs == 2  # 71 x 71 columns
    si, sc = isl.get_state(), cc.get_state()
    for name in ("xc", "Rm", "vc", "om"):
        assert getattr(si, name).tobytes() == getattr(sc, name).tobytes(), name
    ki, kc = isl.kept_contacts(), cc.kept_contacts()
    for k in kc:
        assert ki[k].tobytes() == kc[k].tobytes(), k
    check_cc10k(si, isl.contact_forces(), ki)


def _digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a, np.float32).tobytes())
    return h.hexdigest()


def _box_pair(me, oracle_mod, sc, vit, pit, mu):
    e = me.BoxContactEngine(mu=mu, vit=vit, pit=pit, color_cap=32)
    o = oracle_mod.BoxOracle(mu=mu, vit=vit, pit=pit)
    for c, d, m, de in zip(sc["centers"], sc["dims"], sc["mu"], sc["density"]):
        e.add_box(c, dims=d, density=de, mu=m)
        o.add_box(c, dims=d, density=de, mu=m)
    return e, o


def _gpu_state(e):
    st = e.get_state_packed().numpy()
    return st[0, :, :3], st[1], st[2, :, :3], st[3, :, :3]


def _lockstep(e, o, steps, every, substeps=2):
    for t in range(steps):
        e.step(DT, substeps)
        o.step(DT, substeps)
        if t % every == every - 1 or t == steps - 1:
            assert _digest(*_gpu_state(e)) == _digest(*o.body_state()), f"state differs at step {t}"
            he, ho = e.check_errors(), o.stats()
            for k in ("n_kept", "n_pairs", "n_colors"):
                assert he[k] == ho[k], (t, k, he[k], ho[k])


def test_boxes10k_matches_oracle(me, oracle_mod):
    """The bench's default workload: 10 000 random boxes (edges U[0.2, 0.6], per-body mu
    U[0.3, 0.8]) through the 300 set-up steps in which the pile forms and 20 steps of the timed
    window, 2 substeps x (16 + 10) sweeps, bitwise against the oracle every 20 steps.  Then the
    GPU's next substep against its FP64 re-solve from the GPU's own state and warm store: the
    impulses within 1e-5 of the largest FP64 impulse of their row, velocities within
    1e-3 g dt (the bounds of tests/test_fp64_resolve.py)."""
    sc = importlib.import_module("motion_engine_b200.scenes").random_boxes(n=10000)
    e, o = _box_pair(me, oracle_mod, sc, 16, 10, 0.55)
    _lockstep(e, o, 320, 20)
    assert e.header_dict()["n_kept"] > 30000  # the pile has formed
    st, wm = _gpu_state(e), e.warm_store()
    e.step(DT / 2, 1)

    def make64():
        o64 = oracle_mod.BoxOracle(mu=0.55, vit=16, pit=10, precision="float64")
        for c, d, m, de in zip(sc["centers"], sc["dims"], sc["mu"], sc["density"]):
            o64.add_box(c, dims=d, density=de, mu=m)
        return o64
    o64 = resolve_from_store(make64, st, wm, DT / 2)
    r = compare(e.kept_contacts(), _gpu_state(e), o64.kept_contacts(), o64.body_state(), 9.81 * DT / 2)
    print("boxes10k GPU substep vs FP64 re-solve:", r)
    assert r["matched"] == 1.0
    for f in ("jn", "jt1", "jt2", "jp"):
        assert r[f] <= 1e-5, (f, r[f])
    assert r["v"] <= 1e-3 and r["w"] <= 1e-2


def test_stress100k_first_steps_match_oracle(me, oracle_mod):
    """The 100 000-cube stress lattice (edge 0.25, mu 0.6, 2 substeps x (16 + 16) sweeps): its
    first 80 steps -- the lowest layer on the ground from the start, the upper layers landing on
    it from about step 60 -- bitwise against the oracle every 20 steps."""
    sc = importlib.import_module("motion_engine_b200.scenes").box_lattice(n=100000)
    e, o = _box_pair(me, oracle_mod, sc, 16, 16, 0.6)
    _lockstep(e, o, 80, 20)
    assert e.header_dict()["n_kept"] > 10000


def test_batched512_first_steps_match_oracle(me, oracle_mod):
    """The 512-scene batch (about 180 000 bodies) in one engine: its first steps bitwise equal
    to the oracle run over the same bodies and scene ids."""
    sc = importlib.import_module("motion_engine_b200.scenes")
    scenes = sc.batched_scenes()
    g = me.BatchedBoxEngine(scenes, mu=0.55, vit=16, pit=10, color_cap=32)
    o = oracle_mod.BoxOracle(mu=0.55, vit=16, pit=10)
    for k, s in enumerate(scenes):
        for c, d, de, m in zip(s["centers"], s["dims"], s["density"], s["mu"]):
            o.add_box(c, dims=d, density=de, mu=m, scene=k)
    _lockstep(g, o, 3, 1)
