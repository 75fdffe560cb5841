"""Float32 tolerances stated against an FP64 re-solve (tests/fp64.py): one substep of the float32
oracle -- bitwise the CUDA kernels -- repeated in float64 on the same inputs.

Bounds asserted here, after the stated iterations:
  * impulses jn, jt1, jt2, jp: within 1e-5 of the row's largest FP64 magnitude;
  * velocities: within 1e-5 g dt (bead lattice) and 1e-3 g dt (box piles, whose stacked boxes
    of up to 27x the lightest one's mass carry larger impulses into the same float32 velocity
    words); angular velocities ten times that, in rad/s.
The measured figures are printed (pytest -s) and quoted beside these bounds in the design notes."""
import importlib

import numpy as np

from conftest import DIMS, DT, lattice
from fp64 import compare, resolve_from_store, resolve_injected

IMPULSE_BOUND = 1e-5


def test_color_cache_lattice_against_fp64_resolve(oracle_mod):
    mk = lambda p: oracle_mod.ColoredOracle(mode="color_cache", dims=DIMS, mu=0.5, vit=40, pit=20, precision=p)
    e = mk("float32")
    for c in lattice(1000):
        e.add_body(c)
    for _ in range(39):
        e.step(DT, 1)
    st = e.body_state()
    e.step(DT, 1)

    def make64():
        o = mk("float64")
        for c in lattice(1000):
            o.add_body(c)
        return o
    o = resolve_injected(make64, st, e.kept_contacts(), e.pre_solve_impulses(), DT)
    r = compare(e.kept_contacts(), e.body_state(), o.kept_contacts(), o.body_state(), 9.81 * DT)
    print("lattice1000 vs FP64 re-solve:", r)
    assert r["matched"] == 1.0
    for f in ("jn", "jt1", "jt2", "jp"):
        assert r[f] <= IMPULSE_BOUND, (f, r[f])
    assert r["v"] <= 1e-5 and r["w"] <= 1e-4


def test_box_pile_against_fp64_resolve(me, oracle_mod):
    sc = importlib.import_module("motion_engine_b200.scenes").random_boxes(n=300, box=(5.0, 5.0, 4.0))

    def mk(p):
        o = oracle_mod.BoxOracle(mu=0.5, vit=16, pit=10, precision=p)
        for c, d, m, de in zip(sc["centers"], sc["dims"], sc["mu"], sc["density"]):
            o.add_box(c, dims=d, density=de, mu=m)
        return o
    e = mk("float32")
    for _ in range(2 * 239 + 1):  # 240 steps of 2 substeps, the last substep re-solved
        e.step(DT / 2, 1)
    st, wm = e.body_state(), e.warm_store()
    e.step(DT / 2, 1)
    o = resolve_from_store(lambda: mk("float64"), st, wm, DT / 2)
    r = compare(e.kept_contacts(), e.body_state(), o.kept_contacts(), o.body_state(), 9.81 * DT / 2)
    print("box pile vs FP64 re-solve:", r)
    assert r["matched"] == 1.0
    for f in ("jn", "jt1", "jt2", "jp"):
        assert r[f] <= IMPULSE_BOUND, (f, r[f])
    assert r["v"] <= 1e-3 and r["w"] <= 1e-2


def test_fp64_build_is_the_same_algorithm(me, oracle_mod):
    """The float64 build follows the float32 one: over the first steps of a box drop (the first
    ground contacts, no box-box contact yet, no contact set that a rounding can change) the two
    trajectories agree to float32 rounding."""
    sc = importlib.import_module("motion_engine_b200.scenes").random_boxes(n=300, box=(5.0, 5.0, 4.0))
    a, b = (oracle_mod.BoxOracle(mu=0.5, vit=16, pit=10, precision=p) for p in ("float32", "float64"))
    for c, d, m, de in zip(sc["centers"], sc["dims"], sc["mu"], sc["density"]):
        a.add_box(c, dims=d, density=de, mu=m)
        b.add_box(c, dims=d, density=de, mu=m)
    for _ in range(30):
        a.step(DT, 2)
        b.step(DT, 2)
    assert a.stats()["n_kept"] == b.stats()["n_kept"] > 0
    sa, sb = a.body_state(), b.body_state()
    assert np.abs(sa[0].astype(np.float64) - sb[0]).max() < 1e-6
    assert np.abs(sa[2].astype(np.float64) - sb[2]).max() < 1e-5
