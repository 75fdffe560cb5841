"""The coloured-chain oracle against the reference's golden arrays (ColorCache and pair-chunk
engines, reports/cross_hardware_l4.npz).  lattice1000: bit-exact for all 40 steps.  stack8:
bit-exact up to the first one-ulp quaternion flip (step 100 ColorCache, step 71 pair chunks),
then within the stated tolerance of the reference's positions."""
import hashlib

import numpy as np
import pytest

from conftest import DIMS, DT, SCENES

NAMES = ("xc", "Rm", "vc", "om", "force")
# (engine, scene): steps that must be bit-exact, absolute xc tolerance afterwards
EXACT = {("color_cache", "stack8"): 100, ("color_cache", "lattice1000"): 40,
         ("pair_chunks", "stack8"): 71, ("pair_chunks", "lattice1000"): 40}
XC_TOL = {"color_cache": 1e-8, "pair_chunks": 1e-6}     # metres, |xc| <= 1.6 m -> relative < 1e-5


def _digests(state, force):
    arrs = (state.xc, state.Rm, state.vc, state.om, force)
    return [hashlib.sha256(np.ascontiguousarray(a).tobytes()).digest() for a in arrs]


@pytest.mark.parametrize("engine", ["color_cache", "pair_chunks"])
@pytest.mark.parametrize("scene", ["stack8", "lattice1000"])
def test_oracle_colored_against_reference(engine, scene, golden, oracle_mod):
    make, steps = SCENES[scene]
    e = oracle_mod.ColoredOracle(mode=engine, dims=DIMS, mu=0.5, vit=40, pit=10)
    for c in make():
        e.add_body(c)
    dig = golden[f"{engine}__{scene}__digest"]
    contacts = golden[f"{engine}__{scene}__contacts"]
    sel = list(golden[f"{engine}__{scene}__steps"])
    exact = EXACT[(engine, scene)]
    for t in range(steps):
        e.step(DT, 1)
        st = e.get_state()
        if t < exact:
            assert e.n_contacts == contacts[t], f"step {t}: contact count"
            got = _digests(st, e.contact_forces())
            for k, n in enumerate(NAMES):
                assert got[k] == dig[t, k].tobytes(), f"{engine} {scene} step {t}: {n} differs"
        elif t in sel:
            g = golden[f"{engine}__{scene}__xc"][sel.index(t)]
            assert np.abs(st.xc.astype(np.float64) - g).max() < XC_TOL[engine], f"step {t}"


def test_oracle_color_cache_lattice10k_against_receipt(oracle_mod):
    """The reference's 10 000-body ColorCache receipt (reports/innovation_color_cache_profile_v2.npz):
    40 steps of lattice(10000), vit 40, pit 20.  Positions, the selected contacts and the
    position impulses are bitwise; the rest within the bounds of tests/cc10k.py.  The receipt
    holds the last step only, so the first step where a velocity bit departs is not visible;
    the contact geometry of step 40 being bitwise says that every position up to step 39 was."""
    from cc10k import check_cc10k, receipt
    from conftest import lattice
    from fp64 import compare, resolve_injected
    e = oracle_mod.ColoredOracle(mode="color_cache", dims=DIMS, mu=0.5, vit=40, pit=20)
    for c in lattice(10000):
        e.add_body(c)
    for _ in range(39):
        e.step(DT, 1)
    before = e.body_state()
    e.step(DT, 1)
    st = e.stats()
    assert (st["n_contacts"], st["n_kept"], st["n_pairs"], st["n_colors"], st["hits"], st["misses"]) == \
        (87716, 40000, 10000, 2, 35, 2)  # the receipt's counts
    kept = e.kept_contacts()
    check_cc10k(e.get_state(), e.contact_forces(), kept)
    # the last step's solve repeated in float64 on the same contacts: this float32 run and the
    # reference's receipt both sit within float32 rounding of it
    def make64():
        o = oracle_mod.ColoredOracle(mode="color_cache", dims=DIMS, mu=0.5, vit=40, pit=20, precision="float64")
        for c in lattice(10000):
            o.add_body(c)
        return o
    o = resolve_injected(make64, before, kept, e.pre_solve_impulses(), DT)
    ours = compare(kept, e.body_state(), o.kept_contacts(), o.body_state(), 9.81 * DT)
    g = receipt()
    ref_state = (g["xc"], None, g["vc"], g["om"])
    theirs = compare({k: g[k] for k in kept}, ref_state, o.kept_contacts(), o.body_state(), 9.81 * DT)
    print("10k lattice vs FP64 re-solve: this run", ours, "the reference's receipt", theirs)
    for r in (ours, theirs):
        assert r["matched"] == 1.0
        for f in ("jn", "jt1", "jt2", "jp"):
            assert r[f] <= 1e-5, (f, r[f])
        assert r["v"] <= 1e-5


def test_oracle_m5_stack16_against_receipt(oracle_mod):
    """The reference's M5 gate on the ColorCache engine (K = 16, vit 40, pit 10, 600 steps):
    PASS, within 5 % of the receipt's max pen / R = 0.19564 (reports/innovation_stack_color_cache_l4.json)."""
    import importlib
    import __graft_entry__ as ge
    ge.load_package()
    metrics = importlib.import_module("motion_engine_b200.metrics")
    e = oracle_mod.ColoredOracle(mode="color_cache", dims=DIMS, mu=0.5, vit=40, pit=10)
    for k in range(16):
        e.add_body([0, 0, 0.101 + k * 0.205])
    pens = []
    for _ in range(600):
        e.step(DT, 1)
        z = np.sort(e.get_state().xc[:, 2])
        pens.append(float(np.max(np.float32(0.205) - np.diff(z))))
    q = metrics.m5(pens)
    assert q["status"] == "PASS"
    assert abs(q["max_pen_over_R"] - 0.19563645124435425) < 0.05 * 0.19563645124435425, q


def test_oracle_reduced_set_keeps_m5_on_the_k8_stack(oracle_mod):
    """GraphColoredContactEngine(manifold_reduce=True) without pair chunks: the reduced set coloured
    contact by contact.  The reference picks vit = 40 for this path as "the lowest of the sweep at
    which the reduced K=8 stack keeps M5" (contact_engine_gpu_colored.py:801-802); the restated
    path keeps M5 there too."""
    import importlib
    import __graft_entry__ as ge
    ge.load_package()
    metrics = importlib.import_module("motion_engine_b200.metrics")
    e = oracle_mod.ColoredOracle(mode="reduced", dims=DIMS, mu=0.5, vit=40, pit=20)
    for k in range(8):
        e.add_body([0, 0, 0.101 + k * 0.205])
    pens = []
    for _ in range(600):
        e.step(DT, 1)
        z = np.sort(e.get_state().xc[:, 2])
        pens.append(float(np.max(np.float32(0.205) - np.diff(z))))
    q = metrics.m5(pens)
    assert q["status"] == "PASS", q
