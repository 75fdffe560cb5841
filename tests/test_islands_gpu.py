"""The island solve on the GPU (IslandSolveContactEngine, contact_engine_gpu_island_solve.py:
7-34, 253-287): the device partition against the oracle's, and the engine against the
reference's golden ColorCache arrays, the CPU oracle and the ColorCache engine, bit for bit --
the reference's island engine gives its ColorCache bits (its island probe's exact_reference
gate), so the ColorCache oracle is the island engine's oracle too."""
import hashlib

import numpy as np
import pytest

from conftest import DIMS, DT, SCENES, lattice, stack

pytestmark = pytest.mark.gpu
NAMES = ("xc", "Rm", "vc", "om", "force")


def _random_graph(rng, n, P, static_frac=0.15, ground_frac=0.1, chain=0):
    mass = np.where(rng.random(n) < static_frac, 0.0, rng.uniform(0.1, 2.0, n))
    a = rng.integers(0, n, P)
    b = rng.integers(0, n, P)
    b[rng.random(P) < ground_frac] = -1
    if chain:  # a long chain of dynamic bodies: one island of `chain` links
        idx = np.flatnonzero(mass > 0)[:chain + 1]
        a[:chain], b[:chain] = idx[:-1], idx[1:]
    return a, b, mass, rng.permutation(P)


@pytest.mark.parametrize("case", ["known", "sparse", "dense", "chain", "all_static"])
def test_device_partition_equals_oracle(case, me):
    from oracle.oracle_islands import partition_pairs as oracle_partition
    rng = np.random.default_rng(7)
    if case == "known":
        args = (np.array([0, 1, 0, 2]), np.array([3, 3, 1, -1]), np.array([1., 1., 1., 0.]), np.array([3, 1, 0, 2]))
    elif case == "sparse":
        args = _random_graph(rng, 5000, 3000)
    elif case == "dense":
        args = _random_graph(rng, 800, 6000)
    elif case == "chain":
        args = _random_graph(rng, 6000, 5000, static_frac=0.05, chain=3000)
    else:
        a, b, _, order = _random_graph(rng, 500, 700)
        args = (a, b, np.zeros(500), order)
    got = me.partition_pairs(*args)
    want = oracle_partition(*args)
    for g, w, name in zip(got, want, ("packed", "starts", "counts")):
        assert np.array_equal(g, w), f"{case}: {name} differs from the oracle"


def _engines(me, scene, **kw):
    kw.setdefault("dims", DIMS)
    kw.setdefault("mu", 0.5)
    isl = me.IslandSolveContactEngine(**kw)
    cc = me.ColorCacheContactEngine(**kw)
    for c in scene:
        isl.add_body(c)
        cc.add_body(c)
    return isl, cc


@pytest.mark.parametrize("scene", ["stack8", "lattice1000"])
def test_island_engine_against_reference(scene, golden, me):
    """The reference's golden ColorCache arrays (cross_hardware_l4), bit for bit while the
    ColorCache engine is bit-exact to them."""
    make, steps = SCENES[scene]
    e = me.IslandSolveContactEngine(dims=DIMS, mu=0.5, vit=40, pit=10)
    for c in make():
        e.add_body(c)
    dig = golden[f"color_cache__{scene}__digest"]
    contacts = golden[f"color_cache__{scene}__contacts"]
    exact = {"stack8": 100, "lattice1000": 40}[scene]
    for t in range(min(steps, exact)):
        e.step(DT, 1)
        assert e.island_solve_active
        assert e.n_contacts == contacts[t]
        st = e.get_state()
        got = [hashlib.sha256(np.ascontiguousarray(a).tobytes()).digest()
               for a in (st.xc, st.Rm, st.vc, st.om, e.contact_forces())]
        for k, n in enumerate(NAMES):
            assert got[k] == dig[t, k].tobytes(), f"{scene} step {t}: {n} differs from the reference"


def test_island_engine_matches_oracle(me, oracle_mod):
    """Jittered 3-high columns of mixed density, two substeps: bitwise the ColorCache oracle."""
    rng = np.random.default_rng(3)
    centers, dens = [], []
    for ix in range(3):
        for iy in range(3):
            base = np.array([ix * 0.33, iy * 0.33, 0.0]) + np.r_[rng.uniform(-0.02, 0.02, 2), 0]
            for k in range(3):
                centers.append(list(base + [rng.uniform(-0.03, 0.03), rng.uniform(-0.03, 0.03),
                                            0.101 + 0.205 * k + rng.uniform(0, 0.01)]))
                dens.append(float(rng.uniform(300, 1500)))
    e = me.IslandSolveContactEngine(dims=DIMS, mu=0.6, vit=16, pit=10)
    o = oracle_mod.ColoredOracle(mode="color_cache", dims=DIMS, mu=0.6, vit=16, pit=10)
    for c, d in zip(centers, dens):
        e.add_body(c, density=d)
        o.add_body(c, density=d)
    for t in range(60):
        e.step(DT, 2)
        o.step(DT, 2)
        se, so = e.get_state(), o.get_state()
        for n in ("xc", "Rm", "vc", "om"):
            a, b = getattr(se, n), getattr(so, n)
            assert a.tobytes() == b.tobytes(), f"step {t} {n}: max |d| {np.abs(a - b).max():.3e}"
        assert e.contact_forces().tobytes() == o.contact_forces().tobytes()
    packed, starts, counts = _pairs_partition(e)
    assert e.island_solve_active and e.island_count == len(counts) > 1


def _pairs_partition(e):
    from oracle.oracle_islands import partition_pairs as oracle_partition
    h = e.header_dict()
    P = h["n_pairs"]
    pb = e.p_bufs
    a = pb["pbi"][:P].cpu().numpy()
    b = pb["pbj"][:P].cpu().numpy()
    order = pb["porder"][:P].cpu().numpy()
    return oracle_partition(a, b, e.invM.cpu().numpy(), order)


def _pressed_stack(K):
    return [[0.0, 0.0, 0.099 + 0.198 * k] for k in range(K)]


@pytest.mark.parametrize("scene,active", [("lattice", True), ("stack16", True), ("stack70", False),
                                          ("mixed", False)])
def test_island_engine_equals_color_cache(scene, active, me):
    """Island solve (islands of <= 64 pairs) and its fall-back to the colour-phase solve (a
    70-high stack is one island of 70 pairs) give the ColorCache engine's bits, step by step;
    the engine's island statistics equal the oracle partition of its pairs."""
    if scene == "lattice":
        bodies, steps = lattice(1000), 30
    elif scene == "stack16":
        bodies, steps = stack(16), 120
    elif scene == "stack70":  # pressed together (pitch 0.198 < 0.2): one island of 70 pairs from the start
        bodies, steps = _pressed_stack(70), 20
    else:
        bodies, steps = lattice(200) + [[10.0 + c[0], c[1], c[2]] for c in _pressed_stack(66)], 20
    isl, cc = _engines(me, bodies, vit=20, pit=10)
    for t in range(steps):
        isl.step(DT, 2)
        cc.step(DT, 2)
        a, b = isl.get_state(), cc.get_state()
        for n in ("xc", "Rm", "vc", "om"):
            assert getattr(a, n).tobytes() == getattr(b, n).tobytes(), f"{scene} step {t}: {n}"
        assert isl.contact_forces().tobytes() == cc.contact_forces().tobytes()
    packed, starts, counts = _pairs_partition(isl)
    assert isl.island_count == len(counts)
    assert isl.max_island_pairs == int(counts.max())
    assert isl.island_solve_active == active == (int(counts.max()) <= 64)
    assert isl.island_rebuilds == isl.color_cache_misses >= 1


def test_island_engine_runs_repeat_bit_identical(me):
    runs = []
    for _ in range(2):
        e = me.IslandSolveContactEngine(dims=DIMS, mu=0.5, vit=16, pit=8)
        for c in lattice(600):
            e.add_body(c)
        for _ in range(25):
            e.step(DT, 2)
        runs.append(e.get_state())
    for n in ("xc", "Rm", "vc", "om"):
        assert getattr(runs[0], n).tobytes() == getattr(runs[1], n).tobytes(), n


def _box_pair(me, sc, islands_kw, **kw):
    engines = []
    for isl in (True, False):
        e = me.BoxContactEngine(mu=0.6, vit=16, pit=10, islands=isl, **kw)
        for c, d, m, de in zip(sc["centers"], sc["dims"], sc["mu"], sc["density"]):
            e.add_box(c, dims=d, density=de, mu=m)
        engines.append(e)
    return engines


@pytest.mark.parametrize("scene,active", [("stress_lattice", True), ("pile", False)])
def test_box_engine_island_solve_equals_colour_phases(scene, active, me):
    """The box engine's row form with the island solve: a stress-style cube lattice that falls
    into separate columns (islands of a few pairs: the island kernel runs) and a random pile (one
    island above 64 pairs: the colour phases run) give the bits of the engine without it."""
    from importlib import import_module
    scenes = import_module("motion_engine_b200.scenes")
    if scene == "stress_lattice":
        sc = scenes.box_lattice(n=600, edge=0.25, extent=(10.0, 10.0, 2.0))
        steps = 90
    else:
        sc = scenes.jittered_boxes(300, height=3.0, rng=np.random.default_rng(5))
        steps = 240
    isl, ref = _box_pair(me, sc, True)
    for t in range(steps):
        isl.step(1 / 240, 2)
        ref.step(1 / 240, 2)
        a, b = isl.get_state_packed().numpy(), ref.get_state_packed().numpy()
        assert a.tobytes() == b.tobytes(), f"{scene} step {t}"
    assert isl.contact_forces().tobytes() == ref.contact_forces().tobytes()
    assert isl.island_solve_active == active
    assert isl.island_count > (50 if active else 0)


def test_device_partition_equals_the_reference_partition(me):
    """The device partition against the reference's own partition_pairs outputs
    (tests/golden/islands_golden.npz), array for array."""
    import os
    from conftest import ROOT
    g = np.load(os.path.join(ROOT, "tests", "golden", "islands_golden.npz"))
    for k in range(int(g["n_cases"])):
        args = [g[f"c{k}/{x}"] for x in ("a", "b", "mass", "order")]
        got = me.partition_pairs(*args)
        for arr, name in zip(got, ("packed", "starts", "counts")):
            assert np.array_equal(arr, g[f"c{k}/{name}"]), (k, name)
