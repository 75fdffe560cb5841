"""Relaxed-Jacobi engine on the GPU: bit-exact against the reference's golden arrays and the
CPU oracle, bit-identical run to run and captured vs uncaptured, and the reference's own
contract checks (contact_engine_gpu.py:303-345)."""
import hashlib

import numpy as np
import pytest

from conftest import DIMS, DT, SCENES, lattice, stack

pytestmark = pytest.mark.gpu
NAMES = ("xc", "Rm", "vc", "om", "force")


def _digests(state, force):
    arrs = (state.xc, state.Rm, state.vc, state.om, force)
    return [hashlib.sha256(np.ascontiguousarray(a).tobytes()).digest() for a in arrs]


def _engine(me, centers, **kw):
    e = me.RelaxedJacobiContactEngine(dims=kw.pop("dims", DIMS), mu=kw.pop("mu", 0.5), **kw)
    for c in centers:
        e.add_body(c)
    return e


@pytest.mark.parametrize("scene", ["stack8", "lattice1000"])
def test_jacobi_bit_exact_to_reference(scene, golden, me):
    make, steps = SCENES[scene]
    e = _engine(me, make(), vit=40, pit=10)
    dig = golden[f"jacobi__{scene}__digest"]
    contacts = golden[f"jacobi__{scene}__contacts"]
    for t in range(steps):
        e.step(DT, 1)
        assert e.n_contacts == contacts[t], f"step {t}: contact count {e.n_contacts} != {contacts[t]}"
        got = _digests(e.get_state(), e.contact_forces())
        for k, n in enumerate(NAMES):
            assert got[k] == dig[t, k].tobytes(), f"{scene} step {t}: {n} differs from the reference"


def _random_scene(seed, n_cols=3):
    rng = np.random.default_rng(seed)
    centers, dens = [], []
    for ix in range(n_cols):
        for iy in range(n_cols):
            base = np.array([ix * 0.33, iy * 0.33, 0.0]) + np.r_[rng.uniform(-0.02, 0.02, 2), 0]
            for k in range(3):
                centers.append(list(base + [rng.uniform(-0.03, 0.03), rng.uniform(-0.03, 0.03),
                                            0.101 + 0.205 * k + rng.uniform(0, 0.01)]))
                dens.append(float(rng.uniform(300, 1500)))
    return centers, dens


@pytest.mark.parametrize("seed", [0, 1])
def test_jacobi_matches_oracle_on_random_piles(seed, me, oracle_mod):
    """Jittered 3x3 columns of 3 boxes with mixed densities: off-centre contacts, rotations,
    body-body contacts across columns.  Bit-exact against the CPU oracle every step."""
    centers, dens = _random_scene(seed)
    e = me.RelaxedJacobiContactEngine(dims=DIMS, mu=0.6, vit=12, pit=6)
    o = oracle_mod.JacobiOracle(dims=DIMS, mu=0.6, vit=12, pit=6)
    for c, d in zip(centers, dens):
        e.add_body(c, density=d)
        o.add_body(c, density=d)
    for t in range(80):
        e.step(DT, 2)
        o.step(DT, 2)
        se, so = e.get_state(), o.get_state()
        assert e.n_contacts == o.n_contacts, f"step {t}"
        for n in ("xc", "Rm", "vc", "om"):
            a, b = getattr(se, n), getattr(so, n)
            assert a.tobytes() == b.tobytes(), f"seed {seed} step {t} {n}: max |d| {np.abs(a - b).max():.3e}"
        assert e.contact_forces().tobytes() == o.contact_forces().tobytes()


def test_jacobi_graph_equals_eager_and_runs_repeat(me):
    runs = []
    for graph in (True, False, True):
        e = _engine(me, lattice(200), vit=20, pit=10, graph=graph)
        for _ in range(40):
            e.step(DT, 2)
        runs.append(e.get_state())
    for r in runs[1:]:
        for n in ("xc", "Rm", "vc", "om"):
            assert getattr(r, n).tobytes() == getattr(runs[0], n).tobytes(), n


def test_protocol_and_contract_checks(me):
    """contact_engine_gpu.py:303-345: K=8 stack stable, resting force = Mg, set_kinematic."""
    e = _engine(me, stack(8))
    assert isinstance(e, me.ContactEngine)
    for _ in range(400):
        e.step(1 / 240)
    st = e.get_state()
    ke = float(np.sum(0.5 * e._M[:, None] * st.vc ** 2))
    zs = sorted(st.xc[:, 2])
    seps = [zs[i + 1] - zs[i] for i in range(7)]
    assert ke < 0.5 and all(0.15 < s < 0.25 for s in seps)
    e2 = _engine(me, [[0, 0, 0.101]])
    for _ in range(200):
        e2.step(1 / 240)
    Fz = e2.contact_forces()[0, 2]
    Mg = e2._M[0] * 9.81
    assert abs(Fz - Mg) / Mg * 100 < 8
    e3 = _engine(me, [[0, 0, 0.5]])
    e3.set_kinematic(0, [0, 0, 0.5])
    for _ in range(120):
        e3.step(1 / 240)
    z_stay = e3.get_state().xc[0, 2]
    e3.set_kinematic(0, [0.1, 0, 0.5])
    e3.step(1 / 240)
    assert abs(z_stay - 0.5) < 1e-6 and abs(e3.get_state().xc[0, 0] - 0.1) < 1e-6
    assert e3.contact_forces()[0].tolist() == [0.0, 0.0, 0.0]


def test_contact_capacity_overflow_raises(me):
    """The reference silently truncates at _MAXC (contact_engine_gpu.py:264); here the overflow
    is an error bit in the device header and the host raises on the next call."""
    e = _engine(me, stack(4), contact_capacity=5)
    for _ in range(3):
        e.step(DT)
    e.step(DT)  # first step with 9 ground contacts
    with pytest.raises(RuntimeError, match="capacity"):
        e.step(DT)


def test_unit_cube_stack16_matches_oracle_and_reports_m5(me, oracle_mod):
    """The plain relaxed-Jacobi workload of 16 unit cubes (1 m, 1 kg: 1000 beads each; seeded 1 mm
    xy jitter), mu 0.5, 40 / 20 iterations, 240 steps: bitwise against the oracle at every step,
    and the reference's M5 penetration series computed from the same trajectory.

    The series is the oracle's too, so no target is asserted: with 100 coplanar bead contacts
    per face and relax 0.2, one Jacobi iteration over-corrects the face about twentyfold, the
    accumulated-impulse clamp undoes it on the next, and an even iteration count ends where it
    began.  The stack sinks through the ground in the reference's arithmetic as here; the
    figure is reported, not hidden."""
    from importlib import import_module
    scenes, metrics = import_module("motion_engine_b200.scenes"), import_module("motion_engine_b200.metrics")
    e = me.RelaxedJacobiContactEngine(dims=(1.0, 1.0, 1.0), mu=0.5, vit=40, pit=20)
    o = oracle_mod.JacobiOracle(dims=(1.0, 1.0, 1.0), mu=0.5, vit=40, pit=20)
    for c in scenes.unit_cube_stack(16):
        e.add_body(c, density=1.0)
        o.add_body(c, density=1.0)
    pens = []
    for t in range(240):
        e.step(DT, 1)
        o.step(DT, 1)
        se, so = e.get_state(), o.get_state()
        for n in ("xc", "vc", "om", "Rm"):
            assert getattr(se, n).tobytes() == getattr(so, n).tobytes(), f"step {t}: {n}"
        pens.append(metrics.stack_penetration(se.xc[:, 2], 1.0, ground=0.5))
    q = metrics.m5(pens)
    assert q["steps"] == 240 and np.isfinite(q["max_pen_m"])
