"""The CPU oracle against the reference's golden arrays (reports/cross_hardware_l4.npz):
relaxed Jacobi must be bit-exact at every step (xc, Rm, vc, om, contact forces) and produce
the receipt's raw contact counts; the host body setup must reproduce the receipt's initial
array fingerprints."""
import hashlib

import numpy as np
import pytest

from conftest import DIMS, DT, SCENES

NAMES = ("xc", "Rm", "vc", "om", "force")


def _digests(state, force):
    arrs = (state.xc, state.Rm, state.vc, state.om, force)
    return [hashlib.sha256(np.ascontiguousarray(a).tobytes()).digest() for a in arrs]


@pytest.mark.parametrize("scene", ["stack8", "lattice1000"])
def test_oracle_jacobi_bit_exact(scene, golden, oracle_mod):
    make, steps = SCENES[scene]
    e = oracle_mod.JacobiOracle(dims=DIMS, mu=0.5, vit=40, pit=10)
    for c in make():
        e.add_body(c)
    dig = golden[f"jacobi__{scene}__digest"]
    contacts = golden[f"jacobi__{scene}__contacts"]
    for t in range(steps):
        e.step(DT, 1)
        assert e.n_contacts == contacts[t], f"step {t}: contact count"
        got = _digests(e.get_state(), e.contact_forces())
        for k, n in enumerate(NAMES):
            assert got[k] == dig[t, k].tobytes(), f"{scene} step {t}: {n} differs from the reference"


def test_oracle_initial_arrays(golden, oracle_mod):
    from conftest import stack
    b = oracle_mod.build_bodies(stack(8), [700.0] * 8, [0] * 8, DIMS)
    arrays = dict(xc=b.xc, q=b.q, v=b.v, w=b.w, invM=b.invM, IbInv=b.IbInv, rest=b.rest)
    for n, a in arrays.items():
        assert hashlib.sha256(np.ascontiguousarray(a).tobytes()).digest() == \
            golden[f"initial__jacobi__stack8__{n}"].tobytes(), n


def test_product_host_setup_matches_reference(golden, me):
    """The product's numpy body setup (host side of the engine) reproduces the reference's
    built arrays byte for byte."""
    from conftest import lattice, stack
    for scene, centers in (("stack8", stack(8)), ("lattice1000", lattice(1000))):
        A = me.engine.body_arrays(centers, [700.0] * len(centers), [0] * len(centers), DIMS)
        for n in ("xc", "q", "v", "w", "invM", "IbInv", "rest"):
            assert hashlib.sha256(np.ascontiguousarray(A[n]).tobytes()).digest() == \
                golden[f"initial__jacobi__{scene}__{n}"].tobytes(), (scene, n)


def test_oracle_quat_to_R_matches_golden(golden, me):
    """Host quaternion -> matrix of get_state: identity quaternions give the golden Rm."""
    q = np.tile(np.array([0, 0, 0, 1], np.float32), (8, 1))
    assert me.quat_to_R(q).tobytes() == golden["jacobi__stack8__Rm"][0].tobytes()
