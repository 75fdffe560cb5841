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
