"""Derivatives of the exact-cone NCP solve on the device (float64).

* Implicit form (b2c_ncp_adjoint) at the converged impulses, and the recorded form
  (b2c_ncp_sweeps_record + b2c_ncp_adjoint_unrolled) through 4000 sweeps from zero, against the
  reference's own fixed-branch implicit-function sensitivities (ncp_ref.py: classify +
  sensitivity; tests/golden/ncp_sens_golden.npz, tests/golden/make_ncp_sens_golden.py) on its
  well-posed scenes: lam_bar^T dlam/db and lam_bar^T dlam/dmu.
* Recorded form through a few unconverged sweeps against central finite differences of the
  same float64 sweeps, for every input it differentiates: bias, v_free, mu, the Jacobian blocks,
  Minv (through the contact velocities, the velocity changes and the step sizes rho) and the
  warm start.
"""
import importlib
import os
from dataclasses import replace

import numpy as np
import pytest

from conftest import ROOT, cuda_ok
from ncp_scenes import WELLPOSED, scene

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_ok(), reason="needs a CUDA device")]

SENS = os.path.join(ROOT, "tests", "golden", "ncp_sens_golden.npz")


@pytest.fixture(scope="module")
def ncp(me):
    return importlib.import_module("motion_engine_b200.ncp")


def _rel(a, b):
    a, b = np.ravel(a), np.ravel(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("name", WELLPOSED)
def test_adjoints_match_reference_sensitivity(ncp, name):
    g = np.load(SENS)
    bs = scene(name, ncp.BlockScene)
    n_c = bs.n_c
    rng = np.random.default_rng(5)
    lb = rng.normal(size=(n_c, 3))
    want_b = g[f"{name}/dlam_db"].T @ lb.ravel()
    want_mu = g[f"{name}/dlam_dmu"].T @ lb.ravel()
    J = bs.jacobian()
    s = ncp.NCPSolverB200(bs.n_b, n_c, dtype="float64")
    s.solve(bs, iters=4000)
    imp = s.vjp_implicit(lb, 4000)
    rec = s.vjp_recorded(bs, lb, 4000)
    for out in (imp, rec):
        assert _rel(out["bias"], want_b) < 1e-8
        assert _rel(out["mu"], want_mu) < 1e-8
        # v_free enters through b = J v_free + bias
        assert _rel(out["vfree"].ravel(), J.T @ out["bias"].ravel()) < 1e-10
    # 4000 sweeps forget where they started
    assert np.abs(rec["lam0"]).max() < 1e-8 * np.abs(lb).max()


def _perturbed(bs, field, d, eps):
    return replace(bs, **{field: np.asarray(getattr(bs, field), np.float64) + eps * d})


def _agrees(an, f, eps, floor):
    """Central differences at eps and eps / 4: their gap bounds the difference's own error (the
    O(eps^2) term and the rounding of the fixed-point velocity sums); the adjoint must sit within
    twice that gap of the finer one, and the gap itself must be small."""
    f1, f2 = f(eps), f(eps / 4)
    gap = abs(f1 - f2)
    return gap <= 1e-3 * max(abs(f2), floor) and abs(an - f2) <= 2 * gap + 1e-9 * max(abs(f2), floor), (an, f1, f2)


@pytest.mark.parametrize("name", WELLPOSED[:2])
def test_recorded_adjoint_matches_finite_differences(ncp, name):
    """d<lam_bar, lam_K>/d(.) for K = 6 sweeps from a warm start, along a random direction of each
    input, against central differences of the same float64 sweeps."""
    bs = scene(name, ncp.BlockScene)
    n_c, n_b = bs.n_c, bs.n_b
    K = 6
    rng = np.random.default_rng(11)
    lb = rng.normal(size=(n_c, 3))
    s = ncp.NCPSolverB200(n_b, n_c, dtype="float64", color_cache=False)
    warm = s.solve(bs, iters=3).lam  # a warm start that is not the solution
    rec = s.vjp_recorded(bs, lb, K, warm=warm)
    sym = lambda m: 0.5 * (m + np.swapaxes(m, -1, -2))
    dirs = {"bias": rng.normal(size=(n_c, 3)), "v_free": rng.normal(size=(n_b, 6)), "mu": rng.normal(size=n_c) * 0.1,
            "Ja": rng.normal(size=(n_c, 3, 6)) * (np.asarray(bs.Ja) != 0),
            "Jb": rng.normal(size=(n_c, 3, 6)) * (np.asarray(bs.Jb) != 0),
            "Minv": sym(rng.normal(size=(n_b, 6, 6))) * 0.1 * np.abs(np.asarray(bs.Minv)).max() * (np.asarray(bs.Minv) != 0)}
    key = {"bias": "bias", "v_free": "vfree", "mu": "mu", "Ja": "Ja", "Jb": "Jb", "Minv": "Minv"}
    floor = 1e-3 * np.abs(lb).max()
    for field, d in dirs.items():
        an = float(np.sum(rec[key[field]] * d))
        f = lambda e: float(np.sum(lb * (s.solve(_perturbed(bs, field, d, e), iters=K, warm=warm).lam -
                                         s.solve(_perturbed(bs, field, d, -e), iters=K, warm=warm).lam)) / (2 * e))
        ok, info = _agrees(an, f, 1e-4, floor)
        assert ok, (field, info)
    dw = rng.normal(size=(n_c, 3)) * 0.01
    an = float(np.sum(rec["lam0"] * dw))
    f = lambda e: float(np.sum(lb * (s.solve(bs, iters=K, warm=warm + e * dw).lam -
                                     s.solve(bs, iters=K, warm=warm - e * dw).lam)) / (2 * e))
    ok, info = _agrees(an, f, 1e-4, floor)
    assert ok, ("warm", info)
