"""The batched ADMM oracle (oracle/oracle_badmm.py, the reference's BatchProxADMMGPU restated in
numpy) pinned on the CPU: its grad_affine against the reference's own implicit sensitivities
(ncp_ref.sensitivity, golden vectors made by the reference's code), on the all-slip scenes of the
reference's batched-adjoint test (its bar: 1e-9) and the random / tripod scenes; its forward
against the reference's converged PGS impulses; the int64 accumulation order-free."""
import numpy as np
import pytest

from conftest import ROOT

import os

from oracle.oracle_badmm import BatchADMMOracle, proj, round_away

ADMM = os.path.join(ROOT, "tests", "golden", "admm_golden.npz")
SENS = os.path.join(ROOT, "tests", "golden", "sens_golden.npz")


def _scene_batch(G, b, mu, B):
    n = len(b)
    return BatchADMMOracle(np.tile(np.eye(n), (B, 1, 1)), np.tile(G, (B, 1, 1)), np.tile(b, (B, 1)),
                           np.tile(mu, B), 0.01)


@pytest.mark.parametrize("n_c", [1, 2, 4, 8])
def test_all_slip_grad_affine_matches_the_reference_ift(n_c):
    """tests/test_ncp_batch_adjoint.py's procedure: one problem per b-direction, the impulses
    from the reference's PGS, u = G lam + b, dlam/db against ncp_ref.sensitivity within 1e-9."""
    g = np.load(ADMM)
    name = f"all_slip_{n_c}"
    G, b, mu, lam, db = (g[f"{name}/{k}"] for k in ("G", "b", "mu", "lam", "db"))
    n = len(b)
    o = _scene_batch(G, b, mu, n)
    d = o.grad_db(np.tile(lam, (n, 1)), np.tile(G @ lam + b, (n, 1)), np.eye(n), cg=60)
    assert (o.nslip == n_c).all()
    assert np.abs(d.reshape(n, n).T - db).max() <= 1e-9


def test_grad_affine_matches_the_reference_on_its_scenes():
    s = np.load(SENS)
    checked = 0
    for name in s["names"]:
        G, b, mu, lam, db, sing = (s[f"{name}/{k}"] for k in ("G", "b", "mu", "lam", "db", "singular"))
        if int(sing) or not np.isfinite(db).all():
            continue
        n = len(b)
        o = _scene_batch(G, b, mu, n)
        d = o.grad_db(np.tile(lam, (n, 1)), np.tile(G @ lam + b, (n, 1)), np.eye(n), cg=120)
        scale = max(1.0, np.abs(db).max())
        assert np.abs(d.reshape(n, n).T - db).max() <= 1e-9 * scale, name
        checked += 1
    assert checked >= 10


def test_forward_reaches_the_reference_impulses():
    s = np.load(SENS)
    for name in ("random_3", "random_7", "random_11", "random6_21", "tripod"):
        G, b, mu, lam = (s[f"{name}/{k}"] for k in ("G", "b", "mu", "lam"))
        o = _scene_batch(G, b, mu, 1).set_rho("regime")
        o.forward(n_iter=400, cg_iters=8, refresh_every=4, tol=1e-12)
        assert np.abs(o.lam[0].ravel() - lam).max() < 1e-6 * max(1.0, np.abs(lam).max()), name


def test_projection_and_rounding():
    mu = np.array([0.5, 0.5, 0.5])
    z = np.array([[1.0, 0.2, 0.1], [-1.0, 0.1, 0.0], [0.1, 1.0, 0.0]])
    p = proj(z, mu)
    assert np.array_equal(p[0], z[0]) and np.array_equal(p[1], np.zeros(3))
    assert np.isclose(np.hypot(p[2, 1], p[2, 2]), 0.5 * p[2, 0])
    assert np.array_equal(round_away(np.array([0.5, -0.5, 1.5, -2.5, 0.49])), [1.0, -1.0, 2.0, -3.0, 0.0])


def test_int64_products_do_not_depend_on_the_contact_order():
    """M^-1 J^T x summed in int64: permuting the contacts (rows of J and entries of x together)
    leaves w bit for bit."""
    rng = np.random.default_rng(3)
    B, C, NV = 4, 4, 18
    J = rng.standard_normal((B, 3 * C, NV))
    A = rng.standard_normal((B, NV, NV))
    Minv = np.linalg.inv(A @ A.transpose(0, 2, 1) + NV * np.eye(NV))
    x = rng.standard_normal((B, C, 3))
    o = BatchADMMOracle(J, Minv, rng.standard_normal((B, NV)), 0.5, 0.01)
    o.matvec(x, False)
    w0 = o.wv.copy()
    perm = rng.permutation(C)
    Jp = J.reshape(B, C, 3, NV)[:, perm].reshape(B, 3 * C, NV)
    o2 = BatchADMMOracle(Jp, Minv, np.zeros((B, NV)), 0.5, 0.01)
    o2.kap = o.kap
    o2.matvec(x[:, perm], False)
    assert o2.wv.tobytes() == w0.tobytes()
