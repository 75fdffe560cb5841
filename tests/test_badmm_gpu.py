"""The batched ADMM on the GPU (b2c_admm_solve, the reference's BatchProxADMMGPU,
ncp/ncp_batch_gpu.py:918-1313): its grad_affine against the reference's own implicit
sensitivities with the reference test's procedure and bar, the whole step and gradient against
the ADMM oracle on the legged-stance batch, a problem alone = the same problem in the batch bit
for bit (the reference's claim, NB:41-43), two runs bit-identical."""
import os

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu
ADMM = os.path.join(ROOT, "tests", "golden", "admm_golden.npz")
SENS = os.path.join(ROOT, "tests", "golden", "sens_golden.npz")


def _badmm():
    import __graft_entry__ as ge
    ge.load_package()
    from motion_engine_b200 import badmm
    return badmm


def _given(G, b, mu, lam, cg=60):
    badmm = _badmm()
    n, nc = len(b), len(mu)
    s = badmm.BatchProxADMM(n, n, nc).upload(np.tile(np.eye(n), (n, 1, 1)), np.tile(G, (n, 1, 1)), np.tile(b, (n, 1)),
                                              np.tile(mu, n), 0.01)
    d = s.grad_given(np.tile(lam, (n, 1)), np.tile(G @ lam + b, (n, 1)), np.eye(n).reshape(n, nc, 3), cg=cg)
    return d.reshape(n, n).T, s


@pytest.mark.parametrize("n_c", [1, 2, 4, 8])
def test_all_slip_batched_adjoint_matches_the_reference_ift(n_c):
    g = np.load(ADMM)
    name = f"all_slip_{n_c}"
    G, b, mu, lam, db = (g[f"{name}/{k}"] for k in ("G", "b", "mu", "lam", "db"))
    d1, s = _given(G, b, mu, lam)
    d2, _ = _given(G, b, mu, lam)
    assert (s.nslip.cpu().numpy() == n_c).all()
    assert d1.tobytes() == d2.tobytes(), "two runs differ"
    assert np.abs(d1 - db).max() <= 1e-9


def test_batched_adjoint_matches_the_reference_on_its_scenes():
    s = np.load(SENS)
    for name in s["names"]:
        G, b, mu, lam, db, sing = (s[f"{name}/{k}"] for k in ("G", "b", "mu", "lam", "db", "singular"))
        if int(sing) or not np.isfinite(db).all():
            continue
        d, _ = _given(G, b, mu, lam, cg=120)
        assert np.abs(d - db).max() <= 1e-9 * max(1.0, np.abs(db).max()), name


def _stance(B, seed=8):
    import __graft_entry__ as ge
    me = ge.load_package()
    from importlib import import_module
    return import_module("motion_engine_b200.scenes").stance_batch(B=B, nv=18, nc=4, mu=0.5, seed=seed)


def test_step_and_gradient_match_the_oracle():
    """200 ADMM iterations (regime rho, 8 CG steps, refresh every 4) and both gradient
    directions on 48 sliding-stance problems: the device equals the oracle to 1e-9 of each
    output's scale (the two differ only in summation order; the int64 sums are exact)."""
    from oracle.oracle_badmm import BatchADMMOracle
    badmm = _badmm()
    J, Minv, v, mu = _stance(48)
    s = badmm.BatchProxADMM(48, 18, 4).upload(J, Minv, v, mu, 1 / 240).set_rho("regime")
    s.step_and_grad(200, 8, 4, 1e-8, n_calls=6, grad_cg=60)
    o = BatchADMMOracle(J, Minv, v, mu, 1 / 240).set_rho("regime").forward(200, 8, 4, 1e-8)
    o.gradient(n_calls=6, grad_cg=60)
    assert np.allclose(s.rho.cpu().numpy(), o.rho, rtol=1e-12, atol=0)
    assert np.array_equal(s.labels.cpu().numpy(), o.labels)
    for dev_t, ref in ((s.lam, o.lam), (s.u, o.u), (s.v_plus, o.vplus), (s.dlam_tau, o.dlam_tau),
                       (s.dv_tau, o.dv_tau), (s.dlam_mu, o.dlam_mu)):
        got = dev_t.cpu().numpy()
        assert np.abs(got - ref).max() <= 1e-9 * max(1.0, np.abs(ref).max())
    assert np.array_equal(s.mask.cpu().numpy(), o.mask)


def test_problem_alone_equals_problem_in_batch_and_runs_repeat():
    badmm = _badmm()
    J, Minv, v, mu = _stance(32, seed=5)
    outs = []
    for _ in range(2):
        s = badmm.BatchProxADMM(32, 18, 4).upload(J, Minv, v, mu, 1 / 240).set_rho("regime")
        s.step_and_grad(120, 8, 4, 1e-8, n_calls=6, grad_cg=40)
        outs.append([t.cpu().numpy().copy() for t in (s.lam, s.v_plus, s.dlam_tau, s.dv_tau, s.dlam_mu)])
    for a, b in zip(*outs):
        assert a.tobytes() == b.tobytes()
    for e in (0, 7, 31):
        s1 = badmm.BatchProxADMM(1, 18, 4).upload(J[e:e + 1], Minv[e:e + 1], v[e:e + 1], mu[e:e + 1], 1 / 240)
        s1.set_rho("regime").step_and_grad(120, 8, 4, 1e-8, n_calls=6, grad_cg=40)
        for t, full in zip((s1.lam, s1.v_plus, s1.dlam_tau, s1.dv_tau, s1.dlam_mu), outs[0]):
            assert t.cpu().numpy()[0].tobytes() == full[e].tobytes()


def test_forward_converges_to_the_reference_impulses():
    s_ = np.load(SENS)
    badmm = _badmm()
    for name in ("random_3", "random_7", "random6_21", "tripod"):
        G, b, mu, lam = (s_[f"{name}/{k}"] for k in ("G", "b", "mu", "lam"))
        n, nc = len(b), len(mu)
        s = badmm.BatchProxADMM(1, n, nc).upload(np.eye(n)[None], G[None], b[None], mu[None], 0.01)
        f = s.set_rho("regime").forward(n_iter=400, cg_iters=8, refresh_every=4, tol=1e-12, chunk=400)
        assert np.abs(f.lam[0].ravel() - lam).max() < 1e-6 * max(1.0, np.abs(lam).max()), name
        assert f.resenv[0] < 1e-7


def test_bad_sizes_are_rejected():
    badmm = _badmm()
    with pytest.raises(ValueError):
        badmm.BatchProxADMM(4, 40, 4)
    with pytest.raises(ValueError):
        badmm.BatchProxADMM(4, 18, 9)
