"""Batched exact-cone NCP and its implicit adjoint on the GPU (b2c_bncp_*): the reference's own
solutions and sensitivities (golden), the oracle, finite differences through torch.autograd,
bit identity and padding invariance, and a 4096-problem batch."""
import importlib
import os

import numpy as np
import pytest

from conftest import cuda_ok

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_ok(), reason="needs a CUDA device")]

G_ = dict(np.load(os.path.join(os.path.dirname(__file__), "golden", "sens_golden.npz")))
NAMES = [str(x) for x in G_["names"]]


def _rel(a, f):
    return float(np.max(np.abs(a - f)) / max(float(np.max(np.abs(f))), 1e-30))


@pytest.fixture(scope="module")
def bn(me):
    return importlib.import_module("motion_engine_b200.bncp")


def _batch(names):
    import torch
    nmax = max(len(G_[f"{n}/b"]) for n in names)
    B = len(names)
    G = np.zeros((B, nmax, nmax)); b = np.zeros((B, nmax)); mu = np.zeros((B, nmax // 3)); nc = np.zeros(B, np.int32)
    for e, n in enumerate(names):
        k = len(G_[f"{n}/b"])
        G[e, :k, :k] = G_[f"{n}/G"]; b[e, :k] = G_[f"{n}/b"]; mu[e, :k // 3] = G_[f"{n}/mu"]; nc[e] = k // 3
    t = lambda a: torch.from_numpy(a).cuda()
    return t(G), t(b), t(mu), t(nc), nmax


def test_solve_and_sensitivity_match_reference(bn):
    G, b, mu, nc, nmax = _batch(NAMES)
    s = bn.BatchNCP(G, b, mu, nc)
    lam = s.solve(20000, 1e-14).cpu().numpy()
    assert (s.iters.cpu().numpy() < 20000).all() and (s.res.cpu().numpy() < 1e-13).all()
    dmu, db = (x.cpu().numpy() for x in s.sensitivity())
    status, labels = s.status.cpu().numpy(), s.labels.cpu().numpy()
    for e, n in enumerate(NAMES):
        k = len(G_[f"{n}/b"])
        if G_[f"{n}/singular"]:
            assert status[e] & 1 and np.isnan(dmu[e, :k, :k // 3]).all() and np.isnan(db[e, :k, :k]).all()
            continue
        assert status[e] == 0, n
        assert np.max(np.abs(lam[e, :k] - G_[f"{n}/lam"])) < 1e-11, n
        np.testing.assert_array_equal(labels[e, :k // 3], G_[f"{n}/labels"])
        assert _rel(dmu[e, :k, :k // 3], G_[f"{n}/dmu"]) < 1e-9, n
        assert _rel(db[e, :k, :k], G_[f"{n}/db"]) < 1e-9, n
        assert _rel(db[e, :k, :k], G_[f"{n}/fd_b"]) < 1e-5, n


def test_vjp_matches_oracle_and_autograd_matches_fd(bn, oracle_mod):
    import torch
    from oracle import oracle_bncp as OB
    names = [n for n in NAMES if not G_[f"{n}/singular"] and len(G_[f"{n}/b"]) == 12]
    G, b, mu, nc, nmax = _batch(names)
    w = torch.from_numpy(np.random.default_rng(1).normal(size=(len(names), nmax))).cuda()
    bb, mm = b.clone().requires_grad_(True), mu.clone().requires_grad_(True)
    lam = bn.ncp_solve(G, bb, mm, 20000, 1e-15)
    (lam * w).sum().backward()
    gb, gmu = bb.grad.cpu().numpy(), mm.grad.cpu().numpy()
    for e, n in enumerate(names):
        ob, om = OB.vjp(G_[f"{n}/lam"], G_[f"{n}/G"], G_[f"{n}/b"], G_[f"{n}/mu"], w[e].cpu().numpy())
        assert _rel(gb[e], ob) < 1e-9 and _rel(gmu[e], om) < 1e-9, n
    # central finite differences of sum(w * lambda) on the GPU solver itself
    h = 1e-6
    fd_b = np.zeros_like(gb)
    for j in range(nmax):
        lp = bn.ncp_solve(G, b + h * torch.eye(nmax, device="cuda", dtype=torch.float64)[j], mu, 20000, 1e-15)
        lm = bn.ncp_solve(G, b - h * torch.eye(nmax, device="cuda", dtype=torch.float64)[j], mu, 20000, 1e-15)
        fd_b[:, j] = ((lp - lm) * w).sum(1).cpu().numpy() / (2 * h)
    for e in range(len(names)):
        assert _rel(gb[e], fd_b[e]) < 1e-5


def test_bit_identity_and_padding_invariance(bn):
    import torch
    G, b, mu, nc, nmax = _batch(NAMES)
    r = []
    for _ in range(2):
        s = bn.BatchNCP(G, b, mu, nc)
        r.append(s.solve(20000, 1e-14).cpu().numpy().tobytes())
    assert r[0] == r[1]
    lam_b = bn.BatchNCP(G, b, mu, nc).solve(20000, 1e-14).cpu().numpy()
    e = NAMES.index("random_7")
    k = len(G_["random_7/b"])
    one = bn.BatchNCP(G[e:e + 1, :k, :k].contiguous(), b[e:e + 1, :k].contiguous(), mu[e:e + 1, :k // 3].contiguous())
    np.testing.assert_array_equal(one.solve(20000, 1e-14).cpu().numpy()[0], lam_b[e, :k])


def test_large_batch_converges(bn):
    import torch
    rng = np.random.default_rng(7)
    B, ncon, nv = 4096, 4, 18
    J = torch.from_numpy(rng.normal(size=(B, 3 * ncon, nv))).cuda()
    Minv = torch.diag_embed(torch.from_numpy(np.exp(rng.uniform(-1, 1, (B, nv)))).cuda())
    vf = torch.from_numpy(rng.normal(size=(B, nv)) * 0.3).cuda()
    vf[:, 2::6] -= 0.5
    G, b = bn.delassus(J, Minv, vf)
    mu = torch.full((B, ncon), 0.4, dtype=torch.float64, device="cuda")
    s = bn.BatchNCP(G, b, mu)
    lam = s.solve(5000, 1e-12)
    it, res = s.iters.cpu().numpy(), s.res.cpu().numpy()
    assert (res[it < 5000] < 1e-12).all() and (it < 5000).mean() > 0.99
    from oracle import oracle_bncp as OB
    for e in (0, 1, 2, 4095):
        ref, _ = OB.pgs(G[e].cpu().numpy(), b[e].cpu().numpy(), mu[e].cpu().numpy(), 20000, 1e-14)
        assert np.max(np.abs(lam[e].cpu().numpy() - ref)) < 1e-9


def test_stance_batch_matches_oracle(bn, oracle_mod):
    """The shape of the batched-adjoint workload (legged stance: a floating base and 4 legs of 3
    joints, nv = 18, 4 contacts, sliding, mu 0.5), 64 problems: the solve and a vector-Jacobian
    product against the oracle's PGS and fixed-branch VJP, problem by problem."""
    import torch
    from importlib import import_module
    from oracle import oracle_bncp as OB
    S = import_module("motion_engine_b200.scenes")
    J, Minv, vf, mu = S.stance_batch(B=64, nv=18, nc=4, mu=0.5)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    G, b = bn.delassus(t(J), t(Minv), t(vf))
    w = t(np.random.default_rng(2).normal(size=tuple(b.shape)))
    bb, mm = b.clone().requires_grad_(True), t(mu).requires_grad_(True)
    lam = bn.ncp_solve(G, bb, mm, 20000, 1e-14)
    (lam * w).sum().backward()
    lam, gb, gm = lam.detach().cpu().numpy(), bb.grad.cpu().numpy(), mm.grad.cpu().numpy()
    Gh, bh = G.cpu().numpy(), b.cpu().numpy()
    checked = 0
    for e in range(64):
        ref, _ = OB.pgs(Gh[e], bh[e], mu[e], 20000, 1e-14)
        assert np.max(np.abs(lam[e] - ref)) < 1e-9, e
        dmu, db, _, status = OB.sensitivity(ref, Gh[e], bh[e], mu[e])
        if status:  # a singular or boundary branch: no derivative (NaN in both)
            continue
        we = w[e].cpu().numpy()
        ob, om = db.T @ we, dmu.T @ we
        assert _rel(gb[e], ob) < 1e-7 and _rel(gm[e], om) < 1e-7, e
        checked += 1
    assert checked >= 48
