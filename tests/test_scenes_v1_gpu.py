"""The reference's canonical contact-scene-v1 problems (data/ncp/scenes, read by scenes_v1.py)
on the device solvers: the rigid body-contact scenes through the exact-cone NCP solver, bit for
bit the oracle's PGS in float64; the floating-base stance and humanoid operators through the
batched ADMM, equal to the ADMM oracle."""
import gzip
import importlib
import json
import os

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu
FILES = os.path.join(ROOT, "tests", "golden", "scenes_v1.json.gz")
RIGID = (0, 1, 2, 3, 4, 5, 6, 7, 13, 14)


@pytest.fixture(scope="module")
def sv1(me):
    return importlib.import_module("motion_engine_b200.scenes_v1")


@pytest.fixture(scope="module")
def package():
    with gzip.open(FILES, "rt") as f:
        return {int(k): v for k, v in json.load(f).items()}


@pytest.mark.parametrize("i", RIGID)
def test_rigid_scene_matches_the_oracle_bitwise(i, sv1, package, oracle_mod):
    ncp = importlib.import_module("motion_engine_b200.ncp")
    bs = sv1.block_scene(sv1.read_scene(package[i]))
    r = ncp.NCPSolverB200(bs.n_b, bs.n_c, dtype="float64").solve(bs, iters=400)
    o = oracle_mod.ncp_solve(bs, 400, dtype="float64")
    assert r.n_colors == o["n_colors"]
    np.testing.assert_array_equal(r.lam, o["lam"])
    np.testing.assert_array_equal(r.v, o["v"])
    assert r.residual == o["residual"]


@pytest.mark.parametrize("i", (0, 6, 7))
def test_well_conditioned_scenes_converge(i, sv1, package):
    ncp = importlib.import_module("motion_engine_b200.ncp")
    sc = sv1.read_scene(package[i])
    bs = sv1.block_scene(sc)
    r = ncp.NCPSolverB200(bs.n_b, bs.n_c, dtype="float64").solve(bs, iters=2000)
    assert r.residual < 1e-8
    u = sc.delassus() @ r.lam.reshape(-1) + sc.b
    assert np.all(r.lam[:, 0] >= 0) and np.all(u.reshape(-1, 3)[:, 0] > -1e-6)


def test_stance_and_humanoid_operators_match_the_admm_oracle(sv1, package):
    from motion_engine_b200 import badmm
    from oracle.oracle_badmm import BatchADMMOracle
    for group in ((15, 16, 18, 19, 20), (17,)):
        scs = [sv1.read_scene(package[i]) for i in group]
        J, Mi, vf, mu, b = sv1.admm_problem(scs)
        B, nv, nc = len(scs), J.shape[2], scs[0].n_c
        s = badmm.BatchProxADMM(B, nv, nc).upload(J, Mi, vf, mu, scs[0].dt, b=b).set_rho("regime")
        s.step_and_grad(400, 8, 4, 1e-10, n_calls=nc + 2, grad_cg=60)
        o = BatchADMMOracle(J, Mi, vf, mu, scs[0].dt, b=b).set_rho("regime").forward(400, 8, 4, 1e-10)
        o.gradient(n_calls=nc + 2, grad_cg=60)
        for dev_t, ref in ((s.lam, o.lam), (s.u, o.u), (s.dlam_tau, o.dlam_tau), (s.dlam_mu, o.dlam_mu)):
            got = dev_t.cpu().numpy()
            assert np.abs(got - ref).max() <= 1e-9 * max(1.0, np.abs(ref).max()), group
        res = s.res.cpu().numpy()
        for k, i in enumerate(group):
            if i in (15, 17, 18):  # the sticking stances and the humanoid converge in 400 iterations
                assert res[k] < 1e-9, (i, res[k])
