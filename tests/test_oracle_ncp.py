"""The oracle's exact-cone NCP solve against the reference's float64 CPU solver (ncp_ref.py
solve_ncp_pgs, driven to convergence; golden fixture made by the reference itself).

Well-posed scenes (3 n_c <= 6 n_b, full-rank J) have a unique lambda: compared in lambda, with
the reference test's bounds (tests/test_ncp_gpu_cone.py:111-127: 1e-6 float64, 1e-5 float32).
The pushed cube and the resting stack are statically indeterminate: lambda is not unique, the
contact velocity u = G lambda + b and the net wrench J^T lambda are (test_ncp_gpu_cone.py:130-153)."""
import numpy as np
import pytest

from ncp_scenes import INDETERMINATE, WELLPOSED, golden, scene, with_sep
from oracle import oracle as O

ITERS = 5000


@pytest.mark.parametrize("name", WELLPOSED)
@pytest.mark.parametrize("dtype,tol", [("float64", 1e-6), ("float32", 1e-5)])
def test_lambda_matches_reference(name, dtype, tol):
    g = golden()
    r = O.ncp_solve(scene(name), ITERS, dtype=dtype)
    assert np.max(np.abs(r["lam"] - g[f"{name}/lam_ref"])) < tol
    assert r["residual"] < (1e-9 if dtype == "float64" else 1e-6)


@pytest.mark.parametrize("name", INDETERMINATE)
def test_contact_velocity_and_wrench_match_reference(name):
    g = golden()
    bs = scene(name)
    r = O.ncp_solve(bs, ITERS, dtype="float64")
    G, b, lam_ref = g[f"{name}/G"], g[f"{name}/b"], g[f"{name}/lam_ref"].reshape(-1)
    lam = r["lam"].reshape(-1)
    du = np.max(np.abs((G @ lam + b) - (G @ lam_ref + b)))
    J = np.zeros((3 * len(bs.mu), 6 * len(bs.Minv)))
    for c, (a, bb) in enumerate(bs.body_pairs):
        if a >= 0:
            J[3 * c:3 * c + 3, 6 * a:6 * a + 6] += bs.Ja[c]
        if bb >= 0:
            J[3 * c:3 * c + 3, 6 * bb:6 * bb + 6] += bs.Jb[c]
    dw = np.max(np.abs(J.T @ (lam - lam_ref)))
    assert du < 1e-5 and dw < 1e-4


def test_pushed_cube_has_four_colours():
    assert O.ncp_solve(scene("pushed_cube"), 1)["n_colors"] == 4


def test_velocity_is_v_free_plus_rounded_minv_jt_lambda():
    """acc holds sum_c round(1e10 Minv J_c^T lambda_c): v - (v_free + Minv J^T lambda) stays below
    (contacts on a body) quanta however many iterations ran (test_ncp_gpu_cone.py:156-184)."""
    bs = scene("pushed_cube")
    drift = []
    for it in (500, 5000, 20000):
        r = O.ncp_solve(bs, it, dtype="float64")
        v = np.asarray(bs.v_free, np.float64).copy()
        for c, (a, _) in enumerate(bs.body_pairs):
            v[a] += bs.Minv[a] @ (bs.Ja[c].T @ r["lam"][c])
        drift.append(np.max(np.abs(r["v"] - v)))
    assert max(drift) < len(bs.mu) * 1e-10


def test_warm_restart_is_bit_identical():
    """v is a pure function of lambda: 3 x 400 warm-restarted iterations == 1 x 1200."""
    bs = scene("synthetic_256_64_7")
    a = O.ncp_solve(bs, 1200, dtype="float64")
    r = O.ncp_solve(bs, 400, dtype="float64")
    for _ in range(2):
        r = O.ncp_solve(bs, 400, dtype="float64", warm=r["lam"])
    assert a["lam"].tobytes() == r["lam"].tobytes() and a["v"].tobytes() == r["v"].tobytes()


def test_soft_step_params_match_reference():
    from importlib import import_module
    import __graft_entry__ as ge
    ge.load_package()
    ncp = import_module("motion_engine_b200.ncp")
    g = golden()
    np.testing.assert_allclose(ncp.SoftStep().params(1.0 / 240.0), g["soft/params_240"], rtol=1e-15, atol=0)
    assert tuple(ncp.SoftStep().split(16)) == tuple(g["soft/split_16"])


def test_soft_step_runs_and_relax_converges():
    g = golden()
    bs = with_sep(scene("wellposed_8_8_1"))
    soft = g["soft/params_240"]
    r1 = O.ncp_solve(bs, 300, dtype="float64", softp=soft, use_bias=True)
    r2 = O.ncp_solve(bs, 3000, dtype="float64", softp=soft, use_bias=False, warm=r1["lam"])
    assert np.all(np.isfinite(r1["lam"])) and r2["residual"] < 1e-8


def test_lattice_fixture_matches_the_reference_record(me):
    """The restated LatticeWorld fixture (N = 10 000, n_c = 40 000, float64) reproduces the
    reference's own record of it: 8 colours and a natural residual of 7.778e-05 after 40 PGS
    sweeps (reproducibility/p2/data/reference/lattice_producer_shared.txt, first line)."""
    from motion_engine_b200 import ncp, scenes
    bs = ncp.BlockScene(**scenes.ncp_lattice())
    assert (bs.n_b, bs.n_c) == (10000, 40000)
    r = O.ncp_solve(bs, 40, dtype="float64")
    assert r["n_colors"] == 8
    assert abs(r["residual"] - 7.778e-05) < 5e-9
