"""Exact-cone NCP solve on the GPU (b2c_ncp_*): bitwise against the oracle, against the
reference's CPU solution, and the reference test file's gates (tests/test_ncp_gpu_cone.py:
bit identity, input-permutation invariance, proper colouring, drift, warm restart)."""
import importlib

import numpy as np
import pytest

from conftest import cuda_ok
from ncp_scenes import INDETERMINATE, SYNTHETIC, WELLPOSED, golden, scene, with_sep

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_ok(), reason="needs a CUDA device")]


@pytest.fixture(scope="module")
def ncp(me):
    return importlib.import_module("motion_engine_b200.ncp")


@pytest.mark.parametrize("name", WELLPOSED + INDETERMINATE + SYNTHETIC)
@pytest.mark.parametrize("dtype", ["float32", "float64"])
def test_matches_oracle_bitwise(ncp, oracle_mod, name, dtype):
    bs = scene(name, ncp.BlockScene)
    iters = 300 if name in SYNTHETIC else 1000
    s = ncp.NCPSolverB200(bs.n_b, bs.n_c, dtype=dtype)
    r = s.solve(bs, iters=iters)
    o = oracle_mod.ncp_solve(bs, iters, dtype=dtype)
    nt = np.float32 if dtype == "float32" else np.float64
    assert r.n_colors == o["n_colors"]
    np.testing.assert_array_equal(r.lam.astype(nt), o["lam"])
    np.testing.assert_array_equal(r.v.astype(nt), o["v"])
    assert r.residual == pytest.approx(o["residual"], rel=0, abs=0)


def test_warm_and_soft_match_oracle_bitwise(ncp, oracle_mod):
    g = golden()
    bs = with_sep(scene("synthetic_256_64_7", ncp.BlockScene))
    soft = g["soft/params_240"]
    warm = np.random.default_rng(3).uniform(0.0, 0.05, (bs.n_c, 3))
    warm[:, 1:] *= 0.1
    for dtype in ("float32", "float64"):
        s = ncp.NCPSolverB200(bs.n_b, bs.n_c, dtype=dtype)
        r = s.solve(bs, iters=200, warm=warm, soft=soft, relax_iters=50)
        o1 = oracle_mod.ncp_solve(bs, 200, dtype=dtype, warm=warm, softp=soft, use_bias=True)
        o2 = oracle_mod.ncp_solve(bs, 50, dtype=dtype, warm=o1["lam"], softp=soft, use_bias=False)
        nt = np.float32 if dtype == "float32" else np.float64
        np.testing.assert_array_equal(r.v_bias.astype(nt), o1["v"])
        np.testing.assert_array_equal(r.lam.astype(nt), o2["lam"])
        np.testing.assert_array_equal(r.v.astype(nt), o2["v"])


@pytest.mark.parametrize("name", WELLPOSED)
def test_matches_cpu_reference_lambda(ncp, name):
    """test_ncp_gpu_cone.py:111-127: converged lambda within 1e-6 (float64) / 1e-5 (float32)."""
    g = golden()
    bs = scene(name, ncp.BlockScene)
    for dtype, tol in (("float64", 1e-6), ("float32", 1e-5)):
        r = ncp.solve_scene_gpu(bs, iters=5000, dtype=dtype)
        assert np.max(np.abs(r.lam - g[f"{name}/lam_ref"])) < tol, dtype


def test_pushed_cube_wrench_matches_reference(ncp):
    """test_ncp_gpu_cone.py:130-153: indeterminate scene, compare u and the net wrench."""
    g = golden()
    bs = scene("pushed_cube", ncp.BlockScene)
    r = ncp.solve_scene_gpu(bs, iters=5000, dtype="float64")
    G, b, lam_ref = g["pushed_cube/G"], g["pushed_cube/b"], g["pushed_cube/lam_ref"].reshape(-1)
    lam = r.lam.reshape(-1)
    Jt = np.zeros((6, 3 * bs.n_c))
    for c in range(bs.n_c):
        Jt[:, 3 * c:3 * c + 3] = bs.Ja[c].T
    assert np.max(np.abs((G @ lam + b) - (G @ lam_ref + b))) < 1e-5
    assert np.max(np.abs(Jt @ (lam - lam_ref))) < 1e-4
    assert r.n_colors == 4


@pytest.mark.parametrize("dtype", ["float32", "float64"])
def test_bit_identical_two_runs(ncp, dtype):
    bs = scene("synthetic_256_64_7", ncp.BlockScene)
    out = []
    for _ in range(2):
        s = ncp.NCPSolverB200(bs.n_b, bs.n_c, dtype=dtype)
        s.solve(bs, iters=300)
        out.append(s.raw_bytes())
    assert out[0] == out[1]


def test_bit_identical_under_input_permutation(ncp):
    bs = scene("synthetic_256_64_7", ncp.BlockScene)
    p = np.random.default_rng(5).permutation(bs.n_c)
    bp = ncp.BlockScene(Ja=bs.Ja[p], Jb=bs.Jb[p], Minv=bs.Minv, v_free=bs.v_free, mu=bs.mu[p],
                        body_pairs=bs.body_pairs[p], dt=bs.dt, bias=bs.bias[p], feature=bs.feature[p])
    r1 = ncp.NCPSolverB200(bs.n_b, bs.n_c).solve(bs, iters=300)
    r2 = ncp.NCPSolverB200(bs.n_b, bs.n_c).solve(bp, iters=300)
    assert r1.lam[p].tobytes() == r2.lam.tobytes() and r1.v.tobytes() == r2.v.tobytes()


def test_coloring_is_proper_and_cached(ncp):
    bs = scene("synthetic_1024_128_2", ncp.BlockScene)
    s = ncp.NCPSolverB200(bs.n_b, bs.n_c)
    r = s.solve(bs, iters=10, measure_residual=False)
    col, order, cstart, ccount = s.coloring()
    for ci in range(s.n_colors):
        idx = order[cstart[ci]:cstart[ci] + ccount[ci]]
        bodies = np.concatenate([bs.body_pairs[idx, 0], bs.body_pairs[idx, 1]])
        bodies = bodies[bodies >= 0]
        assert len(np.unique(bodies)) == len(bodies)
    assert sum(ccount) == bs.n_c and not r.cache_hit
    r2 = s.solve(bs, iters=10, measure_residual=False)
    assert r2.cache_hit and s.cache_hits == 1 and s.cache_misses == 1


def test_warm_restart_bit_identical(ncp):
    bs = scene("synthetic_256_64_7", ncp.BlockScene)
    ra = ncp.NCPSolverB200(bs.n_b, bs.n_c, dtype="float64").solve(bs, iters=1200)
    s2 = ncp.NCPSolverB200(bs.n_b, bs.n_c, dtype="float64")
    rb = s2.solve(bs, iters=400)
    for _ in range(2):
        rb = s2.solve(bs, iters=400, warm=rb.lam)
    assert ra.lam.tobytes() == rb.lam.tobytes() and ra.v.tobytes() == rb.v.tobytes()


def test_cluster_block_and_grid_forms_agree(ncp):
    """One CTA, a cluster and a cooperative grid give the same bits: within a colour the
    contacts write disjoint bodies' accumulators."""
    bs = scene("synthetic_1024_128_2", ncp.BlockScene)
    r1 = ncp.NCPSolverB200(bs.n_b, bs.n_c, solve_blocks=1).solve(bs, iters=100)
    for form in (-8, 148, 5):
        r2 = ncp.NCPSolverB200(bs.n_b, bs.n_c, solve_blocks=form).solve(bs, iters=100)
        assert r1.lam.tobytes() == r2.lam.tobytes() and r1.v.tobytes() == r2.v.tobytes(), form


def test_history_and_dense_scene(ncp):
    bs = scene("wellposed_8_8_1", ncp.BlockScene)
    r = ncp.NCPSolverB200(bs.n_b, bs.n_c).solve(bs, iters=300, history_every=100)
    assert r.history["iter"] == [0, 100, 200, 300] and len(r.history["lam"]) == 4
    assert r.history["res"][-1] <= r.history["res"][0]
    sc = ncp.Scene(J=bs.jacobian(), Minv=np.kron(np.eye(bs.n_b), np.eye(6)) * 0 + _block_diag(bs.Minv),
                   v_free=bs.v_free.reshape(-1), mu=bs.mu, body_pairs=bs.body_pairs, dt=bs.dt,
                   bias=bs.bias.reshape(-1), feature=bs.feature)
    r1 = ncp.solve_scene_gpu(bs, iters=500)
    r2 = ncp.solve_scene_gpu(sc.blocks(), iters=500)
    assert r1.lam.tobytes() == r2.lam.tobytes()


def _block_diag(M):
    n = len(M)
    out = np.zeros((6 * n, 6 * n))
    for i in range(n):
        out[6 * i:6 * i + 6, 6 * i:6 * i + 6] = M[i]
    return out


def test_resident_resolve_equals_full_solve(me):
    """solve_resident (the scene kept on the device, the colour cache hit) gives the same bytes
    as a full solve of the same scene."""
    from motion_engine_b200 import ncp, scenes
    bs = ncp.BlockScene(**scenes.ncp_lattice(n=2000))
    s = ncp.NCPSolverB200(bs.n_b, bs.n_c, dtype="float64")
    s.solve(bs, iters=40)
    lam0, v0 = s.raw_bytes()
    s.solve_resident(40)
    lam1, v1 = s.raw_bytes()
    assert lam0 == lam1 and v0 == v1
