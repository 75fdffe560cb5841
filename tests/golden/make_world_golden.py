"""Golden trajectory of the reference's exact-cone box world, for BoxWorldB200.

Source (read-only, in the reference checkout): src/motion_engine/ncp/ncp_gpu.py BoxWorld
(:1237-1413) -- box/plane and box/box SAT contacts, build_scene, integration -- run on the host
with its NCPSolverGPU (Warp, not installed) replaced by the reference's own float64 CPU solver,
ncp_ref.solve_ncp_pgs (src/motion_engine/ncp/ncp_ref.py), driven to a natural residual of 1e-11 (at most 3000 sweeps):
a converged solve, so the result does not depend on the sweep order.  Scene: nine boxes -- a
stack of three, four dropped from heights up to 0.5 m, three of them tilted so that box-box edge and
face contacts both occur, one sliding -- on the ground, mu 0.5, dt 1/240, one substep, 90 steps.
No box lands flat on another with its face turned about the normal: that clips more than four
points at one depth, and "keep the 4 deepest" then depends on the last bits of the state.

Written here: world_golden.npz with the scene (half, mass, x0, q0, v0) and per step x, q, v, w and
the contact count.

Run:  python tests/golden/make_world_golden.py /path/to/reference   (or with B2C_REFERENCE set)
"""
import os
import sys

import numpy as np


def scene():
    half = np.array([[0.1, 0.1, 0.1], [0.1, 0.1, 0.1], [0.1, 0.1, 0.1], [0.15, 0.1, 0.05], [0.08, 0.12, 0.1],
                     [0.1, 0.1, 0.1], [0.2, 0.05, 0.05], [0.1, 0.1, 0.15], [0.06, 0.06, 0.06]])
    mass = np.array([1.0, 1.0, 1.0, 2.0, 0.7, 1.5, 0.9, 1.2, 0.4])
    x0 = np.array([[0.0, 0.0, 0.1], [0.003, -0.002, 0.3005], [-0.004, 0.002, 0.501], [0.6, 0.0, 0.3],
                   [0.65, 0.02, 0.5], [-0.6, 0.1, 0.4], [-0.55, 0.1, 0.65], [0.0, 0.7, 0.3], [0.05, 0.72, 0.6]])
    q0 = np.tile([0.0, 0.0, 0.0, 1.0], (len(half), 1))
    for i, (axis, ang) in ((4, ([1.0, 0.0, 0.0], 0.3)), (6, ([0.3, 1.0, 0.2], 0.5)), (8, ([1.0, 1.0, 0.0], 0.2))):
        a = np.array(axis) / np.linalg.norm(axis)
        q0[i] = np.r_[np.sin(ang / 2) * a, np.cos(ang / 2)]
    v0 = np.zeros((len(half), 3))
    v0[5] = [0.4, 0.0, 0.0]
    return half, mass, x0, q0, v0


class _ConvergedCpuSolver:
    """NCPSolverGPU.solve's contract (ncp_gpu.py:974-1063) over ncp_ref.solve_ncp_pgs."""

    def __init__(self, R, G):
        self.R, self.G = R, G

    def solve(self, bs, iters=200, warm=None, history_every=0, **kw):
        Gm, b = bs.delassus(), bs.rhs()
        lam = self.R.solve_ncp_pgs(Gm, b, bs.mu, iters=3000, tol=1e-11)[0].reshape(-1, 3)
        v = np.array(bs.v_free, float).copy()
        for c, (ia, ib) in enumerate(bs.body_pairs):
            v[ia] += bs.Minv[ia] @ (bs.Ja[c].T @ lam[c])
            if ib >= 0:
                v[ib] += bs.Minv[ib] @ (bs.Jb[c].T @ lam[c])
        return self.G.SolveResult(lam=lam, v=v, residual=float(self.R.natural_residual(lam.ravel(), Gm, b, bs.mu)),
                                  iters=0, n_colors=0, cache_hit=False)


def reference_root():
    """The reference checkout: the first argument, else $B2C_REFERENCE."""
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("B2C_REFERENCE")
    if not ref:
        raise SystemExit(f"usage: python {os.path.basename(__file__)} /path/to/reference  (or set B2C_REFERENCE)")
    return ref


def main(ref):
    sys.path.insert(0, os.path.join(ref, "src"))
    from motion_engine.ncp import ncp_gpu as G
    from motion_engine.ncp import ncp_ref as R
    half, mass, x0, q0, v0 = scene()
    w = G.BoxWorld(dt=1.0 / 240.0, mu=0.5, iters=1)
    for i in range(len(half)):
        w.add(half[i], mass[i], x0[i], v=v0[i])
        w.bodies[i].q = q0[i].copy()
    w._solver = _ConvergedCpuSolver(R, G)
    T = 90
    out = {k: [] for k in ("x", "q", "v", "w", "contacts")}
    for _ in range(T):
        w.step()
        out["x"].append([b.x.copy() for b in w.bodies])
        out["q"].append([b.q.copy() for b in w.bodies])
        out["v"].append([b.v.copy() for b in w.bodies])
        out["w"].append([b.w.copy() for b in w.bodies])
        out["contacts"].append(w.n_contacts)
    here = os.path.dirname(os.path.abspath(__file__))
    np.savez_compressed(os.path.join(here, "world_golden.npz"), half=half, mass=mass, x0=x0, q0=q0, v0=v0,
                        **{k: np.array(v) for k, v in out.items()})
    print("wrote world_golden.npz; contacts per step:", out["contacts"][::10])


if __name__ == "__main__":
    main(reference_root())
