"""Golden vectors for the exact-cone NCP solve, made by the reference's own host code.

Scenes come from the reference's generators and rigid-body world (src/motion_engine/ncp/ncp_gpu.py:
random_wellposed_scene, synthetic_scene, BoxWorld.build_scene); the reference solutions from its
float64 CPU solver (src/motion_engine/ncp/ncp_ref.py: solve_ncp_pgs with de Saxce, driven to
convergence, and natural_residual).  Soft-step parameters from SoftStep.params.  Everything
imported here is numpy-only (Warp is not needed).

Run:  python tests/golden/make_ncp_golden.py /path/to/reference   (or with B2C_REFERENCE set)
"""
import os
import sys

import numpy as np


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
    out = {}

    def put(name, bs, solve=True):
        out[f"{name}/Ja"] = bs.Ja
        out[f"{name}/Jb"] = bs.Jb
        out[f"{name}/Minv"] = bs.Minv
        out[f"{name}/v_free"] = bs.v_free
        out[f"{name}/mu"] = bs.mu
        out[f"{name}/pairs"] = bs.body_pairs
        out[f"{name}/bias"] = bs.bias
        out[f"{name}/feature"] = bs.feature
        out[f"{name}/dt"] = np.float64(bs.dt)
        if bs.sep is not None:
            out[f"{name}/sep"] = bs.sep
        if solve:
            Gm, b = bs.delassus(), bs.rhs()
            lam = R.solve_ncp_pgs(Gm, b, bs.mu, iters=5000, tol=1e-14)[0]
            out[f"{name}/G"] = Gm
            out[f"{name}/b"] = b
            out[f"{name}/lam_ref"] = lam.reshape(-1, 3)
            out[f"{name}/res_ref"] = np.float64(R.natural_residual(lam, Gm, b, bs.mu))

    for (nc, nb, seed) in ((8, 8, 1), (16, 8, 2), (6, 6, 3), (12, 10, 4)):
        put(f"wellposed_{nc}_{nb}_{seed}", G.random_wellposed_scene(n_c=nc, n_b=nb, seed=seed))
    w = G.BoxWorld(dt=0.004, mu=0.5, iters=1)
    w.add([0.1, 0.1, 0.1], 15.0, [0.0, 0.0, 0.1])
    put("pushed_cube", w.build_scene(f_ext=lambda i: np.array([100.0, 0.0, 0.0])))
    # a small resting stack of three boxes: box/box and box/plane manifolds of the reference world
    w3 = G.BoxWorld(dt=1.0 / 240.0, mu=0.5, iters=1)
    for k in range(3):
        w3.add([0.1, 0.1, 0.1], 1.0, [0.002 * k, -0.001 * k, 0.1 + 0.2 * k - 1e-4 * k])
    put("stack3", w3.build_scene())
    put("synthetic_256_64_7", G.synthetic_scene(256, n_b=64, seed=7), solve=False)
    put("synthetic_1024_128_2", G.synthetic_scene(1024, n_b=128, seed=2), solve=False)
    soft = G.SoftStep()
    out["soft/params_240"] = soft.params(1.0 / 240.0)
    out["soft/split_16"] = np.array(soft.split(16), np.int32)
    here = os.path.dirname(os.path.abspath(__file__))
    np.savez_compressed(os.path.join(here, "ncp_golden.npz"), **out)
    for k in sorted(out):
        if k.endswith("/res_ref"):
            print(k, float(out[k]))


if __name__ == "__main__":
    main(reference_root())
