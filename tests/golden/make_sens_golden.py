"""Golden vectors for the batched exact-cone NCP solve and its implicit sensitivity, made by the
reference's own CPU code (src/motion_engine/ncp/ncp_ref.py: scene_random, scene_tripod,
solve_ncp_pgs, classify, sensitivity (the fixed-branch implicit-function response, :907-959)
and sensitivity_fd (central finite differences, :962-987)).  numpy only.

Run:  python tests/golden/make_sens_golden.py /path/to/reference   (or with B2C_REFERENCE set)
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
    from motion_engine.ncp import ncp_ref as R
    out = {}
    cases = []
    for seed in (3, 7, 11, 13, 17):
        cases.append((f"random_{seed}", R.scene_random(n_c=4, n_b=2, mu=0.4, seed=seed)))
    for seed in (21, 22, 23):
        cases.append((f"random6_{seed}", R.scene_random(n_c=6, n_b=3, mu=0.35, seed=seed)))
    cases.append(("tripod", R.scene_tripod(mu=0.4)))
    cases.append(("tripod_stick", R.scene_tripod(mu=2.0, vx=0.01, vy=0.0)))
    for seed in (5, 6):
        cases.append((f"random_stick_{seed}", R.scene_random(n_c=4, n_b=2, mu=2.5, seed=seed)))
    names = []
    for name, sc in cases:
        G, b, mu = sc.delassus(), sc.b(), np.asarray(sc.mu, np.float64)
        lam, hist, labels = R.solve_ncp_pgs(G, b, mu, 5000, 1e-14)
        dmu, db, info = R.sensitivity(lam, G, b, mu, labels)
        fmu, fdb = R.sensitivity_fd(G, b, mu, lam, h_mu=1e-6, h_b=1e-6)
        code = np.array([{"open": 0, "stick": 1, "slip": 2}[x] for x in labels], np.int32)
        out.update({f"{name}/G": G, f"{name}/b": b, f"{name}/mu": mu, f"{name}/lam": lam,
                    f"{name}/labels": code, f"{name}/dmu": dmu, f"{name}/db": db, f"{name}/fd_mu": fmu,
                    f"{name}/fd_b": fdb, f"{name}/singular": np.int32(info["singular"]),
                    f"{name}/boundary": np.int32(len(info["boundary"]) > 0),
                    f"{name}/res": np.float64(hist[-1])})
        names.append(name)
        print(name, list(labels), "singular", info["singular"], "boundary", info["boundary"], "res %.1e" % hist[-1])
    out["names"] = np.array(names)
    here = os.path.dirname(os.path.abspath(__file__))
    np.savez_compressed(os.path.join(here, "sens_golden.npz"), **out)


if __name__ == "__main__":
    main(reference_root())
