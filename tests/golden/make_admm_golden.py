"""Golden vectors for the batched ADMM adjoint (grad_affine), made by the reference's own CPU
code: the all-slip scenes of its batched-adjoint test (tests/test_ncp_batch_adjoint.py:26-46:
contact c couples body c to body c + 1, the last to the ground; every contact slips), solved by
src/motion_engine/ncp/ncp_ref.py's solve_ncp_pgs (2000 sweeps, tol 1e-15, as that test does),
classified, and differentiated by its fixed-branch implicit sensitivity (ncp_ref.sensitivity,
:907-959).  numpy only.

Run:  python tests/golden/make_admm_golden.py /path/to/reference   (or with B2C_REFERENCE set)
"""
import os
import sys

import numpy as np


def all_slip_scene(n_c):
    n = 3 * n_c
    J = np.zeros((n, n))
    for c in range(n_c):
        J[3 * c:3 * c + 3, 3 * c:3 * c + 3] = np.eye(3)
        if c + 1 < n_c:
            J[3 * c:3 * c + 3, 3 * (c + 1):3 * (c + 1) + 3] = -np.eye(3)
    m = 1.0 + 0.5 * np.arange(n_c)
    Minv = np.diag(np.repeat(1.0 / m, 3))
    G = J @ Minv @ J.T
    mu = np.full(n_c, 0.3)
    b = np.zeros(n)
    for c in range(n_c):
        b[3 * c + 0] = -1.0 - 0.1 * c
        b[3 * c + 1] = 0.9 + 0.2 * c
        b[3 * c + 2] = -0.7 + 0.1 * c
    return G, b, mu


def reference_root():
    """The reference checkout: the first argument, else $B2C_REFERENCE."""
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("B2C_REFERENCE")
    if not ref:
        raise SystemExit(f"usage: python {os.path.basename(__file__)} /path/to/reference  (or set B2C_REFERENCE)")
    return ref


def main(ref):
    sys.path.insert(0, os.path.join(ref, "src"))
    from motion_engine.ncp import ncp_ref as R
    out, names = {}, []
    for n_c in (1, 2, 4, 8):
        G, b, mu = all_slip_scene(n_c)
        lam = R.solve_ncp_pgs(G, b, mu, 2000, 1e-15)[0]
        labels = R.classify(lam, G, b, mu)
        dmu, db, info = R.sensitivity(lam, G, b, mu, labels)
        name = f"all_slip_{n_c}"
        out.update({f"{name}/G": G, f"{name}/b": b, f"{name}/mu": mu, f"{name}/lam": lam, f"{name}/db": db,
                    f"{name}/dmu": dmu, f"{name}/res": np.float64(R.natural_residual(lam, G, b, mu)),
                    f"{name}/labels": np.array([{"open": 0, "stick": 1, "slip": 2}[x] for x in labels], np.int32)})
        names.append(name)
        print(name, list(labels), "res %.2e" % R.natural_residual(lam, G, b, mu))
    out["names"] = np.array(names)
    np.savez_compressed(os.path.join(os.path.dirname(os.path.abspath(__file__)), "admm_golden.npz"), **out)


if __name__ == "__main__":
    main(reference_root())
