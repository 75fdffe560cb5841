"""Golden sensitivities of the exact-cone NCP, made by the reference's own host code.

For the well-posed block scenes of ncp_golden.npz (the reference's random_wellposed_scene,
src/motion_engine/ncp/ncp_gpu.py) at the reference's converged impulses lam_ref, the reference's
fixed-branch implicit-function derivatives (src/motion_engine/ncp/ncp_ref.py: classify, then
sensitivity -> dlam/dmu (3 n_c, n_c) and dlam/db (3 n_c, 3 n_c), b = J v_free + bias) and its
diagnostics (singular, boundary).  numpy only.

Run:  python tests/golden/make_ncp_sens_golden.py /path/to/reference   (or with B2C_REFERENCE set)
"""
import os
import sys

import numpy as np

SCENES = ("wellposed_8_8_1", "wellposed_16_8_2", "wellposed_6_6_3", "wellposed_12_10_4")
LABELS = {"open": 0, "stick": 1, "slip": 2}


def reference_root():
    """The reference checkout: the first argument, else $B2C_REFERENCE."""
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("B2C_REFERENCE")
    if not ref:
        raise SystemExit(f"usage: python {os.path.basename(__file__)} /path/to/reference  (or set B2C_REFERENCE)")
    return ref


def main(ref):
    sys.path.insert(0, os.path.join(ref, "src"))
    from motion_engine.ncp import ncp_ref as R
    here = os.path.dirname(os.path.abspath(__file__))
    g = np.load(os.path.join(here, "ncp_golden.npz"))
    out = {}
    for name in SCENES:
        G, b, mu = g[f"{name}/G"], g[f"{name}/b"], g[f"{name}/mu"]
        lam = g[f"{name}/lam_ref"].reshape(-1)
        labels = R.classify(lam, G, b, mu)
        dm, db, info = R.sensitivity(lam, G, b, mu, labels)
        out[f"{name}/dlam_dmu"] = dm
        out[f"{name}/dlam_db"] = db
        out[f"{name}/labels"] = np.array([LABELS[str(x)] for x in labels], np.int32)
        out[f"{name}/singular"] = np.int32(bool(info["singular"]))
        out[f"{name}/boundary"] = np.int32(len(info["boundary"]))
        print(name, "labels", "".join(str(x)[0] for x in labels), "singular", info["singular"],
              "boundary", info["boundary"], "finite", bool(np.isfinite(dm).all() and np.isfinite(db).all()))
    np.savez_compressed(os.path.join(here, "ncp_sens_golden.npz"), **out)


if __name__ == "__main__":
    main(reference_root())
