"""Extract the reference's 10 000-body ColorCache fixture.

Source (read-only, in the reference checkout): reports/innovation_color_cache_profile_v2.npz,
written by probes/innovation_color_cache_profile_v2.py:18-35 on an NVIDIA L4 (Warp 1.13.0):
ColorCacheContactEngine(dims=(0.3, 0.3, 0.2), mu=0.5, vit=40, pit=20) over lattice(10000)
(scripts/colored_vs_jacobi.py:104-112), 10 + 30 steps of dt 1/240 with 1 substep.  After the
40th step it stored the body state (xc, Rm, vc, om), contact_forces(), and the selected
contacts of the last step in feature order (ckeys, sbi, sbj, spA, spB, sn, spen and the impulses
jn, jt1, jt2, jp).  The probe ran four workers (two plain, two profiled); its receipt gate
`exact_full_states` says all four wrote the same bytes, which this script checks again.

Written here: cc10k_golden.npz with the arrays of the first plain worker.

Run:  python tests/golden/make_cc10k_golden.py /path/to/reference   (or with B2C_REFERENCE set)
"""
import os
import sys

import numpy as np

FIELDS = ("xc", "Rm", "vc", "om", "force", "ckeys", "sbi", "sbj", "spA", "spB", "sn", "spen", "jn", "jt1", "jt2",
          "jp")
LEGS = ("plain_0", "plain_1", "profiled_0", "profiled_1")


def reference_root():
    """The reference checkout: the first argument, else $B2C_REFERENCE."""
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("B2C_REFERENCE")
    if not ref:
        raise SystemExit(f"usage: python {os.path.basename(__file__)} /path/to/reference  (or set B2C_REFERENCE)")
    return ref


def main(ref):
    src = np.load(os.path.join(ref, "reports/innovation_color_cache_profile_v2.npz"))
    out = {f: np.ascontiguousarray(src[f"plain_0__{f}"]) for f in FIELDS}
    for leg in LEGS[1:]:
        for f in FIELDS:
            if src[f"{leg}__{f}"].tobytes() != out[f].tobytes():
                raise SystemExit(f"{leg}.{f} differs from plain_0.{f}: the receipt is not one trajectory")
    here = os.path.dirname(os.path.abspath(__file__))
    np.savez_compressed(os.path.join(here, "cc10k_golden.npz"), **out)
    print("wrote cc10k_golden.npz:", {f: out[f].shape for f in FIELDS})


if __name__ == "__main__":
    main(reference_root())
