"""Extract the golden vectors for the contact-solve path from the reference's own receipts.

Source (read-only, in the reference checkout):
  reports/cross_hardware_l4.npz / .json -- written by probes/cross_hardware_state_probe.py on an
  NVIDIA L4 (Warp 1.13.0).  Per step, the ContactEngine outputs xc, Rm, vc, om (float32) and
  contact_forces (float64) of three engines (jacobi, pair_chunks, color_cache) on two scenes
  (stack8: 8 boxes x 120 steps; lattice1000: 1000 boxes x 40 steps), fixture dims (0.3, 0.3,
  0.2), mu 0.5, vit 40, pit 10, dt 1/240, 1 substep.  The receipts were bit-identical over two
  legs, and the jacobi arrays are bit-identical across L4 / A10G / H100 / RTX 5070.

Written here: golden_l4.npz with, per engine and scene,
  * `digest`   (T, 5, 32) uint8 -- sha256 of the bytes of xc, Rm, vc, om, force at every step,
  * `contacts` (T,) int32     -- raw generated contact count at every step (from the .json),
  * full arrays at a few steps (all steps for stack8; steps 3, 9, 39 for lattice1000),
plus `initial__<engine>__<scene>__<name>` sha256 of the built body arrays (xc, q, v, w, invM,
IbInv, rest).

Run:  python tests/golden/make_golden.py /path/to/reference   (or with B2C_REFERENCE set)
"""
import hashlib
import json
import os
import sys

import numpy as np

NAMES = ("xc", "Rm", "vc", "om", "force")
ENGINES = ("jacobi", "pair_chunks", "color_cache")
SCENES = {"stack8": None, "lattice1000": (3, 9, 39)}


def reference_root():
    """The reference checkout: the first argument, else $B2C_REFERENCE."""
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("B2C_REFERENCE")
    if not ref:
        raise SystemExit(f"usage: python {os.path.basename(__file__)} /path/to/reference  (or set B2C_REFERENCE)")
    return ref


def main(ref):
    src = np.load(os.path.join(ref, "reports/cross_hardware_l4.npz"))
    meta = json.load(open(os.path.join(ref, "reports/cross_hardware_l4.json")))
    out = {}
    for rec in meta["records"]:
        e, s = rec["engine"], rec["scene"]
        if e not in ENGINES or s not in SCENES:
            continue
        leg = rec["legs"][0]
        pre = f"{e}__{s}__0__"
        T = src[pre + "xc"].shape[0]
        dig = np.zeros((T, len(NAMES), 32), np.uint8)
        for t in range(T):
            for k, n in enumerate(NAMES):
                dig[t, k] = np.frombuffer(hashlib.sha256(np.ascontiguousarray(src[pre + n][t]).tobytes()).digest(),
                                          np.uint8)
        out[f"{e}__{s}__digest"] = dig
        out[f"{e}__{s}__contacts"] = np.array(leg["contacts"], np.int32)
        steps = SCENES[s]
        sel = np.arange(T) if steps is None else np.array(steps)
        out[f"{e}__{s}__steps"] = sel.astype(np.int32)
        for n in NAMES:
            out[f"{e}__{s}__{n}"] = np.ascontiguousarray(src[pre + n][sel])
        for n, fp in leg["initial"].items():
            out[f"initial__{e}__{s}__{n}"] = np.frombuffer(bytes.fromhex(fp["sha256"]), np.uint8)
    here = os.path.dirname(os.path.abspath(__file__))
    np.savez_compressed(os.path.join(here, "golden_l4.npz"), **out)
    print("wrote", os.path.join(here, "golden_l4.npz"), len(out), "arrays")


if __name__ == "__main__":
    main(reference_root())
