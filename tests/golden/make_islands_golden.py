"""Golden vectors for the island partition, made by the reference's own partition_pairs
(src/motion_engine/contact_engine_gpu_island_solve.py:7-34; numpy only, the module imports
without warp) on seeded random pair graphs: static bodies, ground pairs, pairs without a dynamic
body, long chains and random pair orders.

Run:  python tests/golden/make_islands_golden.py /path/to/reference   (or with B2C_REFERENCE set)
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


CASES = [  # (bodies, pairs, static fraction, ground fraction, chain links)
    (10, 12, 0.2, 0.2, 0), (50, 40, 0.1, 0.3, 0), (300, 400, 0.15, 0.1, 0), (800, 3000, 0.05, 0.05, 0),
    (2000, 1500, 0.3, 0.2, 0), (1000, 900, 0.02, 0.1, 600), (400, 350, 1.0, 0.1, 0), (200, 600, 0.0, 0.0, 0),
]


def graph(case, seed):
    n, P, static, ground, chain = case
    rng = np.random.default_rng(seed)
    mass = np.where(rng.random(n) < static, 0.0, rng.uniform(0.1, 2.0, n))
    a = rng.integers(0, n, P)
    b = rng.integers(0, n, P)
    b[rng.random(P) < ground] = -1
    if chain:
        idx = np.flatnonzero(mass > 0)[:chain + 1]
        k = len(idx) - 1
        a[:k], b[:k] = idx[:-1], idx[1:]
    return a, b, mass, rng.permutation(P)


def main(ref):
    sys.path.insert(0, os.path.join(ref, "src"))
    from motion_engine.contact_engine_gpu_island_solve import partition_pairs
    out = {}
    for k, case in enumerate(CASES):
        a, b, mass, order = graph(case, 40 + k)
        packed, starts, counts = partition_pairs(a, b, mass, order)
        out.update({f"c{k}/a": a, f"c{k}/b": b, f"c{k}/mass": mass, f"c{k}/order": order,
                    f"c{k}/packed": packed, f"c{k}/starts": starts, f"c{k}/counts": counts})
        print(k, case, "islands", len(counts), "largest", int(counts.max()) if len(counts) else 0)
    out["n_cases"] = np.int32(len(CASES))
    np.savez_compressed(os.path.join(os.path.dirname(os.path.abspath(__file__)), "islands_golden.npz"), **out)


if __name__ == "__main__":
    main(reference_root())
