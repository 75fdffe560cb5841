"""Golden vectors for the box/plane and box/box narrowphase, made by the reference itself.

Runs the reference's float64 host narrowphase (src/motion_engine/ncp/ncp_gpu.py:1148-1227:
box_plane_contacts, box_box_contacts; importable without Warp) on seeded box pairs and writes
inputs and outputs to sat_golden.npz.  Box states are drawn in float32 and widened, so the GPU
path (float32 state, float64 narrowphase) sees exactly the reference's inputs.

Cases: face-face resting stacks with small tilts and offsets, random orientations at random
separations (touching, overlapping and apart), edge-on-edge crossings, and boxes near the
ground plane.

Run:  python tests/golden/make_sat_golden.py /path/to/reference   (or with B2C_REFERENCE set)
"""
import os
import sys

import numpy as np

MARGIN = 2e-3


def _rand_quat(rng, scale=None):
    if scale is None:
        q = rng.normal(size=4)
    else:
        ax = rng.normal(size=3)
        ax /= np.linalg.norm(ax)
        ang = rng.uniform(-scale, scale)
        q = np.r_[ax * np.sin(ang / 2), np.cos(ang / 2)]
    q /= np.linalg.norm(q)
    return q.astype(np.float32)


def reference_root():
    """The reference checkout: the first argument, else $B2C_REFERENCE."""
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("B2C_REFERENCE")
    if not ref:
        raise SystemExit(f"usage: python {os.path.basename(__file__)} /path/to/reference  (or set B2C_REFERENCE)")
    return ref


def main(ref):
    sys.path.insert(0, os.path.join(ref, "src"))
    from motion_engine.ncp.ncp_gpu import Box, box_box_contacts, box_plane_contacts
    rng = np.random.default_rng(20261203)
    A_half, A_x, A_q, B_half, B_x, B_q = [], [], [], [], [], []
    kinds = []
    n_each = 300
    for kind in ("stacked", "random", "edge"):
        for _ in range(n_each):
            ha = rng.uniform(0.1, 0.3, 3).astype(np.float32)
            hb = rng.uniform(0.1, 0.3, 3).astype(np.float32)
            if kind == "stacked":
                qa = _rand_quat(rng, 0.05)
                qb = _rand_quat(rng, 0.05)
                xa = np.r_[rng.uniform(-1, 1, 2), rng.uniform(0, 1)].astype(np.float32)
                off = np.r_[rng.uniform(-0.15, 0.15, 2), ha[2] + hb[2] + rng.uniform(-0.01, 0.003)]
                xb = (xa + off).astype(np.float32)
            elif kind == "random":
                qa, qb = _rand_quat(rng), _rand_quat(rng)
                xa = rng.uniform(-1, 1, 3).astype(np.float32)
                d = rng.normal(size=3)
                d /= np.linalg.norm(d)
                xb = (xa + d * rng.uniform(0.1, 0.9)).astype(np.float32)
            else:
                qa = _rand_quat(rng, 0.2)
                qb = (np.r_[0.0, 0.0, np.sin(np.pi / 8), np.cos(np.pi / 8)] + rng.normal(scale=0.02, size=4))
                qb = (qb / np.linalg.norm(qb)).astype(np.float32)
                xa = rng.uniform(-1, 1, 3).astype(np.float32)
                xb = (xa + np.r_[rng.uniform(-0.05, 0.05, 2), ha[2] + hb[2] * 0.8]).astype(np.float32)
            A_half.append(ha); A_x.append(xa); A_q.append(qa)
            B_half.append(hb); B_x.append(xb); B_q.append(qb)
            kinds.append(kind)
    # ground cases: box A alone near z = 0
    G_half, G_x, G_q = [], [], []
    for _ in range(300):
        h = rng.uniform(0.1, 0.3, 3).astype(np.float32)
        q = _rand_quat(rng, rng.choice([0.02, 0.3, np.pi]))
        x = np.r_[rng.uniform(-1, 1, 2), rng.uniform(0.0, 0.5)].astype(np.float32)
        G_half.append(h); G_x.append(x); G_q.append(q)

    def box(h, x, q):
        return Box(half=np.asarray(h, float), mass=1.0, x=np.asarray(x, float), q=np.asarray(q, float))

    bb_pair, bb_p, bb_n, bb_g, bb_f = [], [], [], [], []
    for k in range(len(A_half)):
        cs = box_box_contacts(0, box(A_half[k], A_x[k], A_q[k]), 1, box(B_half[k], B_x[k], B_q[k]), MARGIN)
        for (_, _, p, n, g, f) in cs:
            bb_pair.append(k); bb_p.append(p); bb_n.append(n); bb_g.append(g); bb_f.append(f)
    bp_box, bp_p, bp_g, bp_f = [], [], [], []
    for k in range(len(G_half)):
        for (_, _, p, n, g, f) in box_plane_contacts(0, box(G_half[k], G_x[k], G_q[k]), MARGIN):
            bp_box.append(k); bp_p.append(p); bp_g.append(g); bp_f.append(f)
    here = os.path.dirname(os.path.abspath(__file__))
    np.savez_compressed(
        os.path.join(here, "sat_golden.npz"), margin=np.float64(MARGIN),
        A_half=np.array(A_half), A_x=np.array(A_x), A_q=np.array(A_q),
        B_half=np.array(B_half), B_x=np.array(B_x), B_q=np.array(B_q), kind=np.array(kinds),
        bb_pair=np.array(bb_pair, np.int32), bb_p=np.array(bb_p), bb_n=np.array(bb_n), bb_g=np.array(bb_g),
        bb_f=np.array(bb_f, np.int32),
        G_half=np.array(G_half), G_x=np.array(G_x), G_q=np.array(G_q),
        bp_box=np.array(bp_box, np.int32), bp_p=np.array(bp_p), bp_g=np.array(bp_g), bp_f=np.array(bp_f, np.int32))
    print("box-box pairs", len(A_half), "contacts", len(bb_pair), "| box-plane boxes", len(G_half), "contacts",
          len(bp_box))
    print("contacts per box-box pair histogram", np.bincount(np.bincount(bb_pair, minlength=len(A_half))))


if __name__ == "__main__":
    main(reference_root())
