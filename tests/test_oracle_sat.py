"""The oracle's box/plane and box/box narrowphase against golden vectors made by the reference's
own float64 host narrowphase (ncp_gpu.py:1148-1227; tests/golden/make_sat_golden.py).

Contact counts, feature ids, normals and gaps agree to float64 rounding.  Face-face points
agree to rounding too.  An edge-edge point is the midpoint of the two support corners along the
edge axis; when two corners tie along that axis (edges parallel to a face) the reference's
numpy expressions and the scalar oracle may round the tie differently and pick the other
corner, so edge-edge points are compared by their projection on the normal, which is the same
for either corner of a tie."""
import numpy as np
import pytest

from oracle import oracle as O

TOL = 1e-10


@pytest.fixture(scope="module")
def sat():
    return dict(np.load(__import__("os").path.join(__import__("os").path.dirname(__file__), "golden",
                                                   "sat_golden.npz")))


def test_box_plane_golden(sat):
    m = float(sat["margin"])
    n_box = len(sat["G_half"])
    for k in range(n_box):
        p, g, f = O.box_plane(sat["G_half"][k], sat["G_x"][k], sat["G_q"][k], m)
        sel = sat["bp_box"] == k
        assert len(g) == sel.sum(), k
        np.testing.assert_array_equal(f, sat["bp_f"][sel])
        np.testing.assert_allclose(p, sat["bp_p"][sel], rtol=0, atol=TOL)
        np.testing.assert_allclose(g, sat["bp_g"][sel], rtol=0, atol=TOL)


def test_box_box_golden(sat):
    m = float(sat["margin"])
    n_pairs = len(sat["A_half"])
    seen = {"face": 0, "edge": 0, "none": 0}
    for k in range(n_pairs):
        p, n, g, f = O.box_box(sat["A_half"][k], sat["A_x"][k], sat["A_q"][k], sat["B_half"][k], sat["B_x"][k],
                               sat["B_q"][k], m)
        sel = sat["bb_pair"] == k
        assert len(g) == sel.sum(), k
        if not len(g):
            seen["none"] += 1
            continue
        np.testing.assert_array_equal(f, sat["bb_f"][sel])  # local feature ids (face base + n, or 100 + edge)
        nref = sat["bb_n"][sel]
        np.testing.assert_allclose(np.broadcast_to(n, nref.shape), nref, rtol=0, atol=TOL)
        np.testing.assert_allclose(g, sat["bb_g"][sel], rtol=0, atol=TOL)
        if f[0] >= 100:
            seen["edge"] += 1
            np.testing.assert_allclose(p @ n, sat["bb_p"][sel] @ n, rtol=0, atol=TOL)
        else:
            seen["face"] += 1
            np.testing.assert_allclose(p, sat["bb_p"][sel], rtol=0, atol=TOL)
    assert seen["face"] > 300 and seen["edge"] > 20 and seen["none"] > 50, seen
