"""The oracle's batched-NCP restatement against the reference's CPU solver and sensitivity
(golden fixture made by the reference: tests/golden/make_sens_golden.py): lambda, labels, the
fixed-branch responses dlam/dmu and dlam/db (ncp_ref.sensitivity) and the reference's central
finite differences (ncp_ref.sensitivity_fd; the reference test's bound, 1e-5 relative,
tests/test_ncp_reference.py:316-345)."""
import os

import numpy as np
import pytest

from oracle import oracle_bncp as OB

G_ = dict(np.load(os.path.join(os.path.dirname(__file__), "golden", "sens_golden.npz")))
NAMES = [str(x) for x in G_["names"]]


def _rel(a, f):
    return float(np.max(np.abs(a - f)) / max(float(np.max(np.abs(f))), 1e-30))


@pytest.mark.parametrize("name", NAMES)
def test_solution_labels_and_sensitivity(name):
    G, b, mu = G_[f"{name}/G"], G_[f"{name}/b"], G_[f"{name}/mu"]
    lam, it = OB.pgs(G, b, mu, 20000, 1e-14)
    assert OB.residual(lam, G, b, mu) < 1e-13
    singular = bool(G_[f"{name}/singular"])
    if not singular:  # lambda is unique on a non-singular branch
        assert np.max(np.abs(lam - G_[f"{name}/lam"])) < 1e-11
        np.testing.assert_array_equal(OB.classify(lam, mu), G_[f"{name}/labels"])
    dmu, db, labels, status = OB.sensitivity(G_[f"{name}/lam"], G, b, mu)
    if singular:
        assert status & 1 and np.isnan(dmu).all() and np.isnan(db).all()
        return
    assert status == 0
    assert _rel(dmu, G_[f"{name}/dmu"]) < 1e-10 and _rel(db, G_[f"{name}/db"]) < 1e-10
    assert _rel(dmu, G_[f"{name}/fd_mu"]) < 1e-5 and _rel(db, G_[f"{name}/fd_b"]) < 1e-5
