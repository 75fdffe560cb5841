"""The reference's 10 000-body ColorCache receipt (tests/golden/cc10k_golden.npz, cut from
reports/innovation_color_cache_profile_v2.npz) and the bounds a run is held to against it."""
import numpy as np

from conftest import DT, ROOT

G_DT = 9.81 * DT  # the velocity one step of gravity gives, the scale of the velocity bounds
R = 0.05


def receipt():
    """The receipt's arrays (float32 state and contacts, float64 forces)."""
    return np.load(f"{ROOT}/tests/golden/cc10k_golden.npz")


def _cc10k_bounds():
    """Per field: None = bitwise, else the largest admitted |got - receipt|.  The impulses are
    bounded at 1e-5 of the receipt's largest impulse of that row (the stated 1e-5 relative), the
    linear velocities at 1e-5 g dt, the angular ones at 1e-5 g dt / R and the forces at 1e-5 of
    the largest force."""
    g = receipt()
    tol = {k: None for k in ("xc", "ckeys", "sbi", "sbj", "spA", "spB", "sn", "spen", "jp")}
    tol.update(jn=1e-5 * float(np.abs(g["jn"]).max()), jt1=1e-5 * float(np.abs(g["jt1"]).max()),
               jt2=1e-5 * float(np.abs(g["jt2"]).max()), vc=1e-5 * G_DT, om=1e-5 * G_DT / R, Rm=1e-6,
               force=1e-5 * float(np.abs(g["force"]).max()))
    return g, tol


def check_cc10k(state, force, kept):
    """Assert the final state and kept contacts of the 10k lattice run against the receipt;
    returns {field: (differing rows, max |d|)} for the report."""
    g, tol = _cc10k_bounds()
    got = dict(xc=state.xc, Rm=state.Rm, vc=state.vc, om=state.om, force=force, **kept)
    out = {}
    for k, t in tol.items():
        a, b = got[k], g[k]
        assert a.shape == b.shape, (k, a.shape, b.shape)
        rows = int((a != b).reshape(len(a), -1).any(1).sum())
        d = float(np.abs(a.astype(np.float64) - b.astype(np.float64)).max()) if a.dtype.kind == "f" else float(rows)
        out[k] = (rows, d)
        if t is None:
            assert rows == 0, f"{k}: {rows} rows differ from the reference receipt"
        else:
            assert d <= t, f"{k}: max |d| {d:.3e} above the bound {t:.3e}"
    return out
