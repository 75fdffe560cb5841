"""Quality figures reported beside the timing: the reference's M5 penetration gate.

The reference's M5 (scripts/engine_metrics.py:265-293) runs a vertical stack, records per step
the penetration max(rest pitch - spacing of adjacent bodies) and then
  * max_pen_over_R = max over the run / R (R = 0.05 m, the bead radius),
  * the drift class from the least-squares slope over the second half of the run: "secular"
    when |slope| x (half the steps) > R / 10, else "bounded",
  * PASS when max_pen_over_R < 0.5 and the drift is bounded.
`m5` applies that rule to any per-step penetration series.  Two series feed it here:
  * `stack_penetration` -- the reference's own per-step figure for a vertical stack (adjacent
    spacing against the rest pitch, and the lowest body against the ground);
  * the deepest solved contact of every step (BoxContactEngine / bead engines
    `max_depth_device`), the same quantity for piles that are not a single stack.
"""
from __future__ import annotations

import numpy as np

R = 0.05            # bead radius of the reference's engines (contact_engine_gpu.py:25)
PEN_OVER_R_MAX = 0.5
DRIFT_FRAC = 0.1    # secular drift: extrapolated change over the second half > R / 10


def stack_penetration(z, pitch, ground=None) -> float:
    """Penetration of a vertical stack from its body heights: max(pitch - diff(sorted z))
    (engine_metrics.py:274-276); with `ground` (the rest height of the lowest body) also
    ground - min(z)."""
    zs = np.sort(np.asarray(z, np.float64))
    pen = float(np.max(pitch - np.diff(zs))) if len(zs) > 1 else -np.inf
    if ground is not None:
        pen = max(pen, float(ground - zs[0]))
    return pen


def m5(pens) -> dict:
    """The M5 gate over a per-step penetration series (metres)."""
    p = np.asarray(pens, np.float64)
    if len(p) < 4:
        raise ValueError("m5: needs at least 4 steps")
    h = len(p) // 2
    tail = p[h:]
    slope = float(np.polyfit(np.arange(len(tail)), tail, 1)[0])
    drift = "secular" if abs(slope) * h > DRIFT_FRAC * R else "bounded"
    mx = float(p.max())
    ok = bool(mx / R < PEN_OVER_R_MAX and drift == "bounded")
    return {"max_pen_m": mx, "max_pen_over_R": mx / R, "final_pen_m": float(p[-1]), "drift_class": drift,
            "drift_slope_m_per_step": slope, "threshold_pen_over_R": PEN_OVER_R_MAX, "steps": int(len(p)),
            "status": "PASS" if ok else "FAIL"}
