"""The FP64 re-solve: the float32 step's own solve repeated in float64 (oracle/liboracle64.so, the
oracle's source compiled in double precision) on the same inputs, so that a float32 error is
measured against the same algorithm in exact-ish arithmetic on the same contacts -- not against
a different trajectory, which in a pile or a lattice parts from it at the first contact that
appears, disappears or changes its selected points under a rounding.

* Coloured bead engines: the float32 step's kept contacts, with the impulses its solve started
  from (warm-started and reduced), are handed to the float64 oracle (`inject`), which solves
  them from the same body state (one substep).
* Box engine: the float64 oracle runs one substep from the same body state and warm store; its
  narrowphase is float64 in both builds, so the contact set is the same (checked by key).

`compare` reports per impulse row the largest |f32 - f64| over the matched contacts relative to
the row's largest f64 magnitude, and the velocities' largest |d| relative to a velocity scale."""
import numpy as np

IMPULSES = ("jn", "jt1", "jt2", "jp")


def resolve_injected(make64, state, kept, start, dt):
    """Float64 oracle (make64()) solving `kept` from the impulses `start`, one substep of dt from
    `state` (xc, q, v, w)."""
    o = make64()
    o.set_body_state(*state)
    o.inject(kept, start)
    o.step(dt, 1)
    return o


def resolve_from_store(make64, state, warm, dt):
    """Float64 oracle advanced one substep of dt from `state` and the warm store `warm`."""
    o = make64()
    o.set_body_state(*state)
    o.set_warm_store(warm)
    o.step(dt, 1)
    return o


def compare(kept32, state32, kept64, state64, v_scale):
    common, i32, i64 = np.intersect1d(kept32["ckeys"], kept64["ckeys"], return_indices=True)
    out = {"matched": len(common) / max(len(kept32["ckeys"]), len(kept64["ckeys"]), 1)}
    for f in IMPULSES:
        a = kept32[f][i32].astype(np.float64)
        b = kept64[f][i64].astype(np.float64)
        out[f] = float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30)) if len(b) else 0.0
    _, _, v32, w32 = (np.asarray(x, np.float64) for x in state32)
    _, _, v64, w64 = (np.asarray(x, np.float64) for x in state64)
    out["v"] = float(np.abs(v32 - v64).max() / v_scale)
    out["w"] = float(np.abs(w32 - w64).max() / v_scale)
    return out
