"""The rollout adjoint of the device box world (rollout.BoxRollout behind torch.autograd) against
central finite differences of the same float64 rollouts, and its memory.

A rollout is piecewise smooth: the contact set, the kept manifold points and the colouring are
discrete, and the reference's velocity bias has a kink at zero gap (g / h for an open contact, 0
inside the 0.1 mm penetration allowance).  A box that lands closes its gap to zero exactly and
then rests on that kink, where the two one-sided derivatives differ by 1 / h; central
differences there average them.  The scenes here start every contact inside the penetration
allowance (or well open) and keep the discrete structure, so differences are a valid reference:
a sliding box, a stack with a sliding top, a box sliding half across another (points clipped
where an edge crosses the reference face), and slowly moving pyramids of the pushed-pyramid
workload."""
import numpy as np
import pytest
import torch

from conftest import cuda_ok

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_ok(), reason="needs a CUDA device")]

IN = 5e-5  # start 0.05 mm deep, inside the 0.1 mm allowance


def _mods(me):
    from importlib import import_module
    return import_module("motion_engine_b200.world"), import_module("motion_engine_b200.rollout")


def _grads(RO, w, v0, mu, target, steps):
    ro = RO.BoxRollout(w)
    v0r = v0.clone().requires_grad_(True)
    mur = mu.clone().requires_grad_(True)
    x = RO.rollout(ro, v0r, mur, steps)
    ((x - target) ** 2).sum().backward()
    return ro, v0r.grad.clone(), mur.grad.clone()


def _check(RO, ro, v0, mu, target, steps, gv, gm, dv, dm, eps, rel):
    """The adjoint's directional derivative against central differences at eps and eps / 3, both
    within `rel` of the gradient's largest component.  eps is large enough to clear the rounding
    of the fixed-point velocity sums (1e-10 m/s: at eps 1e-6 it moves a difference by ~1e-3
    relative) and small enough to keep the structure."""
    loss = lambda xx: ((xx - target) ** 2).sum()
    an = float((gv * dv).sum() + (gm * dm).sum())
    f1 = float(RO.fd_directional(ro, v0, mu, steps, loss, dv, dm, eps))
    f2 = float(RO.fd_directional(ro, v0, mu, steps, loss, dv, dm, eps / 3))
    scale = max(float(gv.abs().max()), float(gm.abs().max()), abs(an))
    assert abs(an - f1) <= rel * scale and abs(an - f2) <= rel * scale, (an, f1, f2, scale)


def _unit(like, idx):
    d = torch.zeros_like(like)
    d[idx] = 1.0
    return d


def test_sliding_box(me):
    """A box sliding on the ground (four corner contacts, slipping all along): v0 and mu."""
    W, RO = _mods(me)
    w = W.BoxWorldB200(dt=1 / 240, mu=0.4, iters=16, substeps=2, warm_start=True)
    w.add([0.1, 0.15, 0.05], 2.0, [0.0, 0.0, 0.05 - IN])
    w._build()
    dev = w.dev
    v0 = torch.tensor([[0.8, 0.3, 0.0]], dtype=torch.float64, device=dev)
    mu = torch.tensor([0.4], dtype=torch.float64, device=dev)
    target = torch.tensor([[0.1, 0.1, 0.05]], dtype=torch.float64, device=dev)
    ro, gv, gm = _grads(RO, w, v0, mu, target, 20)
    zv, zm = torch.zeros_like(v0), torch.zeros_like(mu)
    for dv, dm in ((_unit(v0, (0, 0)), zm), (_unit(v0, (0, 1)), zm), (zv, _unit(mu, 0))):
        _check(RO, ro, v0, mu, target, 20, gv, gm, dv, dm, 1e-3, 1e-5)


def test_stack_with_a_sliding_top(me):
    """Two boxes face on face (redundant contacts: the impulses the sweeps reach depend on the
    warm start), both pushed, 200 sweeps a substep, 20 steps: every component of the v0
    gradient and mu."""
    W, RO = _mods(me)
    w = W.BoxWorldB200(dt=1 / 240, mu=0.5, iters=200, substeps=2, warm_start=True)
    w.add([0.1] * 3, 1.0, [0, 0, 0.1 - IN])
    w.add([0.1] * 3, 1.0, [0.002, 0.001, 0.3 - 2 * IN])
    w._build()
    dev = w.dev
    rng = np.random.default_rng(0)
    v0 = torch.tensor([[0.1, 0.0, 0.0], [0.0, 0.4, 0.0]], dtype=torch.float64, device=dev)
    mu = torch.full((2,), 0.5, dtype=torch.float64, device=dev)
    target = w.x[:2].clone() + torch.tensor(rng.normal(0, 0.05, (2, 3)), device=dev)
    ro, gv, gm = _grads(RO, w, v0, mu, target, 20)
    zv, zm = torch.zeros_like(v0), torch.zeros_like(mu)
    for i in range(2):
        for k in range(3):
            _check(RO, ro, v0, mu, target, 20, gv, gm, _unit(v0, (i, k)), zm, 1e-4, 3e-5)
        _check(RO, ro, v0, mu, target, 20, gv, gm, zv, _unit(mu, i), 1e-4, 3e-5)


def test_offset_box_sliding_on_a_box(me):
    """A box resting half across another of the same size and sliding over it: the faces
    overlap in a rectangle whose corners are edge crossings of the two faces, so the contact
    points move along the edges as the boxes move -- the three-plane point model of the
    adjoint."""
    W, RO = _mods(me)
    w = W.BoxWorldB200(dt=1 / 240, mu=0.3, iters=64, substeps=2, warm_start=True)
    w.add([0.1, 0.1, 0.1], 1.0, [0.0, 0.0, 0.1 - IN])
    w.add([0.1, 0.1, 0.1], 0.6, [0.05, 0.03, 0.3 - 2 * IN])
    w._build()
    dev = w.dev
    rng = np.random.default_rng(3)
    v0 = torch.tensor([[0.0, 0.0, 0.0], [-0.12, 0.05, 0.0]], dtype=torch.float64, device=dev)
    mu = torch.full((2,), 0.3, dtype=torch.float64, device=dev)
    target = w.x[:2].clone() + torch.tensor(rng.normal(0, 0.05, (2, 3)), device=dev)
    ro, gv, gm = _grads(RO, w, v0, mu, target, 20)
    zv, zm = torch.zeros_like(v0), torch.zeros_like(mu)
    for k in range(2):
        _check(RO, ro, v0, mu, target, 20, gv, gm, _unit(v0, (1, k)), zm, 3e-4, 1e-4)
    _check(RO, ro, v0, mu, target, 20, gv, gm, zv, _unit(mu, 1), 3e-4, 1e-4)


def test_moving_pyramid(me):
    """Two pyramids of the pushed-pyramid workload (64 boxes, layers 8-4-2-1-1 in four slices,
    1 mm side gaps: open contacts inside the margin; +-0.3 mm jitter, so the faces overlap in
    offset rectangles; many colours; 16 sweeps a substep, 2 substeps), every face-on-face
    contact inside the allowance, the plate out of reach, the boxes moving at a tenth of the
    workload's initial velocities: directional derivatives in v0 over 10 steps.  (Boxes that
    start at rest fall together: the first substep's box-on-box contacts then have z = 0 exactly,
    the apex of the friction cone, where the projection has no derivative -- central
    differences average its one-sided slopes, the adjoint takes the cone's interior.)  Here the
    differences themselves scatter by about 1 % between steps of 3e-6 and 1e-6 (the 1e-10 m/s
    rounding of the velocity sums over 5 000 contact updates a substep), hence the bound."""
    W, RO = _mods(me)
    from importlib import import_module
    S = import_module("motion_engine_b200.scenes")
    d = S.pushed_pyramids(n_scenes=2, jitter=3e-4)
    x = d["x"].copy()
    h = 0.1
    dyn = d["kin"] == 0
    layer = np.rint((x[:, 2] - h) / (2 * h + 1e-3)).astype(int)
    x[dyn, 2] = h - IN + layer[dyn] * (2 * h - IN)
    x[~dyn, 0] -= 0.2  # keep the plate away for the whole rollout
    w = W.BoxWorldB200(dt=1 / 240, mu=0.5, iters=16, substeps=2, warm_start=True)
    for i in range(len(d["half"])):
        w.add(d["half"][i], float(d["mass"][i]), x[i], kin=int(d["kin"][i]), v_kin=d["v_kin"][i],
              mu=float(d["mu"][i]), scene=int(d["scene"][i]))
    w._build()
    dev = w.dev
    mu = torch.tensor(d["mu"], device=dev)
    target = torch.tensor(d["target"], device=dev)
    rng = np.random.default_rng(4)
    dmask = torch.tensor(dyn, device=dev, dtype=torch.float64)
    v = 0.1 * torch.tensor(d["v0"], device=dev)
    ro, gv, gm = _grads(RO, w, v, mu, target, 10)
    for _ in range(2):
        dv = torch.tensor(rng.normal(0, 1, (w.n, 3)), device=dev) * dmask[:, None]
        _check(RO, ro, v, mu, target, 10, gv, gm, dv, torch.zeros_like(mu), 3e-6, 2e-2)


def test_device_memory_is_flat_in_the_rollout_length(me):
    """Per-substep checkpoints live in pinned host memory: the device's peak over forward and
    backward does not grow with the number of steps."""
    W, RO = _mods(me)
    from importlib import import_module
    S = import_module("motion_engine_b200.scenes")
    d = S.pushed_pyramids(n_scenes=2)
    w = W.BoxWorldB200(dt=1 / 240, mu=0.5, iters=16, substeps=2, warm_start=True)
    for i in range(len(d["half"])):
        w.add(d["half"][i], float(d["mass"][i]), d["x"][i], kin=int(d["kin"][i]), v_kin=d["v_kin"][i],
              mu=float(d["mu"][i]), scene=int(d["scene"][i]))
    w._build()
    dev = w.dev
    ro = RO.BoxRollout(w)
    v0 = torch.tensor(d["v0"], device=dev)
    mu = torch.tensor(d["mu"], device=dev)
    target = torch.tensor(d["target"], device=dev)
    peaks = []
    for steps in (15, 30, 60):
        torch.cuda.synchronize()
        torch.cuda.reset_peak_memory_stats(dev)
        v0r = v0.clone().requires_grad_(True)
        mur = mu.clone().requires_grad_(True)
        x = RO.rollout(ro, v0r, mur, steps)
        ((x - target) ** 2).sum().backward()
        torch.cuda.synchronize()
        # the sweep record of one substep is sized by the most contacts a substep had
        peaks.append(torch.cuda.max_memory_allocated(dev) - 8 * ro.trace.numel())
        assert len(ro.checkpoints) == steps * 2
    print("device peak bytes (less the one-substep sweep record) at 15 / 30 / 60 steps:", peaks)
    assert max(peaks) - min(peaks) <= 1024 * 1024
