"""Differentiable rollouts of the box world: a hand-written adjoint of the substep loop behind a
torch.autograd.Function.

    x_final = rollout(ro, v0, mu, steps)           # torch tensors on the world's device
    loss(x_final).backward()                        # -> v0.grad, mu.grad

Forward: `steps` macro steps of the world (BoxWorldB200: SAT contacts, build_scene, the exact-cone
NCP, integration) from the world's initial positions and orientations, the initial velocities
v0 (n, 3) and the per-body friction mu (n).  Before every substep the state it starts from --
positions, quaternions, velocities, angular velocities and the warm-start store -- is copied to
pinned host memory: one checkpoint per substep, so the device memory of a rollout does not grow
with its length.

Backward, substep by substep from the last: the substep is recomputed from its checkpoint (the
same contacts, the same warm start, the same sweeps, bitwise: the same impulses), this time
recording where every contact update of every sweep started from; then its adjoint runs on the
device --
  * the integration in reverse (x' = x + v' h, q' = normalize(q + 0.5 h (w', 0) q));
  * lambda_bar = J Minv V_bar through V' = v_free + Minv J^T lambda, plus the next substep's
    warm-start adjoint for the contacts of the same key (b2c_world_warm_adjoint);
  * the recorded sweeps in reverse (b2c_ncp_adjoint_unrolled): the exact derivative of the
    impulses the sweeps computed -- converged or not -- with respect to the free velocity, the
    bias, the friction, the Jacobian blocks, Minv, the step sizes and the warm start;
  * the bias through the contact gaps to the poses, the friction of each contact to its bodies
    (sqrt(mu_a mu_b), ground mu_a), the blocks through the lever arms, the contact point and
    frame, Minv through the world inertia, and v_free = [v + g h, w] to the velocities.
The contact set, the clipping of the manifold and the colouring are held at the substep's values
(they are piecewise constant).

Gradients come back as float64 tensors shaped like v0 and mu.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .engine import _ptr


class _Checkpoint:
    """Pinned host copy of the state a substep starts from."""

    def __init__(self, world):
        n = world.n
        self.state = torch.empty((n, 13), dtype=torch.float64, pin_memory=True)
        self.have_warm = False
        self.warm_n = 0
        self.warm_keys = None
        self.warm_lam = None

    def save(self, world, buf):
        n = world.n
        torch.cat([world.x[:n], world.q[:n], world.v[:n], world.w[:n]], dim=1, out=buf)
        self.state.copy_(buf, non_blocking=True)
        self.have_warm = world._have_warm
        if world.warm_start and world._have_warm:
            k = int(world.warm_n.item())
            self.warm_n = k
            self.warm_keys = torch.empty(max(k, 1), dtype=torch.int64, pin_memory=True)
            self.warm_lam = torch.empty((max(k, 1), 3), dtype=torch.float64, pin_memory=True)
            self.warm_keys[:k].copy_(world.warm_keys[:k], non_blocking=True)
            self.warm_lam[:k].copy_(world.warm_lam[:k], non_blocking=True)

    def restore(self, world):
        n = world.n
        st = self.state.to(world.dev, non_blocking=True)
        world.x[:n].copy_(st[:, 0:3])
        world.q[:n].copy_(st[:, 3:7])
        world.v[:n].copy_(st[:, 7:10])
        world.w[:n].copy_(st[:, 10:13])
        world._have_warm = self.have_warm
        if world.warm_start and self.have_warm:
            k = self.warm_n
            world.warm_n.fill_(k)
            world.warm_keys[:k].copy_(self.warm_keys[:k], non_blocking=True)
            world.warm_lam[:k].copy_(self.warm_lam[:k], non_blocking=True)


class BoxRollout:
    """The rollout machinery of one world: initial poses, substep checkpoints, forward and
    adjoint."""

    def __init__(self, world):
        if not world._built:
            world._build()
        self.world = world
        n = world.n
        self.x0 = world.x[:n].clone()
        self.q0 = world.q[:n].clone()
        self.w0 = world.w[:n].clone()
        self.checkpoints = []
        self._buf = torch.empty((n, 13), dtype=torch.float64, device=world.dev)
        dev, MC = world.dev, world.MC
        f64 = lambda *s: torch.zeros(*s, dtype=torch.float64, device=dev)
        self.xb, self.qb, self.vb, self.wb = f64(n, 3), f64(n, 4), f64(n, 3), f64(n, 3)
        self.xb_in, self.qb_in = f64(n, 3), f64(n, 4)
        self.Vb, self.vfree_b, self.Vscr = f64(n, 6), f64(n, 6), f64(n, 6)
        self.lam_b, self.bias_b, self.mu_b = f64(MC, 3), f64(MC, 3), f64(MC)
        self.Ja_b, self.Jb_b, self.Minv_b = f64(MC, 18), f64(MC, 18), f64(n, 36)
        self.mub_body = f64(n)
        self.acc = torch.zeros((max(n, 1), 8), dtype=torch.float64, device=dev)
        # the warm-start adjoint handed from a substep to the one before it, by contact key
        self.adj_keys = torch.zeros(MC, dtype=torch.int64, device=dev)
        self.adj_lam = f64(MC, 3)
        self.adj_n = torch.zeros(1, dtype=torch.int32, device=dev)
        self.trace = f64(1)
        self.words = int(world.L.b2c_ncp_trace_words())
        self.max_c = 0

    def _size_trace(self):
        """The sweep record of one substep (b2c_ncp_trace_words() doubles per contact and sweep),
        sized once per backward by the most contacts a substep of the forward had."""
        need = self.words * self.world.iters * max(self.max_c, 1)
        if self.trace.numel() < need:
            self.trace = None
            self.trace = torch.empty(need, dtype=torch.float64, device=self.world.dev)

    def _reset(self, v0, mu):
        w, n = self.world, self.world.n
        w.x[:n].copy_(self.x0)
        w.q[:n].copy_(self.q0)
        w.v[:n].copy_(v0.to(w.dev, torch.float64))
        w.w[:n].copy_(self.w0)
        w.body_mu[:n].copy_(mu.to(w.dev, torch.float64))
        w._have_warm = False
        w.warm_n.zero_()

    def forward(self, v0, mu, steps, checkpoint=True):
        """Run the rollout; returns the final positions (n, 3) float64 on the device."""
        w = self.world
        self._reset(v0, mu)
        h = w.dt / max(1, w.substeps)
        self.checkpoints = []
        self.max_c = 0
        for _ in range(int(steps) * max(1, w.substeps)):
            if checkpoint:
                cp = _Checkpoint(w)
                cp.save(w, self._buf)
                self.checkpoints.append(cp)
            w._substep(h)
            self.max_c = max(self.max_c, w.n_contacts)
        self.h = h
        return w.x[:w.n].clone()

    def backward(self, x_bar):
        """Adjoint of the last forward: gradients of <x_bar, x_final> with respect to v0 (n, 3)
        and mu (n), float64 on the device."""
        w, L = self.world, self.world.L
        s = w.solver
        st = w._stream()
        n = w.n
        self.xb.copy_(x_bar.to(w.dev, torch.float64))
        self.qb.zero_()
        self.vb.zero_()
        self.wb.zero_()
        self.mub_body.zero_()
        self.acc.zero_()
        self.adj_n.zero_()
        params = s._params(None, True)
        h = self.h
        p = lambda t: ctypes.c_void_p(_ptr(t))
        self._size_trace()
        for cp in reversed(self.checkpoints):
            cp.restore(w)
            C = w.contacts_device()
            w.scene_device(C, h)
            warm = False
            if C:
                warm = w.warm_start and w._have_warm
                trace = self.trace[:self.words * w.iters * C]
                w.solve_device(C, w.iters, warm, trace=trace)
                V6 = s.v
            else:
                V6 = s.vfree
            _lib.check(L.b2c_world_adj_begin(ctypes.byref(w.c_world), ctypes.byref(s.c_scene), p(V6), float(h),
                                             p(self.xb), p(self.qb), p(self.vb), p(self.wb), p(self.xb_in),
                                             p(self.qb_in), p(self.Vb), p(self.vfree_b), p(self.lam_b), st),
                       "b2c_world_adj_begin")
            if C:
                if w.warm_start:
                    _lib.check(L.b2c_world_warm_adjoint(ctypes.byref(w.c_world), C, p(self.adj_keys), p(self.adj_lam),
                                                        p(self.adj_n), p(self.lam_b), st), "b2c_world_warm_adjoint")
                self.bias_b[:C].zero_()
                self.mu_b[:C].zero_()
                self.Ja_b[:C].zero_()
                self.Jb_b[:C].zero_()
                self.Minv_b.zero_()
                _lib.check(L.b2c_ncp_adjoint_unrolled(ctypes.byref(s.c_scene), ctypes.byref(s.c_state),
                                                      ctypes.byref(params), w.iters, p(trace), trace.numel(),
                                                      p(self.lam_b), p(self.Vscr), p(self.vfree_b), p(self.bias_b),
                                                      p(self.mu_b), p(self.Ja_b), p(self.Jb_b), p(self.Minv_b), st),
                           "b2c_ncp_adjoint_unrolled")
                if warm:  # this substep started from the previous one's impulses of the same keys
                    self.adj_keys[:C].copy_(w.key[:C])
                    self.adj_lam[:C].copy_(self.lam_b[:C])
                    self.adj_n.fill_(C)
                else:
                    self.adj_n.zero_()
            else:
                self.adj_n.zero_()
            self.xb.copy_(self.xb_in)
            self.qb.copy_(self.qb_in)
            _lib.check(L.b2c_world_adj_end(ctypes.byref(w.c_world), ctypes.byref(s.c_scene), p(s.lam), p(V6),
                                           p(self.Vb), float(h), p(self.bias_b), p(self.mu_b), p(self.vfree_b),
                                           p(self.Ja_b), p(self.Jb_b), p(self.Minv_b), p(self.acc), p(self.xb),
                                           p(self.qb), p(self.vb), p(self.wb), p(self.mub_body), st),
                       "b2c_world_adj_end")
            if C:
                s._check_stats()
        return self.vb[:n].clone(), self.mub_body[:n].clone()


class _RolloutFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, v0, mu, ro, steps):
        x = ro.forward(v0.detach(), mu.detach(), steps, checkpoint=True)
        ctx.ro = ro
        ctx.dtypes = (v0.dtype, mu.dtype)
        return x

    @staticmethod
    def backward(ctx, gx):
        gv, gmu = ctx.ro.backward(gx.detach())
        return gv.to(ctx.dtypes[0]), gmu.to(ctx.dtypes[1]), None, None


def rollout(ro: BoxRollout, v0: torch.Tensor, mu: torch.Tensor, steps: int) -> torch.Tensor:
    """Final positions (n, 3) after `steps` macro steps from initial velocities v0 (n, 3) and
    per-body friction mu (n); differentiable in v0 and mu through the hand-written adjoint."""
    return _RolloutFn.apply(v0, mu, ro, int(steps))


def fd_directional(ro: BoxRollout, v0, mu, steps, loss_fn, dv, dmu, eps=1e-3):
    """Central finite difference (loss(+eps d) - loss(-eps d)) / (2 eps) of a per-scene loss
    vector along the direction (dv, dmu), on the same float64 forward."""
    with torch.no_grad():
        lp = loss_fn(ro.forward(v0 + eps * dv, mu + eps * dmu, steps, checkpoint=False))
        lm = loss_fn(ro.forward(v0 - eps * dv, mu - eps * dmu, steps, checkpoint=False))
    return (lp - lm) / (2 * eps)
