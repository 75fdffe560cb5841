"""Batched proximal ADMM and its adjoint on the device: the reference's ``BatchProxADMMGPU``
(src/motion_engine/ncp/ncp_batch_gpu.py:918-1313) behind its own method names.

B independent contact problems of nc point contacts on nv generalised velocities (a legged
stance: J (B, 3 nc, nv), M^-1 (B, nv, nv), v_free (B, nv), mu (B, nc)) are solved matrix-free
with int64-accumulated M^-1 J^T products, by ADMM with a preconditioned CG x-step and a
per-problem convergence mask, then differentiated by grad_affine.  ``b2c_admm_solve`` runs the
whole of it -- set-up, iterations, refreshes, active set, both gradient directions -- with one
warp per problem in ONE launch (the reference: 133 launches per ADMM iteration).

    s = BatchProxADMM(B, nv, nc).upload(J, Minv, v_free, mu, dt)
    s.set_rho("regime")
    fwd = s.forward(n_iter=200, cg_iters=8)              # Fwd(lam, u, resenv, iters, n_active, ms, rho)
    out = s.step_and_grad(200, 8, 4, 1e-8, grad_cg=60)   # + dlam_tau, dv_tau, dlam_mu, v_plus
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib


@dataclass
class Fwd:
    lam: np.ndarray
    u: np.ndarray
    resenv: np.ndarray
    iters: int
    n_active: int
    ms: float
    rho: np.ndarray


class BatchProxADMM:
    def __init__(self, B, nv, nc, device="cuda"):
        if not torch.cuda.is_available():
            raise RuntimeError("BatchProxADMM: no CUDA device; b2c_admm_solve runs only on the GPU")
        if not (1 <= int(nc) <= _lib.ADMM_MAX_CONTACTS and 1 <= int(nv) <= _lib.ADMM_MAX_DOFS):
            raise ValueError(f"BatchProxADMM: nc must be in 1..{_lib.ADMM_MAX_CONTACTS} and nv in "
                             f"1..{_lib.ADMM_MAX_DOFS} (got nc={nc}, nv={nv})")
        self.L = _lib.load()
        self.dev = torch.device(device)
        self.B, self.NV, self.C = int(B), int(nv), int(nc)
        B_, C, NV = self.B, self.C, self.NV
        f64 = lambda *s: torch.zeros(s, dtype=torch.float64, device=self.dev)
        i32 = lambda *s: torch.zeros(s, dtype=torch.int32, device=self.dev)
        self.lam, self.u, self.v_plus = f64(B_, C, 3), f64(B_, C, 3), f64(B_, NV)
        self.res, self.mask, self.rho = f64(B_), i32(B_), f64(B_)
        self.nslip, self.labels = i32(B_), i32(B_, C)
        self.dlam_tau, self.dv_tau, self.dlam_mu = f64(B_, C, 3), f64(B_, NV), f64(B_, C, 3)
        self.dbv = f64(B_, C, 3)
        self.rho_mode = _lib.ADMM_RHO["regime"]
        self.dt = 1.0
        self.alpha_eta, self.jacobi_sweeps = 0.0, 10
        self._in = None
        self._b = None

    def _t(self, a, shape):
        t = torch.as_tensor(a, dtype=torch.float64)
        return t.reshape(shape).to(self.dev).contiguous()

    def upload(self, J, Minv, v_free, mu, dt, alpha_eta=0.0, jacobi_sweeps=10, b=None):
        """NB:974-1000.  Arrays may be numpy or torch (host or device).  `b` (B, nc, 3), when
        given, is the free contact velocity itself (a stored problem's q) instead of J v_free."""
        B_, C, NV = self.B, self.C, self.NV
        self._b = None if b is None else self._t(b, (B_, C, 3))
        mu_t = torch.as_tensor(mu, dtype=torch.float64).reshape(-1)
        mu_t = mu_t.expand(B_ * C) if mu_t.numel() == 1 else mu_t
        self._in = (self._t(J, (B_, 3 * C, NV)), self._t(Minv, (B_, NV, NV)), self._t(v_free, (B_, NV)),
                    self._t(mu_t, (B_, C)))
        self.dt = float(dt)
        self.alpha_eta, self.jacobi_sweeps = float(alpha_eta), int(jacobi_sweeps)
        return self

    def set_rho(self, mode):
        """NB:1013-1022: 'sqrt' | 'lmin' | 'lmax' | 'regime' (the bilateral test); computed on the
        device at the start of each solve."""
        if mode == "regime_probe":
            raise ValueError("BatchProxADMM.set_rho: 'regime_probe' (rho from an ADMM probe's labels) is not "
                             "provided; 'regime' reads the regime from the bilateral solution")
        self.rho_mode = _lib.ADMM_RHO[mode]
        return self

    def set_rho_host(self, rho_vec):
        self.rho.copy_(self._t(rho_vec, (self.B,)))
        self.rho_mode = _lib.ADMM_RHO["given"]
        return self

    def _struct(self, dbv=None):
        p = lambda t: t.data_ptr()
        J, Mi, vf, mu = self._in
        return _lib.Admm(self.B, self.C, self.NV, p(J), p(Mi), p(vf), p(mu), p(self.lam), p(self.u), p(self.v_plus),
                         p(self.res), p(self.mask), p(self.rho), p(self.nslip), p(self.labels), p(self.dlam_tau),
                         p(self.dv_tau), p(self.dlam_mu), p(dbv) if dbv is not None else None,
                         p(self._b) if self._b is not None else None)

    def launch(self, flags, n_iter=0, cg_iters=8, refresh_every=4, tol=1e-8, chunk=0, desax=True, jdir=0,
               n_calls=None, grad_cg=60, do_mu=True, dbv=None, stream=None):
        """One b2c_admm_solve launch on `stream` (default: the current stream), asynchronous."""
        if self._in is None:
            raise RuntimeError("BatchProxADMM: upload() first")
        prm = _lib.AdmmParams(int(flags), int(n_iter), int(cg_iters), int(refresh_every), float(tol), int(chunk),
                              1 if desax else 0, int(self.rho_mode), self.jacobi_sweeps, self.alpha_eta, self.dt,
                              int(jdir), int(n_calls) if n_calls else 0, int(grad_cg), 1 if do_mu else 0)
        st = stream if stream is not None else torch.cuda.current_stream(self.dev)
        a = self._struct(dbv)
        _lib.check(self.L.b2c_admm_solve(ctypes.byref(a), ctypes.byref(prm), ctypes.c_void_p(st.cuda_stream)),
                   "b2c_admm_solve")

    def forward(self, n_iter=100, cg_iters=8, refresh_every=4, tol=1e-8, chunk=25, desax=True, readback=True):
        """NB:1112-1143: the set-up and n_iter iterations from zero, the refresh count restarting
        every `chunk` iterations as in the reference's chunked graph."""
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        self.launch(_lib.ADMM_FORWARD, n_iter, cg_iters, refresh_every, tol, chunk=min(int(chunk), int(n_iter)),
                    desax=desax)
        b.record()
        b.synchronize()
        if not readback:
            return Fwd(None, None, None, int(n_iter), -1, a.elapsed_time(b), None)
        return Fwd(lam=self.lam.cpu().numpy(), u=self.u.cpu().numpy(), resenv=self.res.cpu().numpy(),
                   iters=int(n_iter), n_active=int(self.mask.sum().item()), ms=a.elapsed_time(b),
                   rho=self.rho.cpu().numpy())

    def step_and_grad(self, n_iter, cg_iters=8, refresh_every=4, tol=1e-8, n_calls=None, grad_cg=60, do_mu=True,
                      jdir=0, stream=None):
        """NB's captured step-and-gradient (capture_step_grad, NB:1103-1110 with _fwd_part and
        _grad_part): the forward in one block, v+, then d/dtau_jdir and d/dmu.  Asynchronous."""
        self.launch(_lib.ADMM_FORWARD | _lib.ADMM_GRADIENT, n_iter, cg_iters, refresh_every, tol, chunk=0,
                    jdir=jdir, n_calls=n_calls, grad_cg=grad_cg, do_mu=do_mu, stream=stream)
        return self

    def grad_given(self, lam, u, dbv, n_calls=None, cg=60):
        """grad_affine at given impulses and contact velocities for the b-directions dbv (B, nc, 3),
        the reference's own adjoint test (tests/test_ncp_batch_adjoint.py:55-76)."""
        self.lam.copy_(self._t(lam, (self.B, self.C, 3)))
        self.u.copy_(self._t(u, (self.B, self.C, 3)))
        self.dbv.copy_(self._t(dbv, (self.B, self.C, 3)))
        self.launch(_lib.ADMM_GRAD_GIVEN, n_calls=n_calls, grad_cg=cg, dbv=self.dbv)
        return self.dlam_tau.cpu().numpy()
