"""Batched exact-cone NCP with an implicit adjoint, over libb2c's b2c_bncp_* entry points.

The host mirror of the reference's batched solver and adjoint (BatchProxADMMGPU,
src/motion_engine/ncp/ncp_batch_gpu.py:918-1313: many small contact problems solved in one
launch, with a convergence mask, and the gradient of the solution through the implicit-function
theorem on the fixed contact branch, grad_affine :1172-1186) and of the CPU sensitivity it is
checked against (src/motion_engine/ncp/ncp_ref.py:907-959).  Problems are given in Delassus form
G = J Minv J^T, b = J v_free + bias; `delassus` builds them from Jacobians in torch, so gradients
reach J's inputs through torch's own autograd.

`ncp_solve(G, b, mu)` is differentiable in b and mu (a torch.autograd.Function whose backward is
the batched vector-Jacobian product).  The derivative is that of the exact NCP solution on its
current branch: NaN when the branch is singular (redundant contacts) or on a branch boundary, as
the reference's guarded response reports.
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib

STATUS_SINGULAR = 1
STATUS_BOUNDARY = 2
LABELS = ("open", "stick", "slip")


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


class BatchNCP:
    """One batch of small contact problems on the GPU (float64)."""

    def __init__(self, G: torch.Tensor, b: torch.Tensor, mu: torch.Tensor, nc: torch.Tensor = None):
        """G (B, n, n), b (B, n), mu (B, n/3) float64 CUDA tensors; nc (B,) the contacts of each
        problem when fewer than n/3 (rows and columns beyond 3 nc are ignored)."""
        self.L = _lib.load()
        if G.dim() != 3 or G.shape[1] != G.shape[2] or G.shape[1] % 3:
            raise ValueError("BatchNCP: G must be (B, n, n) with n a multiple of 3")
        B, n = G.shape[0], G.shape[1]
        if n > int(self.L.b2c_bncp_max_rows()):
            raise ValueError(f"BatchNCP: {n // 3} contacts per problem exceeds {self.L.b2c_bncp_max_rows() // 3}")
        dev = G.device
        f64 = lambda t: t.detach().to(dev, torch.float64).contiguous()
        self.G, self.b, self.mu = f64(G), f64(b.reshape(B, n)), f64(mu.reshape(B, n // 3))
        self.nc = (torch.full((B,), n // 3, dtype=torch.int32, device=dev) if nc is None
                   else nc.to(dev, torch.int32).contiguous())
        self.B, self.n = B, n
        self.lam = torch.zeros((B, n), dtype=torch.float64, device=dev)
        self.res = torch.zeros(B, dtype=torch.float64, device=dev)
        self.iters = torch.zeros(B, dtype=torch.int32, device=dev)
        self.labels = torch.zeros((B, n // 3), dtype=torch.int32, device=dev)
        self.status = torch.zeros(B, dtype=torch.int32, device=dev)
        self.c = _lib.Bncp(B, n, *(_ptr(t).value for t in (self.nc, self.G, self.b, self.mu, self.lam, self.res,
                                                             self.iters, self.labels, self.status)))

    def _stream(self):
        return ctypes.c_void_p(torch.cuda.current_stream(self.G.device).cuda_stream)

    def solve(self, max_iters: int = 5000, tol: float = 1e-14, check: int = 10, warm: torch.Tensor = None):
        """Solve every problem; returns lambda (B, n).  `iters` < max_iters marks the converged."""
        if warm is None:
            self.lam.zero_()
        else:
            self.lam.copy_(warm.reshape(self.B, self.n))
        _lib.check(self.L.b2c_bncp_solve(ctypes.byref(self.c), int(max_iters), float(tol), int(check),
                                         self._stream()), "b2c_bncp_solve")
        return self.lam

    def sensitivity(self):
        """(dlam/dmu (B, n, n/3), dlam/db (B, n, n)) at the current lambda; NaN on singular or
        boundary branches (status)."""
        dmu = torch.empty((self.B, self.n, self.n // 3), dtype=torch.float64, device=self.G.device)
        db = torch.empty((self.B, self.n, self.n), dtype=torch.float64, device=self.G.device)
        _lib.check(self.L.b2c_bncp_sensitivity(ctypes.byref(self.c), _ptr(dmu), _ptr(db), self._stream()),
                   "b2c_bncp_sensitivity")
        return dmu, db

    def vjp(self, glam: torch.Tensor):
        """(gb, gmu) = ((dlam/db)^T glam, (dlam/dmu)^T glam) at the current lambda."""
        g = glam.detach().to(torch.float64).reshape(self.B, self.n).contiguous()
        gb = torch.empty((self.B, self.n), dtype=torch.float64, device=self.G.device)
        gmu = torch.empty((self.B, self.n // 3), dtype=torch.float64, device=self.G.device)
        _lib.check(self.L.b2c_bncp_vjp(ctypes.byref(self.c), _ptr(g), _ptr(gb), _ptr(gmu), self._stream()),
                   "b2c_bncp_vjp")
        return gb, gmu


class _NCPSolve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, G, b, mu, max_iters, tol):
        s = BatchNCP(G, b, mu)
        lam = s.solve(max_iters, tol).clone()
        ctx.solver = s
        return lam

    @staticmethod
    def backward(ctx, glam):
        gb, gmu = ctx.solver.vjp(glam)
        return None, gb, gmu, None, None


def ncp_solve(G: torch.Tensor, b: torch.Tensor, mu: torch.Tensor, max_iters: int = 5000, tol: float = 1e-14):
    """lambda (B, n) of the exact-cone NCP (de Saxce) for every problem, differentiable in b and mu."""
    return _NCPSolve.apply(G, b, mu, max_iters, tol)


def delassus(J: torch.Tensor, Minv: torch.Tensor, v_free: torch.Tensor, bias: torch.Tensor = None):
    """G = J Minv J^T, b = J v_free + bias for batched dense J (B, n, nv), Minv (B, nv, nv),
    v_free (B, nv) in torch (differentiable)."""
    G = J @ Minv @ J.transpose(1, 2)
    b = (J @ v_free.unsqueeze(-1)).squeeze(-1)
    if bias is not None:
        b = b + bias
    return G, b
