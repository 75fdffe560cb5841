"""CPU oracle of the batched proximal ADMM and its adjoint -- TEST INFRASTRUCTURE ONLY.

Only the tests and the bench's CPU-baseline leg may import this module.  It restates, in numpy
float64 vectorised over the batch, the reference's ``BatchProxADMMGPU``
(src/motion_engine/ncp/ncp_batch_gpu.py:918-1313, abbreviated NB below) so that the device
solver (csrc/badmm.cu, one warp per problem) can be checked against it:

* set-up (NB:974-1000): b = J v_free, the int64 scale bound kappa, M^-1 J^T (k_mj NB:149-157),
  the dense Delassus G (k_gdense NB:160-167), its spectrum by cyclic Jacobi (k_jacobi
  NB:170-202), the diagonal blocks and their largest eigenvalue (k_gd3 NB:291-300, f_eigmax
  NB:130-146), eta and the per-contact step (k_eta NB:303-313), the bilateral regime test
  (k_bilat NB:205-258) and rho (k_rho NB:261-288), the block-Jacobi preconditioner (k_pjac
  NB:316-322);
* the matrix-free product G x + (eta + rho) x with the int64 accumulation of M^-1 J^T x at a
  power-of-two scale per problem (k_scale / k_jt / k_mscat / k_acc2w / k_gath NB:326-388);
* ADMM with a preconditioned CG x-step, the cone projection z-step and the dual update, the
  Cadoux refresh of the slip speed, the natural residual and the per-problem convergence mask
  (NB:466-543, 1048-1099);
* the active set (k_active NB:556-598, k_slipidx, k_sjac) and grad_affine: the affine de Saxce
  sigma map solved by 1 + n_slip + 1 applications (NB:629-769, 1145-1186), for the tau direction
  db = dt J M^-1 e_j and the mu direction at each problem's first slip contact (NB:771-808,
  1190-1206).

Where the restatement differs from NB, by design and without effect beyond rounding: the scale
exponent is taken from the float's exponent (floor(log2 v) = ilogb v) instead of log2, and the
3x3 inverses are the adjugate over the determinant.  Rounding to int64 is half away from zero
(Warp's round).
"""
from __future__ import annotations

import numpy as np

TINY = 1e-300
SCALE_BOUND = 4.503599627370496e15


def proj(z, mu):
    """f_proj (NB:113-126): projection onto the cone of friction mu; z (..., 3), mu (...)."""
    zn = z[..., 0]
    zt = np.sqrt(z[..., 1] * z[..., 1] + z[..., 2] * z[..., 2])
    inside = zt <= mu * zn
    polar = ~inside & (mu * zt <= -zn)
    with np.errstate(divide="ignore", invalid="ignore"):
        s = (zn + mu * zt) / (1.0 + mu * mu)
        f = mu * s / zt
    out = np.stack([s, f * z[..., 1], f * z[..., 2]], axis=-1)
    out = np.where(inside[..., None], z, out)
    return np.where(polar[..., None], 0.0, out)


def eigmax3(A):
    """f_eigmax (NB:130-146): largest eigenvalue of symmetric 3x3 blocks, closed form."""
    p1 = A[..., 0, 1] ** 2 + A[..., 0, 2] ** 2 + A[..., 1, 2] ** 2
    q = (A[..., 0, 0] + A[..., 1, 1] + A[..., 2, 2]) / 3.0
    out = np.maximum(A[..., 0, 0], np.maximum(A[..., 1, 1], A[..., 2, 2]))
    p2 = (A[..., 0, 0] - q) ** 2 + (A[..., 1, 1] - q) ** 2 + (A[..., 2, 2] - q) ** 2 + 2.0 * p1
    p = np.sqrt(p2 / 6.0)
    ok = (p1 > 0) & (p > 1e-300)
    with np.errstate(divide="ignore", invalid="ignore"):
        Bm = (A - q[..., None, None] * np.eye(3)) / p[..., None, None]
        r = np.clip(np.linalg.det(Bm) / 2.0, -1.0, 1.0)
        val = q + 2.0 * p * np.cos(np.arccos(r) / 3.0)
    return np.where(ok, val, out)


def inv3(A):
    """3x3 inverses by the adjugate over the determinant (zero where singular)."""
    a = A
    c00 = a[..., 1, 1] * a[..., 2, 2] - a[..., 1, 2] * a[..., 2, 1]
    c01 = a[..., 0, 2] * a[..., 2, 1] - a[..., 0, 1] * a[..., 2, 2]
    c02 = a[..., 0, 1] * a[..., 1, 2] - a[..., 0, 2] * a[..., 1, 1]
    c10 = a[..., 1, 2] * a[..., 2, 0] - a[..., 1, 0] * a[..., 2, 2]
    c11 = a[..., 0, 0] * a[..., 2, 2] - a[..., 0, 2] * a[..., 2, 0]
    c12 = a[..., 0, 2] * a[..., 1, 0] - a[..., 0, 0] * a[..., 1, 2]
    c20 = a[..., 1, 0] * a[..., 2, 1] - a[..., 1, 1] * a[..., 2, 0]
    c21 = a[..., 0, 1] * a[..., 2, 0] - a[..., 0, 0] * a[..., 2, 1]
    c22 = a[..., 0, 0] * a[..., 1, 1] - a[..., 0, 1] * a[..., 1, 0]
    det = a[..., 0, 0] * c00 + a[..., 0, 1] * c10 + a[..., 0, 2] * c20
    adj = np.stack([np.stack([c00, c01, c02], -1), np.stack([c10, c11, c12], -1),
                    np.stack([c20, c21, c22], -1)], -2)
    with np.errstate(divide="ignore", invalid="ignore"):
        out = adj / det[..., None, None]
    return np.where((det != 0)[..., None, None], out, 0.0)


def jacobi_eigs(G, sweeps):
    """k_jacobi (NB:170-202): cyclic Jacobi rotations in the fixed pair order; the diagonal."""
    A = G.copy()
    B, M, _ = A.shape
    for _ in range(sweeps):
        for p in range(M - 1):
            for q in range(p + 1, M):
                apq = A[:, p, q]
                act = np.abs(apq) > TINY
                if not act.any():
                    continue
                app, aqq = A[:, p, p], A[:, q, q]
                with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
                    th = (aqq - app) / (2.0 * apq)
                    t = 1.0 / (np.abs(th) + np.sqrt(th * th + 1.0))
                t = np.where(th < 0, -t, t)
                c = 1.0 / np.sqrt(t * t + 1.0)
                sn = t * c
                c = np.where(act, c, 1.0)
                sn = np.where(act, sn, 0.0)
                akp, akq = A[:, :, p].copy(), A[:, :, q].copy()
                A[:, :, p] = c[:, None] * akp - sn[:, None] * akq
                A[:, :, q] = sn[:, None] * akp + c[:, None] * akq
                apk, aqk = A[:, p, :].copy(), A[:, q, :].copy()
                A[:, p, :] = c[:, None] * apk - sn[:, None] * aqk
                A[:, q, :] = sn[:, None] * apk + c[:, None] * aqk
    return np.einsum("bii->bi", A)


def bilateral_binds(G, b, mu, C):
    """k_bilat (NB:205-258): 1 when the bilateral solution -G^-1 b leaves the cone.  Cholesky
    with the pivots floored at 1e-300, as NB's, so a singular G still gives an answer."""
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        return _bilateral_binds(G, b, mu, C)


def _bilateral_binds(G, b, mu, C):
    B, M, _ = G.shape
    L = np.zeros_like(G)
    for k in range(M):
        d = G[:, k, k] - (L[:, k, :k] ** 2).sum(axis=1)
        d = np.sqrt(np.maximum(d, TINY))
        L[:, k, k] = d
        for i in range(k + 1, M):
            L[:, i, k] = (G[:, i, k] - (L[:, i, :k] * L[:, k, :k]).sum(axis=1)) / d
    y = np.zeros((B, M))
    rhs = -b
    for i in range(M):
        y[:, i] = (rhs[:, i] - (L[:, i, :i] * y[:, :i]).sum(axis=1)) / L[:, i, i]
    x = np.zeros((B, M))
    for i in reversed(range(M)):
        x[:, i] = (y[:, i] - (L[:, i + 1:, i] * x[:, i + 1:]).sum(axis=1)) / L[:, i, i]
    lam = x.reshape(-1, C, 3)
    lt = np.sqrt(lam[..., 1] ** 2 + lam[..., 2] ** 2)
    return ((lam[..., 0] <= 0) | (lt > mu * lam[..., 0])).any(axis=1).astype(np.int32)


def round_away(x):
    return np.where(x >= 0, np.floor(x + 0.5), -np.floor(-x + 0.5))


class BatchADMMOracle:
    """NB's BatchProxADMMGPU restated: upload / set_rho / forward / gradient, per problem."""

    def __init__(self, J, Minv, v_free, mu, dt, alpha_eta=0.0, jacobi_sweeps=10, b=None):
        J = np.ascontiguousarray(J, np.float64)
        self.B, self.M, self.NV = J.shape
        self.C = self.M // 3
        B, C, NV, M = self.B, self.C, self.NV, self.M
        self.J = J
        self.Mi = np.ascontiguousarray(Minv, np.float64).reshape(B, NV, NV)
        self.vfree = np.ascontiguousarray(v_free, np.float64).reshape(B, NV)
        self.mu = np.broadcast_to(np.asarray(mu, np.float64).reshape(-1), (B * C,)).reshape(B, C).copy()
        self.dt = float(dt)
        self.bb = (np.einsum("bik,bk->bi", J, self.vfree) if b is None
                   else np.asarray(b, np.float64).reshape(B, M).copy())
        self.kap = (C * np.abs(self.Mi).sum(axis=2).max(axis=1)
                    * np.abs(J.reshape(B, C, 3, NV)).sum(axis=2).max(axis=(1, 2)) + 1e-300)
        self.MJ = np.einsum("bkl,bil->bik", self.Mi, J)
        self.G = np.einsum("bik,bjk->bij", J, self.MJ)
        self.ev = jacobi_eigs(self.G, jacobi_sweeps)
        idx = np.arange(C)
        blk = self.G.reshape(B, C, 3, C, 3)[:, idx, :, idx, :].transpose(1, 0, 2, 3)
        self.Gd = np.ascontiguousarray(blk)  # (B, C, 3, 3)
        gnorm = eigmax3(self.Gd)
        self.eta = alpha_eta * gnorm
        s = gnorm + self.eta
        with np.errstate(divide="ignore"):
            self.rhoc = np.where(s > 0, 1.0 / s, 1.0)
        self.rho = np.zeros(B)

    # ---- rho (k_rho NB:261-288) ----
    def set_rho(self, mode="regime", relt=1e-12):
        mx = self.ev.max(axis=1)
        thr = relt * mx
        cand = np.where(self.ev > thr[:, None], self.ev, np.inf)
        mn = np.minimum(cand.min(axis=1), mx)
        if mode == "sqrt":
            r = np.sqrt(mn * mx)
        elif mode == "lmin":
            r = mn
        elif mode == "lmax":
            r = mx
        else:
            r = np.where(bilateral_binds(self.G, self.bb, self.mu, self.C) > 0, mx, mn)
        self.rho = r
        return self

    # ---- matrix-free product (NB:326-388, 1030-1038) ----
    def matvec(self, x, use_rho):
        """x (B, C, 3) -> G x + (eta + rho) x, with w = M^-1 J^T x accumulated in int64."""
        B, C, NV = self.B, self.C, self.NV
        m = np.abs(x).reshape(B, -1).max(axis=1)
        t = self.kap * m
        v = np.where(t > 0, SCALE_BOUND / np.where(t > 0, t, 1.0), 1.0)
        e = np.clip(np.frexp(v)[1] - 1, -1000, 1000)  # floor(log2 v), exactly
        scal = np.where(t > 0, np.ldexp(1.0, e), 1.0)
        yt = np.einsum("bcrk,bcr->bck", self.J.reshape(B, C, 3, NV), x)
        s = np.einsum("bkl,bcl->bck", self.Mi, yt)
        acc = round_away(s * scal[:, None, None]).astype(np.int64).sum(axis=1)
        self.wv = acc.astype(np.float64) / scal[:, None]
        u = np.einsum("bik,bk->bi", self.J, self.wv).reshape(B, C, 3)
        r = self.rho[:, None] if use_rho else 0.0
        return u + ((self.eta + r)[..., None]) * x

    @staticmethod
    def _dot(a, b):
        return (a * b).sum(axis=(1, 2))

    def _pcg(self, rhs, x, n_it, op, P, warm_zero, mask=None):
        if warm_zero:
            x[:] = 0.0
            r = rhs.copy()
        else:
            r = rhs - op(x)
        zz = np.einsum("bcij,bcj->bci", P, r)
        p = zz.copy()
        s0 = self._dot(r, zz)
        for _ in range(int(n_it)):
            Ap = op(p)
            s1 = self._dot(p, Ap)
            with np.errstate(divide="ignore", invalid="ignore"):
                s2 = np.where(s1 != 0, s0 / np.where(s1 != 0, s1, 1.0), 0.0)
            upd = s2[:, None, None] * p
            if mask is None:
                x += upd
            else:
                x += np.where(mask[:, None, None] != 0, upd, 0.0)
            r = r - s2[:, None, None] * Ap
            zz = np.einsum("bcij,bcj->bci", P, r)
            s3 = self._dot(r, zz)
            with np.errstate(divide="ignore", invalid="ignore"):
                s4 = np.where(s0 != 0, s3 / np.where(s0 != 0, s0, 1.0), 0.0)
            p = zz + s4[:, None, None] * p
            s0 = s3
        return x

    # ---- forward (NB:1075-1143, 1190-1195) ----
    def forward(self, n_iter=200, cg_iters=8, refresh_every=4, tol=1e-8, desax=True, chunk=0):
        B, C = self.B, self.C
        bb = self.bb.reshape(B, C, 3)
        I3 = np.eye(3)
        self.Pj = inv3(self.Gd + (self.eta + self.rho[:, None])[..., None, None] * I3)
        self.gam = np.zeros((B, C, 3))
        self.zv = np.zeros((B, C, 3))
        self.x = np.zeros((B, C, 3))
        self.s = np.zeros((B, C))
        self.u = np.zeros((B, C, 3))
        self.mask = np.ones(B, np.int32)
        self.resenv = np.full(B, np.nan)
        rho = self.rho[:, None, None]
        for i in range(int(n_iter)):
            g = bb.copy()
            g[..., 0] += self.mu * self.s
            rhs = -(g + self.gam - rho * self.zv)
            self._pcg(rhs, self.x, cg_iters, lambda v: self.matvec(v, True), self.Pj, False, self.mask)
            act = self.mask[:, None, None] != 0
            znew = proj(self.x + self.gam / rho, self.mu)
            self.zv = np.where(act, znew, self.zv)
            self.gam = np.where(act, self.gam + rho * (self.x - self.zv), self.gam)
            k = (i % chunk) if chunk else i
            if refresh_every and (k + 1) % refresh_every == 0:
                self._refresh(tol, desax)
        self.lam = self.zv.copy()
        self.matvec(self.lam, False)
        self.vplus = self.vfree + self.wv
        return self

    def _refresh(self, tol, desax):
        self.u = self.matvec(self.zv, False) + self.bb.reshape(self.B, self.C, 3)
        ut = np.sqrt(self.u[..., 1] ** 2 + self.u[..., 2] ** 2)
        self.s = ut
        w = self.u.copy()
        if desax:
            w[..., 0] = w[..., 0] + self.mu * ut
        d = self.zv - proj(self.zv - self.rhoc[..., None] * w, self.mu)
        res = np.abs(d).max(axis=2)
        m = np.where(np.isnan(res).any(axis=1), np.nan, res.max(axis=1))
        self.resenv = m
        self.mask = np.where((self.mask == 1) & (m < tol), 0, self.mask).astype(np.int32)

    # ---- active set and gradient (NB:1145-1206) ----
    def build_active(self, tol_lam=1e-10, tol_rel=1e-6):
        B, C = self.B, self.C
        L, u, mu = self.lam, self.u, self.mu
        lsc = np.maximum(1e-30, np.abs(L).reshape(B, -1).max(axis=1))[:, None]
        ln = L[..., 0]
        lt = np.sqrt(L[..., 1] ** 2 + L[..., 2] ** 2)
        openc = ln <= tol_lam + tol_rel * lsc
        slip = ~openc & (lt >= mu * ln * (1.0 - tol_rel) - tol_lam)
        nw = np.maximum(np.sqrt(u[..., 1] ** 2 + u[..., 2] ** 2), 1e-300)
        h1, h2 = u[..., 1] / nw, u[..., 2] / nw
        Z = np.zeros((B, C, 3, 3))
        Z[...] = np.eye(3)
        Zs = np.zeros((B, C, 3, 3))
        Zs[..., 0, 0] = 1.0
        Zs[..., 1, 0] = -mu * h1
        Zs[..., 2, 0] = -mu * h2
        Zs[..., 1, 1] = -h2
        Zs[..., 2, 1] = h1
        Z = np.where(slip[..., None, None], Zs, Z)
        Z = np.where(openc[..., None, None], 0.0, Z)
        D = np.zeros((B, C, 3))
        D[openc] = 1.0
        Ds = np.stack([np.zeros_like(nw), nw / np.maximum(mu * ln, 1e-300), np.ones_like(nw)], -1)
        D = np.where(slip[..., None], Ds, D)
        self.Z, self.D = Z, D
        self.slipf = slip.astype(np.float64)
        self.what = np.where(slip[..., None], np.stack([np.zeros_like(h1), h1, h2], -1), 0.0)
        self.labels = np.where(openc, 0, np.where(slip, 2, 1)).astype(np.int32)
        self.nslip = slip.sum(axis=1).astype(np.int32)
        self.sidx = np.full((B, C), -1, np.int32)
        for e in range(B):
            k = np.flatnonzero(slip[e])
            self.sidx[e, :len(k)] = k
        A = np.einsum("bcji,bcjk,bckl->bcil", Z, self.Gd + self.eta[..., None, None] * np.eye(3), Z)
        A = A + np.einsum("bci,ij->bcij", D, np.eye(3))
        self.Ps = inv3(A)
        return self

    def _sopv(self, y):
        t = self.matvec(np.einsum("bcij,bcj->bci", self.Z, y), False)
        return np.einsum("bcji,bcj->bci", self.Z, t) + self.D * y

    def _grad_once(self, cg):
        v = -self.ZtHp
        v[..., 0] -= np.where(self.slipf > 0.5, self.mu * self.sig, 0.0)
        y = np.zeros_like(v)
        self._pcg(v, y, cg, self._sopv, self.Ps, True)
        self.dlam = np.einsum("bcij,bcj->bci", self.Z, y) + self.pinh
        Hd = self.matvec(self.dlam, False)
        so = self.what[..., 1] * (Hd[..., 1] + self.dbv[..., 1]) + self.what[..., 2] * (Hd[..., 2] + self.dbv[..., 2])
        self.sigo = np.where(self.slipf > 0.5, so, 0.0)

    def grad_affine(self, n_calls, cg):
        B, C = self.B, self.C
        K = int(n_calls) - 2
        Hp = self.matvec(self.pinh, False) + self.dbv
        self.ZtHp = np.einsum("bcji,bcj->bci", self.Z, Hp)
        self.sig = np.zeros((B, C))
        self._grad_once(cg)
        a = self.sigo.copy()
        Bm = np.zeros((B, C, C))
        rows = np.arange(B)
        for j in range(K):
            self.sig = np.zeros((B, C))
            has = j < self.nslip
            self.sig[rows[has], self.sidx[has, j]] = 1.0
            self._grad_once(cg)
            for e in np.flatnonzero(has):
                n = self.nslip[e]
                c = self.sidx[e, :n]
                Bm[e, :n, j] = self.sigo[e, c] - a[e, c]
        self.sig = np.zeros((B, C))
        for e in range(B):
            n = int(self.nslip[e])
            if n == 0:
                continue
            c = self.sidx[e, :n]
            A = np.eye(n) - Bm[e, :n, :n]
            self.sig[e, c] = np.linalg.solve(A, a[e, c])
        self._grad_once(cg)
        return self.dlam

    def gradient(self, n_calls=None, grad_cg=60, do_mu=True, jdir=0):
        """NB's _grad_part (NB:1197-1206): d/dtau_j (db = dt J M^-1 e_j) and d/dmu at each
        problem's first slip contact."""
        B, C = self.B, self.C
        self.build_active()
        if n_calls is None:
            n_calls = int(self.nslip.max()) + 2
        self.pinh = np.zeros((B, C, 3))
        self.dbv = self.dt * self.MJ[:, :, jdir].reshape(B, C, 3)
        self.grad_affine(n_calls, grad_cg)
        self.matvec(self.dlam, False)
        self.dv_tau = self.dt * self.Mi[:, :, jdir] + self.wv
        self.dlam_tau = self.dlam.copy()
        self.dlam_mu = np.zeros((B, C, 3))
        if do_mu:
            self.pinh = np.zeros((B, C, 3))
            for e in np.flatnonzero(self.nslip > 0):
                c = self.sidx[e, 0]
                self.pinh[e, c] = [0.0, -self.lam[e, c, 0] * self.what[e, c, 1], -self.lam[e, c, 0] * self.what[e, c, 2]]
            self.dbv = np.zeros((B, C, 3))
            self.grad_affine(n_calls, grad_cg)
            self.dlam_mu = self.dlam.copy()
        return self

    def grad_db(self, lam, u, dbv, n_calls=None, cg=60):
        """NB's grad_affine from given impulses and velocities (the reference's own test,
        tests/test_ncp_batch_adjoint.py:55-76): dlam for the b-directions dbv (B, C, 3)."""
        self.lam = np.asarray(lam, np.float64).reshape(self.B, self.C, 3).copy()
        self.u = np.asarray(u, np.float64).reshape(self.B, self.C, 3).copy()
        self.build_active()
        if n_calls is None:
            n_calls = int(self.nslip.max()) + 2
        self.pinh = np.zeros((self.B, self.C, 3))
        self.dbv = np.asarray(dbv, np.float64).reshape(self.B, self.C, 3).copy()
        return self.grad_affine(n_calls, cg).copy()
