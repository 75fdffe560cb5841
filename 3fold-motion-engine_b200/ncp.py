"""Exact-cone NCP solve on the GPU: the host mirror of the reference's NCPSolverGPU
(src/motion_engine/ncp/ncp_gpu.py:784-1063) over libb2c's b2c_ncp_* entry points.

The contract types mirror the reference's (ncp_gpu.py:191-339): a BlockScene holds per-contact
3x6 Jacobian blocks of the two bodies (the minus sign of the relative velocity baked into Jb),
per-body 6x6 inverse masses, the free velocity, friction, the bias added to u and stable
feature ids; a SolveResult the impulses in the contact frame (n, t1, t2), the velocity after
them and the natural-map residual.  SoftStep gives the soft-step constants of the published
box2d / box3d soft constraint (the reference's src/motion_engine/soft_step.py:35-49).
"""
from __future__ import annotations

import ctypes
import math
import time
from dataclasses import dataclass, field
from typing import Optional

import numpy as np
import torch

from . import _lib

SCALE = 1.0e10
FEATBITS = 20
NCOLMAX = 1024
CONTACT_HERTZ = 30.0
CONTACT_DAMPING_RATIO = 10.0
CONTACT_SPEED = 3.0


@dataclass
class BlockScene:
    """u_c = Ja_c v_a + Jb_c v_b + bias_c (ncp_gpu.py:191-197)."""
    Ja: np.ndarray            # (n_c, 3, 6)
    Jb: np.ndarray            # (n_c, 3, 6)
    Minv: np.ndarray          # (n_b, 6, 6)
    v_free: np.ndarray        # (n_b, 6)
    mu: np.ndarray            # (n_c,)
    body_pairs: np.ndarray    # (n_c, 2) int32, -1 = static
    dt: float
    bias: np.ndarray          # (n_c, 3)
    feature: np.ndarray       # (n_c,) int32
    sep: Optional[np.ndarray] = None   # (n_c,) separation, soft step only

    @property
    def n_c(self) -> int:
        return int(np.shape(self.Ja)[0])

    @property
    def n_b(self) -> int:
        return int(np.shape(self.Minv)[0])

    def jacobian(self) -> np.ndarray:
        J = np.zeros((3 * self.n_c, 6 * self.n_b))
        for c in range(self.n_c):
            a, b = int(self.body_pairs[c, 0]), int(self.body_pairs[c, 1])
            if a >= 0:
                J[3 * c:3 * c + 3, 6 * a:6 * a + 6] += self.Ja[c]
            if b >= 0:
                J[3 * c:3 * c + 3, 6 * b:6 * b + 6] += self.Jb[c]
        return J

    def delassus(self) -> np.ndarray:
        """G = J Minv J^T, dense float64 (host, for comparisons)."""
        J = self.jacobian()
        M = np.zeros((6 * self.n_b, 6 * self.n_b))
        for i in range(self.n_b):
            M[6 * i:6 * i + 6, 6 * i:6 * i + 6] = self.Minv[i]
        return J @ M @ J.T

    def rhs(self) -> np.ndarray:
        """b = J v_free + bias, float64."""
        return (self.jacobian() @ np.asarray(self.v_free, np.float64).reshape(-1)
                + np.asarray(self.bias, np.float64).reshape(-1))


@dataclass
class Scene:
    """The dense contract (ncp_gpu.py:263-307): J (3 n_c, 6 n_b), Minv dense or diagonal."""
    J: np.ndarray
    Minv: np.ndarray
    v_free: np.ndarray
    mu: np.ndarray
    body_pairs: np.ndarray
    dt: float
    bias: Optional[np.ndarray] = None
    feature: Optional[np.ndarray] = None
    sep: Optional[np.ndarray] = None

    def blocks(self) -> BlockScene:
        J = np.asarray(self.J, np.float64)
        n_c, n_v = J.shape[0] // 3, J.shape[1]
        if n_v % 6:
            raise ValueError(f"Scene.blocks: n_v={n_v} is not a multiple of 6 (6-DOF rigid bodies)")
        n_b = n_v // 6
        Mi = np.asarray(self.Minv, np.float64)
        if Mi.ndim == 1:
            Mi = np.diag(Mi)
        pairs = np.asarray(self.body_pairs, np.int32).reshape(n_c, 2)
        Ja, Jb = np.zeros((n_c, 3, 6)), np.zeros((n_c, 3, 6))
        for c in range(n_c):
            a, b = int(pairs[c, 0]), int(pairs[c, 1])
            if a >= 0:
                Ja[c] = J[3 * c:3 * c + 3, 6 * a:6 * a + 6]
            if b >= 0:
                Jb[c] = J[3 * c:3 * c + 3, 6 * b:6 * b + 6]
        Minv = np.stack([Mi[6 * i:6 * i + 6, 6 * i:6 * i + 6] for i in range(n_b)]) if n_b else np.zeros((0, 6, 6))
        return BlockScene(Ja=Ja, Jb=Jb, Minv=Minv, v_free=np.asarray(self.v_free, np.float64).reshape(n_b, 6),
                          mu=np.asarray(self.mu, np.float64).reshape(n_c), body_pairs=pairs, dt=float(self.dt),
                          bias=(np.zeros((n_c, 3)) if self.bias is None
                                else np.asarray(self.bias, np.float64).reshape(n_c, 3)),
                          feature=(np.arange(n_c, dtype=np.int32) if self.feature is None
                                   else np.asarray(self.feature, np.int32)),
                          sep=None if self.sep is None else np.asarray(self.sep, np.float64).reshape(n_c))


@dataclass
class SolveResult:
    lam: np.ndarray           # (n_c, 3) impulses in the contact frame (n, t1, t2)
    v: np.ndarray             # (n_b, 6) velocity after the contact impulses
    residual: float           # max_c |lambda_c - proj_K(lambda_c - rho_c (u_c + Gamma(u_c)))|
    iters: int
    n_colors: int
    cache_hit: bool
    ms: dict = field(default_factory=dict)
    history: Optional[dict] = None
    v_bias: Optional[np.ndarray] = None   # velocity after the biased pass (soft step with relax)
    contact_model: str = "NCP_RIGID"
    bias_applied: bool = True


def make_soft(hertz: float, zeta: float, h: float):
    """Soft constraint of a discrete implicit spring (box2d / box3d MakeSoft):
    (bias_rate, mass_scale, impulse_scale), mass_scale + impulse_scale = 1."""
    if hertz <= 0.0:
        return 0.0, 0.0, 0.0
    omega = 2.0 * math.pi * hertz
    a1 = 2.0 * zeta + h * omega
    a2 = h * omega * a1
    a3 = 1.0 / (1.0 + a2)
    return omega / a1, a2 * a3, a3


def contact_hertz(inv_h: float, world_hertz: float = CONTACT_HERTZ) -> float:
    """Stiffness capped at a quarter of the substep Nyquist frequency."""
    return min(world_hertz, 0.125 * inv_h)


@dataclass
class SoftStep:
    """Soft-step configuration (ncp_gpu.py:167-188)."""
    hertz: float = CONTACT_HERTZ
    zeta: float = CONTACT_DAMPING_RATIO
    contact_speed: float = CONTACT_SPEED
    relax_frac: float = 0.25

    def params(self, h: float) -> np.ndarray:
        """(bias_rate, mass_scale, impulse_scale, inv_h, contact_speed) for a substep h."""
        inv_h = 1.0 / h
        br, ms, isc = make_soft(contact_hertz(inv_h, self.hertz), self.zeta, h)
        return np.array([br, ms, isc, inv_h, self.contact_speed], dtype=np.float64)

    def split(self, iters: int):
        """(biased iterations, relax iterations) of a per-substep budget."""
        iters = max(1, int(iters))
        relax = min(iters - 1, max(1, int(round(self.relax_frac * iters)))) if iters > 1 else 0
        return iters - relax, relax


def _ptr(t: torch.Tensor) -> int:
    return t.data_ptr()


class NCPSolverB200:
    """Persistent exact-cone NCP solver (the reference's NCPSolverGPU interface).  Capacity is
    fixed at construction; the colour cache lives across solve() calls.  All sweeps of a solve
    run in one persistent kernel launch, so there is no per-colour launch to capture."""

    def __init__(self, n_bodies: int, max_contacts: int, dtype: str = "float32", device: Optional[str] = None,
                 desaxce: bool = True, graph_capture: bool = True, color_cache: bool = True, solve_blocks: int = 0):
        if dtype not in ("float32", "float64"):
            raise ValueError(f"dtype must be 'float32' or 'float64', got {dtype!r}")
        if not torch.cuda.is_available():
            raise RuntimeError("NCPSolverB200: no CUDA device; the b2c NCP solver runs only on the GPU")
        self.L = _lib.load()
        self.dev = torch.device(device or "cuda")
        self.dtype = dtype
        self.tdt = torch.float32 if dtype == "float32" else torch.float64
        self.np_t = np.float32 if dtype == "float32" else np.float64
        self.NB, self.MC = int(n_bodies), int(max_contacts)
        self.desaxce = 1 if desaxce else 0
        self.use_cache = bool(color_cache)
        self.solve_blocks = int(solve_blocks)
        MC, NB, dev, t = max(self.MC, 1), max(self.NB, 1), self.dev, self.tdt
        z = lambda *shape, dtype=t: torch.zeros(*shape, dtype=dtype, device=dev)
        i32 = torch.int32
        self.Ja, self.Jb = z(MC, 3, 6), z(MC, 3, 6)
        self.Minv, self.vfree = z(NB, 6, 6), z(NB, 6)
        self.mu, self.bias, self.sep = z(MC), z(MC, 3), z(MC)
        self.pa, self.pb, self.feat = z(MC, dtype=i32), z(MC, dtype=i32), z(MC, dtype=i32)
        self.rho, self.lam, self.v = z(MC), z(MC, 3), z(NB, 6)
        self.acc = z(NB * 6, dtype=torch.int64)
        self.res, self.u = z(MC), z(MC, 3)
        self.col, self.order = z(MC, dtype=i32), z(MC, dtype=i32)
        self.cstart, self.ccount = z(NCOLMAX, dtype=i32), z(NCOLMAX, dtype=i32)
        self.claim = z(NB, dtype=torch.int64)
        self.dyn = z(NB, dtype=i32)
        self.c_pa, self.c_pb, self.c_feat = z(MC, dtype=i32), z(MC, dtype=i32), z(MC, dtype=i32)
        self.c_minv = z(NB, 4)
        self.stats = z(8, dtype=i32)
        self.res_max = z(1, dtype=torch.int64)
        self.barrier = z(int(self.L.b2c_barrier_words()), dtype=i32)
        self.c_state = _lib.NcpState(MC, NB, NCOLMAX, *(_ptr(x) for x in (
            self.rho, self.lam, self.v, self.acc, self.res, self.u, self.col, self.order, self.cstart, self.ccount,
            self.claim, self.dyn, self.c_pa, self.c_pb, self.c_feat, self.c_minv, self.stats, self.res_max,
            self.barrier)))
        self.C = 0
        self.n_colors = 0
        self.cache_hits = 0
        self.cache_misses = 0
        self.prof = {}

    # ---- helpers ----
    def _t(self, name, fn):
        torch.cuda.synchronize(self.dev)
        t0 = time.perf_counter()
        out = fn()
        torch.cuda.synchronize(self.dev)
        self.prof[name] = (time.perf_counter() - t0) * 1e3
        return out

    def upload(self, bs: BlockScene):
        C, NB = bs.n_c, bs.n_b
        if C > self.MC:
            raise ValueError(f"NCPSolverB200: {C} contacts exceeds capacity {self.MC}")
        if NB != self.NB:
            raise ValueError(f"NCPSolverB200: scene has {NB} bodies, solver built for {self.NB}")
        pairs = np.ascontiguousarray(bs.body_pairs, np.int32).reshape(C, 2)
        feat = np.ascontiguousarray(bs.feature, np.int32).reshape(C)
        if C and (feat.min() < 0 or feat.max() >= (1 << FEATBITS)):
            raise ValueError(f"NCPSolverB200: feature ids must lie in [0, 2^{FEATBITS})")
        if C and (pairs.min() < -1 or pairs.max() >= NB):
            raise ValueError("NCPSolverB200: body index out of range")
        key = ((pairs[:, 0].astype(np.int64) + 1) * (NB + 1) + pairs[:, 1] + 1) * (1 << FEATBITS) + feat
        if len(np.unique(key)) != C:
            raise ValueError("NCPSolverB200: (body_a, body_b, feature) keys must be unique")
        nt, dev = self.np_t, self.dev
        put = lambda dst, src: dst[:len(src)].copy_(torch.from_numpy(np.ascontiguousarray(src)).to(dev))
        if C:
            put(self.Ja, np.asarray(bs.Ja, nt).reshape(C, 3, 6))
            put(self.Jb, np.asarray(bs.Jb, nt).reshape(C, 3, 6))
            put(self.mu, np.asarray(bs.mu, nt).reshape(C))
            put(self.bias, np.asarray(bs.bias, nt).reshape(C, 3))
            put(self.sep, (np.zeros(C) if bs.sep is None else np.asarray(bs.sep, np.float64)).astype(nt))
            put(self.pa, pairs[:, 0].copy())
            put(self.pb, pairs[:, 1].copy())
            put(self.feat, feat)
        if NB:
            put(self.Minv, np.asarray(bs.Minv, nt).reshape(NB, 6, 6))
            put(self.vfree, np.asarray(bs.v_free, nt).reshape(NB, 6))
        self.C = C
        self.c_scene = _lib.NcpScene(C, NB, 4 if nt == np.float32 else 8, *(_ptr(x) for x in (
            self.Ja, self.Jb, self.Minv, self.vfree, self.mu, self.bias, self.sep, self.pa, self.pb, self.feat)))

    def _params(self, soft, use_bias):
        p = _lib.NcpParams()
        p.desaxce = self.desaxce
        p.soft = 1 if soft is not None else 0
        p.use_bias = 1 if use_bias else 0
        p.color_cache = 1 if self.use_cache else 0
        p.solve_blocks = self.solve_blocks
        if soft is not None:
            for k in range(5):
                p.softp[k] = float(soft[k])
        p.barrier_timeout_ns = 1_000_000_000
        return p

    def _stream(self):
        return ctypes.c_void_p(torch.cuda.current_stream(self.dev).cuda_stream)

    def _sweeps(self, params, n):
        _lib.check(self.L.b2c_ncp_sweeps(ctypes.byref(self.c_scene), ctypes.byref(self.c_state),
                                         ctypes.byref(params), int(n), self._stream()), "b2c_ncp_sweeps")

    def _residual(self, params) -> float:
        _lib.check(self.L.b2c_ncp_residual(ctypes.byref(self.c_scene), ctypes.byref(self.c_state),
                                           ctypes.byref(params), self._stream()), "b2c_ncp_residual")
        bits = int(self.res_max.item())
        return float(np.array([bits], np.int64).view(np.float64)[0])

    def _check_stats(self):
        st = self.stats.cpu().numpy()
        if st[7]:
            bits = int(st[7])
            self.stats[7] = 0
            raise RuntimeError("NCPSolverB200: " + ("colour count exceeds capacity" if bits & 1 else
                                                    "colouring did not terminate" if bits & 2 else
                                                    "a sweep barrier timed out"))
        return st

    # ---- solve ----
    def solve(self, bs: BlockScene, iters: int = 200, warm: Optional[np.ndarray] = None,
              measure_residual: bool = True, history_every: int = 0, soft: Optional[np.ndarray] = None,
              relax_iters: int = 0) -> SolveResult:
        self._t("upload", lambda: self.upload(bs))
        C = self.C
        if C == 0:
            return SolveResult(np.zeros((0, 3)), np.asarray(bs.v_free, np.float64).copy(), 0.0, 0, 0, False,
                               dict(self.prof), v_bias=np.asarray(bs.v_free, np.float64).copy())
        params = self._params(soft, True)
        s = self._stream()

        def setup():
            if warm is not None:
                self.lam[:C].copy_(torch.from_numpy(np.asarray(warm, self.np_t).reshape(C, 3)).to(self.dev))
            _lib.check(self.L.b2c_ncp_setup(ctypes.byref(self.c_scene), ctypes.byref(self.c_state),
                                            1 if warm is not None else 0, s), "b2c_ncp_setup")
        self._t("setup", setup)

        def color():
            self.stats[3] = 0
            _lib.check(self.L.b2c_ncp_color(ctypes.byref(self.c_scene), ctypes.byref(self.c_state),
                                            ctypes.byref(params), s), "b2c_ncp_color")
            return self._check_stats()
        st = self._t("color", color)
        self.n_colors, hit = int(st[0]), bool(st[3])
        self.cache_hits, self.cache_misses = int(st[4]), int(st[5])
        hist = None

        def run():
            nonlocal hist
            if history_every > 0:
                hist = {"iter": [0], "res": [self._residual(params)],
                        "lam": [self.lam[:C].double().cpu().numpy().copy()]}
                done = 0
                while done < iters:
                    n = min(history_every, iters - done)
                    self._sweeps(params, n)
                    done += n
                    hist["iter"].append(done)
                    hist["res"].append(self._residual(params))
                    hist["lam"].append(self.lam[:C].double().cpu().numpy().copy())
            else:
                self._sweeps(params, iters)
            vb = None
            if relax_iters > 0:
                vb = self.v.double().cpu().numpy().copy()
                self._sweeps(self._params(soft, False), relax_iters)
            return vb
        v_bias = self._t("iter", run)
        self._check_stats()
        r = 0.0
        if measure_residual:
            r = self._t("resid", lambda: self._residual(self._params(soft, relax_iters <= 0)))
        return SolveResult(lam=self.lam[:C].double().cpu().numpy().copy(), v=self.v.double().cpu().numpy().copy(),
                           residual=r, iters=int(iters) + int(relax_iters), n_colors=self.n_colors, cache_hit=hit,
                           ms=dict(self.prof), history=hist, v_bias=v_bias,
                           contact_model="SOFT_STEP" if soft is not None else ("NCP_RIGID" if self.desaxce else "CCP"),
                           bias_applied=relax_iters <= 0)

    def solve_resident(self, iters: int, soft: Optional[np.ndarray] = None) -> None:
        """Solve the last uploaded scene again on the device, without host transfers: setup
        (lambda from zero), the colouring through the colour cache, and `iters` sweeps.  The
        results stay in self.lam and self.v."""
        if self.C == 0:
            return
        params = self._params(soft, True)
        s = self._stream()
        _lib.check(self.L.b2c_ncp_setup(ctypes.byref(self.c_scene), ctypes.byref(self.c_state), 0, s),
                   "b2c_ncp_setup")
        _lib.check(self.L.b2c_ncp_color(ctypes.byref(self.c_scene), ctypes.byref(self.c_state),
                                        ctypes.byref(params), s), "b2c_ncp_color")
        self._sweeps(params, iters)

    def residual(self, soft: Optional[np.ndarray] = None) -> float:
        """Natural-map residual of the current lambda (one device reduction)."""
        return self._residual(self._params(soft, True))

    def coloring(self):
        """(colour per contact, colour-grouped order, per-colour offset, per-colour count)."""
        C, k = self.C, self.n_colors
        return (self.col[:C].cpu().numpy().copy(), self.order[:C].cpu().numpy().copy(),
                self.cstart[:k].cpu().numpy().copy(), self.ccount[:k].cpu().numpy().copy())

    def raw_bytes(self):
        """Raw device bytes of lambda and v (the bit-identity gate)."""
        return self.lam[:self.C].cpu().numpy().tobytes(), self.v.cpu().numpy().tobytes()

    def contact_velocity(self):
        return self.u[:self.C].double().cpu().numpy().copy()

    # ---- derivatives (float64 scenes) ----
    def _adj_buffers(self):
        C, NB, dev = self.C, self.NB, self.dev
        z = lambda *shape: torch.zeros(*shape, dtype=torch.float64, device=dev)
        return dict(vscr=z(max(NB, 1), 6), vfree=z(max(NB, 1), 6), bias=z(max(C, 1), 3), mu=z(max(C, 1)))

    def vjp_implicit(self, lam_bar: np.ndarray, iters: int) -> dict:
        """The implicit-function derivative at the impulses of the last solve (b2c_ncp_adjoint):
        for lam_bar (n_c, 3), the adjoints of v_free (n_b, 6), bias (n_c, 3) and mu (n_c) --
        lam_bar^T dlam*/d(.) -- as `iters` reverse sweeps at lam*.  The solve should have
        converged; the Jacobian blocks and Minv are held."""
        if self.dtype != "float64":
            raise ValueError("vjp_implicit: float64 solvers only")
        C = self.C
        params = self._params(None, True)
        s = self._stream()
        _lib.check(self.L.b2c_ncp_residual(ctypes.byref(self.c_scene), ctypes.byref(self.c_state),
                                           ctypes.byref(params), s), "b2c_ncp_residual")
        b = self._adj_buffers()
        gl = torch.from_numpy(np.ascontiguousarray(lam_bar, np.float64).reshape(C, 3)).to(self.dev)
        _lib.check(self.L.b2c_ncp_adjoint(ctypes.byref(self.c_scene), ctypes.byref(self.c_state),
                                          ctypes.byref(params), int(iters), ctypes.c_void_p(_ptr(gl)),
                                          ctypes.c_void_p(_ptr(b["vscr"])), ctypes.c_void_p(_ptr(b["vfree"])),
                                          ctypes.c_void_p(_ptr(b["bias"])), ctypes.c_void_p(_ptr(b["mu"])), s),
                   "b2c_ncp_adjoint")
        self._check_stats()
        return dict(vfree=b["vfree"][:self.NB].cpu().numpy(), bias=b["bias"][:C].cpu().numpy(),
                    mu=b["mu"][:C].cpu().numpy())

    def vjp_recorded(self, bs: BlockScene, lam_bar: np.ndarray, iters: int, warm: Optional[np.ndarray] = None) -> dict:
        """The exact derivative of `iters` sweeps from `warm` (or from zero): the solve runs again
        recording every contact update (b2c_ncp_sweeps_record), then in reverse
        (b2c_ncp_adjoint_unrolled).  For lam_bar (n_c, 3) the adjoints of v_free, bias, mu, the
        blocks Ja, Jb (n_c, 3, 6), Minv (n_b, 6, 6) and the warm start (lam0, n_c x 3).  Also
        returns the impulses of the solve (lam)."""
        if self.dtype != "float64":
            raise ValueError("vjp_recorded: float64 solvers only")
        self.upload(bs)
        C, NB, dev = self.C, self.NB, self.dev
        params = self._params(None, True)
        s = self._stream()
        if warm is not None:
            self.lam[:C].copy_(torch.from_numpy(np.asarray(warm, np.float64).reshape(C, 3)).to(dev))
        _lib.check(self.L.b2c_ncp_setup(ctypes.byref(self.c_scene), ctypes.byref(self.c_state),
                                        1 if warm is not None else 0, s), "b2c_ncp_setup")
        self.stats[3] = 0
        _lib.check(self.L.b2c_ncp_color(ctypes.byref(self.c_scene), ctypes.byref(self.c_state),
                                        ctypes.byref(params), s), "b2c_ncp_color")
        trace = torch.empty(int(self.L.b2c_ncp_trace_words()) * int(iters) * max(C, 1), dtype=torch.float64,
                            device=dev)
        _lib.check(self.L.b2c_ncp_sweeps_record(ctypes.byref(self.c_scene), ctypes.byref(self.c_state),
                                                ctypes.byref(params), int(iters), ctypes.c_void_p(_ptr(trace)),
                                                trace.numel(), s), "b2c_ncp_sweeps_record")
        lam = self.lam[:C].cpu().numpy().copy()
        b = self._adj_buffers()
        z = lambda *shape: torch.zeros(*shape, dtype=torch.float64, device=dev)
        Jab, Jbb, Mb = z(max(C, 1), 18), z(max(C, 1), 18), z(max(NB, 1), 36)
        gl = torch.from_numpy(np.ascontiguousarray(lam_bar, np.float64).reshape(C, 3)).to(dev)
        _lib.check(self.L.b2c_ncp_adjoint_unrolled(ctypes.byref(self.c_scene), ctypes.byref(self.c_state),
                                                   ctypes.byref(params), int(iters), ctypes.c_void_p(_ptr(trace)),
                                                   trace.numel(), ctypes.c_void_p(_ptr(gl)),
                                                   ctypes.c_void_p(_ptr(b["vscr"])),
                                                   ctypes.c_void_p(_ptr(b["vfree"])), ctypes.c_void_p(_ptr(b["bias"])),
                                                   ctypes.c_void_p(_ptr(b["mu"])), ctypes.c_void_p(_ptr(Jab)),
                                                   ctypes.c_void_p(_ptr(Jbb)), ctypes.c_void_p(_ptr(Mb)), s),
                   "b2c_ncp_adjoint_unrolled")
        self._check_stats()
        return dict(lam=lam, vfree=b["vfree"][:NB].cpu().numpy(), bias=b["bias"][:C].cpu().numpy(),
                    mu=b["mu"][:C].cpu().numpy(), Ja=Jab[:C].reshape(C, 3, 6).cpu().numpy(),
                    Jb=Jbb[:C].reshape(C, 3, 6).cpu().numpy(), Minv=Mb[:NB].reshape(NB, 6, 6).cpu().numpy(),
                    lam0=gl[:C].cpu().numpy())


def solve_scene_gpu(bs: BlockScene, iters: int = 200, dtype: str = "float32", **kw) -> SolveResult:
    s = NCPSolverB200(bs.n_b, max(bs.n_c, 1), dtype=dtype, **kw)
    return s.solve(bs, iters=iters)
