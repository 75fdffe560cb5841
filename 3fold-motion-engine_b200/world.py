"""The exact-cone box world on the device: the reference's BoxWorld (src/motion_engine/ncp/
ncp_gpu.py:1237-1413) with every substep on the B200, in float64.

A substep is the reference's: SAT box/plane and box/box contacts (b2c_world_contacts: the box
engine's broadphase proposes candidate pairs, the float64 narrowphase finds the contacts),
build_scene (b2c_world_scene: frame, 3x6 blocks, Baumgarte bias, Minv, v_free), the exact-cone
NCP solve (b2c_ncp_setup / _color / _sweeps of NCPSolverB200's arrays), and the integration
(b2c_world_integrate).  The one host read per substep is the contact count, which sizes the NCP
launches.

Beyond the reference: many independent scenes in one world (the `scene` of add; bodies of
different scenes never touch), per-body friction (pair: sqrt(mu_a mu_b), ground: mu_a) and
kinematic bodies that move with a prescribed velocity (a pushing plate).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .engine import _ptr
from .ncp import NCPSolverB200

G = 9.81


class BoxWorldB200:
    """Boxes on a static ground plane at z = 0, stepped on the device (float64 state)."""

    def __init__(self, dt=1.0 / 240.0, mu=0.5, gravity=True, iters=200, margin=2e-3, desaxce=True, substeps=1,
                 warm_start=False, device="cuda", max_contacts=None, cand_per_body=16, solve_blocks=0):
        if not torch.cuda.is_available():
            raise RuntimeError("BoxWorldB200: no CUDA device; the box world runs only on the GPU")
        self.L = _lib.load()
        self.dev = torch.device(device)
        self.dt, self.mu, self.gravity = float(dt), float(mu), bool(gravity)
        self.iters, self.margin, self.desaxce = int(iters), float(margin), bool(desaxce)
        self.substeps, self.warm_start = int(substeps), bool(warm_start)
        self.max_contacts = max_contacts
        self.cand_per_body = int(cand_per_body)
        self.solve_blocks = int(solve_blocks)
        self._half, self._mass, self._x, self._v, self._w, self._q = [], [], [], [], [], []
        self._kin, self._vkin, self._mu, self._scene = [], [], [], []
        self._built = False
        self.n_contacts = 0
        self.n_colors = 0
        self._have_warm = False

    # ---- bodies ----
    def add(self, half, mass, x, v=None, w=None, q=None, kin=False, v_kin=None, mu=None, scene=0) -> int:
        """A box of half extents `half` and `mass` at `x` (BoxWorld.add, :1270-1273).  kin=True makes
        it kinematic: zero inverse mass, moving with v_kin (6: linear then angular)."""
        self._half.append(np.asarray(half, float).reshape(3))
        self._mass.append(float(mass))
        self._x.append(np.asarray(x, float).reshape(3))
        self._v.append(np.zeros(3) if v is None else np.asarray(v, float).reshape(3))
        self._w.append(np.zeros(3) if w is None else np.asarray(w, float).reshape(3))
        self._q.append(np.array([0.0, 0.0, 0.0, 1.0]) if q is None else np.asarray(q, float).reshape(4))
        self._kin.append(1 if kin else 0)
        self._vkin.append(np.zeros(6) if v_kin is None else np.asarray(v_kin, float).reshape(6))
        self._mu.append(self.mu if mu is None else float(mu))
        self._scene.append(int(scene))
        self._built = False
        return len(self._half) - 1

    @property
    def n(self) -> int:
        return len(self._half)

    def _build(self):
        N, dev = self.n, self.dev
        d = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float64)).to(dev)
        i32 = lambda n: torch.zeros(max(int(n), 1), dtype=torch.int32, device=dev)
        half = np.array(self._half).reshape(N, 3)
        mass = np.array(self._mass)
        e = 2.0 * half
        Ib = (mass / 12.0)[:, None] * np.stack([e[:, 1] ** 2 + e[:, 2] ** 2, e[:, 0] ** 2 + e[:, 2] ** 2,
                                                e[:, 0] ** 2 + e[:, 1] ** 2], axis=1)
        self.x, self.q = d(np.array(self._x)), d(np.array(self._q))
        self.v, self.w = d(np.array(self._v)), d(np.array(self._w))
        self.half, self.mass, self.Ib = d(half), d(mass), d(Ib)
        self.kin = torch.from_numpy(np.array(self._kin, np.int32)).to(dev)
        self.vkin = d(np.array(self._vkin))
        self.body_mu = d(np.array(self._mu))
        # broadphase of the box engine over a float32 mirror of the centres
        sc = np.array(self._scene, np.int32)
        self.scene_t = torch.from_numpy(sc).to(dev) if N and sc.max() > 0 else None
        hmax = float(np.max(np.linalg.norm(half, axis=1))) if N else 0.5
        cell = 1.01 * (2.0 * hmax + self.margin)
        dims = (16, 16, 8) if N <= 2000 else (32, 32, 16) if N <= 20000 else (64, 64, 32)
        nbk = dims[0] * dims[1] * dims[2]
        cap = max(self.cand_per_body * N + N, 64)
        self.cand_cap = cap
        MC = int(self.max_contacts) if self.max_contacts else 8 * cap
        self.MC = MC
        self.half32 = torch.zeros((max(N, 1), 4), dtype=torch.float32, device=dev)
        self.half32[:N, :3] = torch.from_numpy(half.astype(np.float32)).to(dev)
        self.bx_bufs = dict(bucket=i32(N), start=i32(nbk + 1), cursor=i32(nbk + 1), sorted=i32(N), cand_count=i32(N + 1),
                            cand_offset=i32(N + 1), cand_a=i32(cap), cand_b=i32(cap), cont_count=i32(cap + 1),
                            cont_offset=i32(cap + 1), pair_flag=i32(cap + 1), pair_offset=i32(cap + 1),
                            scan_tmp=i32(self.L.b2c_scan_scratch_ints(max(nbk, N, cap) + 1)))
        b = self.bx_bufs
        self.c_boxes = _lib.Boxes(N, _ptr(self.half32), None, self.margin, cell, dims[0], dims[1], dims[2], cap,
                                  *(_ptr(b[k]) for k in ("bucket", "start", "cursor", "sorted", "cand_count",
                                                         "cand_offset", "cand_a", "cand_b", "cont_count", "cont_offset",
                                                         "pair_flag", "pair_offset")),
                                  None, None, None, _ptr(b["scan_tmp"]),
                                  _ptr(self.scene_t) if self.scene_t is not None else None)
        self.header = torch.zeros(8, dtype=torch.int32, device=dev)
        # the NCP (its scene arrays are the world's scene)
        self.solver = NCPSolverB200(N, MC, dtype="float64", device=dev, desaxce=self.desaxce,
                                    solve_blocks=self.solve_blocks)
        s = self.solver
        f64 = lambda *shape: torch.zeros(*shape, dtype=torch.float64, device=dev)
        self.xc32 = torch.zeros((max(N, 1), 4), dtype=torch.float32, device=dev)
        self.x4, self.half4 = f64(max(N, 1), 4), f64(max(N, 1), 4)
        self.slot_p, self.slot_n, self.slot_f = f64(cap * 8, 4), f64(cap, 4), i32(cap * 8)
        self.fid = i32(MC)
        self.key = torch.zeros(MC, dtype=torch.int64, device=dev)
        self.p, self.nrm, self.gap = f64(MC, 3), f64(MC, 3), f64(MC)
        self.attach = i32(MC)
        self.count = i32(1)
        self.warm_keys = torch.zeros(MC, dtype=torch.int64, device=dev)
        self.warm_lam, self.warm_n = f64(MC, 3), i32(1)
        self.c_world = _lib.World(N, MC, _ptr(self.x), _ptr(self.q), _ptr(self.v), _ptr(self.w), _ptr(self.half),
                                  _ptr(self.mass), _ptr(self.Ib), _ptr(self.kin), _ptr(self.vkin), _ptr(self.body_mu),
                                  self.mu, _ptr(self.xc32), _ptr(self.x4), _ptr(self.half4), _ptr(self.slot_p),
                                  _ptr(self.slot_n), _ptr(self.slot_f), _ptr(s.pa), _ptr(s.pb), _ptr(self.fid),
                                  _ptr(self.key), _ptr(self.p), _ptr(self.nrm), _ptr(self.gap), _ptr(self.attach),
                                  _ptr(self.count),
                                  _ptr(self.warm_keys), _ptr(self.warm_lam), _ptr(self.warm_n))
        self._have_warm = False
        self._built = True

    def _stream(self):
        return ctypes.c_void_p(torch.cuda.current_stream(self.dev).cuda_stream)

    # ---- one substep: the pieces, so the adjoint can run them again ----
    def contacts_device(self) -> int:
        """Contacts of the current state into the world's arrays; returns their count."""
        if not self._built:
            self._build()
        L, s = self.L, self._stream()
        _lib.check(L.b2c_world_contacts(ctypes.byref(self.c_world), ctypes.byref(self.c_boxes),
                                        ctypes.c_void_p(_ptr(self.header)), s), "b2c_world_contacts")
        C = int(self.count.item())
        if C > self.MC:
            raise RuntimeError(f"BoxWorldB200: {C} contacts exceed the capacity {self.MC}")
        if int(self.header[6].item()):
            raise RuntimeError("BoxWorldB200: broadphase candidate capacity exceeded")
        return C

    def scene_device(self, C: int, dt: float):
        """build_scene on the device; returns the NCP scene struct for the first C contacts."""
        s, L = self.solver, self.L
        _lib.check(L.b2c_world_scene(ctypes.byref(self.c_world), C, float(dt), 1 if self.gravity else 0,
                                     ctypes.c_void_p(_ptr(s.Ja)), ctypes.c_void_p(_ptr(s.Jb)),
                                     ctypes.c_void_p(_ptr(s.Minv)), ctypes.c_void_p(_ptr(s.vfree)),
                                     ctypes.c_void_p(_ptr(s.bias)), ctypes.c_void_p(_ptr(s.mu)),
                                     ctypes.c_void_p(_ptr(s.feat)), self._stream()), "b2c_world_scene")
        s.C = C
        s.c_scene = _lib.NcpScene(C, self.n, 8, *(_ptr(t) for t in (s.Ja, s.Jb, s.Minv, s.vfree, s.mu, s.bias)),
                                  None, _ptr(s.pa), _ptr(s.pb), _ptr(s.feat))
        return s.c_scene

    def solve_device(self, C: int, iters: int, warm: bool, trace=None):
        """The NCP solve of the scene just built: setup (from the warm store when `warm`), the
        colouring, `iters` sweeps.  The impulses stay in solver.lam, velocities in solver.v.
        With `trace` (a float64 device tensor of at least b2c_ncp_trace_words() iters C elements) the sweeps also
        record where every contact update started from (b2c_ncp_sweeps_record), bitwise the
        same solve, for the adjoint."""
        s, L, st = self.solver, self.L, self._stream()
        if warm:
            _lib.check(L.b2c_world_warm(ctypes.byref(self.c_world), C, ctypes.c_void_p(_ptr(s.lam)), st),
                       "b2c_world_warm")
        _lib.check(L.b2c_ncp_setup(ctypes.byref(s.c_scene), ctypes.byref(s.c_state), 1 if warm else 0, st),
                   "b2c_ncp_setup")
        params = s._params(None, True)
        s.stats[3] = 0
        _lib.check(L.b2c_ncp_color(ctypes.byref(s.c_scene), ctypes.byref(s.c_state), ctypes.byref(params), st),
                   "b2c_ncp_color")
        if trace is None:
            _lib.check(L.b2c_ncp_sweeps(ctypes.byref(s.c_scene), ctypes.byref(s.c_state), ctypes.byref(params),
                                        int(iters), st), "b2c_ncp_sweeps")
        else:
            _lib.check(L.b2c_ncp_sweeps_record(ctypes.byref(s.c_scene), ctypes.byref(s.c_state), ctypes.byref(params),
                                               int(iters), ctypes.c_void_p(_ptr(trace)), trace.numel(), st),
                       "b2c_ncp_sweeps_record")

    def _substep(self, dt):
        C = self.contacts_device()
        self.scene_device(C, dt)
        s, L, st = self.solver, self.L, self._stream()
        if C:
            warm = self.warm_start and self._have_warm
            self.solve_device(C, self.iters, warm)
            stats = s._check_stats()
            self.n_colors = int(stats[0])
            if self.warm_start:
                _lib.check(L.b2c_world_store(ctypes.byref(self.c_world), C, ctypes.c_void_p(_ptr(s.lam)), st),
                           "b2c_world_store")
                self._have_warm = True
            v6 = s.v
        else:
            self.n_colors = 0
            if self.warm_start:
                self.warm_n.zero_()
            v6 = s.vfree
        _lib.check(L.b2c_world_integrate(ctypes.byref(self.c_world), ctypes.c_void_p(_ptr(v6)), float(dt), st),
                   "b2c_world_integrate")
        self.n_contacts = C

    def step(self):
        """One macro step of `substeps` substeps of dt / substeps (BoxWorld.step, :1333-1339)."""
        if not self._built:
            self._build()
        for _ in range(max(1, self.substeps)):
            self._substep(self.dt / max(1, self.substeps))

    # ---- data out ----
    def get_state(self):
        """(x, q, v, w) float64 numpy copies."""
        if not self._built:
            self._build()
        return tuple(t[:self.n].cpu().numpy().copy() for t in (self.x, self.q, self.v, self.w))

    def set_state(self, x, q, v, w):
        if not self._built:
            self._build()
        for dst, src in ((self.x, x), (self.q, q), (self.v, v), (self.w, w)):
            dst[:self.n].copy_(torch.as_tensor(np.asarray(src, np.float64), device=self.dev).reshape(dst[:self.n].shape))

    def contact_arrays(self) -> dict:
        """The last substep's contacts: pa, pb, point, normal (from pb to pa), gap, feature, key."""
        C = self.n_contacts
        return dict(pa=self.solver.pa[:C].cpu().numpy(), pb=self.solver.pb[:C].cpu().numpy(),
                    p=self.p[:C].cpu().numpy(), n=self.nrm[:C].cpu().numpy(), gap=self.gap[:C].cpu().numpy(),
                    fid=self.fid[:C].cpu().numpy(), key=self.key[:C].cpu().numpy())

    def penetration(self) -> float:
        """Deepest penetration of the current configuration (BoxWorld.penetration, :1407-1410)."""
        C = self.contacts_device()
        return max(0.0, float((-self.gap[:C]).max().item())) if C else 0.0
