"""ContactEngine protocol engines backed by the b2c CUDA library.

Mirror of the reference's drop-in boundary (src/motion_engine/contact_engine.py:39-55):
``BodyState`` plus the runtime-checkable ``ContactEngine`` protocol (``name``, ``step``,
``get_state``, ``set_kinematic``, ``contact_forces``), with the reference engines' extra
surface (``add_body``, ``com``, the diagnostics counters).  Device buffers are torch tensors
owned by the engine; every computation runs in libb2c.so kernels on the engine's CUDA stream.
There is no CPU path: constructing an engine without a CUDA device raises.

The host-side body setup (bead offsets, masses, bead inertia, its inverse) is the reference's
own numpy arithmetic (contact_engine_gpu.py:186-239), done once at build time; everything per
step is on the device.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Protocol, runtime_checkable

import numpy as np
import torch

from . import _lib

G = 9.81
R = 0.05
MAXC = 400000  # contact capacity, the reference's _MAXC (contact_engine_gpu.py:25)


@dataclass
class BodyState:
    """Rigid-body state as plain data: xc (N,3) centre of mass, Rm (N,3,3) orientation,
    vc (N,3) linear velocity, om (N,3) angular velocity (contact_engine.py:39-45)."""
    xc: np.ndarray
    Rm: np.ndarray
    vc: np.ndarray
    om: np.ndarray


@runtime_checkable
class ContactEngine(Protocol):
    """The reference's interchangeable contact-solver contract (contact_engine.py:48-55)."""
    name: str

    def step(self, dt: float, substeps: int = 1) -> None: ...

    def get_state(self) -> BodyState: ...

    def set_kinematic(self, i: int, xc) -> None: ...

    def contact_forces(self) -> np.ndarray: ...


def voxbox(w, h, d, res=R * 2):
    """Bead rest offsets of a w x h x d box at pitch 2R, x fastest (contact_engine_gpu.py:186-188)."""
    a = lambda L: np.arange(-L / 2 + res / 2, L / 2, res)
    return np.array([[x, y, z] for z in a(d) for y in a(h) for x in a(w)], float)


def quat_to_R(q: np.ndarray) -> np.ndarray:
    """Quaternion (x, y, z, w) -> rotation matrix, float32 arithmetic as the reference's
    get_state does it on the host (contact_engine_gpu.py:283-287)."""
    x, y, z, w = (np.ascontiguousarray(q[:, k]) for k in range(4))
    one = np.float32(1)
    two = np.float32(2)
    Rm = np.empty((len(q), 3, 3), np.float32)
    Rm[:, 0, 0] = one - two * (y * y + z * z)
    Rm[:, 0, 1] = two * (x * y - z * w)
    Rm[:, 0, 2] = two * (x * z + y * w)
    Rm[:, 1, 0] = two * (x * y + z * w)
    Rm[:, 1, 1] = one - two * (x * x + z * z)
    Rm[:, 1, 2] = two * (y * z - x * w)
    Rm[:, 2, 0] = two * (x * z - y * w)
    Rm[:, 2, 1] = two * (y * z + x * w)
    Rm[:, 2, 2] = one - two * (x * x + y * y)
    return Rm


def body_arrays(centers, dens, kin, dims, who="engine") -> dict:
    """Host body setup of the bead engines (contact_engine_gpu.py:209-239): per-bead mass
    mp = density * vol / P, M = mp * P, bead point-mass inertia Ib = sum mp (r.r I - r r^T)
    built once from body 0 and scaled per body, IbInv by np.linalg.inv (identity for kinematic
    bodies), identity quaternions.  Float64 arithmetic, cast to float32 where the reference's
    wp.array casts.  Returns xc (N,3), q (N,4), v, w, invM (N,), IbInv (N,3,3) float32, rest
    (P,3) float32, kin (N,) int32, M (N,) float64."""
    rest64 = voxbox(*dims)
    P = len(rest64)
    N = len(centers)
    w_, h_, d_ = dims
    vol = w_ * h_ * d_
    mp = np.array(dens, float) * vol / P
    M = mp * P
    kinarr = np.array(kin, int)
    invM = np.where(kinarr == 1, 0.0, 1.0 / M)
    Ib = sum(mp[0] * ((r @ r) * np.eye(3) - np.outer(r, r)) for r in rest64)
    IbInv = np.array([np.linalg.inv((mp[i] / mp[0]) * Ib) if kinarr[i] == 0 else np.eye(3) for i in range(N)])
    if not np.all(np.isfinite(IbInv)):
        raise ValueError(f"{who}._build: IbInv contains non-finite (NaN/inf) entries -- "
                         "degenerate body mass/inertia; refusing to build a corrupted rigid-body sim")
    return dict(xc=np.array(np.array(centers, float), np.float32).reshape(N, 3),
                q=np.tile(np.array([0, 0, 0, 1.0], np.float32), (N, 1)),
                v=np.zeros((N, 3), np.float32), w=np.zeros((N, 3), np.float32),
                invM=invM.astype(np.float32), IbInv=IbInv.astype(np.float32).reshape(N, 3, 3),
                rest=rest64.astype(np.float32), kin=kinarr.astype(np.int32), M=M.astype(np.float64))


def _ptr(t: torch.Tensor) -> int:
    return t.data_ptr()


def _pad4(a: np.ndarray) -> np.ndarray:
    out = np.zeros((a.shape[0], 4), np.float32)
    out[:, :a.shape[1]] = a
    return out


class _BeadEngineBase:
    """Shared body store, bead setup and state I/O of the bead-model engines."""
    name = "b2c_base"

    def __init__(self, dims=(0.3, 0.3, 0.2), mu=0.5, device="cuda", graph=True):
        if not torch.cuda.is_available():
            raise RuntimeError(f"{type(self).__name__}: no CUDA device; the b2c engines run only on the GPU")
        self.L = _lib.load()
        self.dev = torch.device(device)
        self.dims = tuple(float(x) for x in dims)
        self.rest_np = voxbox(*self.dims)
        self.P = len(self.rest_np)
        self.mu = float(mu)
        self.graph = bool(graph)
        self._centers, self._dens, self._kin = [], [], []
        self._built = False
        self.n_graph_captures = 0
        self._graphs = {}
        self.kernels_per_step = {}  # graph key -> kernel nodes of the captured step
        self._force_dt = None

    # ---- construction (data in) ----
    def add_body(self, center, density=700.0, kin=False):
        self._centers.append(list(center))
        self._dens.append(float(density))
        self._kin.append(1 if kin else 0)
        self._built = False
        return len(self._centers) - 1

    def _setup_bodies(self):
        """contact_engine_gpu.py:209-239 / contact_engine_gpu_colored.py:836-862."""
        A = body_arrays(self._centers, self._dens, self._kin, self.dims, type(self).__name__)
        N = len(self._centers)
        self.N = N
        self._M = A["M"]
        self._kinarr = A["kin"].astype(int)
        dev = self.dev
        f32 = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(dev)
        # positions, quaternions, velocities and angular velocities as the four contiguous
        # (N, 4) planes of one tensor, so the whole state moves in one copy (set/get_state_packed)
        self.state = torch.zeros((4, N, 4), dtype=torch.float32, device=dev)
        self.xc, self.q, self.v, self.w = self.state[0], self.state[1], self.state[2], self.state[3]
        self.xc.copy_(f32(_pad4(A["xc"])))
        self.q.copy_(f32(A["q"]))
        z4 = lambda: torch.zeros((N, 4), dtype=torch.float32, device=dev)
        self.pv, self.po = z4(), z4()
        self.vgrav = z4()
        self.invM = f32(A["invM"])
        Ib12 = np.zeros((N, 3, 4), np.float32)
        Ib12[:, :, :3] = A["IbInv"]
        self.IbInv = f32(Ib12.reshape(N, 12))
        self.kin = torch.from_numpy(A["kin"]).to(dev)
        self.invIw = torch.zeros((N, 12), dtype=torch.float32, device=dev)
        # beads, body-major (bead gid = body * P + p), as k_worldp indexes them
        NB = N * self.P
        self.NB = NB
        self.rest = f32(_pad4(np.tile(self.rest_np.astype(np.float32), (N, 1))))
        self.owner = torch.from_numpy(np.repeat(np.arange(N, dtype=np.int32), self.P)).to(dev)
        self.bead_start = torch.from_numpy((np.arange(N + 1) * self.P).astype(np.int32)).to(dev)
        self.world = torch.zeros((NB, 4), dtype=torch.float32, device=dev)
        self.header = torch.zeros(8, dtype=torch.int32, device=dev)
        self._hdr_host = torch.zeros(8, dtype=torch.int32, pin_memory=True)

    def _auto_grid_dims(self, budget=1 << 22):
        """Hash-grid dims for the scene as added: enough cells of 2R per axis to cover the bodies'
        initial extent plus a margin without wrapping (a power of two, at least 8), within
        `budget` buckets (the widest axis halved until it fits).  Buckets that alias only cost
        time: the contact set, and its order after the per-bead sort, do not depend on the dims."""
        c = np.asarray(self._centers, np.float64).reshape(-1, 3)
        half = 0.5 * max(self.dims) + 2.0 * R
        ext = (c.max(axis=0) - c.min(axis=0)) + 2.0 * half if len(c) else np.zeros(3)
        cells = np.ceil(ext / (2.0 * R)).astype(np.int64) + 4
        dims = [max(8, 1 << int(np.ceil(np.log2(max(int(n), 1))))) for n in cells]
        dims = [min(d, cap) for d, cap in zip(dims, (1024, 1024, 256))]
        while dims[0] * dims[1] * dims[2] > budget:
            k = int(np.argmax(dims))
            dims[k] //= 2
        return tuple(int(d) for d in dims)

    def _setup_grid(self, dims=None):
        if dims is None:
            dims = self._auto_grid_dims()
        self.grid_dims_used = tuple(int(x) for x in dims)
        dev = self.dev
        nbk = dims[0] * dims[1] * dims[2]
        i32 = lambda n: torch.zeros(n, dtype=torch.int32, device=dev)
        self.g_bucket, self.g_start, self.g_cursor, self.g_sorted = i32(max(self.NB, 1)), i32(nbk + 1), i32(nbk + 1), \
            i32(max(self.NB, 1))
        self.g_scan = i32(max(self.L.b2c_scan_scratch_ints(nbk + 1), 1))
        self.g_spos = torch.zeros((max(self.NB, 1), 4), dtype=torch.float32, device=dev)
        self.c_grid = _lib.Grid(dims[0], dims[1], dims[2], 2.0 * R, _ptr(self.g_bucket), _ptr(self.g_start),
                                _ptr(self.g_cursor), _ptr(self.g_sorted), _ptr(self.g_scan), _ptr(self.g_spos))

    def _setup_contacts(self, cap=MAXC):
        dev = self.dev
        i32 = lambda: torch.zeros(cap, dtype=torch.int32, device=dev)
        f4 = lambda: torch.zeros((cap, 4), dtype=torch.float32, device=dev)
        self.cbi, self.cbj, self.cfa, self.cfb = i32(), i32(), i32(), i32()
        self.cpA, self.cpB, self.cn, self.cimp = f4(), f4(), f4(), f4()
        self.c_contacts = _lib.Contacts(cap, _ptr(self.cbi), _ptr(self.cbj), _ptr(self.cpA), _ptr(self.cpB),
                                        _ptr(self.cn), _ptr(self.cfa), _ptr(self.cfb), _ptr(self.cimp))

    def _struct_bodies(self):
        self.c_bodies = _lib.Bodies(self.N, _ptr(self.xc), _ptr(self.q), _ptr(self.v), _ptr(self.w), _ptr(self.pv),
                                    _ptr(self.po), _ptr(self.invM), _ptr(self.IbInv), _ptr(self.kin),
                                    _ptr(self.invIw))
        self.c_beads = _lib.Beads(self.NB, _ptr(self.rest), _ptr(self.owner), _ptr(self.world),
                                  _ptr(self.bead_start))

    def _stream(self):
        return torch.cuda.current_stream(self.dev)

    # ---- per-step header: one small async read-back per step, checked lazily ----
    def _fetch_header(self):
        self._hdr_host.copy_(self.header, non_blocking=True)
        ev = torch.cuda.Event()
        ev.record(torch.cuda.current_stream(self.dev))
        self._hdr_event = ev
        self._hdr_cache = None

    def header_dict(self) -> dict:
        """Device counters of the last substep (waits for that step to finish)."""
        if getattr(self, "_hdr_cache", None) is None:
            ev = getattr(self, "_hdr_event", None)
            if ev is None:
                return dict.fromkeys(_lib.HEADER_FIELDS, 0)
            ev.synchronize()
            self._hdr_cache = dict(zip(_lib.HEADER_FIELDS, (int(x) for x in self._hdr_host.tolist())))
        return self._hdr_cache

    def check_errors(self):
        """Raise RuntimeError for any error bit the kernels set (capacity, colour cap, timeout)."""
        h = self.header_dict()
        if h["error"]:
            bits = [m for b, m in _lib.ERR_BITS.items() if h["error"] & b]
            self.header.zero_()
            self._hdr_cache = None
            self._hdr_event = None
            raise RuntimeError(f"{self.name}: device error: {'; '.join(bits)}")
        return h

    @property
    def n_contacts(self):
        return self.header_dict()["n_raw"]

    @property
    def n_contacts_solved(self):
        return self.header_dict()["n_kept" if getattr(self, "_has_manifold", False) else "n_contacts"]

    @property
    def n_pairs(self):
        return self.header_dict()["n_pairs"]

    @property
    def n_colors(self):
        return self.header_dict()["n_colors"]

    def _graph_step(self, key, launch):
        """Run one step's launches; with graph=True the launch sequence of a key is captured once
        into a CUDA graph and replayed on later steps (the first step runs eagerly, the capture
        itself executes nothing, so the state advances exactly once per step)."""
        if not self.graph:
            launch()
            return
        g = self._graphs.get(key)
        if g is not None:
            g.replay()
            return
        launch()
        g = torch.cuda.CUDAGraph(keep_graph=True)
        cs = torch.cuda.Stream(self.dev)
        cs.wait_stream(torch.cuda.current_stream(self.dev))
        with torch.cuda.graph(g, stream=cs):
            launch()
        torch.cuda.current_stream(self.dev).wait_stream(cs)
        self.kernels_per_step[key] = int(self.L.b2c_graph_kernel_nodes(ctypes.c_void_p(g.raw_cuda_graph())))
        g.instantiate()
        if len(self._graphs) >= 8:
            self._graphs.clear()
        self._graphs[key] = g
        self.n_graph_captures += 1

    # ---- live kinematic update (contact_engine_gpu.py:241-249) ----
    def set_kinematic(self, i, xc):
        self._kin[i] = 1
        self._centers[i] = list(xc)
        if self._built:
            self.xc[i, :3] = torch.tensor(np.array(xc, np.float32), device=self.dev)
            self.invM[i] = 0.0
            self.v[i] = 0.0
            self.w[i] = 0.0
            self.kin[i] = 1
            self._kinarr[i] = 1
            self._M[i] = np.inf

    # ---- host state I/O ----
    def set_body_state(self, xc, q, v, w):
        """Overwrite the body state from host arrays ((N,3), (N,4), (N,3), (N,3) float32; pinned
        torch tensors are copied asynchronously on the engine's stream)."""
        if not self._built:
            self._build()
        for dst, src, k in ((self.xc, xc, 3), (self.q, q, 4), (self.v, v, 3), (self.w, w, 3)):
            t = src if isinstance(src, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(src, np.float32))
            dst[:, :k].copy_(t, non_blocking=True)

    def set_state_packed(self, state):
        """Overwrite the whole body state with one (4, N, 4) float32 array: the planes are the
        positions, the quaternions (x, y, z, w), the velocities and the angular velocities, each
        row padded to four floats (the kernels read the first three of a vector row).  One copy;
        a pinned torch tensor is copied asynchronously on the current stream."""
        if not self._built:
            self._build()
        t = state if isinstance(state, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(state, np.float32))
        self.state.copy_(t.reshape(self.state.shape), non_blocking=True)

    def get_state_packed(self, out=None):
        """The whole body state as one (4, N, 4) float32 array (see set_state_packed): a new host
        tensor, or copied into `out` (asynchronously when it is pinned)."""
        if not self._built:
            self._build()
        if out is None:
            return self.state.cpu()
        out.copy_(self.state, non_blocking=True)
        return out

    # ---- data out ----
    def get_state(self) -> BodyState:
        if not self._built:
            self._build()
        torch.cuda.synchronize(self.dev)
        xc = self.xc[:, :3].cpu().numpy()
        q = self.q.cpu().numpy()
        return BodyState(xc=xc, Rm=quat_to_R(q), vc=self.v[:, :3].cpu().numpy(), om=self.w[:, :3].cpu().numpy())

    def contact_forces(self) -> np.ndarray:
        """M (v_after - v_before) / dt in float64 for the last substep; kinematic rows are 0."""
        f = np.zeros((len(self._centers), 3))
        if not self._built or self._force_dt is None:
            return f
        torch.cuda.synchronize(self.dev)
        after = self.v[:, :3].cpu().numpy()
        before = self.vgrav[:, :3].cpu().numpy()
        nk = self._kinarr == 0
        f[nk] = self._M[nk, None] * (after[nk] - before[nk]) / self._force_dt
        return f

    def com(self, i):
        return self.xc[i, :3].cpu().numpy()

    def kept_contacts(self) -> dict:
        """The contacts the last substep solved, in feature order, as numpy arrays named like
        the reference engine's attributes (contact_engine_gpu_colored.py:1095-1103): ckeys, sbi,
        sbj, spA, spB, sn, spen (depth) and the impulses after the solve jn, jt1, jt2, jp.  For
        the manifold engines and the box engine these are the kept contacts.  The relaxed-Jacobi
        engine solves every generated contact in the order the atomic append left them, has no
        feature keys (ckeys is -1) and keeps no impulses per contact (zeros)."""
        if not self._built:
            self._build()
        h = self.header_dict()
        if hasattr(self, "k_keys"):
            C = h["n_kept"]
            keys, bi, bj, pA, pB, nrm, imp = (self.k_keys, self.k_bi, self.k_bj, self.k_pA, self.k_pB, self.k_n,
                                              self.k_imp)
        else:
            C = h["n_contacts"]
            keys = torch.full((max(C, 1),), -1, dtype=torch.int64)
            bi, bj, pA, pB, nrm, imp = self.cbi, self.cbj, self.cpA, self.cpB, self.cn, self.cimp
        pA_ = pA[:C].cpu().numpy()
        imp_ = imp[:C].cpu().numpy()
        return dict(ckeys=keys[:C].cpu().numpy(), sbi=bi[:C].cpu().numpy(), sbj=bj[:C].cpu().numpy(),
                    spA=np.ascontiguousarray(pA_[:, :3]), spB=pB[:C, :3].cpu().numpy(),
                    sn=nrm[:C, :3].cpu().numpy(), spen=np.ascontiguousarray(pA_[:, 3]),
                    jn=np.ascontiguousarray(imp_[:, 0]), jt1=np.ascontiguousarray(imp_[:, 1]),
                    jt2=np.ascontiguousarray(imp_[:, 2]), jp=np.ascontiguousarray(imp_[:, 3]))

    def warm_store(self) -> dict:
        """The warm-start store the next substep looks its impulses up in (engines that keep
        one): feature keys ascending, and jn, jt1, jt2 as stored."""
        if not self._built:
            self._build()
        torch.cuda.synchronize(self.dev)
        n = int(self.w_n[0].item())
        imp = self.w_imp[:n].cpu().numpy()
        return dict(keys=self.w_keys[:n].cpu().numpy(), jn=imp[:, 0].copy(), jt1=imp[:, 1].copy(),
                    jt2=imp[:, 2].copy())

    def max_depth_device(self) -> torch.Tensor:
        """The deepest penetration among the last substep's solved contacts, as a 0-d float32
        device tensor computed on the engine's stream without a host read (0 without
        contacts).  The quality figure beside a timed step."""
        if hasattr(self, "k_pA"):
            depth, n = self.k_pA[:, 3], self.header[_lib.HEADER_FIELDS.index("n_kept")]
        else:
            depth, n = self.cpA[:, 3], self.header[_lib.HEADER_FIELDS.index("n_contacts")]
        live = torch.arange(depth.shape[0], device=depth.device, dtype=torch.int32) < n
        return torch.where(live, depth, torch.zeros((), dtype=depth.dtype, device=depth.device)).max()


class RelaxedJacobiContactEngine(_BeadEngineBase):
    """Relaxed Jacobi with int64 fixed-point accumulation on bead bodies: the B200 build of the
    reference's RelaxedJacobiContactEngine (contact_engine_gpu.py:191-299).  Bit-exact to the
    reference on the same inputs and bit-identical run to run."""
    name = "relaxed_jacobi_b200"

    def __init__(self, dims=(0.3, 0.3, 0.2), relax=0.2, vit=40, pit=20, mu=0.5, device="cuda", graph=True,
                 contact_capacity=MAXC, grid_dims=None):
        super().__init__(dims=dims, mu=mu, device=device, graph=graph)
        self.relax = float(relax)
        self.vit = int(vit)
        self.pit = int(pit)
        self.contact_capacity = int(contact_capacity)
        # buckets of the bead hash grid (cell 2R, wrapping): a performance choice only -- the
        # Jacobi sum is order free, so the contacts and the results do not depend on it
        self.grid_dims = None if grid_dims is None else tuple(int(x) for x in grid_dims)

    def _build(self):
        self._setup_bodies()
        self._setup_grid(self.grid_dims)
        self._setup_contacts(self.contact_capacity)
        self.acc = torch.zeros((6, self.N), dtype=torch.int64, device=self.dev)
        self._struct_bodies()
        self.c_params = _lib.JacobiParams(self.vit, self.pit, self.relax, self.mu)
        self._graphs = {}
        self._built = True

    def _launch_step(self, sdt: float, substeps: int):
        s = torch.cuda.current_stream(self.dev).cuda_stream
        L = self.L
        for _ in range(substeps):
            rc = L.b2c_jacobi_substep(ctypes.byref(self.c_bodies), ctypes.byref(self.c_beads),
                                      ctypes.byref(self.c_grid), ctypes.byref(self.c_contacts),
                                      ctypes.c_void_p(_ptr(self.header)), ctypes.c_void_p(_ptr(self.acc)),
                                      ctypes.byref(self.c_params), ctypes.c_float(sdt),
                                      ctypes.c_void_p(_ptr(self.vgrav)), ctypes.c_void_p(s))
            _lib.check(rc, "b2c_jacobi_substep")

    def solve_sample(self, sdt: float):
        """One b2c_jacobi_solve on the current contacts between CUDA events (it moves the state on:
        call it last).  Returns (milliseconds, algorithmic bytes, counts).  Bytes per launch
        sequence, each array element read or written once per launch: a velocity iteration
        (k_jacobi_velocity + k_jacobi_apply) moves 68 C + (76 + 16 x 12) E + 144 N, a position
        iteration 56 C + (76 + 16 x 6) E + 144 N -- C contacts, E their dynamic endpoints (a
        body's xc, invM, invIw, v, w and its 6 int64 accumulators, 12 atomics per endpoint in the
        velocity pass), N bodies (apply: 6 int64 read and cleared, v, w read and written)."""
        h = self.header_dict()
        C = min(int(h["n_contacts"]), self.contact_capacity)
        bi = self.cbi[:C].long()
        bj = self.cbj[:C].long()
        dyn = self.invM > 0
        E = int(dyn[bi].sum()) + int(((bj >= 0) & dyn[bj.clamp(min=0)]).sum())
        N = self.N
        vel = 68 * C + (76 + 16 * 12) * E + 144 * N
        pos = 56 * C + (76 + 16 * 6) * E + 144 * N
        s = torch.cuda.current_stream(self.dev)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(self.dev)
        a.record(s)
        _lib.check(self.L.b2c_jacobi_solve(ctypes.byref(self.c_bodies), ctypes.byref(self.c_contacts),
                                           ctypes.c_void_p(_ptr(self.header)), ctypes.c_void_p(_ptr(self.acc)),
                                           ctypes.byref(self.c_params), ctypes.c_float(sdt),
                                           ctypes.c_void_p(s.cuda_stream)), "b2c_jacobi_solve")
        b.record(s)
        b.synchronize()
        return a.elapsed_time(b), self.vit * vel + self.pit * pos, dict(contacts=C, endpoints=E, bodies=N,
                                                                         vit=self.vit, pit=self.pit)

    def step(self, dt, substeps=1):
        if not self._built:
            self._build()
        self.check_errors()
        sdt = dt / substeps
        self._graph_step(("jacobi", float(sdt), int(substeps)), lambda: self._launch_step(sdt, substeps))
        self._force_dt = sdt
        self._fetch_header()
