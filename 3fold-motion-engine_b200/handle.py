"""ContactEngine over the library-owned engine handle (b2c_create ... b2c_destroy).

The reference's drop-in boundary is the ContactEngine protocol (src/motion_engine/contact_engine.py:48-55).
BoxContactEngine implements it with PyTorch owning the device arrays; this class implements it
over ctypes and numpy arrays only: libb2c.so owns the device memory of the handle and runs the
same substep launches (b2c_box_substep), so the two give the same bits over the same bodies.
Its calls are the binding a caller without a tensor library would write.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .engine import BodyState, quat_to_R

MARGIN = 2e-3


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


class HandleBoxEngine:
    """The box engine (solid boxes, float64 SAT contacts, the ColorCache pair solve) through the
    engine handle.  Keywords as BoxContactEngine; `flags` overrides the B2C_COLOR_* set."""
    name = "box_color_cache_handle_b200"

    def __init__(self, dims=(0.3, 0.3, 0.2), mu=0.5, vit=16, pit=10, margin=MARGIN, color_cap=512, solve_blocks=0,
                 barrier_timeout_s=1.0, cand_per_body=16, flags=None, graph=True, device=0):
        self.L = _lib.load()
        c = _lib.Config()
        self.L.b2c_config_init(ctypes.byref(c))
        c.device, c.vit, c.pit, c.mu = int(device), int(vit), int(pit), float(mu)
        for k in range(3):
            c.dims[k] = float(dims[k])
        c.margin, c.color_cap, c.solve_blocks = float(margin), int(color_cap), int(solve_blocks)
        c.cand_per_body, c.barrier_timeout_ns, c.graph = int(cand_per_body), int(barrier_timeout_s * 1e9), int(graph)
        if flags is not None:
            c.flags = int(flags)
        self.config = c
        self.dims = tuple(float(x) for x in dims)
        self.mu = float(mu)
        self._h = ctypes.c_void_p()
        rc = self.L.b2c_create(ctypes.byref(c), ctypes.byref(self._h))
        if rc == 1:
            raise ValueError(f"{self.name}: {self.L.b2c_last_error().decode()}")
        _lib.check(rc, "b2c_create")

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self.L.b2c_destroy(ctypes.byref(self._h))

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _call(self, rc, what):
        if rc == 1:
            raise ValueError(f"{what}: {self.L.b2c_last_error().decode()}")
        _lib.check(rc, what)

    # ---- construction ----
    @property
    def N(self) -> int:
        return int(self.L.b2c_body_count(self._h))

    def add_body(self, center, density=700.0, kin=False):
        return self.add_box(center, dims=self.dims, density=density, kin=kin)

    def add_box(self, center, dims=None, density=1000.0, mu=None, kin=False, scene=0):
        return int(self.add_boxes([center], None if dims is None else [dims], [density],
                                  None if mu is None else [mu], [bool(kin)], [scene])[0])

    def add_boxes(self, centers, dims=None, density=None, mu=None, kin=None, scene=None) -> np.ndarray:
        """Appends n boxes at once; returns their indices."""
        c = np.ascontiguousarray(np.asarray(centers, np.float64).reshape(-1, 3))
        n, first = len(c), self.N
        d = None if dims is None else np.ascontiguousarray(np.asarray(dims, np.float64).reshape(n, 3))
        rho = None if density is None else np.ascontiguousarray(np.broadcast_to(np.asarray(density, np.float64), (n,)))
        k = None if kin is None else np.ascontiguousarray(np.asarray(kin, bool).astype(np.int32).reshape(n))
        self._call(self.L.b2c_add_bodies(self._h, n, _dptr(c), None if rho is None else _dptr(rho),
                                         None if d is None else _dptr(d), None if k is None else _dptr(k)),
                   "b2c_add_bodies")
        if mu is not None:
            m = np.ascontiguousarray(np.broadcast_to(np.asarray(mu, np.float64), (n,)))
            self._call(self.L.b2c_set_body_mu(self._h, first, n, _dptr(m)), "b2c_set_body_mu")
        if scene is not None:
            s = np.ascontiguousarray(np.broadcast_to(np.asarray(scene, np.int32), (n,)))
            if np.any(s):
                self._call(self.L.b2c_set_body_scene(self._h, first, n, _dptr(s)), "b2c_set_body_scene")
        return np.arange(first, first + n)

    # ---- stepping and diagnostics ----
    def step(self, dt, substeps=1):
        """Advance; raises RuntimeError when the previous step set a device error bit."""
        _lib.check(self.L.b2c_step(self._h, float(dt), int(substeps), None), "b2c_step")

    def header(self) -> dict:
        h = _lib.StepHeader()
        _lib.check(self.L.b2c_sync_header(self._h, ctypes.byref(h)), "b2c_sync_header")
        out = dict(zip(_lib.HEADER_FIELDS, (int(x) for x in h.last)))
        out.update(color_cache_hits=h.color_cache_hits, color_cache_misses=h.color_cache_misses,
                   n_graph_captures=h.graph_captures, kernels_per_step=h.kernels_per_step, bodies=h.bodies,
                   built=h.built)
        return out

    @property
    def n_contacts(self):
        return self.header()["n_raw"]

    @property
    def n_contacts_solved(self):
        return self.header()["n_kept"]

    @property
    def n_pairs(self):
        return self.header()["n_pairs"]

    @property
    def n_colors(self):
        return self.header()["n_colors"]

    @property
    def color_cache_hits(self):
        return self.header()["color_cache_hits"]

    @property
    def color_cache_misses(self):
        return self.header()["color_cache_misses"]

    @property
    def n_graph_captures(self):
        return self.header()["n_graph_captures"]

    # ---- state ----
    def get_state(self) -> BodyState:
        n = self.N
        xc, q = np.empty((n, 3), np.float32), np.empty((n, 4), np.float32)
        v, w = np.empty((n, 3), np.float32), np.empty((n, 3), np.float32)
        _lib.check(self.L.b2c_get_state(self._h, _dptr(xc), _dptr(q), _dptr(v), _dptr(w)), "b2c_get_state")
        return BodyState(xc=xc, Rm=quat_to_R(q), vc=v, om=w)

    def get_state_packed(self) -> np.ndarray:
        """(4, N, 4) float32: planes xc, q, v, w."""
        out = np.empty((4, self.N, 4), np.float32)
        _lib.check(self.L.b2c_get_state_packed(self._h, _dptr(out), None), "b2c_get_state_packed")
        return out

    def set_state_packed(self, state):
        s = np.ascontiguousarray(np.asarray(state, np.float32).reshape(4, self.N, 4))
        _lib.check(self.L.b2c_set_state_packed(self._h, _dptr(s), None), "b2c_set_state_packed")

    def set_kinematic(self, i, xc):
        x = np.ascontiguousarray(np.asarray(xc, np.float64).reshape(3))
        self._call(self.L.b2c_set_kinematic(self._h, int(i), _dptr(x)), "b2c_set_kinematic")

    def contact_forces(self) -> np.ndarray:
        f = np.zeros((self.N, 3))
        _lib.check(self.L.b2c_contact_forces(self._h, _dptr(f)), "b2c_contact_forces")
        return f

    def com(self, i):
        return self.get_state().xc[i]

    # ---- checkpoint ----
    def state_save(self) -> bytes:
        n = ctypes.c_size_t(0)
        _lib.check(self.L.b2c_state_save(self._h, None, ctypes.byref(n)), "b2c_state_save")
        buf = ctypes.create_string_buffer(n.value)
        _lib.check(self.L.b2c_state_save(self._h, buf, ctypes.byref(n)), "b2c_state_save")
        return buf.raw[:n.value]

    def state_load(self, blob: bytes):
        self._call(self.L.b2c_state_load(self._h, blob, len(blob)), "b2c_state_load")
