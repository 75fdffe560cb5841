"""CPU oracle for the contact-solve hot path -- TEST INFRASTRUCTURE ONLY.

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may
import this module.  It is the checker the CUDA product is compared against, never part of
the product: the product package does not import it and fails loudly without its CUDA
library.

Python half of the oracle: the host-side body setup of the reference (numpy, float64 then
cast to float32 exactly where the reference's ``wp.array(...)`` casts) and ctypes bindings to
``liboracle.so`` (``oracle_contact.c``), which restates the reference's float32 kernels.

Reference anchors:
  * ``_voxbox``                        src/motion_engine/contact_engine_gpu.py:186-188
  * ``RelaxedJacobiContactEngine._build`` src/motion_engine/contact_engine_gpu.py:209-239
  * ``RelaxedJacobiContactEngine.step``  src/motion_engine/contact_engine_gpu.py:252-280
  * ``_quat2R`` / ``get_state``          src/motion_engine/contact_engine_gpu.py:283-293
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

R = 0.05
MAXC = 400000

# variant indices of oracle_contact.c (g_fv[])
FV_NAMES = ["DOT", "CROSS", "MATVEC", "MATMUL", "QROT", "QMUL", "QNORM", "VNORM", "SITE_GRAV", "SITE_VT",
            "SITE_T1", "SITE_MAG", "SITE_JT", "SITE_APPLY", "SITE_INTX", "SITE_INTQ", "SITE_IMP", "QDOT",
            "SITE_VUPD", "SITE_WUPD", "SITE_BIAS"]
FV = {n: i for i, n in enumerate(FV_NAMES)}

# The contraction pattern that reproduces the reference's golden arrays bit for bit.
PINNED_VARIANTS = {n: (1 if n.startswith("SITE_") else 0) for n in FV_NAMES}
PINNED_VARIANTS.update(SITE_WUPD=0, SITE_BIAS=0)


def build(force: bool = False) -> str:
    """Compile liboracle.so and its FP64 re-solve build liboracle64.so beside this file (gcc,
    contraction off)."""
    so = os.path.join(_HERE, "liboracle.so")
    srcs = [os.path.join(_HERE, f) for f in ("oracle_contact.c", "oracle_ncp.c", "f64_prelude.h", "Makefile")]
    newest = max(os.path.getmtime(f) for f in srcs)
    outs = [so, os.path.join(_HERE, "liboracle64.so")]
    if force or any(not os.path.exists(o) or os.path.getmtime(o) < newest for o in outs):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return so


def lib():
    global _LIB
    if _LIB is None:
        so = build()
        L = ctypes.CDLL(so)
        P = ctypes.c_void_p
        L.or_set_variant.argtypes = [ctypes.c_int, ctypes.c_int]
        L.or_get_variant.argtypes = [ctypes.c_int]
        L.or_get_variant.restype = ctypes.c_int
        L.or_jacobi_step.argtypes = [ctypes.c_int, ctypes.c_int, P, P, P, P, P, P, P, P, P, P, P, P,
                                     ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_float, ctypes.c_float, ctypes.c_int, P, P]
        L.or_jacobi_step.restype = ctypes.c_int
        _LIB = L
        set_variants(PINNED_VARIANTS)
    return _LIB


_LIB64 = None


def lib64():
    """liboracle64.so: the coloured / ColorCache chain and the box engine compiled in float64
    (f64_prelude.h), the FP64 re-solve the float32 tolerances are stated against."""
    global _LIB64
    if _LIB64 is None:
        build()
        L = ctypes.CDLL(os.path.join(_HERE, "liboracle64.so"))
        L.or_set_variant.argtypes = [ctypes.c_int, ctypes.c_int]
        for k, v in PINNED_VARIANTS.items():
            L.or_set_variant(FV[k], int(v))
        _col_sigs(L, ctypes.c_double)
        _box_sigs(L, ctypes.c_double)
        L._col_ready = True
        _LIB64 = L
    return _LIB64


def _precision(precision):
    """(numpy dtype, library) of an oracle precision, "float32" (the restatement of the
    reference's arithmetic) or "float64" (the FP64 re-solve)."""
    if precision == "float32":
        return np.float32, lib()
    if precision == "float64":
        return np.float64, lib64()
    raise ValueError(f"precision is 'float32' or 'float64', not {precision!r}")


def set_variants(d: dict) -> None:
    L = lib()
    for k, v in d.items():
        L.or_set_variant(FV[k], int(v))


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def voxbox(w, h, d, res=R * 2):
    """Bead rest offsets of a box (contact_engine_gpu.py:186-188): per axis
    arange(-L/2 + res/2, L/2, res), x fastest, then y, then z; float64."""
    a = lambda L: np.arange(-L / 2 + res / 2, L / 2, res)
    return np.array([[x, y, z] for z in a(d) for y in a(h) for x in a(w)], float)


@dataclass
class BodySetup:
    """Device-ready body arrays, exactly as RelaxedJacobiContactEngine._build lays them out."""
    rest: np.ndarray     # (P, 3) f32 per-bead rest offsets (uniform over bodies)
    xc: np.ndarray       # (N, 3) f32
    q: np.ndarray        # (N, 4) f32, (x, y, z, w)
    v: np.ndarray
    w: np.ndarray
    invM: np.ndarray     # (N,) f32
    IbInv: np.ndarray    # (N, 3, 3) f32
    kin: np.ndarray      # (N,) int32
    M: np.ndarray        # (N,) f64 (inf for bodies made kinematic after the build)


def build_bodies(centers, dens, kin, dims) -> BodySetup:
    """contact_engine_gpu.py:209-239 (also contact_engine_gpu_colored.py:836-850):
    mass = density*vol, bead point-mass inertia Ib = sum mp (r.r I - r r^T), IbInv by
    np.linalg.inv per body (identity for kinematic), identity quaternion."""
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
        raise ValueError("IbInv contains non-finite entries: degenerate body mass/inertia")
    return BodySetup(rest=rest64.astype(np.float32),
                     xc=np.array(np.array(centers, float), np.float32).reshape(N, 3),
                     q=np.tile(np.array([0, 0, 0, 1.0], np.float32), (N, 1)),
                     v=np.zeros((N, 3), np.float32), w=np.zeros((N, 3), np.float32),
                     invM=invM.astype(np.float32), IbInv=IbInv.astype(np.float32).reshape(N, 3, 3),
                     kin=kinarr.astype(np.int32), M=M.astype(np.float64))


def _cast_bodies(b: BodySetup, F) -> BodySetup:
    """The body arrays in the oracle's precision: the float32 setup values themselves, widened
    for the FP64 re-solve (so both precisions start from the same inputs)."""
    if F is np.float32:
        return b
    return BodySetup(rest=b.rest.astype(F), xc=b.xc.astype(F), q=b.q.astype(F), v=b.v.astype(F), w=b.w.astype(F),
                     invM=b.invM.astype(F), IbInv=b.IbInv.astype(F), kin=b.kin, M=b.M)


def quat_to_R(q: np.ndarray) -> np.ndarray:
    """Host quaternion -> matrix of get_state (contact_engine_gpu.py:283-287), float32
    arithmetic on float32 inputs as numpy does it there."""
    x, y, z, w = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    one = np.float32(1); two = np.float32(2)
    Rm = np.empty((len(q), 3, 3), np.float32)
    Rm[:, 0, 0] = one - two * (y * y + z * z); Rm[:, 0, 1] = two * (x * y - z * w); Rm[:, 0, 2] = two * (x * z + y * w)
    Rm[:, 1, 0] = two * (x * y + z * w); Rm[:, 1, 1] = one - two * (x * x + z * z); Rm[:, 1, 2] = two * (y * z - x * w)
    Rm[:, 2, 0] = two * (x * z - y * w); Rm[:, 2, 1] = two * (y * z + x * w); Rm[:, 2, 2] = one - two * (x * x + y * y)
    return Rm


@dataclass
class State:
    xc: np.ndarray
    Rm: np.ndarray
    vc: np.ndarray
    om: np.ndarray


class JacobiOracle:
    """CPU restatement of RelaxedJacobiContactEngine (contact_engine_gpu.py:191-299)."""
    name = "relaxed_jacobi_oracle"

    def __init__(self, dims=(0.3, 0.3, 0.2), relax=0.2, vit=40, pit=20, mu=0.5):
        self.dims = dims; self.relax = relax; self.vit = vit; self.pit = pit; self.mu = mu
        self._centers = []; self._dens = []; self._kin = []
        self.b = None
        self.n_contacts = 0

    def add_body(self, center, density=700.0, kin=False):
        self._centers.append(list(center)); self._dens.append(float(density)); self._kin.append(1 if kin else 0)
        self.b = None
        return len(self._centers) - 1

    def _build(self):
        self.b = build_bodies(self._centers, self._dens, self._kin, self.dims)
        N = len(self._centers); P = len(self.b.rest)
        self.N = N; self.P = P
        self.rest_all = np.ascontiguousarray(np.tile(self.b.rest, (N, 1)))
        self.owner = np.repeat(np.arange(N, dtype=np.int32), P)
        self.force = np.zeros((N, 3))
        self.pv = np.zeros((N, 3), np.float32); self.po = np.zeros((N, 3), np.float32)

    def set_kinematic(self, i, xc):
        self._kin[i] = 1; self._centers[i] = list(xc)
        if self.b is not None:
            self.b.xc[i] = np.array(xc, np.float32); self.b.invM[i] = 0.0
            self.b.v[i] = 0.0; self.b.w[i] = 0.0; self.b.kin[i] = 1; self.b.M[i] = np.inf

    def step(self, dt, substeps=1):
        if self.b is None:
            self._build()
        b = self.b
        force = np.zeros((self.N, 3))
        nc = np.zeros(substeps, np.int32)
        rc = lib().or_jacobi_step(self.N, self.N * self.P, _p(self.rest_all), _p(self.owner), _p(b.xc), _p(b.q),
                                  _p(b.v), _p(b.w), _p(self.pv), _p(self.po), _p(b.invM), _p(b.IbInv), _p(b.kin), _p(b.M), float(dt),
                                  int(substeps), int(self.vit), int(self.pit), float(self.relax), float(self.mu),
                                  MAXC, _p(force), _p(nc))
        if rc != 0:
            raise RuntimeError(f"oracle jacobi step failed with status {rc}")
        self.force = force
        self.n_contacts = int(nc[-1])

    def get_state(self) -> State:
        if self.b is None:
            self._build()
        return State(xc=self.b.xc.copy(), Rm=quat_to_R(self.b.q), vc=self.b.v.copy(), om=self.b.w.copy())

    def contact_forces(self):
        return self.force.copy()


def _col_sigs(L, F=ctypes.c_float):
    P = ctypes.c_void_p
    L.or_col_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, F, F, ctypes.c_int,
                                ctypes.c_int]
    L.or_col_create.restype = P
    L.or_col_destroy.argtypes = [P]
    L.or_col_stats.argtypes = [P, P]
    L.or_col_step.argtypes = [P, ctypes.c_int, ctypes.c_int, P, P, P, P, P, P, P, P, P, P, P, ctypes.c_double,
                              ctypes.c_int, P]
    L.or_col_step.restype = ctypes.c_int
    L.or_col_kept.argtypes = [P] * 12
    L.or_col_kept.restype = ctypes.c_int
    L.or_col_warm_get.argtypes = [P] * 5
    L.or_col_warm_get.restype = ctypes.c_int
    L.or_col_warm_set.argtypes = [P, ctypes.c_int, P, P, P, P]
    L.or_col_warm_set.restype = ctypes.c_int
    L.or_col_pre.argtypes = [P] * 4
    L.or_col_pre.restype = ctypes.c_int
    L.or_col_inject.argtypes = [P, ctypes.c_int, P, P, P, P]
    L.or_col_inject.restype = ctypes.c_int


class ColoredOracle:
    """CPU restatement of the coloured pair-chunk engines.

    mode="pair_chunks": GraphColoredContactEngine(manifold_reduce=True, graph_capture=True,
        pair_chunks=True) -- contact_engine_gpu_colored.py:793-1410, slip-basis chunk sweep.
    mode="plain": GraphColoredContactEngine() -- per-contact colouring, no manifold reduction
        (contact_engine_gpu_colored.py:903-936, 1105-1137, 188-320).
    mode="reduced": GraphColoredContactEngine(manifold_reduce=True) -- the device manifold
        reduction, then the kept contacts coloured one by one with k_prio_manifold's priority
        (contact_engine_gpu_colored.py:776-787, 1105-1113).
    mode="color_cache": ColorCacheContactEngine -- contact_engine_gpu_color_cache.py:21-54 on top of
        DeferredForce / AppliedWarm / FixedFrame (fixed tangent frame, warm impulses applied once per
        colour before the sweeps, colouring reused while the pair graph and masses are unchanged).
    """

    def __init__(self, mode="color_cache", dims=(0.3, 0.3, 0.2), vit=40, pit=20, mu=0.5, max_points=4,
                 t2_damp=1.0, cap=MAXC, precision="float32"):
        assert mode in ("pair_chunks", "color_cache", "plain", "reduced")
        self.mode = mode
        self.precision = precision
        self.F, self.L = _precision(precision)
        self.name = f"{mode}_oracle"
        self.dims = dims; self.vit = vit; self.pit = pit; self.mu = mu; self.mx = max_points; self.t2d = t2_damp
        self.cap = cap
        self._centers = []; self._dens = []; self._kin = []
        self.b = None
        self._h = None
        self._force_dt = None

    def add_body(self, center, density=700.0, kin=False):
        self._centers.append(list(center)); self._dens.append(float(density)); self._kin.append(1 if kin else 0)
        self.b = None
        return len(self._centers) - 1

    def _build(self):
        L = self.L
        if not hasattr(L, "_col_ready"):
            _col_sigs(L); L._col_ready = True
        self.b = _cast_bodies(build_bodies(self._centers, self._dens, self._kin, self.dims), self.F)
        N = len(self._centers); P = len(self.b.rest)
        self.N = N; self.P = P
        self.rest_all = np.ascontiguousarray(np.tile(self.b.rest, (N, 1)))
        self.owner = np.repeat(np.arange(N, dtype=np.int32), P)
        self.pv = np.zeros((N, 3), self.F); self.po = np.zeros((N, 3), self.F)
        self.vgrav = np.zeros((N, 3), self.F)
        if self._h:
            L.or_col_destroy(self._h)
        self._h = L.or_col_create({"pair_chunks": 0, "color_cache": 1, "plain": 2, "reduced": 3}[self.mode], self.vit,
                                  self.pit,
                                  self.mx, self.mu,
                                  self.t2d, self.cap, N)

    def __del__(self):
        try:
            if self._h:
                self.L.or_col_destroy(self._h)
        except Exception:
            pass

    def set_kinematic(self, i, xc):
        self._kin[i] = 1; self._centers[i] = list(xc)
        if self.b is not None:
            self.b.xc[i] = np.array(np.array(xc, np.float32), self.F); self.b.invM[i] = 0.0
            self.b.v[i] = 0.0; self.b.w[i] = 0.0; self.b.kin[i] = 1; self.b.M[i] = np.inf

    def step(self, dt, substeps=1):
        if self.b is None:
            self._build()
        b = self.b
        rc = self.L.or_col_step(self._h, self.N, self.N * self.P, _p(self.rest_all), _p(self.owner), _p(b.xc), _p(b.q),
                               _p(b.v), _p(b.w), _p(self.pv), _p(self.po), _p(b.invM), _p(b.IbInv), _p(b.kin),
                               float(dt), int(substeps), _p(self.vgrav))
        if rc != 0:
            raise RuntimeError(f"oracle coloured step failed with status {rc}")
        self._force_dt = dt / substeps

    def stats(self):
        out = np.zeros(7, np.int32)
        self.L.or_col_stats(self._h, _p(out))
        return dict(zip(("n_contacts", "n_kept", "n_pairs", "n_colors", "hits", "misses", "seg_overflow"),
                        out.tolist()))

    @property
    def n_contacts(self):
        return self.stats()["n_contacts"]

    def kept_contacts(self) -> dict:
        """The last substep's kept contacts in feature order, named as the reference's engine
        attributes (ckeys, sbi, sbj, spA, spB, sn, spen, jn, jt1, jt2, jp; COL:1095-1103)."""
        L, F = self.L, self.F
        C = int(L.or_col_kept(self._h, *([None] * 11)))
        out = dict(ckeys=np.zeros(C, np.int64), sbi=np.zeros(C, np.int32), sbj=np.zeros(C, np.int32),
                   spA=np.zeros((C, 3), F), spB=np.zeros((C, 3), F), sn=np.zeros((C, 3), F),
                   spen=np.zeros(C, F), jn=np.zeros(C, F), jt1=np.zeros(C, F), jt2=np.zeros(C, F), jp=np.zeros(C, F))
        if C:
            L.or_col_kept(self._h, *(_p(out[k]) for k in ("ckeys", "sbi", "sbj", "spA", "spB", "sn", "spen", "jn",
                                                          "jt1", "jt2", "jp")))
        return out

    def pre_solve_impulses(self) -> dict:
        """jn, jt1, jt2 (float64 copies) of the last substep's kept contacts as its solve received
        them: warm-started and, in the manifold engines, reduced onto the kept points."""
        n = int(self.L.or_col_pre(self._h, None, None, None))
        d = dict(jn=np.zeros(n), jt1=np.zeros(n), jt2=np.zeros(n))
        self.L.or_col_pre(self._h, _p(d["jn"]), _p(d["jt1"]), _p(d["jt2"]))
        return d

    def inject(self, kept: dict, start: dict) -> None:
        """Make the next substep solve `kept` (ckeys, sbi, sbj, spA, spB, sn, spen) from the
        impulses `start` (jn, jt1, jt2) instead of the contacts it selects itself (one substep,
        coloured engines): the FP64 re-solve of a float32 step on the float32 step's contacts."""
        if self.b is None:
            self._build()
        n = len(kept["ckeys"])
        f = np.zeros((n, 13))
        f[:, 0:3], f[:, 3:6], f[:, 6:9] = kept["spA"], kept["spB"], kept["sn"]
        f[:, 9] = kept["spen"]
        f[:, 10], f[:, 11], f[:, 12] = start["jn"], start["jt1"], start["jt2"]
        keys = np.ascontiguousarray(kept["ckeys"], np.int64)
        bi, bj = (np.ascontiguousarray(kept[k], np.int32) for k in ("sbi", "sbj"))
        if self.L.or_col_inject(self._h, n, _p(keys), _p(bi), _p(bj), _p(np.ascontiguousarray(f))) != 0:
            raise ValueError("injected contacts exceed the oracle's capacity")

    def warm_store(self) -> dict:
        """The warm-start store the next substep looks its impulses up in: keys (int64) and
        jn, jt1, jt2 (float64 copies of the stored values)."""
        if self.b is None:
            self._build()
        n = int(self.L.or_col_warm_get(self._h, None, None, None, None))
        d = dict(keys=np.zeros(n, np.int64), jn=np.zeros(n), jt1=np.zeros(n), jt2=np.zeros(n))
        self.L.or_col_warm_get(self._h, _p(d["keys"]), _p(d["jn"]), _p(d["jt1"]), _p(d["jt2"]))
        return d

    def set_warm_store(self, d: dict) -> None:
        """Replace the warm-start store (keys ascending; impulses rounded to this precision)."""
        if self.b is None:
            self._build()
        k = np.ascontiguousarray(d["keys"], np.int64)
        a = [np.ascontiguousarray(d[f], np.float64) for f in ("jn", "jt1", "jt2")]
        if self.L.or_col_warm_set(self._h, len(k), _p(k), *(_p(x) for x in a)) != 0:
            raise ValueError("warm store larger than the oracle's capacity")

    def body_state(self):
        """(xc, q, v, w) copies in the oracle's precision."""
        if self.b is None:
            self._build()
        return self.b.xc.copy(), self.b.q.copy(), self.b.v.copy(), self.b.w.copy()

    def set_body_state(self, xc, q, v, w):
        """Overwrite positions, quaternions (x, y, z, w) and velocities (the warm store is kept)."""
        if self.b is None:
            self._build()
        for dst, src in ((self.b.xc, xc), (self.b.q, q), (self.b.v, v), (self.b.w, w)):
            dst[...] = np.asarray(src, self.F).reshape(dst.shape)

    def get_state(self) -> State:
        if self.b is None:
            self._build()
        return State(xc=self.b.xc.copy(), Rm=quat_to_R(self.b.q), vc=self.b.v.copy(), om=self.b.w.copy())

    def contact_forces(self):
        f = np.zeros((len(self._centers), 3))
        if self.b is None or self._force_dt is None:
            return f
        nk = self.b.kin == 0
        f[nk] = self.b.M[nk, None] * (self.b.v[nk] - self.vgrav[nk]) / self._force_dt
        return f


def _box_sigs(L, F=ctypes.c_float):
    P = ctypes.c_void_p
    L.or_box_step.argtypes = [P, ctypes.c_int, ctypes.c_int, P, P, F, P, P, P, P, P, P, P, P, P,
                              ctypes.c_double, ctypes.c_int, ctypes.c_double, P, P, P]
    L.or_box_step.restype = ctypes.c_int
    L.or_box_box.argtypes = [P, P, P, P, P, P, ctypes.c_double, P, P, P, P]
    L.or_box_box.restype = ctypes.c_int
    L.or_box_plane.argtypes = [P, P, P, ctypes.c_double, P, P, P]
    L.or_box_plane.restype = ctypes.c_int


def box_plane(half, x, q, margin=2e-3):
    """Oracle box_plane_contacts (ncp_gpu.py:1148-1154): (points (m,3), gaps (m,), feature ids)."""
    L = lib(); _box_sigs(L)
    a = [np.ascontiguousarray(v, np.float64) for v in (half, x, q)]
    po, go, fo = np.zeros(24), np.zeros(8), np.zeros(8, np.int32)
    m = L.or_box_plane(*[_p(v) for v in a], float(margin), _p(po), _p(go), _p(fo))
    return po[:3 * m].reshape(m, 3), go[:m], fo[:m]


def box_box(ha, xa, qa, hb, xb, qb, margin=2e-3):
    """Oracle box_box_contacts (ncp_gpu.py:1157-1227): (points (m,3), normal B->A, gaps, feature ids)."""
    L = lib(); _box_sigs(L)
    a = [np.ascontiguousarray(v, np.float64) for v in (ha, xa, qa, hb, xb, qb)]
    po, no, go, fo = np.zeros(12), np.zeros(3), np.zeros(4), np.zeros(4, np.int32)
    m = L.or_box_box(*[_p(v) for v in a], float(margin), _p(po), _p(no), _p(go), _p(fo))
    return po[:3 * m].reshape(m, 3), no, go[:m], fo[:m]


def scene_local_index(scene):
    """Index of every body among the bodies of its scene, in body order."""
    scene = np.asarray(scene, np.int64)
    out = np.zeros(len(scene), np.int32)
    seen = {}
    for i, s in enumerate(scene.tolist()):
        out[i] = seen.get(s, 0)
        seen[s] = out[i] + 1
    return out


class BoxOracle:
    """CPU restatement of the box engine: box/plane + box/box narrowphase (BoxWorld.contacts,
    ncp_gpu.py:1273-1280) over the pairs whose bounding spheres are within the margin, with the
    ColorCache pair solve of the coloured chain and per-body friction.  flags: 1 fixed frame,
    2 applied warm, 4 colour cache, 8 warm start, 32 first-fit colours, 64 row form."""
    name = "box_color_cache_oracle"

    def __init__(self, dims=(0.3, 0.3, 0.2), mu=0.5, vit=16, pit=10, flags=111, margin=2e-3, cap=MAXC,
                 precision="float32"):
        self.precision = precision
        self.F, self.L = _precision(precision)
        self.dims = dims; self.mu = mu; self.vit = vit; self.pit = pit; self.flags = flags; self.margin = margin
        self.cap = cap
        self._centers, self._halves, self._dens, self._mus, self._kin = [], [], [], [], []
        self._scenes = []
        self.b = None; self._h = None; self._force_dt = None

    def add_box(self, center, dims=None, density=1000.0, mu=None, kin=False, scene=0):
        d = self.dims if dims is None else dims
        self._centers.append(list(center)); self._halves.append([0.5 * d[0], 0.5 * d[1], 0.5 * d[2]])
        self._dens.append(float(density)); self._mus.append(self.mu if mu is None else float(mu))
        self._kin.append(1 if kin else 0)
        self._scenes.append(int(scene))
        self.b = None
        return len(self._centers) - 1

    def _build(self):
        L = self.L
        if not hasattr(L, "_col_ready"):
            _col_sigs(L); L._col_ready = True
        if L is lib():
            _box_sigs(L)
        c = np.array(self._centers, float); h = np.array(self._halves, float); N = len(c)
        M = np.array(self._dens) * 8.0 * h[:, 0] * h[:, 1] * h[:, 2]
        e = 2.0 * h
        Ib = (M / 12.0)[:, None] * np.stack([e[:, 1] ** 2 + e[:, 2] ** 2, e[:, 0] ** 2 + e[:, 2] ** 2,
                                             e[:, 0] ** 2 + e[:, 1] ** 2], axis=1)
        kin = np.array(self._kin, int)
        IbInv = np.array([np.eye(3) if kin[i] else np.linalg.inv(np.diag(Ib[i])) for i in range(N)])
        self.N = N
        self.b = BodySetup(rest=np.zeros((0, 3), np.float32), xc=c.astype(np.float32),
                           q=np.tile(np.array([0, 0, 0, 1.0], np.float32), (N, 1)),
                           v=np.zeros((N, 3), np.float32), w=np.zeros((N, 3), np.float32),
                           invM=np.where(kin == 1, 0.0, 1.0 / M).astype(np.float32),
                           IbInv=IbInv.astype(np.float32), kin=kin.astype(np.int32), M=M)
        self.b = _cast_bodies(self.b, self.F)
        F = self.F
        self.half4 = np.zeros((N, 4), np.float32); self.half4[:, :3] = h
        self.half4 = self.half4.astype(F)
        self.mus = np.array(self._mus, np.float32)
        self.per_body = bool(np.any(self.mus != np.float32(self.mu)))
        self.mus = self.mus.astype(F)
        self.pv = np.zeros((N, 3), F); self.po = np.zeros((N, 3), F)
        self.vgrav = np.zeros((N, 3), F)
        sc = np.array(self._scenes, np.int32)
        self.scene = sc if len(sc) and sc.max() > 0 else None
        self.local = scene_local_index(sc)
        self._h = L.or_col_create(1, self.vit, self.pit, 4, self.mu, 1.0, self.cap, N)

    def step(self, dt, substeps=1):
        if self.b is None:
            self._build()
        b = self.b
        rc = self.L.or_box_step(self._h, self.flags, self.N, _p(self.half4), _p(self.mus) if self.per_body else None,
                               float(self.F(np.float32(self.mu))), _p(b.xc), _p(b.q), _p(b.v), _p(b.w), _p(self.pv),
                               _p(self.po),
                               _p(b.invM), _p(b.IbInv), _p(b.kin), float(dt), int(substeps),
                               float(np.float32(self.margin)), _p(self.vgrav),
                               None if self.scene is None else _p(self.scene), _p(self.local))
        if rc != 0:
            raise RuntimeError(f"oracle box step failed with status {rc}")
        self._force_dt = dt / substeps

    def stats(self):
        out = np.zeros(7, np.int32)
        self.L.or_col_stats(self._h, _p(out))
        return dict(zip(("n_contacts", "n_kept", "n_pairs", "n_colors", "hits", "misses", "seg_overflow"),
                        out.tolist()))

    def kept_contacts(self) -> dict:
        """The last substep's kept contacts (see ColoredOracle.kept_contacts)."""
        return ColoredOracle.kept_contacts(self)

    def warm_store(self) -> dict:
        """The warm-start store (see ColoredOracle.warm_store)."""
        return ColoredOracle.warm_store(self)

    def set_warm_store(self, d: dict) -> None:
        ColoredOracle.set_warm_store(self, d)

    def set_body_state(self, xc, q, v, w):
        """Overwrite positions, quaternions (x, y, z, w) and velocities (the warm-start store is kept)."""
        if self.b is None:
            self._build()
        for dst, src in ((self.b.xc, xc), (self.b.q, q), (self.b.v, v), (self.b.w, w)):
            dst[...] = np.asarray(src, self.F).reshape(dst.shape)

    def body_state(self):
        """(xc, q, v, w) float32 copies."""
        if self.b is None:
            self._build()
        return self.b.xc.copy(), self.b.q.copy(), self.b.v.copy(), self.b.w.copy()

    def get_state(self) -> State:
        if self.b is None:
            self._build()
        return State(xc=self.b.xc.copy(), Rm=quat_to_R(self.b.q), vc=self.b.v.copy(), om=self.b.w.copy())

    def contact_forces(self):
        f = np.zeros((len(self._centers), 3))
        if self.b is None or self._force_dt is None:
            return f
        nk = self.b.kin == 0
        f[nk] = self.b.M[nk, None] * (self.b.v[nk] - self.vgrav[nk]) / self._force_dt
        return f


# ---- exact-cone NCP (oracle_ncp.c) ----
def _ncp_sigs(L):
    P = ctypes.c_void_p
    for suf in ("_f", "_d"):
        f = getattr(L, "or_ncp_solve" + suf)
        f.argtypes = [ctypes.c_int, ctypes.c_int] + [P] * 11 + [ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                               ctypes.c_int, P, P, P, P, P]
        f.restype = ctypes.c_double


def ncp_solve(bs, iters, dtype="float64", warm=None, desaxce=True, softp=None, use_bias=True):
    """The oracle's coloured PGS on a block scene (any object with Ja, Jb, Minv, v_free, mu,
    body_pairs, bias, feature, sep).  Returns dict(lam (n_c,3), v (n_b,6), res (n_c), residual,
    col (n_c), n_colors); arrays in the solve's dtype."""
    L = lib()
    _ncp_sigs(L)
    nt = np.float32 if dtype == "float32" else np.float64
    fn = L.or_ncp_solve_f if dtype == "float32" else L.or_ncp_solve_d
    Ja = np.ascontiguousarray(bs.Ja, nt)
    n_c, n_b = Ja.shape[0], np.shape(bs.Minv)[0]
    Jb = np.ascontiguousarray(bs.Jb, nt)
    Minv = np.ascontiguousarray(bs.Minv, nt)
    vf = np.ascontiguousarray(bs.v_free, nt)
    mu = np.ascontiguousarray(bs.mu, nt)
    pairs = np.ascontiguousarray(bs.body_pairs, np.int32).reshape(n_c, 2)
    pa, pb = np.ascontiguousarray(pairs[:, 0]), np.ascontiguousarray(pairs[:, 1])
    feat = np.ascontiguousarray(bs.feature, np.int32)
    bias = np.ascontiguousarray(bs.bias, nt)
    sep = None if getattr(bs, "sep", None) is None else np.ascontiguousarray(bs.sep, nt)
    sp = None if softp is None else np.ascontiguousarray(softp, nt)
    lam = np.zeros((n_c, 3), nt) if warm is None else np.array(warm, nt).reshape(n_c, 3)
    v = np.zeros((n_b, 6), nt)
    res = np.zeros(n_c, nt)
    col = np.zeros(n_c, np.int32)
    ncol = np.zeros(1, np.int32)
    r = fn(n_c, n_b, _p(Ja), _p(Jb), _p(Minv), _p(vf), _p(mu), _p(pa), _p(pb), _p(feat), _p(bias),
           None if sep is None else _p(sep), None if sp is None else _p(sp), 1 if use_bias else 0,
           1 if desaxce else 0, int(iters), 0 if warm is None else 1, _p(lam), _p(v), _p(res), _p(col), _p(ncol))
    return dict(lam=lam, v=v, res=res, residual=float(r), col=col, n_colors=int(ncol[0]))
