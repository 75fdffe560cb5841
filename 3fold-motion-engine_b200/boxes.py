"""Box engine: box/plane + box/box narrowphase contacts solved by the coloured pair-chunk solve.

The reference's box contact model is BoxWorld (src/motion_engine/ncp/ncp_gpu.py:1237-1405):
solid boxes with per-body half extents, vertex-plane contacts against z = 0 and SAT box-box
manifolds (<= 4 points per pair), generated on the host.  Here the same narrowphase (float64)
runs on the device for every candidate pair of a body-AABB broadphase, and the contacts feed the
coloured Gauss-Seidel pair solve of the ColorCache chain (fixed tangent frame, warm impulses
applied once per colour, colouring cached while the pair graph and masses are unchanged).
Per-body sizes and per-body friction (sqrt(mu_a mu_b) per pair, mu_a against the ground) are
the superset the 10 000-random-box workload needs; with one size and a scalar mu it is the
plain setting.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .colored import NCOLMAX
from .engine import _BeadEngineBase, _pad4, _ptr

MARGIN = 2e-3


def scene_local_index(scene):
    """Index of every body among the bodies of its scene, in body order."""
    scene = np.asarray(scene, np.int64)
    out = np.zeros(len(scene), np.int32)
    if len(scene):
        order = np.argsort(scene, kind="stable")
        ss = scene[order]
        first = np.r_[0, np.flatnonzero(np.diff(ss)) + 1]
        run_start = np.repeat(first, np.diff(np.r_[first, len(ss)]))
        out[order] = (np.arange(len(ss)) - run_start).astype(np.int32)
    return out


def box_body_arrays(centers, halves, dens, kin):
    """Solid boxes (Box.Ib, ncp_gpu.py:1105-1109): mass = density * 8 hx hy hz,
    Ib = m/12 diag(h_y^2 + h_z^2, ...) with full edges h = 2 half; float64, cast to float32."""
    c = np.array(centers, float).reshape(-1, 3)
    h = np.array(halves, float).reshape(-1, 3)
    N = len(c)
    M = np.array(dens, float) * 8.0 * h[:, 0] * h[:, 1] * h[:, 2]
    kinarr = np.array(kin, int)
    e = 2.0 * h
    Ib = (M / 12.0)[:, None] * np.stack([e[:, 1] ** 2 + e[:, 2] ** 2, e[:, 0] ** 2 + e[:, 2] ** 2,
                                         e[:, 0] ** 2 + e[:, 1] ** 2], axis=1)
    IbInv = np.zeros((N, 3, 3))
    for i in range(N):
        IbInv[i] = np.eye(3) if kinarr[i] else np.linalg.inv(np.diag(Ib[i]))
    if not np.all(np.isfinite(IbInv)) or np.any(M <= 0):
        raise ValueError("box engine: degenerate box mass / inertia")
    invM = np.where(kinarr == 1, 0.0, 1.0 / M)
    return dict(xc=c.astype(np.float32), half=h.astype(np.float32), M=M, invM=invM.astype(np.float32),
                IbInv=IbInv.astype(np.float32), kin=kinarr.astype(np.int32))


class BoxContactEngine(_BeadEngineBase):
    """ContactEngine over solid boxes (box/plane + box/box contacts) with the ColorCache solve."""
    name = "box_color_cache_b200"

    def __init__(self, dims=(0.3, 0.3, 0.2), mu=0.5, vit=16, pit=10, fixed_frame=True, apply_warm=True,
                 color_cache=True, warm_start=True, margin=MARGIN, device="cuda", color_cap=NCOLMAX,
                 solve_blocks=0, barrier_timeout_s=1.0, cand_per_body=16, first_fit=True, row_form=True,
                 islands=False):
        super().__init__(dims=dims, mu=mu, device=device, graph=True)
        # the island solve (B2C_COLOR_ISLANDS): one thread per island when no island has more than
        # 64 pairs, else the colour phases; the same bits either way
        self.islands = bool(islands)
        self.vit, self.pit = int(vit), int(pit)
        self.fixed_frame, self.apply_warm = bool(fixed_frame), bool(apply_warm)
        self.color_cache, self.warm_start = bool(color_cache), bool(warm_start)
        self.margin = float(margin)
        self.color_cap = int(color_cap)
        self.solve_blocks = int(solve_blocks)
        self.barrier_timeout_ns = int(barrier_timeout_s * 1e9)
        self.cand_per_body = int(cand_per_body)
        self.first_fit = bool(first_fit)
        self.row_form = bool(row_form) and self.fixed_frame
        self._halves, self._mus, self._scenes = [], [], []
        self._has_manifold = True

    def add_body(self, center, density=700.0, kin=False):
        return self.add_box(center, dims=self.dims, density=density, kin=kin)

    def add_box(self, center, dims=None, density=1000.0, mu=None, kin=False, scene=0):
        """Add a solid box.  `scene` groups bodies into independent scenes (a batch): bodies of
        different scenes never touch, whatever their positions."""
        d = self.dims if dims is None else tuple(float(x) for x in dims)
        self._halves.append([0.5 * d[0], 0.5 * d[1], 0.5 * d[2]])
        self._mus.append(self.mu if mu is None else float(mu))
        self._scenes.append(int(scene))
        return super().add_body(center, density=density, kin=kin)

    def _build(self):
        A = box_body_arrays(self._centers, self._halves, self._dens, self._kin)
        N = len(self._centers)
        self.N = N
        self._M = A["M"]
        self._kinarr = A["kin"].astype(int)
        dev = self.dev
        f32 = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(dev)
        i32 = lambda n: torch.zeros(max(int(n), 1), dtype=torch.int32, device=dev)
        # positions, quaternions, velocities, angular velocities: four planes of one tensor
        self.state = torch.zeros((4, N, 4), dtype=torch.float32, device=dev)
        self.xc, self.q, self.v, self.w = self.state[0], self.state[1], self.state[2], self.state[3]
        self.xc.copy_(f32(_pad4(A["xc"])))
        self.q.copy_(f32(np.tile(np.array([0, 0, 0, 1.0], np.float32), (N, 1))))
        z4 = lambda: torch.zeros((N, 4), dtype=torch.float32, device=dev)
        self.pv, self.po, self.vgrav = z4(), z4(), z4()
        self.invM = f32(A["invM"])
        Ib12 = np.zeros((N, 3, 4), np.float32)
        Ib12[:, :, :3] = A["IbInv"]
        self.IbInv = f32(Ib12.reshape(N, 12))
        self.kin = torch.from_numpy(A["kin"]).to(dev)
        self.invIw = torch.zeros((N, 12), dtype=torch.float32, device=dev)
        self.half = f32(_pad4(A["half"]))
        mus = np.array(self._mus, np.float32)
        self.per_body_mu = bool(np.any(mus != np.float32(self.mu)))
        self.body_mu = f32(mus)
        self.header = torch.zeros(8, dtype=torch.int32, device=dev)
        self._hdr_host = torch.zeros(8, dtype=torch.int32, pin_memory=True)
        # broadphase grid over body centres
        hmax = float(np.max(np.linalg.norm(A["half"], axis=1))) if N else 0.5
        cell = 1.01 * (2.0 * hmax + self.margin)  # every sphere-test pair lies in adjacent cells
        dims = (16, 16, 8) if N <= 2000 else (32, 32, 16) if N <= 20000 else (64, 64, 32) if N <= 500000 \
            else (128, 128, 64)
        # scenes of a batch: the scene of every body, and its index among its scene's bodies (the
        # colouring priority uses scene-local indices, so a scene colours alike alone or batched)
        sc = np.array(self._scenes, np.int32)
        self.n_scenes = int(sc.max()) + 1 if N else 0
        self.scene_t = torch.from_numpy(sc).to(dev) if self.n_scenes > 1 else None
        self.local_t = torch.from_numpy(scene_local_index(sc)).to(dev)
        nbk = dims[0] * dims[1] * dims[2]
        cand_cap = max(self.cand_per_body * N + N, 64)
        kept_cap = 4 * cand_cap + 8 * N
        self.bx_bufs = dict(bucket=i32(N), start=i32(nbk + 1), cursor=i32(nbk + 1), sorted=i32(N), cand_count=i32(N + 1),
                            cand_offset=i32(N + 1), cand_a=i32(cand_cap), cand_b=i32(cand_cap),
                            cont_count=i32(cand_cap + 1), cont_offset=i32(cand_cap + 1), pair_flag=i32(cand_cap + 1),
                            pair_offset=i32(cand_cap + 1),
                            slot_p=torch.zeros((cand_cap * 8, 4), dtype=torch.float32, device=dev),
                            slot_n=torch.zeros((cand_cap, 4), dtype=torch.float32, device=dev),
                            slot_f=i32(cand_cap * 8),
                            scan_tmp=i32(self.L.b2c_scan_scratch_ints(max(nbk, N, cand_cap) + 1)))
        b = self.bx_bufs
        self.c_boxes = _lib.Boxes(N, _ptr(self.half), _ptr(self.body_mu), self.margin, cell, dims[0], dims[1], dims[2],
                                  cand_cap, *(_ptr(b[k]) for k in (
                                      "bucket", "start", "cursor", "sorted", "cand_count", "cand_offset", "cand_a",
                                      "cand_b", "cont_count", "cont_offset", "pair_flag", "pair_offset", "slot_p",
                                      "slot_n", "slot_f", "scan_tmp")),
                                  _ptr(self.scene_t) if self.scene_t is not None else None)
        # kept contacts, pairs, colouring, records, warm store
        i64 = lambda n: torch.zeros(max(int(n), 1), dtype=torch.int64, device=dev)
        f4 = lambda n: torch.zeros((max(int(n), 1), 4), dtype=torch.float32, device=dev)
        self.k_bi, self.k_bj, self.k_fa, self.k_fb = i32(kept_cap), i32(kept_cap), i32(kept_cap), i32(kept_cap)
        self.k_pA, self.k_pB, self.k_n, self.k_imp = f4(kept_cap), f4(kept_cap), f4(kept_cap), f4(kept_cap)
        self.k_keys = i64(kept_cap)
        self.c_kept = _lib.Contacts(kept_cap, _ptr(self.k_bi), _ptr(self.k_bj), _ptr(self.k_pA), _ptr(self.k_pB),
                                    _ptr(self.k_n), _ptr(self.k_fa), _ptr(self.k_fb), _ptr(self.k_imp))
        pcap, kslots = cand_cap, 8
        self.p_bufs = dict(pbi=i32(pcap), pbj=i32(pcap), kcount=i32(pcap + 1), pstart=i32(pcap + 1), pidx=i32(kept_cap),
                           col=i32(pcap), porder=i32(pcap), cstart=i32(NCOLMAX), ccount=i32(NCOLMAX), claim=i64(2 * N),
                           cached_a=i32(pcap), cached_b=i32(pcap),
                           cached_mass=torch.zeros(max(N, 1), dtype=torch.float32, device=dev), cache_state=i32(8),
                           body_colors=i64(N), body_slots=i32(64 * N),
                           barrier=torch.zeros(int(self.L.b2c_barrier_words()), dtype=torch.int32, device=dev),
                           rec=torch.zeros(max(int(self.L.b2c_pair_record_floats(pcap, kslots)), 1),
                                           dtype=torch.float32, device=dev))
        pb = self.p_bufs
        self.c_pairs = _lib.Pairs(pcap, NCOLMAX, *(_ptr(pb[k]) for k in (
            "pbi", "pbj", "kcount", "pstart", "pidx", "col", "porder", "cstart", "ccount", "claim", "cached_a",
            "cached_b", "cached_mass", "cache_state", "barrier", "rec")), kslots, _ptr(pb["body_colors"]),
            _ptr(self.local_t), _ptr(pb["body_slots"]))
        # the scene schedule of the solve (one CTA per scene): possible when each scene's bodies
        # are contiguous and the scenes in body order, as a batch adds them
        self.scene_schedule = self.n_scenes > 1 and bool(np.all(np.diff(sc) >= 0))
        if self.scene_schedule:
            counts = np.bincount(sc, minlength=self.n_scenes)
            self.s_bufs = dict(start=torch.from_numpy(np.r_[0, np.cumsum(counts)].astype(np.int32)).to(dev),
                               order=torch.from_numpy(np.argsort(-counts, kind="stable").astype(np.int32)).to(dev),
                               pair_slot=i32(pcap), scene_slots=i32(pcap))
            sb = self.s_bufs
            self.c_pairs.n_scenes = self.n_scenes
            self.c_pairs.scene_body_start, self.c_pairs.scene_order = _ptr(sb["start"]), _ptr(sb["order"])
            self.c_pairs.pair_slot, self.c_pairs.scene_slots = _ptr(sb["pair_slot"]), _ptr(sb["scene_slots"])
        if self.islands:
            pb["isl_work"] = i32(self.L.b2c_island_work_ints(N, pcap))
            self.c_pairs.isl_work = _ptr(pb["isl_work"])
        self.w_keys, self.w_imp, self.w_n = i64(kept_cap), f4(kept_cap), i32(1)
        self.c_warm = _lib.Warm(kept_cap, _ptr(self.w_keys), _ptr(self.w_imp), _ptr(self.w_n))
        self.c_bodies = _lib.Bodies(N, _ptr(self.xc), _ptr(self.q), _ptr(self.v), _ptr(self.w), _ptr(self.pv),
                                    _ptr(self.po), _ptr(self.invM), _ptr(self.IbInv), _ptr(self.kin), _ptr(self.invIw))
        flags = ((_lib.COLOR_FIXED_FRAME if self.fixed_frame else 0) | (_lib.COLOR_APPLY_WARM if self.apply_warm else 0)
                 | (_lib.COLOR_CACHE if self.color_cache else 0) | (_lib.COLOR_WARM_START if self.warm_start else 0)
                 | (_lib.COLOR_FIRST_FIT if self.first_fit else 0) | (_lib.COLOR_ROW_FORM if self.row_form else 0)
                 | (_lib.COLOR_ISLANDS if self.islands else 0))
        self.c_params = _lib.ColorParams(self.vit, self.pit, 8, flags, self.mu, 1.0, min(self.color_cap, NCOLMAX),
                                         self.solve_blocks, self.barrier_timeout_ns,
                                         _ptr(self.body_mu) if self.per_body_mu else None)
        self._graphs = {}
        self._built = True

    def _launch_step(self, sdt, substeps):
        s = torch.cuda.current_stream(self.dev).cuda_stream
        for _ in range(substeps):
            rc = self.L.b2c_box_substep(ctypes.byref(self.c_bodies), ctypes.byref(self.c_boxes),
                                        ctypes.byref(self.c_kept), ctypes.c_void_p(_ptr(self.k_keys)),
                                        ctypes.byref(self.c_pairs), ctypes.byref(self.c_warm),
                                        ctypes.c_void_p(_ptr(self.header)), ctypes.byref(self.c_params),
                                        ctypes.c_float(sdt), ctypes.c_void_p(_ptr(self.vgrav)), ctypes.c_void_p(s))
            _lib.check(rc, "b2c_box_substep")

    def step(self, dt, substeps=1):
        if not self._built:
            self._build()
        self.check_errors()
        sdt = dt / substeps
        self._graph_step(("box", float(sdt), int(substeps)), lambda: self._launch_step(sdt, substeps))
        self._force_dt = sdt
        self._fetch_header()

    def set_solve_blocks(self, n: int):
        """Launch form of the persistent solve: 0 auto, 1 one CTA, n > 1 a cooperative grid of n
        CTAs, -n a cluster of n CTAs, _lib.SOLVE_SCENES one CTA per scene (a batch in the row
        form).  Results do not depend on it.  Drops captured graphs."""
        if int(n) == _lib.SOLVE_SCENES and self._built and not (self.scene_schedule and self.row_form):
            raise ValueError(f"{self.name}: the scene schedule needs several scenes in body order and the row form")
        self.solve_blocks = int(n)
        if self._built:
            self.c_params.solve_blocks = self.solve_blocks
            self._graphs = {}

    def set_kinematic(self, i, xc):
        super().set_kinematic(i, xc)

    @property
    def island_count(self):
        """Islands of the last partition (islands=True)."""
        return int(self.p_bufs["isl_work"][0].item()) if self._built and self.islands else 0

    @property
    def max_island_pairs(self):
        """Pairs of the largest island of the last partition (islands=True)."""
        return int(self.p_bufs["isl_work"][1].item()) if self._built and self.islands else 0

    @property
    def island_solve_active(self):
        return self.islands and self._built and self.max_island_pairs <= _lib.ISLAND_MAX_PAIRS

    @property
    def color_cache_hits(self):
        return int(self.p_bufs["cache_state"][3].item()) if self._built else 0

    @property
    def color_cache_misses(self):
        return int(self.p_bufs["cache_state"][4].item()) if self._built else 0

    # staged substep with CUDA events (profiling); same launches as b2c_box_substep
    STAGES = ("predict", "candidates", "narrowphase", "colour", "solve", "warm_store", "integrate")

    def profile_substep(self, dt):
        if not self._built:
            self._build()
        self.check_errors()
        L, b = self.L, ctypes.byref
        stream = torch.cuda.current_stream(self.dev)
        s = ctypes.c_void_p(stream.cuda_stream)
        hdr = ctypes.c_void_p(_ptr(self.header))
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(len(self.STAGES) + 1)]
        sdt = ctypes.c_float(dt)
        ev[0].record(stream)
        _lib.check(L.b2c_body_predict(b(self.c_bodies), sdt, s), "predict")
        self.vgrav.copy_(self.v)
        self.pv.zero_()
        self.po.zero_()
        ev[1].record(stream)
        _lib.check(L.b2c_box_candidates(b(self.c_bodies), b(self.c_boxes), hdr, s), "candidates")
        ev[2].record(stream)
        _lib.check(L.b2c_box_contacts(b(self.c_bodies), b(self.c_boxes), b(self.c_kept),
                                      ctypes.c_void_p(_ptr(self.k_keys)), b(self.c_pairs), b(self.c_warm), hdr,
                                      b(self.c_params), s), "narrowphase")
        ev[3].record(stream)
        _lib.check(L.b2c_color_pairs(b(self.c_bodies), b(self.c_pairs), hdr, b(self.c_params), s), "colour")
        ev[4].record(stream)
        _lib.check(L.b2c_color_solve(b(self.c_bodies), b(self.c_kept), b(self.c_pairs), hdr, b(self.c_params), sdt, s),
                   "solve")
        ev[5].record(stream)
        _lib.check(L.b2c_warm_store(b(self.c_kept), ctypes.c_void_p(_ptr(self.k_keys)), b(self.c_warm), hdr, s),
                   "warm_store")
        ev[6].record(stream)
        _lib.check(L.b2c_body_integrate(b(self.c_bodies), sdt, s), "integrate")
        ev[7].record(stream)
        self._force_dt = dt
        self._fetch_header()
        ev[7].synchronize()
        return {name: ev[i].elapsed_time(ev[i + 1]) for i, name in enumerate(self.STAGES)}

    def solve_bytes(self) -> dict:
        """Algorithmic bytes of one persistent-solve launch (see GraphColoredContactEngine.solve_bytes)."""
        h = self.header_dict()
        P, Ck = h["n_pairs"], h["n_kept"]
        pbi = self.p_bufs["pbi"][:P].cpu().numpy()
        pbj = self.p_bufs["pbj"][:P].cpu().numpy()
        invM = self.invM.cpu().numpy()
        E = int(np.sum(invM[pbi] > 0) + np.sum((pbj >= 0) & (invM[np.maximum(pbj, 0)] > 0)))
        per_vel = 20 * P + 100 * E + 64 * Ck
        per_pos = 20 * P + 100 * E + 52 * Ck
        # the row form applies the warm start in k_warm_gather_row, outside the solve launch
        warm = per_pos if (self.apply_warm and not self.row_form) else 0
        return dict(pairs=P, kept=Ck, endpoints=E, colors=h["n_colors"],
                    bytes=warm + self.vit * per_vel + self.pit * per_pos)


class BatchedBoxEngine(BoxContactEngine):
    """Many independent box scenes advanced together: one body array, scene ids that keep the
    scenes apart in the broadphase, and every stage of a substep -- the broadphase, the
    narrowphase, the colouring and the persistent solve -- launched once for all scenes.  Each
    scene's slice of the result is bytewise the scene advanced alone (its colouring uses
    scene-local priorities; nothing else couples scenes).  The scenes may overlap in space."""
    name = "box_color_cache_batched_b200"

    def __init__(self, scenes=(), **kw):
        kw.setdefault("cand_per_body", 12)
        super().__init__(**kw)
        self.scene_start = [0]
        for sc in scenes:
            self.add_scene(sc)

    def add_scene(self, sc) -> int:
        """sc: dict(centers, dims, density, mu[, kin]).  Returns the scene index."""
        s = len(self.scene_start) - 1
        kin = sc.get("kin", np.zeros(len(sc["centers"]), bool))
        for c, d, de, m, k in zip(sc["centers"], sc["dims"], sc["density"], sc["mu"], kin):
            self.add_box(c, dims=d, density=de, mu=m, kin=bool(k), scene=s)
        self.scene_start.append(len(self._centers))
        return s

    def scene_slice(self, s) -> slice:
        return slice(self.scene_start[s], self.scene_start[s + 1])

    def scene_state(self, s):
        st = self.get_state()
        sl = self.scene_slice(s)
        return type(st)(xc=st.xc[sl], Rm=st.Rm[sl], vc=st.vc[sl], om=st.om[sl])


_TUNED = {}


def autotune(engine, dt, substeps=1, candidates=(-16, -8, 148, 74), steps=2):
    """Pick the persistent solve's launch form (a cluster of 16 or 8 CTAs, a cooperative grid
    of 148 or 74 CTAs, and for a batch also one CTA per scene) by timing `steps` live steps of
    each.  The launch forms give bit-identical results (the tests check it), so tuning on live
    steps does not change the trajectory.  The choice is cached per (bodies, scenes, colours)
    and applied to the engine."""
    import torch
    h = engine.header_dict() if engine._built else {"n_colors": 0}
    key = (engine.N if engine._built else len(engine._centers), getattr(engine, "n_scenes", 1), h["n_colors"])
    if key in _TUNED:
        engine.set_solve_blocks(_TUNED[key][0])
        return _TUNED[key]
    times = {}
    candidates = list(candidates)
    if getattr(engine, "scene_schedule", False) and engine.row_form and _lib.SOLVE_SCENES not in candidates:
        candidates.append(_lib.SOLVE_SCENES)
    for cand in candidates:
        engine.set_solve_blocks(cand)
        engine.step(dt, substeps)  # capture / first run of this form
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(steps):
            engine.step(dt, substeps)
        b.record()
        b.synchronize()
        times[cand] = a.elapsed_time(b) / steps
        engine.check_errors()
    best = min(times, key=times.get)
    engine.set_solve_blocks(best)
    _TUNED[key] = (best, times)
    return _TUNED[key]


def partition_scenes(counts, parts):
    """Longest-processing-time assignment of scenes (by body count) to `parts` workers (GPUs or
    processes): scenes in decreasing size, each to the currently lightest worker; ties by index.
    Returns one ascending index list per worker.  Scenes are independent, so a shard needs no
    data exchange with the others."""
    load = [0] * parts
    out = [[] for _ in range(parts)]
    for i in sorted(range(len(counts)), key=lambda i: (-counts[i], i)):
        k = min(range(parts), key=lambda k: (load[k], k))
        out[k].append(i)
        load[k] += counts[i]
    return [sorted(x) for x in out]
