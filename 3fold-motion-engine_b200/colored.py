"""Coloured Gauss-Seidel engines on the b2c CUDA library.

Mirrors of the reference's coloured engine family behind the ContactEngine protocol:

* GraphColoredContactEngine  -- contact_engine_gpu_colored.py:793-1410.  Solve paths: the plain
  per-contact colouring (manifold_reduce=False), the reduced set coloured contact by contact
  (manifold_reduce=True, pair_chunks=False: the device manifold's priority, COL:776-787, 1105-1113)
  and the pair-chunk path (manifold_reduce=True, pair_chunks=True).  chunk_mode 'registers' and
  'global' give the same
  states in the reference and are one kernel here; manifold_on_host selects the same points as
  the device path, so it runs the device path.
* FixedFrameContactEngine    -- contact_engine_gpu_fixed_frame.py:82-88 (normal-derived frame).
* AppliedWarmContactEngine   -- contact_engine_gpu_applied_warm.py:57-75 (warm impulses applied
  once per colour before the sweeps).
* DeferredForceContactEngine -- contact_engine_gpu_deferred_force.py:7-74.
* ColorCacheContactEngine    -- contact_engine_gpu_color_cache.py:21-54 (colouring reused while
  the pair graph and the masses are unchanged).
* IslandSolveContactEngine   -- contact_engine_gpu_island_solve.py:253-287 (the pair graph split
  into islands of dynamic bodies; one thread per island runs its sweeps when no island has more
  than 64 pairs).

A whole step (every substep: prediction, bead grid, contacts in feature order, manifold
reduction, pairs, colouring, the persistent chunk solve, warm store, integration) is one fixed
sequence of launches with no host read-back, captured once into a CUDA graph.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .engine import MAXC, _BeadEngineBase, _ptr

NCOLMAX = 512  # capacity of the per-colour arrays (contact_engine_gpu_colored.py:564)


class GraphColoredContactEngine(_BeadEngineBase):
    """Graph-coloured Gauss-Seidel on bead bodies (atomics-free solve, plain writes within a colour)."""
    name = "graph_colored_b200"
    _fixed_frame = False
    _apply_warm = False
    _color_cache = False
    _islands = False

    def __init__(self, dims=(0.3, 0.3, 0.2), vit=None, pit=20, mu=0.5, warm_start=True, t2_damp=1.0,
                 manifold_reduce=False, manifold_max_points=4, manifold_on_host=False, profile=False,
                 graph_capture=False, graph_mode="device", pair_chunks=False, chunk_mode="registers",
                 device="cuda", contact_capacity=MAXC, color_cap=NCOLMAX, solve_blocks=0,
                 barrier_timeout_s=1.0, **kw):
        if graph_mode not in ("device", "spans"):
            raise ValueError("contact_engine_gpu_colored: graph_mode is 'device' or 'spans'")
        if pair_chunks:
            if chunk_mode not in ("registers", "global"):
                raise ValueError("contact_engine_gpu_colored: chunk_mode is 'registers' or 'global'")
            if not (manifold_reduce and not manifold_on_host):
                raise ValueError("contact_engine_gpu_colored: pair_chunks=True needs the device manifold "
                                 "reduction (manifold_reduce=True, manifold_on_host=False): a chunk is the "
                                 "<= manifold_max_points contacts of one body pair")
        if not 1 <= int(manifold_max_points) <= 8:
            raise ValueError("manifold_max_points must be in 1..8")
        super().__init__(dims=dims, mu=mu, device=device, graph=True)
        self.vit = (40 if manifold_reduce else 20) if vit is None else int(vit)
        self.pit = int(pit)
        self.warm_start = bool(warm_start)
        self.t2_damp = float(t2_damp)
        self.manifold_reduce = bool(manifold_reduce)
        self.manifold_max_points = int(manifold_max_points)
        self.manifold_on_host = bool(manifold_on_host)
        self.pair_chunks = bool(pair_chunks)
        self.chunk_mode = chunk_mode
        self.graph_capture = bool(graph_capture)
        self.graph_mode = graph_mode
        self.profile = bool(profile)
        self.prof_ms = {}
        self.contact_capacity = int(contact_capacity)
        self.color_cap = int(color_cap)
        self.solve_blocks = int(solve_blocks)
        self.barrier_timeout_ns = int(barrier_timeout_s * 1e9)
        self._has_manifold = True

    # ---- construction ----
    def _flags(self) -> int:
        f = 0
        if self._fixed_frame:
            f |= _lib.COLOR_FIXED_FRAME
        if self._apply_warm:
            f |= _lib.COLOR_APPLY_WARM
        if self._color_cache:
            f |= _lib.COLOR_CACHE
        if self._islands:
            f |= _lib.COLOR_ISLANDS
        if self.warm_start:
            f |= _lib.COLOR_WARM_START
        if not self.manifold_reduce:
            f |= _lib.COLOR_PER_CONTACT
        elif not self.pair_chunks:
            f |= _lib.COLOR_REDUCED_CONTACTS
        return f

    def _build(self):
        self._setup_bodies()
        self._setup_grid()
        cap = self.contact_capacity
        self._setup_contacts(cap)
        dev = self.dev
        N, NB = self.N, self.NB
        i32 = lambda n: torch.zeros(max(int(n), 1), dtype=torch.int32, device=dev)
        f32 = lambda n: torch.zeros(max(int(n), 1), dtype=torch.float32, device=dev)
        f64 = lambda n: torch.zeros(max(int(n), 1), dtype=torch.float64, device=dev)
        i64 = lambda n: torch.zeros(max(int(n), 1), dtype=torch.int64, device=dev)
        # body pairs: with the manifold reduction a pair keeps <= max_points contacts and the pair
        # graph of boxes is sparse (a few partners per body); the plain engine colours contacts
        chunks = self.manifold_reduce and self.pair_chunks
        pcap = min(cap, 8 * N + 4096) if chunks else cap
        kslots = self.manifold_max_points if chunks else 1
        # kept contacts (feature order) and their keys
        self.k_bi, self.k_bj, self.k_fa, self.k_fb = i32(cap), i32(cap), i32(cap), i32(cap)
        self.k_pA, self.k_pB, self.k_n, self.k_imp = (torch.zeros((cap, 4), dtype=torch.float32, device=dev)
                                                      for _ in range(4))
        self.k_keys = i64(cap)
        self.c_kept = _lib.Contacts(cap, _ptr(self.k_bi), _ptr(self.k_bj), _ptr(self.k_pA), _ptr(self.k_pB),
                                    _ptr(self.k_n), _ptr(self.k_fa), _ptr(self.k_fb), _ptr(self.k_imp))
        # manifold scratch
        scan_n = max(NB + 1, cap + 1, pcap + 1, N + 1)
        self.m_bufs = dict(bead_count=i32(NB + 1), bead_offset=i32(NB + 1), pair_local=i32(cap),
                           pair_first=i32(2 * cap), gorder=i32(cap), body_npairs=i32(N + 1), pair_base=i32(N + 1),
                           praw_start=i32(pcap), praw_count=i32(pcap), jn_in=f64(cap), jn_red=f64(cap),
                           jt_in=f32(2 * cap), keep=i32(cap + 1), kidx=i32(cap + 1),
                           scan_tmp=i32(self.L.b2c_scan_scratch_ints(scan_n)))
        mb = self.m_bufs
        self.c_manifold = _lib.Manifold(cap, pcap, *(_ptr(mb[k]) for k in (
            "bead_count", "bead_offset", "pair_local", "pair_first", "gorder", "body_npairs", "pair_base",
            "praw_start", "praw_count", "jn_in", "jn_red", "jt_in", "keep", "kidx", "scan_tmp")))
        # pairs, colouring, colour cache, barrier
        self.p_bufs = dict(pbi=i32(pcap), pbj=i32(pcap), kcount=i32(pcap + 1), pstart=i32(pcap + 1), pidx=i32(cap),
                           col=i32(pcap), porder=i32(pcap), cstart=i32(NCOLMAX), ccount=i32(NCOLMAX), claim=i64(2 * N),
                           cached_a=i32(pcap), cached_b=i32(pcap), cached_mass=f32(N), cache_state=i32(8),
                           barrier=torch.zeros(int(self.L.b2c_barrier_words()), dtype=torch.int32, device=dev),
                           rec=f32(self.L.b2c_pair_record_floats(pcap, kslots)), prio_hi=i32(pcap))
        pb = self.p_bufs
        self.c_pairs = _lib.Pairs(pcap, NCOLMAX, *(_ptr(pb[k]) for k in (
            "pbi", "pbj", "kcount", "pstart", "pidx", "col", "porder", "cstart", "ccount", "claim", "cached_a",
            "cached_b", "cached_mass", "cache_state", "barrier", "rec")), kslots)
        if self.manifold_reduce and not self.pair_chunks:
            self.c_pairs.prio_hi = _ptr(pb["prio_hi"])
        if self._islands:
            pb["isl_work"] = i32(self.L.b2c_island_work_ints(N, pcap))
            self.c_pairs.isl_work = _ptr(pb["isl_work"])
        # warm store
        self.w_keys, self.w_imp, self.w_n = i64(cap), torch.zeros((cap, 4), dtype=torch.float32, device=dev), i32(1)
        self.c_warm = _lib.Warm(cap, _ptr(self.w_keys), _ptr(self.w_imp), _ptr(self.w_n))
        self._struct_bodies()
        self.c_params = _lib.ColorParams(self.vit, self.pit, self.manifold_max_points, self._flags(), self.mu,
                                         self.t2_damp, min(self.color_cap, NCOLMAX), self.solve_blocks,
                                         self.barrier_timeout_ns)
        self._graphs = {}
        self._built = True

    def set_kinematic(self, i, xc):
        super().set_kinematic(i, xc)

    # ---- advance ----
    def _launch_step(self, sdt: float, substeps: int):
        s = torch.cuda.current_stream(self.dev).cuda_stream
        for _ in range(substeps):
            rc = self.L.b2c_color_substep(
                ctypes.byref(self.c_bodies), ctypes.byref(self.c_beads), ctypes.byref(self.c_grid),
                ctypes.byref(self.c_contacts), ctypes.byref(self.c_manifold), ctypes.byref(self.c_kept),
                ctypes.c_void_p(_ptr(self.k_keys)), ctypes.byref(self.c_pairs), ctypes.byref(self.c_warm),
                ctypes.c_void_p(_ptr(self.header)), ctypes.byref(self.c_params), ctypes.c_float(sdt),
                ctypes.c_void_p(_ptr(self.vgrav)), ctypes.c_void_p(s))
            _lib.check(rc, "b2c_color_substep")

    def step(self, dt, substeps=1):
        if not self._built:
            self._build()
        self.check_errors()
        sdt = dt / substeps
        self._graph_step(("colored", float(sdt), int(substeps)), lambda: self._launch_step(sdt, substeps))
        self._force_dt = sdt
        self._fetch_header()

    # ---- staged substep with CUDA events between the stages (profiling; same launches as
    #      b2c_color_substep, so it advances the state exactly like step(dt, 1)) ----
    STAGES = ("predict", "beads", "grid", "contacts", "manifold", "colour", "solve", "warm_store", "integrate")

    def profile_substep(self, dt):
        """One substep launched stage by stage with CUDA events on the launching stream; returns
        {stage: ms} once the substep has finished (the reference's _stage profile,
        contact_engine_gpu_colored.py:1039-1048, without the device synchronisations)."""
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
        _lib.check(L.b2c_bead_world(b(self.c_bodies), b(self.c_beads), b(self.c_grid), s), "beads")
        ev[2].record(stream)
        _lib.check(L.b2c_grid_build(b(self.c_beads), b(self.c_grid), s), "grid")
        ev[3].record(stream)
        _lib.check(L.b2c_bead_contacts_sorted(b(self.c_beads), b(self.c_grid), b(self.c_contacts),
                                              b(self.c_manifold), hdr, s), "contacts")
        ev[4].record(stream)
        _lib.check(L.b2c_manifold_reduce(b(self.c_bodies), b(self.c_beads), b(self.c_contacts), b(self.c_manifold),
                                         b(self.c_kept), ctypes.c_void_p(_ptr(self.k_keys)), b(self.c_pairs),
                                         b(self.c_warm), hdr, b(self.c_params), s), "manifold")
        ev[5].record(stream)
        _lib.check(L.b2c_color_pairs(b(self.c_bodies), b(self.c_pairs), hdr, b(self.c_params), s), "colour")
        ev[6].record(stream)
        _lib.check(L.b2c_color_solve(b(self.c_bodies), b(self.c_kept), b(self.c_pairs), hdr, b(self.c_params), sdt,
                                     s), "solve")
        ev[7].record(stream)
        _lib.check(L.b2c_warm_store(b(self.c_kept), ctypes.c_void_p(_ptr(self.k_keys)), b(self.c_warm), hdr, s),
                   "warm_store")
        ev[8].record(stream)
        _lib.check(L.b2c_body_integrate(b(self.c_bodies), sdt, s), "integrate")
        ev[9].record(stream)
        self._force_dt = dt
        self._fetch_header()
        ev[9].synchronize()
        return {name: ev[i].elapsed_time(ev[i + 1]) for i, name in enumerate(self.STAGES)}

    def solve_bytes(self) -> dict:
        """Algorithmic bytes of one persistent-solve launch (the last substep's counts): every SoA
        element the sweeps read or write, counted once per sweep.  Per sweep over the colours:
        pairs 20 B (porder, pstart, pcount, pbi, pbj), each dynamic pair endpoint 100 B (xc 12,
        invM 4, invIw 36, v/w read 24 and write 24), each kept contact 64 B in a velocity sweep
        (pidx 4, n 12, pA 12, pB 12, impulses read 12 and write 12) and 52 B in a position sweep
        or the applied warm start."""
        h = self.header_dict()
        P, Ck = h["n_pairs"], h["n_kept"]
        pbi = self.p_bufs["pbi"][:P].cpu().numpy()
        pbj = self.p_bufs["pbj"][:P].cpu().numpy()
        invM = self.invM.cpu().numpy()
        E = int(np.sum(invM[pbi] > 0) + np.sum((pbj >= 0) & (invM[np.maximum(pbj, 0)] > 0)))
        per_vel = 20 * P + 100 * E + 64 * Ck
        per_pos = 20 * P + 100 * E + 52 * Ck
        warm = per_pos if self._apply_warm else 0
        return dict(pairs=P, kept=Ck, endpoints=E, colors=h["n_colors"],
                    bytes=warm + self.vit * per_vel + self.pit * per_pos)

    def set_solve_blocks(self, n: int):
        """Launch form of the persistent solve: 0 auto, 1 one CTA, n > 1 a cooperative grid of n
        CTAs, -n a cluster of n CTAs.  Results do not depend on it.  Drops captured graphs."""
        self.solve_blocks = int(n)
        if self._built:
            self.c_params.solve_blocks = self.solve_blocks
            self._graphs = {}

    # ---- diagnostics ----
    @property
    def color_cache_hits(self):
        return int(self.p_bufs["cache_state"][3].item()) if self._built else 0

    @property
    def color_cache_misses(self):
        return int(self.p_bufs["cache_state"][4].item()) if self._built else 0

    def selection_debug(self):
        """Kept contacts of the last substep as (feature key, body i, body j) (COL:1095-1103)."""
        C = self.header_dict()["n_kept"]
        return np.stack([self.k_keys[:C].cpu().numpy(), self.k_bi[:C].cpu().numpy().astype(np.int64),
                         self.k_bj[:C].cpu().numpy().astype(np.int64)], axis=1)


class FixedFrameContactEngine(GraphColoredContactEngine):
    """Pair chunks with the normal-derived tangent frame (contact_engine_gpu_fixed_frame.py:82-88)."""
    name = "fixed_frame_b200"
    _fixed_frame = True

    def __init__(self, **kwargs):
        kwargs.update(manifold_reduce=True, graph_capture=True, pair_chunks=True, chunk_mode="registers")
        super().__init__(**kwargs)


class AppliedWarmContactEngine(FixedFrameContactEngine):
    """Warm impulses applied once per colour before the sweeps (contact_engine_gpu_applied_warm.py:57-75)."""
    name = "applied_warm_b200"
    _apply_warm = True

    def __init__(self, **kwargs):
        super().__init__(**kwargs)
        if self.t2_damp != 1.0:
            raise ValueError("Applied warm start requires full tangent updates")


class DeferredForceContactEngine(AppliedWarmContactEngine):
    """contact_forces() = M (v_after - v_before) / dt from the pre-solve velocity snapshot
    (contact_engine_gpu_deferred_force.py:7-74)."""
    name = "deferred_force_b200"


class ColorCacheContactEngine(DeferredForceContactEngine):
    """Reuses the pair colouring while (pair count, pbi, pbj, invM) are unchanged, compared on the
    device (contact_engine_gpu_color_cache.py:21-54)."""
    name = "color_cache_b200"
    _color_cache = True


class IslandSolveContactEngine(ColorCacheContactEngine):
    """The ColorCache engine with the island solve (contact_engine_gpu_island_solve.py:253-287).

    The reference partitions the pairs on the host after each colour-cache miss
    (``partition_pairs``) and runs one thread per island when the largest island has at most 64
    pairs, else the coloured chunk launch.  Here the partition runs on the device inside the
    captured step (skipped on a colour-cache hit), and the choice between the island solve and
    the persistent colour-phase solve is made on the device.  Both give the ColorCache engine's
    bits."""
    name = "island_solve_b200"
    _islands = True

    def _island_info(self):
        if not self._built:
            return (0, 0)
        info = self.p_bufs["isl_work"][:2].cpu().numpy()
        return int(info[0]), int(info[1])

    @property
    def island_count(self):
        """Islands of the last partition."""
        return self._island_info()[0]

    @property
    def max_island_pairs(self):
        """Pairs of the largest island of the last partition."""
        return self._island_info()[1]

    @property
    def island_rebuilds(self):
        """Partitions computed: one per colour-cache miss, as in the reference."""
        return self.color_cache_misses

    @property
    def island_solve_active(self):
        """True when the last substep ran the island solve (no island above 64 pairs)."""
        return self._built and self.max_island_pairs <= _lib.ISLAND_MAX_PAIRS
