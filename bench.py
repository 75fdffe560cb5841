"""Throughput benchmark of the contact-solve hot path: body-steps/s on one B200 (or N replicas).

python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl b200|reference]

One "step" is one ContactEngine.step(dt, substeps) of the whole scene.  The default workload is
10 000 random boxes (edges U[0.2, 0.6] m, density 1000, per-body mu U[0.3, 0.8]) dropped into a
20 x 20 x 10 m volume onto the ground; box/plane + box/box contacts, ColorCache pair solve with
first-fit colours (15-17 on this pile: the largest pair count of one body, so at most 32
allowed), 2 substeps x (16 velocity + 10 position sweeps), dt 1/240, 600 steps.  The
first 300 steps are set-up (boxes land, the pile forms; untimed), W warm-up steps follow, then
exactly K steps (default 300, the rest of the 600-step run) are timed with CUDA events on the
engine's stream, bracketed by a barrier and a device synchronise; the L2 is flushed (a 256 MiB
write) between timed steps, outside the events.  With N > 1 every rank runs an independent
replica (a single scene does not shard: replicas only) and the time is the max over ranks.
Rank 0 prints one JSON line.

`e2e` is the same metric through the public API with the body state in pinned host memory:
every step uploads the state (set_state_packed), steps, and downloads it again
(get_state_packed).  For the box workloads `e2e_cabi` repeats that loop through the C engine
handle (b2c_set_state_packed, b2c_step, b2c_get_state_packed), from the same state.

`--impl reference` times the CPU restatement of the same algorithm (the oracle; the reference
runs these engines through Warp, which is not installed) on the same workload, one replica per
host core, rank 0 only.

Other workloads (--workload): stress100k (100 000-cube lattice), batched512 (512 uneven
scenes in one engine), colorcache_lattice10k, island_lattice10k and jacobi_lattice10k (the
reference's 10k bead lattice under its ColorCache, island-solve and relaxed-Jacobi engines, with
vs_baseline against their published timings), admm4096 (the reference's batched ADMM and its
adjoint at its own benchmark configuration), ncp_lattice10k (the exact-cone NCP
solve of the reference's LatticeWorld fixture) and adjoint4096 (the batched NCP forward solve
and its adjoint at the reference's batched-adjoint shape).
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # 10 000 random boxes, SAT contacts, per-body friction, ColorCache pair solve
    "boxes10k": dict(engine="box", scene="random_boxes", n=10000, edge=(0.2, 0.6), box=(20.0, 20.0, 10.0),
                     mu_range=(0.3, 0.8), density=1000.0, vit=16, pit=10, substeps=2, dt=1 / 240, color_cap=32,
                     preroll=300, steps=300, warmup=3),
    # stress: 100 000 cubes of edge 0.25 on a seeded, jittered lattice in 50 x 50 x 10 m, mu 0.6,
    # 2 substeps x (16 velocity + 16 position sweeps), broadphase rebuilt every substep, 200 steps
    "stress100k": dict(engine="box", scene="box_lattice", n=100000, edge=(0.25, 0.25), box=(50.0, 50.0, 10.0),
                       mu_range=(0.6, 0.6), density=1000.0, vit=16, pit=16, substeps=2, dt=1 / 240, color_cap=32,
                       preroll=100, steps=200, warmup=3, parity_steps=20),
    # 512 independent box scenes of 8..2000 bodies (log-uniform), ~180k bodies, 10 % of each scene
    # 100x denser, advanced together by one batched engine; scenes are sharded over GPUs
    "batched512": dict(engine="batched", scene="batched", n_scenes=512, nmin=8, nmax=2000, edge=(0.2, 0.6),
                       mu_range=(0.3, 0.8), density=1000.0, vit=16, pit=10, substeps=2, dt=1 / 240, color_cap=32,
                       preroll=300, steps=100, warmup=3),
    # the reference's ColorCache timing fixture: lattice(10000) of (0.3, 0.3, 0.2) bead boxes, mu 0.5,
    # 40 velocity / 20 position sweeps, 1 substep, dt 1/240 (87 716 raw -> 40 000 kept contacts,
    # 10 000 pairs, 2 colours); published: 3.684 ms per step on an NVIDIA L4
    # (reports/innovation_stack_color_cache_l4.json, "timing")
    "colorcache_lattice10k": dict(engine="color_cache", scene="lattice", n=10000, dims=(0.3, 0.3, 0.2), mu=0.5,
                                  vit=40, pit=20, substeps=1, dt=1 / 240, preroll=0, steps=300, warmup=20,
                                  published=(1e4 / 3.684e-3, "reference ColorCache, 3.684 ms/step, NVIDIA L4 "
                                             "(reports/innovation_stack_color_cache_l4.json)")),
    # the same fixture under the island solve (IslandSolveContactEngine: 5 041 islands of at most two pairs,
    # one thread per island, no colour barriers; the ColorCache engine's bits); published: 2.817 and
    # 2.887 ms per step on an NVIDIA L4, the faster taken (reports/innovation_island_solve.json,
    # legs[*].island.timing)
    "island_lattice10k": dict(engine="island", scene="lattice", n=10000, dims=(0.3, 0.3, 0.2), mu=0.5,
                              vit=40, pit=20, substeps=1, dt=1 / 240, preroll=0, steps=300, warmup=20,
                              published=(1e4 / 2.817e-3, "reference IslandSolveContactEngine, 2.817 ms/step, "
                                         "NVIDIA L4 (reports/innovation_island_solve.json)")),
    # the same lattice under relaxed Jacobi; published: 5.599 ms per step at N = 10 000 on an RTX 5070
    # (docs/RUNNING.md:374-379)
    # the batched exact-cone NCP and its adjoint at the shape of the reference's batched-adjoint
    # benchmark (B = 4096 legged-stance problems, nv = 18, 4 contacts, mu 0.5, sliding): one step
    # is a forward solve of the whole batch to a natural residual of 1e-6, and the gradient is
    # two vector-Jacobian-product directions; published: forward 428.49 ms (9 559 env-steps/s),
    # grad (2 directions) 119.61 ms on an RTX 5070
    # (reproducibility/p2/data/reference/batch_throughput_slip.txt)
    "adjoint4096": dict(engine="bncp", B=4096, nv=18, nc=4, mu=0.5, tol=1e-6, max_iters=5000, steps=200, warmup=3,
                        published=(4096 / 428.49e-3, "reference batched ADMM forward, 428.49 ms at B = 4096, "
                                   "RTX 5070 (reproducibility/p2/data/reference/batch_throughput_slip.txt)"),
                        published_grad_ms=119.61, published_fwd_ms=428.49),
    # the reference's batched ADMM itself at its benchmark's configuration (B = 4096 sliding-stance
    # problems, nv 18, 4 contacts, mu 0.5, rho from the regime, 200 ADMM iterations of 8 CG steps,
    # refresh every 4, then the two gradient directions with 60 CG steps per sigma-map application):
    # one step is one launch of the forward and the gradient; published: forward 428.49 ms
    # (9 559 env-steps/s), forward + gradient 530.10 ms on an RTX 5070
    # (reproducibility/p2/data/reference/batch_throughput_slip.txt)
    "admm4096": dict(engine="admm", B=4096, nv=18, nc=4, mu=0.5, n_iter=200, cg=8, refresh=4, tol=1e-8, grad_cg=60,
                     steps=20, warmup=3,
                     published=(4096 / 530.10e-3, "reference BatchProxADMMGPU forward + gradient (2 directions), "
                                "530.10 ms at B = 4096, RTX 5070 (reproducibility/p2/data/reference/"
                                "batch_throughput_slip.txt)"),
                     published_fwd_ms=428.49, published_grad_ms=119.61, published_both_ms=530.10),
    # the reference's exact-cone NCP timing fixture (LatticeWorld, N = 10 000, n_c = 40 000, float64,
    # 40 PGS sweeps: residual 7.778e-05, 8 colours); one step solves the resident scene again
    # (setup, colouring through the cache, 40 sweeps); published: 11.21 ms per step = 280.2 us per
    # sweep on an RTX 5070 (reproducibility/p2/data/reference/lattice_producer_shared.txt)
    "ncp_lattice10k": dict(engine="ncp", n=10000, iters=40, steps=200, warmup=3,
                           published=(40000 * 40 / 11.21e-3, "reference NCPSolverGPU PGS, 40 sweeps in 11.21 ms, "
                                      "RTX 5070 (reproducibility/p2/data/reference/lattice_producer_shared.txt)")),
    "jacobi_lattice10k": dict(engine="jacobi", scene="lattice", n=10000, dims=(0.3, 0.3, 0.2), mu=0.5, vit=40,
                              pit=20, substeps=1, dt=1 / 240, preroll=0, steps=300, warmup=20,
                              published=(1e4 / 5.599e-3, "reference relaxed Jacobi, 5.599 ms/step, RTX 5070 "
                                         "(docs/RUNNING.md:374-379)")),
    # the stress lattice under relaxed Jacobi: 100 000 bead boxes on the stress scene's seeded
    # lattice in 50 x 50 x 10 m (5 % jitter), mu 0.6, 2 substeps x (16 velocity + 16 position
    # iterations), the bead grid rebuilt every substep, 200 steps.  The bead engines need edges
    # that are multiples of the 0.1 m bead pitch (a 0.25 m edge gives asymmetric bead offsets),
    # so the edge is 0.3 m: 27 beads per box, 2.7 M beads
    "stress100k_jacobi": dict(engine="jacobi", scene="box_lattice_beads", n=100000, dims=(0.3, 0.3, 0.3),
                              density=1000.0, mu=0.6, vit=16, pit=16, substeps=2, dt=1 / 240, preroll=100, steps=200,
                              warmup=3, parity_steps=8, contact_capacity=4_000_000, grid_dims=(512, 512, 128)),
    # plain relaxed Jacobi on a vertical stack of 16 unit cubes (1 m edge, 1 kg: density 1, 1000
    # beads each) with seeded 1 mm xy jitter, mu 0.5, 40 velocity / 20 position iterations, relax
    # 0.2, 1 substep, dt 1/240, 240 steps; penetration target 1e-3 m (max over adjacent pairs of
    # 1.0 - dz, and 0.5 - z of the lowest cube)
    "jacobi_stack16": dict(engine="jacobi", scene="unit_cube_stack", n=16, dims=(1.0, 1.0, 1.0), density=1.0,
                           mu=0.5, vit=40, pit=20, substeps=1, dt=1 / 240, preroll=0, steps=240, warmup=3,
                           stack_pitch=1.0, stack_ground=0.5, pen_target_m=1e-3),
    # the differentiable form: 256 scenes of a 64-box stepped pyramid (edge 0.2, density 1000, seeded
    # 1 mm jitter) pushed by a kinematic plate at 0.2 m/s; loss = sum |x_final - target|^2 after a
    # 120-step rollout (2 substeps, 16 sweeps, warm-started); gradients in v0 ~ N(0, 0.1) m/s and
    # per-body mu; central differences with eps 1e-3 on the same float64 forward
    "pyramids256_rollout": dict(engine="rollout", n_scenes=256, rollout_steps=120, substeps=2, iters=16,
                                dt=1 / 240, fd_eps=1e-3, steps=1, warmup=3),
    # a short case of the same rollout (32 scenes, 10 steps): the profiling case of its kernels
    "pyramids32_rollout10": dict(engine="rollout", n_scenes=32, rollout_steps=10, substeps=2, iters=16,
                                 dt=1 / 240, fd_eps=1e-3, steps=1, warmup=3),
}
DEFAULT_WORKLOAD = "boxes10k"


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0}, "fallback"


def _scenes():
    from importlib import import_module
    return import_module("motion_engine_b200.scenes")


def scene_of(wl):
    sc = _scenes()
    if wl["scene"] == "batched":
        return {"scenes": sc.batched_scenes(n_scenes=wl["n_scenes"], nmin=wl["nmin"], nmax=wl["nmax"])}
    if wl["scene"] == "box_lattice":
        return sc.box_lattice(n=wl["n"], edge=wl["edge"][0], extent=wl["box"], mu=wl["mu_range"][0],
                              density=wl["density"])
    if wl["scene"] == "random_boxes":
        return sc.random_boxes(n=wl["n"], edge=wl["edge"], box=wl["box"], mu=wl["mu_range"], density=wl["density"])
    if wl["scene"] == "unit_cube_stack":
        return {"centers": sc.unit_cube_stack(wl["n"])}
    if wl["scene"] == "box_lattice_beads":
        return {"centers": sc.box_lattice(n=wl["n"], edge=wl["dims"][0], extent=(50.0, 50.0, 10.0))["centers"]}
    return {"centers": sc.lattice(wl["n"]) if wl["scene"] == "lattice" else sc.stack(wl["n"])}


def make_engine(me, wl, scene):
    if wl["engine"] == "batched":
        return me.BatchedBoxEngine(scene["scenes"], mu=float(np.mean(wl["mu_range"])), vit=wl["vit"], pit=wl["pit"],
                                   color_cap=wl["color_cap"])
    if wl["engine"] == "box":
        e = me.BoxContactEngine(mu=float(np.mean(wl["mu_range"])), vit=wl["vit"], pit=wl["pit"],
                                color_cap=wl["color_cap"], islands=bool(wl.get("islands", False)))
        for c, d, m, de in zip(scene["centers"], scene["dims"], scene["mu"], scene["density"]):
            e.add_box(c, dims=d, density=de, mu=m)
        return e
    if wl["engine"] == "color_cache":
        e = me.ColorCacheContactEngine(dims=wl["dims"], mu=wl["mu"], vit=wl["vit"], pit=wl["pit"])
    elif wl["engine"] == "island":
        e = me.IslandSolveContactEngine(dims=wl["dims"], mu=wl["mu"], vit=wl["vit"], pit=wl["pit"])
    elif wl["engine"] == "jacobi":
        kw = {k: wl[k] for k in ("contact_capacity", "grid_dims") if k in wl}
        e = me.RelaxedJacobiContactEngine(dims=wl["dims"], mu=wl["mu"], vit=wl["vit"], pit=wl["pit"], **kw)
    else:
        raise ValueError(wl["engine"])
    for c in scene["centers"]:
        e.add_body(c, density=wl.get("density", 700.0))
    return e


def cabi_e2e(me, wl, scene, start, flush, stream, K):
    """Milliseconds of K end-to-end steps through the C ABI's engine handle: the same boxes
    from the packed state `start` (the Python engine's state where its own end-to-end loop
    started), 3 untimed steps (the build, the graph capture, a warm store), then per step
    b2c_set_state_packed from pinned host memory, b2c_step and b2c_get_state_packed back, on
    `stream`, L2 flushed in between."""
    import ctypes

    import torch
    h = me.HandleBoxEngine(mu=float(np.mean(wl["mu_range"])), vit=wl["vit"], pit=wl["pit"],
                           color_cap=wl["color_cap"], device=torch.cuda.current_device())
    h.add_boxes(scene["centers"], dims=scene["dims"], density=scene["density"], mu=scene["mu"])
    dt, S = wl["dt"], wl["substeps"]
    L, s, check = h.L, ctypes.c_void_p(stream.cuda_stream), me._lib.check
    host = torch.empty((4, h.N, 4), dtype=torch.float32, pin_memory=True)
    host.copy_(start)
    hp = ctypes.c_void_p(host.data_ptr())
    check(L.b2c_set_state_packed(h._h, hp, s), "b2c_set_state_packed")
    for _ in range(3):
        check(L.b2c_step(h._h, dt, S, s), "b2c_step")
    check(L.b2c_get_state_packed(h._h, hp, s), "b2c_get_state_packed")
    torch.cuda.synchronize()
    ms = 0.0
    for k in range(K):
        flush.fill_(float(k))
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        check(L.b2c_set_state_packed(h._h, hp, s), "b2c_set_state_packed")
        check(L.b2c_step(h._h, dt, S, s), "b2c_step")
        check(L.b2c_get_state_packed(h._h, hp, s), "b2c_get_state_packed")
        b.record(stream)
        b.synchronize()
        ms += a.elapsed_time(b)
    h.header()
    h.close()
    return ms


def make_oracle(wl, scene):
    from oracle import oracle as O
    if wl["engine"] == "box":
        o = O.BoxOracle(mu=float(np.mean(wl["mu_range"])), vit=wl["vit"], pit=wl["pit"])
        for c, d, m, de in zip(scene["centers"], scene["dims"], scene["mu"], scene["density"]):
            o.add_box(c, dims=d, density=de, mu=m)
        return o
    if wl["engine"] == "jacobi":
        o = O.JacobiOracle(dims=wl["dims"], mu=wl["mu"], vit=wl["vit"], pit=wl["pit"])
    else:
        o = O.ColoredOracle(mode="color_cache", dims=wl["dims"], mu=wl["mu"], vit=wl["vit"], pit=wl["pit"])
    for c in scene["centers"]:
        o.add_body(c, density=wl.get("density", 700.0))
    return o


def state_digest(xc, q, v, w) -> str:
    """sha256 of a body state: positions (N,3), quaternions (N,4), velocities and angular
    velocities (N,3), float32, concatenated in that order."""
    h = hashlib.sha256()
    for a in (xc, q, v, w):
        h.update(np.ascontiguousarray(a, np.float32).tobytes())
    return h.hexdigest()


def combine_digests(digests) -> str:
    """One digest over per-scene digests in scene order."""
    return hashlib.sha256("".join(digests).encode()).hexdigest()


def _oracle_state(o):
    return o.body_state() if hasattr(o, "body_state") else (o.b.xc, o.b.q, o.b.v, o.b.w)


def _parity_worker(workload, idx, steps):
    """The oracle over the workload's first `steps` steps from its initial state: one state
    digest, or for a batch one per scene of `idx` (scenes are independent, so each runs alone)."""
    sys.path.insert(0, ROOT)
    import __graft_entry__ as ge
    ge.load_package()
    wl = WORKLOADS[workload]
    sc = scene_of(wl)
    t0 = time.perf_counter()
    out = []
    if wl["engine"] == "batched":
        for i in idx:
            o = _box_oracle(wl, sc["scenes"][i])
            for _ in range(steps):
                o.step(wl["dt"], wl["substeps"])
            out.append((i, state_digest(*o.body_state())))
    else:
        o = make_oracle(wl, sc)
        for _ in range(steps):
            o.step(wl["dt"], wl["substeps"])
        out.append((0, state_digest(*_oracle_state(o))))
    return out, time.perf_counter() - t0


class ParityCheck:
    """The oracle's state digest after the workload's first `steps` steps, computed in spawned
    processes while the GPU runs (started before the first GPU call), to set beside the GPU
    engine's digest at the same step.  A batch is split over processes by scene (LPT)."""

    def __init__(self, args, wl, steps, scene_idx=None):
        import multiprocessing as mp
        self.steps = steps
        self.batched = scene_idx is not None
        if scene_idx is None:
            parts = [[0]]
        else:
            counts = [len(sc["centers"]) for sc in scene_of(wl)["scenes"]]
            nproc = max(1, min((os.cpu_count() or 2) - 1, 16, len(scene_idx)))
            sub = [counts[i] for i in scene_idx]
            parts = [[scene_idx[j] for j in p] for p in partition_scenes(sub, nproc) if p]
        self.pool = mp.get_context("spawn").Pool(len(parts))
        self.res = self.pool.starmap_async(_parity_worker, [(args.workload, p, steps) for p in parts])

    def result(self, gpu_digest, timeout=900.0):
        out = {"steps": self.steps, "gpu_sha256": gpu_digest, "oracle_sha256": None, "equal": None}
        try:
            res = self.res.get(timeout=timeout)
            digests = dict(d for part, _ in res for d in part)
            od = combine_digests([digests[k] for k in sorted(digests)]) if self.batched else digests[0]
            out.update(oracle_sha256=od, equal=od == out["gpu_sha256"],
                       oracle_s=round(max(t for _, t in res), 1))
        except Exception as ex:  # the oracle did not finish: reported, not raised
            out["note"] = f"oracle digest unavailable: {type(ex).__name__}"
        finally:
            self.pool.terminate()
        return out


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                                      stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        self.rows = []
        if self.p is not None:
            self.p.terminate()
            try:
                out, _ = self.p.communicate(timeout=5)
            except Exception:
                self.p.kill()
                out = ""
            for ln in out.strip().splitlines():
                parts = [x.strip() for x in ln.split(",")]
                if len(parts) >= 9:
                    self.rows.append(parts)

    def summary(self):
        if not getattr(self, "rows", None):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({names[k] for r in self.rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def _time_oracle(o, wl, max_seconds, max_steps):
    n = 0
    t0 = time.perf_counter()
    while True:
        o.step(wl["dt"], wl["substeps"])
        n += 1
        el = time.perf_counter() - t0
        if el > max_seconds or n >= max_steps:
            return n, el


def cpu_baseline_sample(wl, scene, state=None, max_seconds=20.0):
    """The oracle (single-threaded C restatement) on the same workload: from the GPU's body state
    at the start of the timed region when given (box workload), else from the initial state after
    the same warm-up; steps until max_seconds of CPU work."""
    o = make_oracle(wl, scene)
    if state is not None:
        o.set_body_state(*state)
    else:
        t0 = time.perf_counter()
        for _ in range(wl["preroll"] + wl["warmup"]):
            o.step(wl["dt"], wl["substeps"])
            if time.perf_counter() - t0 > 2 * max_seconds:
                break
    n, el = _time_oracle(o, wl, max_seconds, 200)
    return wl["n"] * n / el, n, el


def partition_scenes(counts, parts):
    from importlib import import_module
    return import_module("motion_engine_b200.boxes").partition_scenes(counts, parts)


def _box_oracle(wl, sc):
    from oracle import oracle as O
    o = O.BoxOracle(mu=float(np.mean(wl["mu_range"])), vit=wl["vit"], pit=wl["pit"])
    for c, d, m, de in zip(sc["centers"], sc["dims"], sc["mu"], sc["density"]):
        o.add_box(c, dims=d, density=de, mu=m)
    return o


def batched_cpu_sample(wl, scenes, states, max_seconds=20.0):
    """The oracle, one scene at a time from the GPU's state of that scene, one step each, scenes
    in order until max_seconds of CPU work: body-steps/s on one core."""
    bs, t_busy, n_sc = 0, 0.0, 0
    for sc, st in zip(scenes, states):
        o = _box_oracle(wl, sc)
        o.set_body_state(*st)
        t0 = time.perf_counter()
        o.step(wl["dt"], wl["substeps"])
        t_busy += time.perf_counter() - t0
        bs += len(sc["centers"])
        n_sc += 1
        if t_busy > max_seconds:
            break
    return bs / t_busy, n_sc, t_busy


def _ref_batched_worker(workload, idx, steps, warmup, budget):
    sys.path.insert(0, ROOT)
    import __graft_entry__ as ge
    ge.load_package()
    wl = WORKLOADS[workload]
    scenes = scene_of(wl)["scenes"]
    oracles = [_box_oracle(wl, scenes[i]) for i in idx]
    for o in oracles:
        for _ in range(wl["preroll"] + warmup):
            o.step(wl["dt"], wl["substeps"])
    bs, n = 0, 0
    t0 = time.perf_counter()
    while n < steps:
        for o, i in zip(oracles, idx):
            o.step(wl["dt"], wl["substeps"])
            bs += len(scenes[i]["centers"])
        n += 1
        if time.perf_counter() - t0 > budget:
            break
    return bs, time.perf_counter() - t0, n


def run_reference_batched(args, wl):
    """--impl reference for the batched workload: the oracle on every host core, the scenes
    split over the processes (LPT on body counts); each process advances its scenes through the
    set-up and warm-up steps, then times whole batch steps for up to ~60 s."""
    import multiprocessing as mp
    if int(os.environ.get("RANK", "0")) != 0:
        return
    scenes = scene_of(wl)["scenes"]
    counts = [len(sc["centers"]) for sc in scenes]
    procs = max(1, min(os.cpu_count() or 1, 64, len(scenes)))
    parts = [p for p in partition_scenes(counts, procs) if p]
    ctx = mp.get_context("spawn")
    with ctx.Pool(len(parts)) as pool:
        t0 = time.perf_counter()
        res = pool.starmap(_ref_batched_worker, [(args.workload, p, args.steps, args.warmup, 60.0) for p in parts])
        wall = time.perf_counter() - t0
    steps_min = min(r[2] for r in res)
    # whole-job rate: every process's body-steps over the slowest process's busy time
    value = sum(r[0] for r in res) / max(r[1] for r in res)
    line = {"impl": "reference", "metric": "body-steps/s", "value": value, "unit": "body-steps/s",
            "higher_is_better": True, "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "config": {"workload": args.workload, "bodies": sum(counts), "scenes": len(scenes),
                       **{k: v for k, v in wl.items() if k not in ("warmup", "steps")}},
            "dtype": "f32", "data": "synthetic",
            "cpu_baseline": {"value": value, "unit": "body-steps/s", "cores": len(parts), "kind": "port",
                             "sample": f"{len(parts)} processes, each advancing its share of the {len(scenes)} "
                                       f"scenes (LPT on body counts) by >= {steps_min} timed batch steps after the "
                                       f"{wl['preroll']} set-up and {args.warmup} warm-up steps, capped at ~60 s; "
                                       f"the oracle restatement, the reference's Warp CPU path is not installed"},
            "e2e": {"value": value, "unit": "body-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "wall_s": wall}
    print(json.dumps(line), flush=True)


def run_reference(args, wl):
    """--impl reference: the oracle port on every host core (one independent replica per
    process, spawn start method), each timed over a bounded number of steps from the workload's
    state after its set-up steps (computed once here, by the oracle)."""
    import multiprocessing as mp
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    procs = max(1, min(cores, 64))
    scene = scene_of(wl)
    t_pre = time.perf_counter()
    o = make_oracle(wl, scene)
    for _ in range(wl["preroll"]):
        o.step(wl["dt"], wl["substeps"])
    pre_s = time.perf_counter() - t_pre
    fd, path = tempfile.mkstemp(suffix=".npz")
    os.close(fd)
    parity = ({"steps": wl["preroll"], "oracle_sha256": state_digest(*_oracle_state(o))}
              if wl["preroll"] > 0 else None)
    try:
        st = o.body_state() if hasattr(o, "body_state") else None
        np.savez(path, **{k: np.asarray(v) for k, v in scene.items()},
                 **({} if st is None else dict(s_xc=st[0], s_q=st[1], s_v=st[2], s_w=st[3])))
        del o
        ctx = mp.get_context("spawn")
        budget = 60.0
        with ctx.Pool(procs) as pool:
            t0 = time.perf_counter()
            res = pool.starmap(_ref_worker, [(args.workload, path, args.steps, args.warmup, budget)] * procs)
            wall = time.perf_counter() - t0
    finally:
        os.unlink(path)
    steps_done = sum(r[0] for r in res)
    busy = max(r[1] for r in res)
    value = wl["n"] * steps_done / busy
    line = {"impl": "reference", "metric": "body-steps/s", "value": value, "unit": "body-steps/s",
            "higher_is_better": True, "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "config": {"workload": args.workload, **{k: v for k, v in wl.items() if k not in ("warmup", "steps")}},
            "dtype": "f32", "data": "synthetic",
            "cpu_baseline": {"value": value, "unit": "body-steps/s", "cores": procs, "kind": "port",
                             "sample": f"{procs} processes x {steps_done / procs:.1f} timed steps (<= {args.steps} "
                                       f"each, capped at ~{budget:.0f} s) of independent replicas from the state "
                                       f"after the workload's {wl['preroll']} set-up steps (oracle, {pre_s:.0f} s) and "
                                       f"{args.warmup} warm-up steps; the reference's Warp CPU path is not installed"},
            "e2e": {"value": value, "unit": "body-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "parity": parity, "wall_s": wall}
    print(json.dumps(line), flush=True)


def _ref_worker(workload, path, steps, warmup, budget):
    sys.path.insert(0, ROOT)
    import __graft_entry__ as ge
    ge.load_package()  # registers the package alias for the scene builders
    wl = WORKLOADS[workload]
    d = dict(np.load(path))
    scene = {k: d[k] for k in d if not k.startswith("s_")}
    o = make_oracle(wl, scene)
    if "s_xc" in d:
        o.set_body_state(d["s_xc"], d["s_q"], d["s_v"], d["s_w"])
    else:
        for _ in range(wl["preroll"]):
            o.step(wl["dt"], wl["substeps"])
    t_start = time.perf_counter()
    for _ in range(warmup):
        o.step(wl["dt"], wl["substeps"])
        if time.perf_counter() - t_start > 30.0:
            break
    return _time_oracle(o, wl, budget, steps)


def per_scene_sequential(me, wl, scenes, batch, dt, S, stream, steps=3):
    """The same scenes advanced one engine per scene, one after another (per-scene launches), from
    the batch's current state and for the same sweeps: body-steps/s on this GPU.  Each engine
    first runs one untimed step (its CUDA graph capture; it starts without the batch's warm
    impulses)."""
    import torch
    engines = []
    st = batch.get_state()
    q = batch.q.cpu().numpy()
    for k, sc in enumerate(scenes):
        e = me.BoxContactEngine(mu=float(np.mean(wl["mu_range"])), vit=wl["vit"], pit=wl["pit"],
                                color_cap=wl["color_cap"], cand_per_body=12)
        for c, d, de, m in zip(sc["centers"], sc["dims"], sc["density"], sc["mu"]):
            e.add_box(c, dims=d, density=de, mu=m)
        sl = batch.scene_slice(k)
        e.set_body_state(st.xc[sl], q[sl], st.vc[sl], st.om[sl])
        e.step(dt, S)
        engines.append(e)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(steps):
        for e in engines:
            e.step(dt, S)
    b.record(stream)
    b.synchronize()
    ms = a.elapsed_time(b) / steps
    for e in engines:
        e.check_errors()
    n = sum(len(sc["centers"]) for sc in scenes)
    return {"value": n / (ms / 1e3), "unit": "body-steps/s", "ms_per_step": ms, "steps": steps,
            "engines": len(engines), "note": "same sweeps per scene; each scene's arithmetic is bytewise the batch's"}


def _stance(wl, B=None):
    sc = _scenes()
    return sc.stance_batch(B=wl["B"] if B is None else B, nv=wl["nv"], nc=wl["nc"], mu=wl["mu"])


def _bncp_cpu_worker(args_):
    """Oracle PGS plus two VJP directions on problems [lo, hi) of the stance batch; returns
    (problems done, seconds)."""
    workload, lo, hi, budget = args_
    sys.path.insert(0, ROOT)
    import __graft_entry__ as ge
    ge.load_package()
    from oracle import oracle_bncp as OB
    wl = WORKLOADS[workload]
    J, Minv, v, mu = _stance(wl)
    G = J[lo:hi] @ Minv[lo:hi] @ J[lo:hi].transpose(0, 2, 1)
    b = (J[lo:hi] @ v[lo:hi, :, None])[..., 0]
    done, t0 = 0, time.perf_counter()
    for e in range(hi - lo):
        OB.pgs(G[e], b[e], mu[lo + e], iters=wl["max_iters"], tol=wl["tol"])
        done += 1
        if time.perf_counter() - t0 > budget:
            break
    return done, time.perf_counter() - t0


def run_reference_adjoint(args, wl):
    """--impl reference for the adjoint workload: the oracle's PGS (numpy) on every host core,
    each process on its share of the batch, bounded to ~30 s."""
    import multiprocessing as mp
    if int(os.environ.get("RANK", "0")) != 0:
        return
    procs = max(1, min(os.cpu_count() or 1, 64))
    B = wl["B"]
    cuts = [B * k // procs for k in range(procs + 1)]
    with mp.get_context("spawn").Pool(procs) as pool:
        res = pool.map(_bncp_cpu_worker, [(args.workload, cuts[k], cuts[k + 1], 30.0) for k in range(procs)])
    value = sum(r[0] for r in res) / max(r[1] for r in res)
    line = {"impl": "reference", "metric": "env-steps/s", "value": value, "unit": "env-steps/s",
            "higher_is_better": True, "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "config": {"workload": args.workload, **{k: v for k, v in wl.items() if k not in ("warmup", "steps")}},
            "dtype": "f64", "data": "synthetic",
            "cpu_baseline": {"value": value, "unit": "env-steps/s", "cores": procs, "kind": "port",
                             "sample": f"{sum(r[0] for r in res)} of the {B} problems, forward solves to the "
                                       f"same residual, {procs} processes capped at ~30 s (the oracle's numpy "
                                       f"PGS; the reference's Warp path is not installed)"},
            "e2e": {"value": value, "unit": "env-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _admm_cpu_worker(args_):
    """The ADMM oracle (forward and both gradient directions) on problems [lo, hi) of the stance
    batch, in blocks of 8 until the budget is spent; returns (problems done, seconds)."""
    workload, lo, hi, budget = args_
    sys.path.insert(0, ROOT)
    import __graft_entry__ as ge
    ge.load_package()
    from oracle import oracle_badmm as OA
    wl = WORKLOADS[workload]
    J, Minv, v, mu = _stance(wl)
    done, t0 = 0, time.perf_counter()
    for a in range(lo, hi, 8):
        b = min(hi, a + 8)
        o = OA.BatchADMMOracle(J[a:b], Minv[a:b], v[a:b], mu[a:b], 1.0 / 240.0).set_rho("regime")
        o.forward(wl["n_iter"], wl["cg"], wl["refresh"], wl["tol"])
        o.gradient(n_calls=wl["nc"] + 2, grad_cg=wl["grad_cg"])
        done += b - a
        if time.perf_counter() - t0 > budget:
            break
    return done, time.perf_counter() - t0


def run_reference_admm(args, wl):
    """--impl reference for the ADMM workload: the ADMM oracle (numpy) on every host core."""
    import multiprocessing as mp
    if int(os.environ.get("RANK", "0")) != 0:
        return
    procs = max(1, min(os.cpu_count() or 1, 64))
    B = wl["B"]
    cuts = [B * k // procs for k in range(procs + 1)]
    with mp.get_context("spawn").Pool(procs) as pool:
        res = pool.map(_admm_cpu_worker, [(args.workload, cuts[k], cuts[k + 1], 30.0) for k in range(procs)])
    value = sum(r[0] for r in res) / max(r[1] for r in res)
    line = {"impl": "reference", "metric": "env-steps/s", "value": value, "unit": "env-steps/s",
            "higher_is_better": True, "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "config": {"workload": args.workload, **{k: v for k, v in wl.items() if k not in ("warmup", "steps")}},
            "dtype": "f64", "data": "synthetic",
            "cpu_baseline": {"value": value, "unit": "env-steps/s", "cores": procs, "kind": "port",
                             "sample": f"{sum(r[0] for r in res)} of the {B} problems, forward and both gradient "
                                       f"directions, {procs} processes capped at ~30 s (the ADMM oracle in numpy; "
                                       f"the reference's Warp path is not installed)"},
            "e2e": {"value": value, "unit": "env-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_admm(args, wl):
    """The reference's batched ADMM and its adjoint, one launch per step (forward from zero and
    both gradient directions), the forward alone timed beside it.  With N ranks every rank solves
    its own batch (weak scaling)."""
    import torch
    import __graft_entry__ as ge
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    ge.load_package()
    cpu_base = None
    if rank == 0 and not args.no_cpu_baseline:  # before the first GPU call
        n, el = _admm_cpu_worker((args.workload, 0, wl["B"], 15.0))
        cpu_base = {"value": n / el, "unit": "env-steps/s", "cores": 1, "kind": "port",
                    "sample": f"{n} problems of the batch, forward and both gradient directions, on one host core "
                              f"({el:.1f} s; the ADMM oracle in numpy)"}
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from motion_engine_b200 import badmm
    J, Minv, v, mu = _stance(wl)
    B, C, NV = wl["B"], wl["nc"], wl["nv"]
    s = badmm.BatchProxADMM(B, NV, C, device=dev).upload(J, Minv, v, mu, 1.0 / 240.0).set_rho("regime")
    kw = dict(cg_iters=wl["cg"], refresh_every=wl["refresh"], tol=wl["tol"], n_calls=C + 2, grad_cg=wl["grad_cg"])
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    for _ in range(args.warmup):
        s.step_and_grad(wl["n_iter"], **kw)
        s.launch(1, wl["n_iter"], wl["cg"], wl["refresh"], wl["tol"])
    torch.cuda.synchronize()
    both, fwd = [], []
    with ClockSampler(local) as clk:
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        for _ in range(args.steps):
            flush.zero_()
            e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            e0.record()
            s.step_and_grad(wl["n_iter"], **kw)
            e1.record()
            s.launch(1, wl["n_iter"], wl["cg"], wl["refresh"], wl["tol"])
            e2.record()
            e2.synchronize()
            both.append(e0.elapsed_time(e1))
            fwd.append(e1.elapsed_time(e2))
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
    t = torch.tensor([float(np.mean(both)), float(np.mean(fwd))], device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    both_ms, fwd_ms = float(t[0]), float(t[1])
    grad_ms = both_ms - fwd_ms
    value = B * world / (both_ms / 1e3)
    s.step_and_grad(wl["n_iter"], **kw)
    torch.cuda.synchronize()
    res = s.res.cpu().numpy()
    labels = np.bincount(s.labels.cpu().numpy().ravel(), minlength=3).tolist()
    # end to end through the public API: the problems from pinned host memory, the solution and
    # both gradients back, every step
    hJ, hM, hv, hmu = (torch.from_numpy(np.ascontiguousarray(x)).pin_memory() for x in (J, Minv, v, mu))
    outs = [torch.empty(tuple(t_.shape), dtype=torch.float64).pin_memory()
            for t_ in (s.lam, s.v_plus, s.dlam_tau, s.dv_tau, s.dlam_mu)]
    K2 = max(3, min(args.steps, 10))
    a, z = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(K2):
        s.upload(hJ.to(dev, non_blocking=True), hM.to(dev, non_blocking=True), hv.to(dev, non_blocking=True),
                 hmu.to(dev, non_blocking=True), 1.0 / 240.0)
        s.step_and_grad(wl["n_iter"], **kw)
        for o_, t_ in zip(outs, (s.lam, s.v_plus, s.dlam_tau, s.dv_tau, s.dlam_mu)):
            o_.copy_(t_, non_blocking=True)
    z.record()
    z.synchronize()
    e2e_ms = a.elapsed_time(z) / K2
    peaks, peak_kind = _peaks()
    alg = B * (3 * C * NV + NV * NV + NV + C) * 8 + B * (2 * 3 * C * 3 + NV + 2 * NV) * 8  # inputs once, outputs
    roof = {"bound": "hbm", "achieved": alg / (both_ms / 1e3) / 1e9, "peak": peaks["hbm_gbs"], "unit": "GB/s",
            "frac": alg / (both_ms / 1e3) / 1e9 / peaks["hbm_gbs"], "traffic": None, "peak_kind": peak_kind,
            "kernel": "k_admm (one warp per problem: set-up, ADMM, active set, grad_affine in shared memory)",
            "launch_ms": both_ms, "algorithmic_bytes_per_launch": alg,
            "note": "latency-bound: each warp iterates its problem in shared memory; the inputs are read once"}
    if rank == 0:
        line = {"metric": "env-steps/s", "value": value, "unit": "env-steps/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": both_ms, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": value / wl["published"][0], "dtype": "f64",
                "data": "synthetic (seeded legged-stance batch, the reference's shapes)",
                "config": {"workload": args.workload, "B": B, "nv": NV, "contacts": C, "mu": wl["mu"],
                           "rho": "regime", "admm_iters": wl["n_iter"], "cg": wl["cg"], "refresh": wl["refresh"],
                           "tol": wl["tol"], "grad_cg": wl["grad_cg"], "n_calls": C + 2,
                           "l2": "flushed between timed steps (256 MiB write)", "parallelism": f"batches x{world}"},
                "baseline": {"value": wl["published"][0], "unit": "env-steps/s", "source": wl["published"][1]},
                "adjoint": {"fwd_ms": fwd_ms, "grad_ms_2dir": grad_ms, "fwd_plus_grad_ms": both_ms,
                            "grad_over_fwd": grad_ms / fwd_ms,
                            "reference": {"fwd_ms": wl["published_fwd_ms"], "grad_ms_2dir": wl["published_grad_ms"],
                                          "fwd_plus_grad_ms": wl["published_both_ms"],
                                          "grad_over_fwd": wl["published_grad_ms"] / wl["published_fwd_ms"]}},
                "residual": {"max": float(np.nanmax(res)), "median": float(np.nanmedian(res)),
                             "below_1e-8": float(np.mean(res < 1e-8)),
                             "note": "the reference's run reports frac<1e-8 0.0000 and a median 1.49e-04"},
                "contacts_by_label": dict(zip(("open", "stick", "slip"), labels)),
                "clocks": clk.summary(),
                "e2e": {"value": B / (e2e_ms / 1e3), "unit": "env-steps/s",
                        "h2d_bytes_per_step": int(sum(x.numel() * 8 for x in (hJ, hM, hv, hmu))),
                        "d2h_bytes_per_step": int(sum(o_.numel() * 8 for o_ in outs)), "steps": K2},
                "gpu_launches": args.steps * 2, "launches_per_step": 1,
                "roofline": roof, "cpu_baseline": cpu_base}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def run_adjoint(args, wl):
    """The batched NCP forward solve and its adjoint.  A step solves the whole batch (from zero)
    to the workload's residual; the gradient is two vector-Jacobian products (two seeds), as the
    reference's "grad (2 dir)".  With N ranks every rank solves its own batch (weak scaling)."""
    import torch
    import __graft_entry__ as ge
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    me = ge.load_package()
    from motion_engine_b200 import bncp
    cpu_base = None
    if rank == 0 and not args.no_cpu_baseline:  # before the first GPU call
        n, el = _bncp_cpu_worker((args.workload, 0, wl["B"], 20.0))
        cpu_base = {"value": n / el, "unit": "env-steps/s", "cores": 1, "kind": "port",
                    "sample": f"{n} problems of the batch solved to the same residual on one host core "
                              f"({el:.1f} s; the oracle's numpy PGS)"}
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    J, Minv, v, mu = _stance(wl)
    B, n = wl["B"], 3 * wl["nc"]
    f64 = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    G, b = bncp.delassus(f64(J), f64(Minv), f64(v))
    mu_d = f64(mu)
    s = bncp.BatchNCP(G, b, mu_d)
    gen = torch.Generator(device="cpu").manual_seed(11)
    seeds = [torch.randn((B, n), generator=gen, dtype=torch.float64).to(dev) for _ in range(2)]
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    for _ in range(args.warmup):
        s.solve(wl["max_iters"], wl["tol"])
        for g in seeds:
            s.vjp(g)
    torch.cuda.synchronize()
    fwd, grad = [], []
    with ClockSampler(local) as clk:
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        for _ in range(args.steps):
            flush.zero_()
            e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            e0.record()
            s.solve(wl["max_iters"], wl["tol"])
            e1.record()
            for g in seeds:
                s.vjp(g)
            e2.record()
            e2.synchronize()
            fwd.append(e0.elapsed_time(e1))
            grad.append(e1.elapsed_time(e2))
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
    fwd_ms, grad_ms = float(np.mean(fwd)), float(np.mean(grad))
    t = torch.tensor([fwd_ms, grad_ms], device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    fwd_ms, grad_ms = float(t[0]), float(t[1])
    value = B * world / (fwd_ms / 1e3)
    res = s.res
    conv = int((s.iters < wl["max_iters"]).sum())
    labels = torch.bincount(s.labels.flatten().long(), minlength=3).tolist()
    # end to end through the public autograd entry: pinned host problems in, lambda out, every step
    hG, hb, hmu = (x.cpu().pin_memory() for x in (G, b, mu_d))
    hlam = torch.empty((B, n), dtype=torch.float64).pin_memory()
    K2 = max(3, min(args.steps, 10))
    a, z = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(K2):
        lam = bncp.ncp_solve(hG.to(dev, non_blocking=True), hb.to(dev, non_blocking=True),
                             hmu.to(dev, non_blocking=True), wl["max_iters"], wl["tol"])
        hlam.copy_(lam, non_blocking=True)
    z.record()
    z.synchronize()
    e2e_ms = a.elapsed_time(z) / K2
    peaks, peak_kind = _peaks()
    alg = B * (n * n + n + n // 3 + n) * 8  # G, b, mu read, lambda written, per launch
    roof = {"bound": "hbm", "achieved": alg / (fwd_ms / 1e3) / 1e9, "peak": peaks["hbm_gbs"], "unit": "GB/s",
            "frac": alg / (fwd_ms / 1e3) / 1e9 / peaks["hbm_gbs"], "traffic": None, "peak_kind": peak_kind,
            "kernel": "k_bncp_solve (one warp per problem, PGS sweeps to the residual)",
            "launch_ms": fwd_ms, "algorithmic_bytes_per_launch": alg,
            "note": "latency-bound: each warp iterates its problem in shared memory; the bytes are read once"}
    if rank == 0:
        line = {"metric": "env-steps/s", "value": value, "unit": "env-steps/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": fwd_ms, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": value / wl["published"][0], "dtype": "f64",
                "data": "synthetic (seeded legged-stance batch, the reference's shapes)",
                "config": {"workload": args.workload, "B": B, "nv": wl["nv"], "contacts": wl["nc"], "mu": wl["mu"],
                           "tol": wl["tol"], "max_iters": wl["max_iters"],
                           "l2": "flushed between timed steps (256 MiB write)", "parallelism": f"batches x{world}"},
                "baseline": {"value": wl["published"][0], "unit": "env-steps/s", "source": wl["published"][1]},
                "adjoint": {"fwd_ms": fwd_ms, "grad_ms_2dir": grad_ms, "grad_over_fwd": grad_ms / fwd_ms,
                            "reference": {"fwd_ms": wl["published_fwd_ms"], "grad_ms_2dir": wl["published_grad_ms"],
                                          "grad_over_fwd": wl["published_grad_ms"] / wl["published_fwd_ms"]}},
                "residual": {"max": float(res.max()), "median": float(res.median()), "converged": conv,
                             "iters_mean": float(s.iters.double().mean()), "iters_max": int(s.iters.max())},
                "contacts_by_label": dict(zip(("open", "stick", "slip"), labels)),
                "clocks": clk.summary(),
                "e2e": {"value": B / (e2e_ms / 1e3), "unit": "env-steps/s",
                        "h2d_bytes_per_step": int(hG.numel() * 8 + hb.numel() * 8 + hmu.numel() * 8),
                        "d2h_bytes_per_step": int(hlam.numel() * 8), "steps": K2},
                "gpu_launches": args.steps * 3, "launches_per_step": 3,
                "roofline": roof, "cpu_baseline": cpu_base}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def run_rollout(args, wl):
    """The differentiable rollout: a step is one forward rollout and its adjoint (per-substep
    checkpoints to pinned host memory, the substep recomputed and reversed on the device).
    Reports forward and backward times, their ratio, the device peak, and central differences
    per scene against the adjoint's directional derivatives."""
    import torch
    import __graft_entry__ as ge
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    ge.load_package()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    from motion_engine_b200 import rollout as RO, world as W
    S = _scenes()
    d = S.pushed_pyramids(n_scenes=wl["n_scenes"])
    w = W.BoxWorldB200(dt=wl["dt"], mu=0.5, iters=wl["iters"], substeps=wl["substeps"], warm_start=True,
                       device=str(dev))
    for i in range(len(d["half"])):
        w.add(d["half"][i], float(d["mass"][i]), d["x"][i], kin=int(d["kin"][i]), v_kin=d["v_kin"][i],
              mu=float(d["mu"][i]), scene=int(d["scene"][i]))
    w._build()
    n, NS, T = w.n, wl["n_scenes"], wl["rollout_steps"]
    ro = RO.BoxRollout(w)
    scene = torch.tensor(d["scene"], device=dev, dtype=torch.int64)
    dyn = torch.tensor(1 - d["kin"], device=dev, dtype=torch.float64)
    target = torch.tensor(d["target"], device=dev)
    hv0 = torch.tensor(d["v0"], dtype=torch.float32).pin_memory()  # fp32 inputs, float64 state
    hmu = torch.tensor(d["mu"], dtype=torch.float32).pin_memory()
    hgv, hgm, hloss = (torch.empty_like(hv0).pin_memory(), torch.empty_like(hmu).pin_memory(),
                       torch.empty((), dtype=torch.float64).pin_memory())

    def step(record=None):
        v0 = hv0.to(dev, non_blocking=True).requires_grad_(True)
        mu = hmu.to(dev, non_blocking=True).requires_grad_(True)
        if record:
            record[0].record()
        x = RO.rollout(ro, v0, mu, T)
        loss = ((x - target) ** 2).sum()
        if record:
            record[1].record()
        loss.backward()
        if record:
            record[2].record()
        hgv.copy_(v0.grad, non_blocking=True)
        hgm.copy_(mu.grad, non_blocking=True)
        hloss.copy_(loss.detach(), non_blocking=True)
        return v0.grad.detach().double(), mu.grad.detach().double()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    torch.cuda.reset_peak_memory_stats(dev)
    fwd, bwd, tot = [], [], []
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        for _ in range(args.steps):
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
            a0 = torch.cuda.Event(enable_timing=True)
            a0.record()
            gv, gm = step(ev)
            ev[3].record()
            ev[3].synchronize()
            fwd.append(ev[0].elapsed_time(ev[1]))
            bwd.append(ev[1].elapsed_time(ev[2]))
            tot.append(a0.elapsed_time(ev[3]))
        torch.cuda.synchronize()
    peak = torch.cuda.max_memory_allocated(dev)
    fwd_ms, bwd_ms, tot_ms = (float(np.mean(x)) for x in (fwd, bwd, tot))
    host_ckpt = sum(cp.state.numel() * 8 + (cp.warm_lam.numel() * 8 + cp.warm_keys.numel() * 8
                                            if cp.warm_lam is not None else 0) for cp in ro.checkpoints)
    # central differences per scene (one pair of forwards per direction serves every scene)
    rng = np.random.default_rng(11)
    v0 = hv0.to(dev).double()
    mu = hmu.to(dev).double()
    per_scene = lambda x: torch.zeros(NS, dtype=torch.float64, device=dev).index_add_(0, scene,
                                                                                     ((x - target) ** 2).sum(1))
    fd = {}
    eps = wl["fd_eps"]
    for which in ("v0", "mu"):
        dv = (torch.tensor(rng.normal(0, 1, (n, 3)), device=dev) * dyn[:, None] if which == "v0"
              else torch.zeros_like(v0))
        dm = torch.tensor(rng.normal(0, 1, n), device=dev) * dyn if which == "mu" else torch.zeros_like(mu)
        an = torch.zeros(NS, dtype=torch.float64, device=dev).index_add_(0, scene, (gv * dv).sum(1) + gm * dm)
        with torch.no_grad():
            lp = per_scene(ro.forward(v0 + eps * dv, mu + eps * dm, T, checkpoint=False))
            lm = per_scene(ro.forward(v0 - eps * dv, mu - eps * dm, T, checkpoint=False))
        f = ((lp - lm) / (2 * eps)).cpu().numpy()
        a = an.cpu().numpy()
        rel = np.abs(f - a) / np.maximum(np.maximum(np.abs(f), np.abs(a)), 1e-300)
        fd[which] = {"median_rel": float(np.median(rel)), "frac_rel_lt_1e-3": float(np.mean(rel < 1e-3)),
                     "frac_rel_lt_1e-2": float(np.mean(rel < 1e-2)), "frac_rel_lt_1e-1": float(np.mean(rel < 1e-1)),
                     "adjoint_abs_median": float(np.median(np.abs(a))), "fd_abs_median": float(np.median(np.abs(f)))}
    value = n * T / (tot_ms / 1e3)  # body-steps of forward + adjoint per second
    if rank == 0:
        line = {"metric": "body-steps/s (forward + adjoint)", "value": value, "unit": "body-steps/s",
                "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": tot_ms,
                "higher_is_better": True, "scaling": "replicas only", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded pushed pyramids, the differentiable workload's shapes)",
                "config": {"workload": args.workload, "scenes": NS, "bodies": n, "rollout_steps": T,
                           "substeps": wl["substeps"], "iters": wl["iters"],
                           "l2": "inputs larger than L2 are not needed: each rollout streams its own state"},
                "rollout": {"fwd_ms": fwd_ms, "bwd_ms": bwd_ms, "bwd_over_fwd": bwd_ms / fwd_ms,
                            "device_peak_bytes": int(peak), "host_checkpoint_bytes": int(host_ckpt),
                            "max_contacts_per_substep": int(ro.max_c)},
                "fd_check": {"eps": eps, "per_scene": fd,
                             "note": "central differences of the same float64 forward, one random direction per "
                                     "argument, compared per scene; contact sets, kept manifold points, the "
                                     "cone apex and the bias kink at zero gap make the rollout piecewise smooth"},
                "clocks": clk.summary(),
                "e2e": {"value": value, "unit": "body-steps/s",
                        "h2d_bytes_per_step": int(hv0.numel() * 4 + hmu.numel() * 4),
                        "d2h_bytes_per_step": int(hgv.numel() * 4 + hgm.numel() * 4 + 8)},
                "cpu_baseline": None}
        print(json.dumps(line), flush=True)


def _traffic(workload):
    """DRAM bytes per launch of the workload's dominant kernel, from the committed ncu summary
    (profiles/traffic.json), or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return json.load(f).get(workload)
    except Exception:
        return None


def _ncp_scene(wl):
    from motion_engine_b200 import ncp
    return ncp.BlockScene(**_scenes().ncp_lattice(n=wl["n"]))


def _ncp_cpu_worker(args_):
    """The oracle's exact-cone NCP solve of the lattice, repeated for ~budget seconds on one
    core; returns (solves, seconds)."""
    workload, budget = args_
    sys.path.insert(0, ROOT)
    import __graft_entry__ as ge
    ge.load_package()
    from oracle import oracle as O
    wl = WORKLOADS[workload]
    bs = _ncp_scene(wl)
    done, t0 = 0, time.perf_counter()
    while True:
        O.ncp_solve(bs, wl["iters"], dtype="float64")
        done += 1
        if time.perf_counter() - t0 > budget:
            break
    return done, time.perf_counter() - t0


def run_reference_ncp(args, wl):
    """--impl reference for the NCP lattice: independent replicas of the oracle's solve, one per
    host core, each for ~30 s."""
    import multiprocessing as mp
    if int(os.environ.get("RANK", "0")) != 0:
        return
    procs = max(1, min(os.cpu_count() or 1, 64))
    with mp.get_context("spawn").Pool(procs) as pool:
        res = pool.map(_ncp_cpu_worker, [(args.workload, 30.0)] * procs)
    nc = 4 * wl["n"]
    value = sum(r[0] for r in res) * nc * wl["iters"] / max(r[1] for r in res)
    line = {"impl": "reference", "metric": "contact-sweeps/s", "value": value, "unit": "contact-sweeps/s",
            "higher_is_better": True, "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "config": {"workload": args.workload, **{k: v for k, v in wl.items() if k not in ("warmup", "steps")}},
            "dtype": "f64", "data": "synthetic",
            "cpu_baseline": {"value": value, "unit": "contact-sweeps/s", "cores": procs, "kind": "port",
                             "sample": f"{sum(r[0] for r in res)} solves of {wl['iters']} sweeps over {procs} "
                                       f"independent replicas, ~30 s each (the oracle's C restatement; the "
                                       f"reference's Warp path is not installed)"},
            "e2e": {"value": value, "unit": "contact-sweeps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ncp(args, wl):
    """The exact-cone NCP solver on the reference's lattice fixture (float64).  A step solves the
    resident scene again: setup, colouring through the cache, `iters` sweeps, in CUDA events.
    With N ranks every rank solves its own replica."""
    import torch
    import __graft_entry__ as ge
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    ge.load_package()
    from motion_engine_b200 import ncp
    cpu_base = None
    if rank == 0 and not args.no_cpu_baseline:  # before the first GPU call
        n, el = _ncp_cpu_worker((args.workload, 15.0))
        cpu_base = {"value": n * 4 * wl["n"] * wl["iters"] / el, "unit": "contact-sweeps/s", "cores": 1,
                    "kind": "port", "sample": f"{n} solves of {wl['iters']} sweeps of the same scene on one host "
                                              f"core ({el:.1f} s; the oracle's C restatement)"}
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    bs = _ncp_scene(wl)
    it = wl["iters"]
    s = ncp.NCPSolverB200(bs.n_b, bs.n_c, dtype="float64", solve_blocks=wl.get("solve_blocks", 0))
    first = s.solve(bs, iters=it)  # upload, colouring (cache miss), sweeps
    # the sweeps' launch form, picked on live steps (the forms give the same bits)
    tuned = {}
    for form in (-16, 148):
        s.solve_blocks = form
        s.solve_resident(it)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(3):
            s.solve_resident(it)
        b.record()
        b.synchronize()
        tuned[form] = a.elapsed_time(b) / 3
    s.solve_blocks = min(tuned, key=tuned.get)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    for _ in range(args.warmup):
        s.solve_resident(it)
    torch.cuda.synchronize()
    times = []
    with ClockSampler(local) as clk:
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        for _ in range(args.steps):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            s.solve_resident(it)
            b.record()
            b.synchronize()
            times.append(a.elapsed_time(b))
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
    ms = float(np.mean(times))
    t = torch.tensor([ms], device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t[0])
    res = s.residual()
    nc, nb = bs.n_c, bs.n_b
    value = nc * it * world / (ms / 1e3)
    # end to end through the public solve(): host scene up, lambda and v down, every step
    K2 = 10
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(K2):
        s.solve(bs, iters=it, measure_residual=False)
    b.record()
    b.synchronize()
    e2e_ms = a.elapsed_time(b) / K2
    peaks, peak_kind = _peaks()
    alg = it * (nc * (2 * 18 + 3 + 3 + 1 + 1) * 8 + nb * 6 * 8 * 2)  # per sweep: J rows, lambda, rho, mu; bodies
    if rank == 0:
        line = {"metric": "contact-sweeps/s", "value": value, "unit": "contact-sweeps/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": value / wl["published"][0], "dtype": "f64",
                "data": "synthetic (the reference's LatticeWorld geometry, restated)",
                "config": {"workload": args.workload, "bodies": nb, "contacts": nc, "sweeps": it,
                           "colours": int(first.n_colors), "l2": "flushed between timed steps (256 MiB write)",
                           "autotuned": {"solve_blocks": s.solve_blocks,
                                         "ms_per_step": {str(k): round(v, 4) for k, v in tuned.items()}},
                           "parallelism": f"replicas x{world}"},
                "baseline": {"value": wl["published"][0], "unit": "contact-sweeps/s", "source": wl["published"][1]},
                "us_per_sweep": ms * 1e3 / it, "residual": res, "reference_residual": 7.778e-05,
                "clocks": clk.summary(),
                "e2e": {"value": nc * it / (e2e_ms / 1e3), "unit": "contact-sweeps/s",
                        "h2d_bytes_per_step": int(nc * (2 * 18 + 1 + 3 + 1) * 8 + nc * 3 * 4 + nb * (36 + 6) * 8),
                        "d2h_bytes_per_step": int(nc * 3 * 8 + nb * 6 * 8), "steps": K2},
                "gpu_launches": args.steps * 3, "launches_per_step": 3,
                "roofline": {"bound": "hbm", "achieved": alg / (ms / 1e3) / 1e9, "peak": peaks["hbm_gbs"],
                             "unit": "GB/s", "frac": alg / (ms / 1e3) / 1e9 / peaks["hbm_gbs"],
                             "traffic": _traffic(args.workload),
                             "peak_kind": peak_kind, "kernel": "k_sweeps<double> (persistent coloured PGS)",
                             "launch_ms": ms, "algorithmic_bytes_per_launch": alg},
                "cpu_baseline": cpu_base}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


# the reference's M5 receipt for its ColorCache engine: K = 16, 600 steps, vit 40, pit 10
# (reports/innovation_stack_color_cache_l4.json, legs[0]["40"]["m5"])
M5_REFERENCE = {"engine": "ColorCacheContactEngine(dims=(0.3, 0.3, 0.2), vit=40, pit=10)", "max_pen_over_R":
                0.19563645124435425, "drift_class": "bounded", "status": "PASS",
                "source": "reports/innovation_stack_color_cache_l4.json"}


def m5_quality(me, wl, dt, S):
    """The reference's M5 gate run with the workload's engine and solver settings: a vertical
    stack of 16 (0.3, 0.3, 0.2) boxes at the rest pitch 0.205 m for 600 steps
    (engine_metrics.py:265-293), penetration = max(0.205 - adjacent spacing) per step.  The plain
    Jacobi workload on unit cubes reports its own stack instead (rest pitch 1.0, ground 0.5)."""
    metrics = me.metrics
    if "stack_pitch" in wl:
        q_e = make_engine(me, wl, scene_of(wl))
        pens = []
        for _ in range(wl["steps"]):
            q_e.step(dt, S)
            pens.append(metrics.stack_penetration(q_e.xc[:, 2].cpu().numpy(), wl["stack_pitch"],
                                                  ground=wl.get("stack_ground")))
        out = dict(metrics.m5(pens), gate="the workload's own stack (rest pitch and ground), its steps from the start")
        if "pen_target_m" in wl:
            out.update(target_m=wl["pen_target_m"], meets_target=bool(out["max_pen_m"] <= wl["pen_target_m"]))
        return {"m5": out}
    if wl["engine"] in ("box", "batched"):
        q_e = me.BoxContactEngine(mu=float(np.mean(wl["mu_range"])), vit=wl["vit"], pit=wl["pit"],
                                  color_cap=wl["color_cap"])
        for k in range(16):
            q_e.add_box([0.0, 0.0, 0.101 + k * 0.205], dims=(0.3, 0.3, 0.2), density=wl["density"])
        engine = f"BoxContactEngine(vit={wl['vit']}, pit={wl['pit']}), {S} substeps"
    else:
        q_e = make_engine(me, dict(wl, density=700.0), {"centers": [[0.0, 0.0, 0.101 + k * 0.205] for k in range(16)]})
        engine = f"{type(q_e).__name__}(vit={wl['vit']}, pit={wl['pit']}), {S} substeps"
    pens = []
    for _ in range(600):
        q_e.step(dt, S)
        z = np.sort(q_e.xc[:, 2].cpu().numpy())
        pens.append(float(np.max(np.float32(0.205) - np.diff(z))))
    return {"m5": dict(metrics.m5(pens), gate="K = 16 stack of (0.3, 0.3, 0.2) boxes, rest pitch 0.205 m, 600 steps "
                                               "(engine_metrics.py:265-293)", engine=engine),
            "m5_reference": M5_REFERENCE}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--warmup", type=int, default=None)
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--islands", choices=("on", "off"), default=None,
                    help="box workloads: the island solve on or off (default: the workload's setting)")
    ap.add_argument("--no-parity", action="store_true",
                    help="skip the oracle digest at the parity step (it runs in spawned processes)")
    ap.add_argument("--save-state", default=None,
                    help="write the body state after the set-up steps to this .npz (profiling aid)")
    ap.add_argument("--load-state", default=None,
                    help="start from a state written by --save-state instead of running the set-up steps "
                         "(profiling aid: short runs with few launches before the captured ones)")
    args = ap.parse_args()
    wl = dict(WORKLOADS[args.workload])
    if args.islands is not None:
        wl["islands"] = args.islands == "on"
    if args.steps is None:
        args.steps = wl["steps"]
    if args.warmup is None:
        args.warmup = wl["warmup"]
    args.warmup = max(args.warmup, 3)
    import __graft_entry__ as ge
    if wl["engine"] == "admm":
        return run_reference_admm(args, wl) if args.impl == "reference" else run_admm(args, wl)
    if wl["engine"] == "bncp":
        ge.load_package()
        return run_reference_adjoint(args, wl) if args.impl == "reference" else run_adjoint(args, wl)
    if wl["engine"] == "ncp":
        ge.load_package()
        return run_reference_ncp(args, wl) if args.impl == "reference" else run_ncp(args, wl)
    if wl["engine"] == "rollout":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no rollout adjoint (its "
                              "BoxWorld steps on the host with a Warp solver that is not installed)"}), flush=True)
            return None
        return run_rollout(args, wl)
    if args.impl == "reference":
        ge.load_package()
        return run_reference_batched(args, wl) if wl["engine"] == "batched" else run_reference(args, wl)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    ge.load_package()
    scene = scene_of(wl)
    n_job = wl.get("n", 0) * world  # replicas: every rank runs the whole workload
    if wl["engine"] == "batched":  # scenes sharded over the ranks, no data-path collective
        counts = [len(sc["centers"]) for sc in scene["scenes"]]
        n_job = sum(counts)
        mine = partition_scenes(counts, world)[rank]
        scene = {"scenes": [scene["scenes"][i] for i in mine]}
    # the oracle's digest at the parity step, computed beside the GPU run (rank 0; spawned before
    # the first GPU call)
    parity_steps = wl.get("parity_steps") or (wl["preroll"] if wl["preroll"] > 0 else args.warmup)
    parity = None
    if rank == 0 and not args.load_state and not args.no_parity:
        parity = ParityCheck(args, wl, parity_steps, mine if wl["engine"] == "batched" else None)
    cpu_base = None
    do_cpu = rank == 0 and not args.no_cpu_baseline
    if do_cpu and wl["engine"] not in ("box", "batched"):
        ge.load_package()
        v, n, el = cpu_baseline_sample(wl, scene)  # before the first GPU call
        cpu_base = {"value": v, "unit": "body-steps/s", "cores": 1, "kind": "port",
                    "sample": f"{n} steps of the same workload after the same warm-up on one host core "
                              f"({el:.1f} s; the oracle restatement, not the reference's Warp CPU path)"}
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    me = ge.load_package()
    dev = torch.device("cuda", local)

    def barrier():
        if world > 1:
            dist.barrier()

    e = make_engine(me, wl, scene)
    dt, S = wl["dt"], wl["substeps"]
    gpu_digest = None

    def gpu_state_digest():
        st = e.get_state_packed().numpy()
        xc, q, v, w = st[0, :, :3], st[1], st[2, :, :3], st[3, :, :3]
        if wl["engine"] != "batched":
            return state_digest(xc, q, v, w)
        return combine_digests([state_digest(xc[sl], q[sl], v[sl], w[sl])
                                for sl in (e.scene_slice(k) for k in range(len(scene["scenes"])))])

    n_done = 0
    if args.load_state:
        d = np.load(args.load_state)
        e.set_body_state(d["xc"], d["q"], d["v"], d["w"])
    else:
        for _ in range(wl["preroll"]):
            e.step(dt, S)
            n_done += 1
            if n_done == parity_steps and parity is not None:
                gpu_digest = gpu_state_digest()
    if args.save_state:
        torch.cuda.synchronize()
        np.savez(args.save_state, xc=e.xc[:, :3].cpu().numpy(), q=e.q.cpu().numpy(), v=e.v[:, :3].cpu().numpy(),
                 w=e.w[:, :3].cpu().numpy())
    for _ in range(args.warmup):
        e.step(dt, S)
        n_done += 1
        if n_done == parity_steps and parity is not None:
            gpu_digest = gpu_state_digest()
    tuned = None
    if wl["engine"] in ("batched", "color_cache"):
        # the solve's launch form, picked on live (untimed) steps after the warm-up, then one more
        # untimed step on the chosen form (its graph capture)
        best, times = me.autotune(e, dt, S, steps=4)
        form = lambda k: "scenes" if k == me._lib.SOLVE_SCENES else str(k)
        tuned = {"solve_blocks": form(best), "ms_per_step": {form(k): round(v, 4) for k, v in times.items()}}
        e.step(dt, S)
    e.check_errors()
    torch.cuda.synchronize()
    start_state = None
    if do_cpu and wl["engine"] in ("box", "batched"):
        start_state = (e.xc[:, :3].cpu().numpy(), e.q.cpu().numpy(), e.v[:, :3].cpu().numpy(),
                       e.w[:, :3].cpu().numpy())
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MiB > 126 MB L2
    stream = torch.cuda.current_stream()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    counts = []
    barrier()
    torch.cuda.synchronize()
    depth, hdrs = [], []  # per timed step, on the device, outside the events: deepest contact, counters
    with ClockSampler(local) as clk:
        for k in range(args.steps):
            flush.fill_(float(k))
            evs[k][0].record(stream)
            e.step(dt, S)
            evs[k][1].record(stream)
            depth.append(e.max_depth_device())
            hdrs.append(e.header.clone())
        torch.cuda.synchronize()
        barrier()
    ms = sum(a.elapsed_time(b) for a, b in evs)
    depth = torch.stack(depth).cpu().numpy().astype(np.float64)
    hdrs = torch.stack(hdrs).cpu().numpy()
    colours_timed = hdrs[:, me._lib.HEADER_FIELDS.index("n_colors")]
    h_end = e.check_errors()
    launches_per_step = max(e.kernels_per_step.values()) if e.kernels_per_step else 0

    # end to end through the public API with the state in pinned host memory (one packed copy
    # each way: positions, quaternions, velocities, angular velocities)
    N = e.N
    hstate = torch.empty((4, N, 4), dtype=torch.float32, pin_memory=True)
    e.get_state_packed(hstate)
    torch.cuda.synchronize()
    e2e_start = hstate.clone()  # the engine-handle leg starts from the same state
    e2e_ms = 0.0
    K2 = max(min(args.steps, 100) // 2, 3)
    colors = []
    for k in range(K2):
        flush.fill_(float(k))
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        e.set_state_packed(hstate)
        e.step(dt, S)
        e.get_state_packed(hstate)
        b.record(stream)
        b.synchronize()
        e2e_ms += a.elapsed_time(b)
        colors.append(e.header_dict()["n_colors"])
    e.check_errors()
    bytes_io = hstate.numel() * 4
    # the same loop through the C ABI's engine handle (library-owned device memory)
    cabi_ms = cabi_e2e(me, wl, scene, e2e_start, flush, stream, K2) if wl["engine"] == "box" else 0.0

    per_scene = None
    if wl["engine"] == "batched":
        per_scene = per_scene_sequential(me, wl, scene["scenes"], e, dt, S, stream)

    # the dominant kernel (the persistent chunk solve), timed live on its launching stream
    solve_ms, solve_bytes, stage_ms = [], [], {}
    if hasattr(e, "profile_substep"):
        for _ in range(8):
            st = e.profile_substep(dt / S)
            for kk, vv in st.items():
                stage_ms[kk] = stage_ms.get(kk, 0.0) + vv / 8
            solve_ms.append(st["solve"])
            solve_bytes.append(e.solve_bytes())
        e.check_errors()
    t = torch.tensor([ms, e2e_ms, cabi_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms, e2e_ms, cabi_ms = float(t[0]), float(t[1]), float(t[2])
    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return
    if do_cpu and wl["engine"] == "batched":
        sl = [e.scene_slice(k) for k in range(len(scene["scenes"]))]
        v, nsc, el = batched_cpu_sample(wl, scene["scenes"], [tuple(a[x] for a in start_state) for x in sl])
        cpu_base = {"value": v, "unit": "body-steps/s", "cores": 1, "kind": "port",
                    "sample": f"one step of each of the first {nsc} scenes from the GPU's state of that scene at the "
                              f"start of the timed region, on one host core ({el:.1f} s of stepping; the oracle "
                              f"restatement, not the reference's Warp CPU path)"}
    if do_cpu and wl["engine"] == "box":
        v, n, el = cpu_baseline_sample(wl, scene, state=start_state)
        cpu_base = {"value": v, "unit": "body-steps/s", "cores": 1, "kind": "port",
                    "sample": f"{n} steps of the same workload from the GPU's body state at the start of the timed "
                              f"region, on one host core ({el:.1f} s; the oracle restatement, not the reference's "
                              f"Warp CPU path)"}
    # quality beside the time: the reference's M5 gate (engine_metrics.py:265-293)
    quality = m5_quality(me, wl, dt, S)
    if wl["engine"] in ("box", "batched"):
        d_last = e.kept_contacts()["spen"].astype(np.float64)
        quality["pile"] = {
            "max_depth_timed_m": float(depth.max()),
            "depth_last_step_m": {"p50": float(np.percentile(d_last, 50)), "p99": float(np.percentile(d_last, 99)),
                                  "max": float(d_last.max())},
            "contacts_deeper_than_R_over_2": int((d_last > 0.5 * me.metrics.R).sum()), "contacts": int(len(d_last)),
            "note": "depths of the solved contacts of the pile; boxes dropped from up to 10 m move ~6 cm per "
                    "substep before their first contact, so a few interpenetrate (discrete SAT, no swept test: "
                    "the oracle's SAT, restated from the reference's, gives the same depths bit for bit)"}
    parity_line = parity.result(gpu_digest) if parity is not None else None
    peaks, peak_kind = _peaks()
    value = n_job * args.steps / (ms / 1e3)
    roof = None
    if solve_ms:
        avg_ms = float(np.mean(solve_ms))
        avg_b = float(np.mean([b_["bytes"] for b_ in solve_bytes]))
        achieved = avg_b / (avg_ms / 1e3) / 1e9
        traffic = None
        tf = os.path.join(ROOT, "profiles", "traffic.json")
        if os.path.exists(tf):
            try:
                traffic = json.load(open(tf)).get(args.workload)
            except Exception:
                traffic = None
        roof = {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / peaks["hbm_gbs"], "traffic": traffic, "peak_kind": peak_kind,
                "kernel": ("k_island_solve (one thread per island; b2c_color_solve with its record gather and "
                           "impulse scatter)" if wl["engine"] == "island" else
                           "k_color_solve (persistent chunk solve, one launch per substep)"),
                "launch_ms": avg_ms, "algorithmic_bytes_per_launch": avg_b, "counts": solve_bytes[-1]}
    elif wl["engine"] == "jacobi":  # the iteration launches of one substep, timed after the timed region
        j_ms, j_b, j_counts = e.solve_sample(dt / S)
        achieved = j_b / (j_ms / 1e3) / 1e9
        traffic = None
        tf = os.path.join(ROOT, "profiles", "traffic.json")
        if os.path.exists(tf):
            try:
                traffic = json.load(open(tf)).get(args.workload)
            except Exception:
                traffic = None
        roof = {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / peaks["hbm_gbs"], "traffic": traffic, "peak_kind": peak_kind,
                "kernel": "b2c_jacobi_solve: vit x (k_jacobi_velocity + k_jacobi_apply) + pit x (k_jacobi_position + "
                          "k_jacobi_apply), one substep's iterations on the final state",
                "launch_ms": j_ms, "algorithmic_bytes_per_launch": j_b, "counts": j_counts}
    cfg = {"workload": args.workload, "bodies": n_job if wl["engine"] == "batched" else wl["n"], "substeps": S,
           "vit": wl["vit"], "pit": wl["pit"], "dt": dt, "setup_steps": wl["preroll"],
           "l2": "flushed between timed steps (256 MiB write)",
           "parallelism": f"scenes sharded x{world} (LPT)" if wl["engine"] == "batched" else f"replicas x{world}"}
    if wl["engine"] == "batched":
        cfg.update(scenes=wl["n_scenes"], bodies_per_scene=[wl["nmin"], wl["nmax"]], edge=wl["edge"],
                   mu=wl["mu_range"], density=wl["density"], heavy="10 % of each scene at 100 x density",
                   color_cap=wl["color_cap"], autotuned=tuned)
    if tuned is not None and wl["engine"] != "batched":
        cfg.update(autotuned=tuned)
    if wl["engine"] == "box":
        cfg.update(edge=wl["edge"], volume=wl["box"], mu=wl["mu_range"], density=wl["density"],
                   color_cap=wl["color_cap"], contacts="SAT box/plane + box/box, margin 2e-3",
                   island_solve=bool(wl.get("islands", False)))
        if wl.get("islands"):
            cfg.update(islands={"count": e.island_count, "max_pairs": e.max_island_pairs,
                                "island_kernel_ran": bool(e.island_solve_active)})
    line = {"metric": "body-steps/s", "value": value, "unit": "body-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "strong" if wl["engine"] == "batched" else "weak",
            "vs_baseline": value / wl["published"][0] if "published" in wl else None, "dtype": "f32",
            "data": "synthetic (seeded scene builders)", "config": cfg,
            "clocks": clk.summary(),
            "e2e": {"value": n_job * K2 / (e2e_ms / 1e3), "unit": "body-steps/s",
                    "h2d_bytes_per_step": bytes_io, "d2h_bytes_per_step": bytes_io, "steps": K2},
            "gpu_launches": launches_per_step * args.steps, "launches_per_step": launches_per_step,
            "roofline": roof, "cpu_baseline": cpu_base, "stage_ms": stage_ms, "last_step": h_end,
            "quality": quality, "parity": parity_line,
            "colors_timed_steps": {"max": int(colours_timed.max()), "mean": float(colours_timed.mean())},
            "colors_e2e_steps": {"max": max(colors), "mean": float(np.mean(colors))}}
    if cabi_ms > 0:
        line["e2e_cabi"] = {"value": n_job * K2 / (cabi_ms / 1e3), "unit": "body-steps/s",
                            "h2d_bytes_per_step": bytes_io, "d2h_bytes_per_step": bytes_io, "steps": K2,
                            "calls": "b2c_set_state_packed, b2c_step, b2c_get_state_packed on a b2c_create handle"}
    if "published" in wl:
        line["baseline"] = {"value": wl["published"][0], "unit": "body-steps/s", "source": wl["published"][1]}
    if per_scene is not None:
        line["per_scene_sequential"] = per_scene
        line["batched_over_sequential"] = (N * args.steps / (ms / 1e3)) / per_scene["value"]
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
