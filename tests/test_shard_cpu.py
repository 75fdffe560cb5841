"""Scene sharding of the batched form over ranks, on CPU: two gloo ranks each advance their LPT
share of the scenes (the oracle stands in for a GPU), all-gather the results, and the union
equals one process advancing every scene -- every scene on exactly one rank, no data-path
exchange needed."""
import importlib
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import __graft_entry__ as ge

STEPS = 20


def _scenes():
    ge.load_package()
    return importlib.import_module("motion_engine_b200.scenes").batched_scenes(n_scenes=7, nmin=4, nmax=40, seed_n=3)


def _advance(sc):
    from oracle import oracle as O
    o = O.BoxOracle(mu=0.55, vit=6, pit=4)
    for c, d, de, m in zip(sc["centers"], sc["dims"], sc["density"], sc["mu"]):
        o.add_box(c, dims=d, density=de, mu=m)
    for _ in range(STEPS):
        o.step(1 / 240, 2)
    return o.body_state()[0]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        me = ge.load_package()
        scenes = _scenes()
        mine = me.partition_scenes([len(s["centers"]) for s in scenes], world)[rank]
        out = {i: _advance(scenes[i]) for i in mine}
        gathered = [None] * world
        dist.all_gather_object(gathered, out)
        if rank == 0:
            q.put(gathered)
    finally:
        dist.destroy_process_group()


def test_partition_is_lpt_and_complete():
    me = ge.load_package()
    counts = [5, 100, 7, 60, 60, 3, 41]
    parts = me.partition_scenes(counts, 3)
    assert sorted(i for p in parts for i in p) == list(range(len(counts)))
    loads = [sum(counts[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(counts)


def test_two_ranks_cover_every_scene_once():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    gathered = q.get(timeout=240)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    union = {}
    for part in gathered:
        assert not set(part) & set(union)
        union.update(part)
    scenes = _scenes()
    assert sorted(union) == list(range(len(scenes)))
    for i, sc in enumerate(scenes):
        np.testing.assert_array_equal(union[i], _advance(sc))
