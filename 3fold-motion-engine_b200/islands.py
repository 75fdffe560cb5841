"""Island partition of a pair graph on the device: ``partition_pairs``
(contact_engine_gpu_island_solve.py:7-34) behind the reference's signature.

The island solve of ``IslandSolveContactEngine`` runs the same partition inside its captured
step; this function exposes it for a caller that holds pair arrays on the host, as the
reference's host function does.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib


def _check(a, b, mass, order):
    """The reference's argument checks (contact_engine_gpu_island_solve.py:8-16), in its order
    and with its messages."""
    if a.ndim != 1 or b.shape != a.shape or order.shape != a.shape or mass.ndim != 1:
        raise ValueError("Invalid partition shapes")
    if not all(np.issubdtype(x.dtype, np.integer) for x in (a, b, order)):
        raise ValueError("Integer pair indices required")
    if not np.isfinite(mass).all() or np.any(mass < 0):
        raise ValueError("Invalid inverse masses")
    n = len(mass)
    if np.any(a < 0) or np.any(a >= n) or np.any(b < -1) or np.any(b >= n):
        raise ValueError("Invalid pair endpoints")
    if not np.array_equal(np.sort(order), np.arange(len(a))):
        raise ValueError("Order must be a permutation")


def partition_pairs(a, b, inverse_mass, order, device="cuda"):
    """Group the pairs (a[p], b[p]) into islands of dynamic bodies (inverse mass > 0).

    Returns (packed, starts, counts) as int32 arrays: ``packed[starts[i]:starts[i]+counts[i]]``
    are the pair indices of island i, in the order they appear in ``order``; islands are
    sorted by their smallest body, and a pair without a dynamic body is an island of its own,
    after all others (keyed len(inverse_mass) + pair).  Computed by ``b2c_island_partition``
    on the device."""
    a = np.asarray(a)
    b = np.asarray(b)
    mass = np.asarray(inverse_mass)
    order = np.asarray(order)
    _check(a, b, mass, order)
    P, N = len(a), len(mass)
    if P == 0:
        e = np.zeros(0, np.int32)
        return e, e.copy(), e.copy()
    if not torch.cuda.is_available():
        raise RuntimeError("partition_pairs: the island partition runs on the GPU (b2c_island_partition); "
                           "no CUDA device is available")
    L = _lib.load()
    dev = torch.device(device)
    i32 = lambda x: torch.from_numpy(np.ascontiguousarray(x, dtype=np.int32)).to(dev)
    ta, tb, to = i32(a), i32(b), i32(order)
    # the partition only asks whether a body is dynamic: pass that exactly, whatever the dtype
    tm = torch.from_numpy((mass > 0).astype(np.float32)).to(dev)
    work = torch.zeros(int(L.b2c_island_work_ints(N, P)), dtype=torch.int32, device=dev)
    packed = torch.zeros(P, dtype=torch.int32, device=dev)
    starts = torch.zeros(P, dtype=torch.int32, device=dev)
    counts = torch.zeros(P, dtype=torch.int32, device=dev)
    info = torch.zeros(4, dtype=torch.int32, device=dev)
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    s = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    _lib.check(L.b2c_island_partition(p(ta), p(tb), p(tm), p(to), P, N, p(work), p(packed), p(starts), p(counts),
                                      p(info), s), "b2c_island_partition")
    n = int(info[0].item())
    return packed.cpu().numpy(), starts[:n].cpu().numpy(), counts[:n].cpu().numpy()
