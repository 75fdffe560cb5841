"""CPU oracle of the island partition -- TEST INFRASTRUCTURE ONLY.

Only the tests may import this module.  It restates ``partition_pairs``
(src/motion_engine/contact_engine_gpu_island_solve.py:7-34) in plain Python so that the
device partition (``b2c_island_partition``, the island solve's partition) can be checked:

* two bodies share an island when a chain of pairs links them and both ends of every link are
  dynamic (inverse mass > 0) -- line 22: only pairs with y >= 0 and both masses > 0 unite;
* an island is keyed by its smallest body (the reference's union keeps min(u, v) as the root,
  line 24), a pair by its first dynamic endpoint's island, and a pair without a dynamic endpoint
  by len(mass) + p (line 28);
* islands come out in key order, each island's pairs in the order they appear in ``order``
  (lines 27-33).

The components are found here by a breadth-first search over the dynamic-dynamic links (not
the reference's union-find), labelled with their smallest body.
"""
from __future__ import annotations

from collections import deque

import numpy as np


def partition_pairs(a, b, inverse_mass, order):
    a = [int(x) for x in np.asarray(a)]
    b = [int(x) for x in np.asarray(b)]
    mass = np.asarray(inverse_mass, dtype=np.float64)
    order = [int(x) for x in np.asarray(order)]
    n = len(mass)
    dyn = [bool(m > 0) for m in mass]
    adj = [[] for _ in range(n)]
    for x, y in zip(a, b):
        if y >= 0 and dyn[x] and dyn[y]:
            adj[x].append(y)
            adj[y].append(x)
    label = [-1] * n
    for s in range(n):  # ascending: the first unvisited body of a component is its smallest
        if label[s] >= 0:
            continue
        label[s] = s
        q = deque([s])
        while q:
            u = q.popleft()
            for v in adj[u]:
                if label[v] < 0:
                    label[v] = s
                    q.append(v)
    groups = {}
    for p in order:
        x, y = a[p], b[p]
        if dyn[x]:
            k = label[x]
        elif y >= 0 and dyn[y]:
            k = label[y]
        else:
            k = n + p
        groups.setdefault(k, []).append(p)
    keys = sorted(groups)
    counts = np.array([len(groups[k]) for k in keys], np.int32)
    starts = (np.concatenate([[0], np.cumsum(counts)[:-1]]).astype(np.int32) if len(counts)
              else np.zeros(0, np.int32))
    packed = np.array([p for k in keys for p in groups[k]], np.int32)
    return packed, starts, counts
