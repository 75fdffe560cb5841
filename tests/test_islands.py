"""Island partition (contact_engine_gpu_island_solve.py:7-34) without a GPU: the oracle against
the reference's own known answers (tests/test_island_partition.py of the reference) and against
scipy's connected components, and the product wrapper's argument checks, which run on the host
before any device call."""
import numpy as np
import pytest

from oracle.oracle_islands import partition_pairs as oracle_partition


def _groups(packed, starts, counts):
    return [packed[s:s + c].tolist() for s, c in zip(starts, counts)]


def test_oracle_known_answers_shared_static_and_order():
    # a static body shared by two dynamic ones does not join them; pairs keep the given order
    a = np.array([0, 1, 0, 2]); b = np.array([3, 3, 1, -1]); mass = np.array([1., 1., 1., 0.])
    assert _groups(*oracle_partition(a, b, mass, np.array([3, 1, 0, 2]))) == [[1, 0, 2], [3]]
    packed, starts, counts = oracle_partition(a[:2], b[:2], mass, np.array([1, 0]))
    assert counts.tolist() == [1, 1]


def test_oracle_known_answers_all_static_and_empty():
    a = np.array([0, 1]); b = np.array([1, 0])
    assert oracle_partition(a, b, np.zeros(2), np.array([1, 0]))[2].tolist() == [1, 1]
    e = np.zeros(0, np.int32)
    assert all(len(x) == 0 for x in oracle_partition(e, e, np.ones(2), e))


@pytest.mark.parametrize("seed", range(5))
def test_oracle_components_match_scipy(seed):
    from scipy.sparse import coo_matrix
    from scipy.sparse.csgraph import connected_components
    rng = np.random.default_rng(seed)
    n, P = 300, 400
    mass = np.where(rng.random(n) < 0.15, 0.0, rng.uniform(0.1, 2.0, n))
    a = rng.integers(0, n, P)
    b = rng.integers(-1, n, P)
    order = rng.permutation(P)
    packed, starts, counts = oracle_partition(a, b, mass, order)
    assert sorted(packed.tolist()) == list(range(P))
    dyn = mass > 0
    link = (b >= 0) & dyn[a] & dyn[np.maximum(b, 0)]
    g = coo_matrix((np.ones(link.sum()), (a[link], b[link])), shape=(n, n))
    _, comp = connected_components(g, directed=False)
    pos = np.empty(P, np.int64)
    pos[order] = np.arange(P)
    for s, c in zip(starts, counts):
        grp = packed[s:s + c]
        assert np.all(np.diff(pos[grp]) > 0), "pairs of an island keep the given order"
        owner = [comp[x] if dyn[x] else (comp[y] if y >= 0 and dyn[y] else -1 - p)
                 for p, x, y in ((p, a[p], b[p]) for p in grp)]
        assert len(set(owner)) == 1, "one island per component"
    keys = []
    for s, c in zip(starts, counts):
        p = packed[s]
        x, y = a[p], b[p]
        if dyn[x]:
            keys.append(np.flatnonzero(comp == comp[x]).min())
        elif y >= 0 and dyn[y]:
            keys.append(np.flatnonzero(comp == comp[y]).min())
        else:
            keys.append(n + p)
    assert keys == sorted(keys) and len(set(keys)) == len(keys)


def test_product_partition_checks_arguments_on_the_host(me):
    a = np.array([0, 1]); b = np.array([1, 0]); order = np.array([1, 0])
    with pytest.raises(ValueError, match="permutation"):
        me.partition_pairs(a, b, np.ones(2), np.array([0, 0]))
    with pytest.raises(ValueError, match="endpoints"):
        me.partition_pairs(a, np.array([-2, 0]), np.ones(2), order)
    with pytest.raises(ValueError, match="shapes"):
        me.partition_pairs(a, b[:1], np.ones(2), order)
    with pytest.raises(ValueError, match="Integer"):
        me.partition_pairs(a.astype(float), b, np.ones(2), order)
    with pytest.raises(ValueError, match="inverse masses"):
        me.partition_pairs(a, b, np.array([1.0, -1.0]), order)
    e = np.zeros(0, np.int32)
    assert all(len(x) == 0 for x in me.partition_pairs(e, e, np.ones(2), e))


def test_oracle_equals_the_reference_partition():
    """The reference's own partition_pairs, run on seeded random graphs
    (tests/golden/make_islands_golden.py): the oracle returns the same arrays."""
    import os
    from conftest import ROOT
    g = np.load(os.path.join(ROOT, "tests", "golden", "islands_golden.npz"))
    for k in range(int(g["n_cases"])):
        args = [g[f"c{k}/{x}"] for x in ("a", "b", "mass", "order")]
        got = oracle_partition(*args)
        for arr, name in zip(got, ("packed", "starts", "counts")):
            assert np.array_equal(arr, g[f"c{k}/{name}"]), (k, name)
