"""The contact-scene-v1 reader (scenes_v1.py) against the reference's own loader
(data/ncp/loader.py rebuild, run here by tests/golden/make_scenes_v1_golden.py) and against the
package's published spectral bounds (scenes/table.json), without a GPU."""
import gzip
import importlib
import json
import os

import numpy as np
import pytest

from conftest import ROOT

GOLD = os.path.join(ROOT, "tests", "golden", "scenes_v1_golden.npz")
FILES = os.path.join(ROOT, "tests", "golden", "scenes_v1.json.gz")


@pytest.fixture(scope="module")
def sv1(me):
    return importlib.import_module("motion_engine_b200.scenes_v1")


@pytest.fixture(scope="module")
def package():
    with gzip.open(FILES, "rt") as f:
        return {int(k): v for k, v in json.load(f).items()}


def test_rebuild_equals_the_reference_loader(sv1, package):
    g = np.load(GOLD)
    assert len(package) == 19
    for i, raw in sorted(package.items()):
        sc = sv1.read_scene(raw)
        k = f"s{i:02d}"
        assert sc.index == i and sc.J.shape == tuple(g[f"{k}/shape"])
        for f in ("b", "mu", "eta"):
            assert np.array_equal(getattr(sc, f), g[f"{k}/{f}"]), (i, f)
        W = sc.delassus()
        scale = max(1.0, float(np.abs(W).max()))
        if f"{k}/G" in g:
            assert np.abs(W - g[f"{k}/G"]).max() <= 1e-14 * scale, i
        r = np.random.default_rng(100 + i).standard_normal(W.shape[0])
        assert np.abs(W @ r - g[f"{k}/Gr"]).max() <= 1e-12 * scale * np.abs(r).sum() / len(r) * 10, i
        assert abs(np.linalg.norm(W) - g[f"{k}/G_fro"]) <= 1e-13 * g[f"{k}/G_fro"], i
        assert abs(np.trace(W) - g[f"{k}/G_trace"]) <= 1e-13 * abs(g[f"{k}/G_trace"]), i


def test_spectral_bounds_equal_the_package_table(sv1, package):
    g = np.load(GOLD)
    for i, raw in sorted(package.items()):
        sc = sv1.read_scene(raw)
        W = sc.delassus()
        if W.shape[0] > 2200:
            continue
        ev = np.linalg.eigvalsh(W)
        lmax = ev.max()
        pos = ev[ev > 1e-10 * lmax]
        assert abs(lmax - g["table/lambda_max"][i]) <= 1e-9 * lmax, i
        assert abs(pos.min() - g["table/lambda_min_pos"][i]) <= 1e-7 * g["table/lambda_min_pos"][i], i


def test_block_scenes_carry_the_same_problem(sv1, me, package):
    ncp = importlib.import_module("motion_engine_b200.ncp")
    for i, raw in sorted(package.items()):
        sc = sv1.read_scene(raw)
        if sc.model != "body_contacts" or np.any(sc.eta):
            with pytest.raises(ValueError):
                sv1.block_scene(sc)
            continue
        bs = sv1.block_scene(sc)
        assert isinstance(bs, ncp.BlockScene)
        W = sc.delassus()
        assert np.abs(bs.delassus() - W).max() <= 1e-13 * max(1.0, np.abs(W).max()), i
        assert np.array_equal(bs.rhs(), sc.b), i


def test_reader_rejects_other_schemas(sv1, package):
    raw = dict(package[0], schema="contact-scene-v0")
    with pytest.raises(ValueError):
        sv1.read_scene(raw)
