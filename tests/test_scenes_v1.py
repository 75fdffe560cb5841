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


def test_hdf5_copies_equal_the_json_reconstruction(sv1, package, tmp_path):
    """The package's own acceptance (data/ncp/loader.py verify): each scene's HDF5 copy, read by
    hdf5_lite, equals its JSON reconstruction -- W to 1e-15 relative (Frobenius), q to 1e-15, mu
    exactly -- on the fifteen small scenes carried in tests/golden/scenes_v1_hdf5.zip."""
    import zipfile
    with zipfile.ZipFile(os.path.join(ROOT, "tests", "golden", "scenes_v1_hdf5.zip")) as z:
        z.extractall(tmp_path)
        names = sorted(z.namelist())
    assert len(names) == 15
    for name in names:
        i = int(name[:2])
        r = sv1.verify(sv1.read_scene(package[i]), os.path.join(tmp_path, name))
        assert r["W_rel_fro"] <= 1e-15 and r["q_abs"] <= 1e-15 and r["mu_abs"] == 0.0, (i, r)


def test_hdf5_reader_structure(me, tmp_path):
    import zipfile
    hl = importlib.import_module("motion_engine_b200.hdf5_lite")
    with zipfile.ZipFile(os.path.join(ROOT, "tests", "golden", "scenes_v1_hdf5.zip")) as z:
        z.extract("00.hdf5", tmp_path)
    f = hl.H5File(os.path.join(tmp_path, "00.hdf5"))
    assert f.keys("/") == ["fclib_local"]
    assert f.keys("fclib_local/W") == ["i", "m", "n", "nz", "nzmax", "p", "x"]
    assert f.attrs("fclib_local/W")["symmetric_packed"] == 1
    n, nzmax = int(f["fclib_local/W/n"][0]), int(f["fclib_local/W/nzmax"][0])
    assert n == 12 and nzmax == n * (n + 1) // 2 == len(f["fclib_local/W/x"])
    with pytest.raises(ValueError):
        hl.H5File(os.path.join(ROOT, "tests", "golden", "scenes_v1.json.gz"))
