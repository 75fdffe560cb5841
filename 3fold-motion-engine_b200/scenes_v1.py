"""Reader of the reference's `contact-scene-v1` contact-problem package (data/ncp/scenes/NN.json,
read by its data/ncp/loader.py), and its problems handed to the device solvers.

A scene describes one contact problem  u = W lambda + q  with  W = J M^-1 J^T + diag(eta)
(eta repeated over a contact's three rows), q = b and per-contact friction mu, either through
bodies and contacts (`model = "body_contacts"`: per contact a frame (normal, t1, t2), its two
bodies a, b (-1 = the static world) and lever arms; per body its inverse mass and inertia, or a
full inverse-mass block) or through the operator itself (`model = "operator"`: J and M^-1,
base64 little-endian float64 or lists).  The HDF5 copy of each scene (the compact FCLIB
local-problem layout: W's lower triangle in CSC under /fclib_local/W with symmetric_packed = 1,
q and mu under /fclib_local/vectors) is read by ``read_hdf5_problem`` through ``hdf5_lite`` (h5py
is not installed in this image); ``verify`` compares the two as the package's loader does.

Device solves:
* body-contact scenes without compliance (eta = 0) become a ``ncp.BlockScene`` (3-DOF point
  bodies embedded as 6-DOF bodies with no rotational mobility; v_free = 0 and the bias = q, so
  u = J M^-1 J^T lambda + q) for the exact-cone ``NCPSolverB200``;
* operator scenes of at most 8 contacts and 32 velocities go to ``badmm.BatchProxADMM`` with
  q passed as the free contact velocity.
"""
from __future__ import annotations

import base64
import json
import os
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

SCHEMA = "contact-scene-v1"


@dataclass
class ContactSceneV1:
    index: int
    name: str
    model: str
    n_b: int
    n_c: int
    dof: int
    dt: float
    mu: np.ndarray            # (n_c,)
    b: np.ndarray             # (3 n_c,) q, rows n, t1, t2 per contact
    eta: np.ndarray           # (n_c,) diagonal compliance per contact
    J: np.ndarray             # (3 n_c, n_v)
    Minv: np.ndarray          # (n_v, n_v)
    body_pairs: Optional[np.ndarray] = None   # (n_c, 2) for body-contact scenes, -1 = static
    provenance: Optional[str] = None
    raw: dict = field(default_factory=dict, repr=False)

    def delassus(self) -> np.ndarray:
        """W = J M^-1 J^T + diag(eta per row), float64 (host; for checks and small problems)."""
        W = self.J @ self.Minv @ self.J.T
        if np.any(self.eta):
            W = W + np.diag(np.repeat(self.eta, 3))
        return W


def _f8(s: str, shape) -> np.ndarray:
    return np.frombuffer(base64.b64decode(s), dtype="<f8").astype(np.float64).reshape(shape)


def _cross_rows(r: np.ndarray, D: np.ndarray) -> np.ndarray:
    """Row k: r x D[k] (the angular part of a contact row acting through lever arm r)."""
    return np.stack([np.cross(r, D[k]) for k in range(D.shape[0])])


def _body_contacts(scene: dict):
    bodies, contacts = scene["bodies"], scene["contacts"]
    dof = int(scene["dof"])
    if dof not in (3, 6):
        raise ValueError(f"contact-scene-v1: body dof {dof} (3 or 6 expected)")
    nb, nc = len(bodies), len(contacts)
    Minv = np.zeros((dof * nb, dof * nb))
    for bd in bodies:
        i = int(bd["id"])
        sl = slice(dof * i, dof * i + dof)
        if "minv_block" in bd:
            Minv[sl, sl] = np.asarray(bd["minv_block"], float).reshape(dof, dof)
        else:
            im = float(bd["inv_mass"])
            diag = [im] * 3 if dof == 3 else [im] * 3 + [float(x) for x in bd["inv_inertia"]]
            Minv[sl, sl] = np.diag(diag)
    J = np.zeros((3 * nc, dof * nb))
    pairs = np.full((nc, 2), -1, np.int32)
    for ct in contacts:
        c = int(ct["id"])
        D = np.array([ct["normal"], ct["t1"], ct["t2"]], float)
        rows = slice(3 * c, 3 * c + 3)
        for side, sign, lever in ((int(ct["a"]), 1.0, "lever_a"), (int(ct["b"]), -1.0, "lever_b")):
            if side < 0:
                continue
            J[rows, dof * side:dof * side + 3] = sign * D
            if dof == 6:
                J[rows, dof * side + 3:dof * side + 6] = sign * _cross_rows(np.asarray(ct[lever], float), D)
        pairs[c] = (int(ct["a"]), int(ct["b"]))
    return J, Minv, pairs


def _operator(scene: dict):
    op = scene["operator"]
    J = _f8(op["J_b64"], tuple(op["J_shape"])) if "J_b64" in op else np.asarray(op["J"], float)
    if "minv_diag" in op:
        Minv = np.diag(np.asarray(op["minv_diag"], float))
    elif "minv_b64" in op:
        Minv = _f8(op["minv_b64"], tuple(op["minv_shape"]))
    else:
        Minv = np.asarray(op["Minv"], float)
    return J, Minv


def read_scene(src) -> ContactSceneV1:
    """A scene from a path to NN.json or from its parsed dict."""
    scene = src
    if not isinstance(src, dict):
        with open(os.fspath(src)) as f:
            scene = json.load(f)
    if scene.get("schema") != SCHEMA:
        raise ValueError(f"contact-scene-v1: schema {scene.get('schema')!r}, expected {SCHEMA!r}")
    model = scene["model"]
    pairs = None
    if model == "body_contacts":
        J, Minv, pairs = _body_contacts(scene)
    elif model == "operator":
        J, Minv = _operator(scene)
    else:
        raise ValueError(f"contact-scene-v1: unknown model {model!r}")
    nc = int(scene["n_c"])
    if J.shape[0] != 3 * nc:
        raise ValueError(f"contact-scene-v1: J has {J.shape[0]} rows for {nc} contacts")
    return ContactSceneV1(index=int(scene["index"]), name=str(scene["scene"]), model=model, n_b=int(scene["n_b"]),
                          n_c=nc, dof=int(scene["dof"]), dt=float(scene["dt"]),
                          mu=np.asarray(scene["mu"], float), b=np.asarray(scene["b"], float),
                          eta=np.asarray(scene["eta"], float), J=J, Minv=Minv, body_pairs=pairs,
                          provenance=scene.get("provenance"), raw=scene)


def read_package(directory) -> list:
    """Every NN.json of a package directory, in index order."""
    names = sorted(f for f in os.listdir(directory) if f.endswith(".json") and f[:-5].isdigit())
    return [read_scene(os.path.join(directory, f)) for f in names]


def block_scene(sc: ContactSceneV1):
    """The scene as an exact-cone NCP problem for ``ncp.NCPSolverB200`` (body-contact scenes
    without compliance)."""
    from .ncp import BlockScene
    if sc.model != "body_contacts":
        raise ValueError(f"{sc.name}: an operator scene has no body blocks; use admm_problem")
    if np.any(sc.eta):
        raise ValueError(f"{sc.name}: compliant contacts (eta > 0) are not a rigid NCP problem")
    d, nb, nc = sc.dof, sc.n_b, sc.n_c
    Ja, Jb = np.zeros((nc, 3, 6)), np.zeros((nc, 3, 6))
    for c in range(nc):
        a, b = (int(x) for x in sc.body_pairs[c])
        rows = slice(3 * c, 3 * c + 3)
        if a >= 0:
            Ja[c, :, :d] = sc.J[rows, d * a:d * a + d]
        if b >= 0:
            Jb[c, :, :d] = sc.J[rows, d * b:d * b + d]
    Minv = np.zeros((nb, 6, 6))
    for i in range(nb):
        Minv[i, :d, :d] = sc.Minv[d * i:d * i + d, d * i:d * i + d]
    return BlockScene(Ja=Ja, Jb=Jb, Minv=Minv, v_free=np.zeros((nb, 6)), mu=sc.mu.copy(), body_pairs=sc.body_pairs,
                      dt=sc.dt, bias=sc.b.reshape(nc, 3).copy(), feature=np.arange(nc, dtype=np.int32))


def admm_problem(scenes):
    """Operator scenes of one shape stacked for ``badmm.BatchProxADMM``: (J, Minv, v_free, mu, b)
    with v_free = 0 and b = q."""
    scenes = list(scenes)
    shapes = {(s.J.shape, s.n_c) for s in scenes}
    if len(shapes) != 1:
        raise ValueError(f"admm_problem: the scenes have different shapes {sorted(shapes)}")
    J = np.stack([s.J for s in scenes])
    Minv = np.stack([s.Minv for s in scenes])
    nv = J.shape[2]
    return J, Minv, np.zeros((len(scenes), nv)), np.stack([s.mu for s in scenes]), np.stack(
        [s.b.reshape(-1, 3) for s in scenes])


def read_hdf5_problem(path):
    """(W, q, mu) of a scene's HDF5 copy (the package loader's read_hdf5_problem)."""
    from .hdf5_lite import H5File
    f = H5File(path)
    n = int(f["fclib_local/W/n"].ravel()[0])
    m = int(f["fclib_local/W/m"].ravel()[0])
    nz = int(f["fclib_local/W/nz"].ravel()[0])
    if nz != -1:
        raise ValueError(f"{path}: compressed-column storage expected (nz = -1), got nz = {nz}")
    x = f["fclib_local/W/x"].astype(np.float64)
    rows = f["fclib_local/W/i"].astype(np.int64)
    colp = f["fclib_local/W/p"].astype(np.int64)
    L = np.zeros((n, m))
    cols = np.repeat(np.arange(len(colp) - 1), np.diff(colp))
    L[rows[:len(cols)], cols] = x[:len(cols)]
    if int(f.attrs("fclib_local/W").get("symmetric_packed") or 0):
        W = L + L.T - np.diag(np.diag(L))
    else:
        W = L
    return W, f["fclib_local/vectors/q"].astype(np.float64), f["fclib_local/vectors/mu"].astype(np.float64)


def verify(sc: ContactSceneV1, hdf5_path) -> dict:
    """The JSON reconstruction against the HDF5 copy: W's relative Frobenius and max-element
    differences, and the largest differences of q and mu (the package's acceptance: W to 1e-15
    relative, q to 1e-15, mu exactly)."""
    W, q, mu = read_hdf5_problem(hdf5_path)
    Wj = sc.delassus()
    scale = float(np.abs(W).max()) or 1.0
    nrm = float(np.linalg.norm(W)) or 1.0
    return dict(W_rel_fro=float(np.linalg.norm(Wj - W) / nrm), W_rel_max=float(np.abs(Wj - W).max() / scale),
                q_abs=float(np.abs(sc.b - q).max()) if q.shape == sc.b.shape else float("nan"),
                mu_abs=float(np.abs(sc.mu - mu).max()) if mu.shape == sc.mu.shape else float("nan"))
