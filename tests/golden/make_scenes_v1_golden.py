"""Golden vectors for the contact-scene-v1 reader, made by the reference's own loader
(data/ncp/loader.py: rebuild, the JSON reconstruction W = J M^-1 J^T + diag(eta), q = b, mu).
The loader imports h5py at module level for its HDF5 comparison, which this image lacks; a
placeholder module is registered under that name only so the import succeeds -- rebuild()
never touches it.  For every scene: b, mu, eta, the Frobenius norm and trace of G, and G r for
a seeded vector r; the full G for scenes of at most 256 rows; the package's published spectral
bounds of G (scenes/table.json: lambda_min_pos, lambda_max).  The scene files themselves
(all but the two largest, 11 and 12, 4 MB of the package's 5.3 MB) are copied into
scenes_v1.json.gz so that the reader's tests run without the reference, and the HDF5 copies of
the fifteen small ones (about 20 kB each; every one holds contiguous and deflate-chunked
datasets) into scenes_v1_hdf5.zip.

Run:  python tests/golden/make_scenes_v1_golden.py /path/to/reference   (or with B2C_REFERENCE set)
"""
import gzip
import io
import importlib.util
import json
import os
import sys
import types
import zipfile

import numpy as np


def reference_root():
    """The reference checkout: the first argument, else $B2C_REFERENCE."""
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("B2C_REFERENCE")
    if not ref:
        raise SystemExit(f"usage: python {os.path.basename(__file__)} /path/to/reference  (or set B2C_REFERENCE)")
    return ref


def main(ref):
    sys.modules.setdefault("h5py", types.ModuleType("h5py"))
    spec = importlib.util.spec_from_file_location("ref_loader", os.path.join(ref, "data", "ncp", "loader.py"))
    L = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(L)
    out, files = {}, {}
    for i in range(L.N_SCENES):
        with open(os.path.join(ref, "data", "ncp", "scenes", f"{i:02d}.json")) as f:
            scene = json.load(f)
        if i not in (11, 12):
            files[f"{i:02d}"] = scene
        G, b, mu, J, Minv = L.rebuild(scene)
        r = np.random.default_rng(100 + i).standard_normal(G.shape[0])
        k = f"s{i:02d}"
        out.update({f"{k}/b": b, f"{k}/mu": mu, f"{k}/eta": np.asarray(scene["eta"], float),
                    f"{k}/G_fro": np.float64(np.linalg.norm(G)), f"{k}/G_trace": np.float64(np.trace(G)),
                    f"{k}/Gr": G @ r, f"{k}/shape": np.array(J.shape)})
        if G.shape[0] <= 256:
            out[f"{k}/G"] = G
        print(i, scene["scene"], G.shape, J.shape)
    with open(os.path.join(ref, "data", "ncp", "scenes", "table.json")) as f:
        table = json.load(f)
    out["table/lambda_min_pos"] = np.array([float(r["lambda_min_pos"]) for r in table])
    out["table/lambda_max"] = np.array([float(r["lambda_max"]) for r in table])
    here = os.path.dirname(os.path.abspath(__file__))
    np.savez_compressed(os.path.join(here, "scenes_v1_golden.npz"), **out)
    with gzip.GzipFile(os.path.join(here, "scenes_v1.json.gz"), "wb", mtime=0) as gz, \
            io.TextIOWrapper(gz, encoding="utf-8") as f:
        json.dump(files, f)
    small = [i for i in range(L.N_SCENES) if i not in range(7, 13)]
    with zipfile.ZipFile(os.path.join(here, "scenes_v1_hdf5.zip"), "w", zipfile.ZIP_STORED) as z:
        for i in small:
            z.write(os.path.join(ref, "data", "ncp", "scenes", f"{i:02d}.hdf5"), f"{i:02d}.hdf5")


if __name__ == "__main__":
    main(reference_root())
