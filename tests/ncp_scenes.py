"""Block scenes of the exact-cone NCP tests, read from the golden fixture (made by the
reference's own generators: tests/golden/make_ncp_golden.py)."""
import os
from types import SimpleNamespace

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ncp_golden.npz")
_G = None


def golden():
    global _G
    if _G is None:
        _G = dict(np.load(GOLDEN))
    return _G


WELLPOSED = ("wellposed_8_8_1", "wellposed_16_8_2", "wellposed_6_6_3", "wellposed_12_10_4")
INDETERMINATE = ("pushed_cube", "stack3")
SYNTHETIC = ("synthetic_256_64_7", "synthetic_1024_128_2")


def scene(name, cls=None):
    """The named scene as `cls` (the package's BlockScene) or a plain namespace."""
    g = golden()
    kw = dict(Ja=g[f"{name}/Ja"], Jb=g[f"{name}/Jb"], Minv=g[f"{name}/Minv"], v_free=g[f"{name}/v_free"],
              mu=g[f"{name}/mu"], body_pairs=g[f"{name}/pairs"], dt=float(g[f"{name}/dt"]), bias=g[f"{name}/bias"],
              feature=g[f"{name}/feature"], sep=g.get(f"{name}/sep"))
    return cls(**kw) if cls is not None else SimpleNamespace(**kw)


def with_sep(bs, seed=0):
    """A copy with seeded separations in [-2e-3, 1e-3] (the soft-step branch reads them)."""
    d = dict(vars(bs)) if isinstance(bs, SimpleNamespace) else dict(bs.__dict__)
    d["sep"] = np.random.default_rng(seed).uniform(-2e-3, 1e-3, len(d["mu"]))
    return type(bs)(**d)
