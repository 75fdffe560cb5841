"""B200-native contact-solve hot path of 3fold-motion-engine.

A drop-in for the reference's GPU contact engines behind its ContactEngine protocol
(src/motion_engine/contact_engine.py:48-55).  Compute runs only in libb2c.so (hand-written
sm_100a CUDA, C ABI in include/b2c.h); this package is the host side that mirrors the
reference's engine classes.

The directory name is not a Python identifier, so the package is imported under the alias
``motion_engine_b200`` (see ``__graft_entry__.load_package``).
"""
from . import _lib, build, metrics
from .boxes import BatchedBoxEngine, BoxContactEngine, autotune, partition_scenes
from .colored import (AppliedWarmContactEngine, ColorCacheContactEngine, DeferredForceContactEngine,
                      FixedFrameContactEngine, GraphColoredContactEngine, IslandSolveContactEngine)
from .engine import BodyState, ContactEngine, RelaxedJacobiContactEngine, quat_to_R, voxbox
from .handle import HandleBoxEngine
from .islands import partition_pairs

__all__ = ["BodyState", "ContactEngine", "RelaxedJacobiContactEngine", "GraphColoredContactEngine",
           "FixedFrameContactEngine", "AppliedWarmContactEngine", "DeferredForceContactEngine",
           "ColorCacheContactEngine", "IslandSolveContactEngine", "partition_pairs", "BoxContactEngine", "BatchedBoxEngine", "HandleBoxEngine", "autotune", "partition_scenes", "quat_to_R", "voxbox", "build", "metrics", "_lib"]
