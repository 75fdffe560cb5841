"""ctypes bindings of libb2c.so (the C ABI declared in include/b2c.h).

The library is the product's only compute path: there is no CPU fallback.  Loading fails
loudly if the library is missing and cannot be built.
"""
from __future__ import annotations

import ctypes
import os

from . import build as _build

c_int32 = ctypes.c_int32
c_float = ctypes.c_float
c_void_p = ctypes.c_void_p


class Bodies(ctypes.Structure):
    _fields_ = [("n", c_int32), ("xc", c_void_p), ("q", c_void_p), ("v", c_void_p), ("w", c_void_p),
                ("pv", c_void_p), ("po", c_void_p), ("invM", c_void_p), ("IbInv", c_void_p), ("kin", c_void_p),
                ("invIw", c_void_p)]


class Beads(ctypes.Structure):
    _fields_ = [("n", c_int32), ("rest", c_void_p), ("owner", c_void_p), ("world", c_void_p),
                ("bead_start", c_void_p)]


class Manifold(ctypes.Structure):
    _fields_ = [("capacity", c_int32), ("pair_capacity", c_int32), ("bead_count", c_void_p),
                ("bead_offset", c_void_p), ("pair_local", c_void_p), ("pair_first", c_void_p), ("gorder", c_void_p),
                ("body_npairs", c_void_p), ("pair_base", c_void_p), ("praw_start", c_void_p),
                ("praw_count", c_void_p), ("jn_in", c_void_p), ("jn_red", c_void_p), ("jt_in", c_void_p),
                ("keep", c_void_p), ("kidx", c_void_p), ("scan_tmp", c_void_p)]


class Pairs(ctypes.Structure):
    _fields_ = [("capacity", c_int32), ("max_colors", c_int32), ("pbi", c_void_p), ("pbj", c_void_p),
                ("kcount", c_void_p), ("pstart", c_void_p), ("pidx", c_void_p), ("col", c_void_p),
                ("porder", c_void_p), ("cstart", c_void_p), ("ccount", c_void_p), ("claim", c_void_p),
                ("cached_a", c_void_p), ("cached_b", c_void_p), ("cached_mass", c_void_p),
                ("cache_state", c_void_p), ("barrier", c_void_p), ("rec", c_void_p), ("kslots", c_int32),
                ("body_colors", c_void_p), ("body_local", c_void_p), ("body_slots", c_void_p),
                ("n_scenes", c_int32), ("scene_body_start", c_void_p), ("scene_order", c_void_p),
                ("pair_slot", c_void_p), ("scene_slots", c_void_p), ("prio_hi", c_void_p), ("isl_work", c_void_p)]


SOLVE_SCENES = 0x100000  # b2c_color_params.solve_blocks: one CTA per scene (B2C_SOLVE_SCENES)


class Warm(ctypes.Structure):
    _fields_ = [("capacity", c_int32), ("keys", c_void_p), ("imp", c_void_p), ("n", c_void_p)]


class ColorParams(ctypes.Structure):
    _fields_ = [("vit", c_int32), ("pit", c_int32), ("max_points", c_int32), ("flags", c_int32), ("mu", c_float),
                ("t2d", c_float), ("color_cap", c_int32), ("solve_blocks", c_int32),
                ("barrier_timeout_ns", ctypes.c_int64), ("body_mu", c_void_p)]


class Boxes(ctypes.Structure):
    _fields_ = [("n", c_int32), ("half", c_void_p), ("mu", c_void_p), ("margin", c_float), ("cell", c_float),
                ("dim_x", c_int32), ("dim_y", c_int32), ("dim_z", c_int32), ("cand_capacity", c_int32),
                ("bucket", c_void_p), ("start", c_void_p), ("cursor", c_void_p), ("sorted", c_void_p),
                ("cand_count", c_void_p), ("cand_offset", c_void_p), ("cand_a", c_void_p), ("cand_b", c_void_p),
                ("cont_count", c_void_p), ("cont_offset", c_void_p), ("pair_flag", c_void_p),
                ("pair_offset", c_void_p), ("slot_p", c_void_p), ("slot_n", c_void_p), ("slot_f", c_void_p),
                ("scan_tmp", c_void_p), ("scene", c_void_p)]


class NcpScene(ctypes.Structure):
    _fields_ = [("n_c", c_int32), ("n_b", c_int32), ("dtype", c_int32), ("Ja", c_void_p), ("Jb", c_void_p),
                ("Minv", c_void_p), ("v_free", c_void_p), ("mu", c_void_p), ("bias", c_void_p), ("sep", c_void_p),
                ("pa", c_void_p), ("pb", c_void_p), ("feature", c_void_p)]


class NcpState(ctypes.Structure):
    _fields_ = [("max_contacts", c_int32), ("n_bodies", c_int32), ("max_colors", c_int32), ("rho", c_void_p),
                ("lam", c_void_p), ("v", c_void_p), ("acc", c_void_p), ("res", c_void_p), ("u", c_void_p),
                ("col", c_void_p), ("order", c_void_p), ("cstart", c_void_p), ("ccount", c_void_p),
                ("claim", c_void_p), ("dyn", c_void_p), ("cache_pa", c_void_p), ("cache_pb", c_void_p),
                ("cache_feat", c_void_p), ("cache_minv", c_void_p), ("stats", c_void_p), ("res_max", c_void_p),
                ("barrier", c_void_p)]


class NcpParams(ctypes.Structure):
    _fields_ = [("desaxce", c_int32), ("soft", c_int32), ("use_bias", c_int32), ("color_cache", c_int32),
                ("solve_blocks", c_int32), ("pad", c_int32), ("softp", ctypes.c_double * 5),
                ("barrier_timeout_ns", ctypes.c_int64)]


class World(ctypes.Structure):
    _fields_ = [("n", c_int32), ("max_contacts", c_int32), ("x", c_void_p), ("q", c_void_p), ("v", c_void_p),
                ("w", c_void_p), ("half", c_void_p), ("mass", c_void_p), ("Ib", c_void_p), ("kin", c_void_p),
                ("vkin", c_void_p), ("body_mu", c_void_p), ("mu", ctypes.c_double), ("xc32", c_void_p),
                ("x4", c_void_p), ("half4", c_void_p), ("slot_p", c_void_p), ("slot_n", c_void_p),
                ("slot_f", c_void_p), ("pa", c_void_p), ("pb", c_void_p), ("fid", c_void_p), ("key", c_void_p),
                ("p", c_void_p), ("nrm", c_void_p), ("gap", c_void_p), ("attach", c_void_p), ("count", c_void_p),
                ("warm_keys", c_void_p),
                ("warm_lam", c_void_p), ("warm_n", c_void_p)]


class Bncp(ctypes.Structure):
    _fields_ = [("n_env", c_int32), ("n_max", c_int32), ("nc", c_void_p), ("G", c_void_p), ("b", c_void_p),
                ("mu", c_void_p), ("lam", c_void_p), ("res", c_void_p), ("iters", c_void_p), ("labels", c_void_p),
                ("status", c_void_p)]


class Admm(ctypes.Structure):
    """b2c_admm"""
    _fields_ = [("n_env", c_int32), ("nc", c_int32), ("nv", c_int32)] + [(k, c_void_p) for k in (
        "J", "Minv", "v_free", "mu", "lam", "u", "v_plus", "res", "mask", "rho", "nslip", "labels", "dlam_tau",
        "dv_tau", "dlam_mu", "dbv_in", "b_in")]


class AdmmParams(ctypes.Structure):
    """b2c_admm_params"""
    _fields_ = [("flags", c_int32), ("n_iter", c_int32), ("cg_iters", c_int32), ("refresh_every", c_int32),
                ("tol", ctypes.c_double), ("chunk", c_int32), ("desax", c_int32), ("rho_mode", c_int32),
                ("jacobi_sweeps", c_int32), ("alpha_eta", ctypes.c_double), ("dt", ctypes.c_double),
                ("jdir", c_int32), ("n_calls", c_int32), ("grad_cg", c_int32), ("do_mu", c_int32)]


ADMM_FORWARD, ADMM_GRADIENT, ADMM_GRAD_GIVEN = 1, 2, 4
ADMM_RHO = {"sqrt": 0, "lmin": 1, "lmax": 2, "regime": 3, "given": 4}
ADMM_MAX_CONTACTS, ADMM_MAX_DOFS = 8, 32

COLOR_FIXED_FRAME = 1
COLOR_APPLY_WARM = 2
COLOR_CACHE = 4
COLOR_WARM_START = 8
COLOR_PER_CONTACT = 16
COLOR_FIRST_FIT = 32
COLOR_ROW_FORM = 64
COLOR_REDUCED_CONTACTS = 128
COLOR_ISLANDS = 256
ISLAND_MAX_PAIRS = 64  # B2C_ISLAND_MAX_PAIRS


class Grid(ctypes.Structure):
    _fields_ = [("dim_x", c_int32), ("dim_y", c_int32), ("dim_z", c_int32), ("cell", c_float),
                ("bucket", c_void_p), ("start", c_void_p), ("cursor", c_void_p), ("sorted", c_void_p),
                ("scan_tmp", c_void_p), ("sorted_pos", c_void_p)]


class Contacts(ctypes.Structure):
    _fields_ = [("capacity", c_int32), ("bi", c_void_p), ("bj", c_void_p), ("pA", c_void_p), ("pB", c_void_p),
                ("n", c_void_p), ("fa", c_void_p), ("fb", c_void_p), ("imp", c_void_p)]


class JacobiParams(ctypes.Structure):
    _fields_ = [("vit", c_int32), ("pit", c_int32), ("relax", c_float), ("mu", c_float)]


HEADER_FIELDS = ("n_raw", "n_contacts", "n_kept", "n_pairs", "n_colors", "cache_hit", "error", "rounds")
ERR_BITS = {1: "contact capacity overflow", 2: "a body pair carries more than 1024 contacts",
            4: "a body pair carries more than 8 kept contacts", 8: "colour count exceeds the colour cap",
            16: "colouring did not finish in its round budget", 32: "a bead has more than 64 neighbours within 2R",
            64: "pair capacity overflow", 128: "a grid barrier of the persistent solve gave up waiting"}

class Config(ctypes.Structure):
    """b2c_config: an engine handle's configuration (b2c_config_init fills the defaults)."""
    _fields_ = [("kind", c_int32), ("device", c_int32), ("vit", c_int32), ("pit", c_int32),
                ("mu", ctypes.c_double), ("dims", ctypes.c_double * 3), ("margin", ctypes.c_double),
                ("flags", c_int32), ("color_cap", c_int32), ("solve_blocks", c_int32), ("cand_per_body", c_int32),
                ("barrier_timeout_ns", ctypes.c_int64), ("graph", c_int32)]


class StepHeader(ctypes.Structure):
    """b2c_step_header: the last substep's counters and the handle's diagnostics."""
    _fields_ = [("last", c_int32 * 8), ("color_cache_hits", c_int32), ("color_cache_misses", c_int32),
                ("graph_captures", c_int32), ("kernels_per_step", c_int32), ("bodies", c_int32),
                ("built", c_int32)]


ENGINE_BOX = 1

_P = ctypes.POINTER
_D = ctypes.c_double
_SIGS = {
    "b2c_version": ([], c_int32),
    "b2c_graph_kernel_nodes": ([c_void_p], c_int32),
    "b2c_pair_record_floats": ([c_int32, c_int32], ctypes.c_int64),
    "b2c_last_error": ([], ctypes.c_char_p),
    "b2c_scan_scratch_ints": ([c_int32], c_int32),
    "b2c_barrier_words": ([], c_int32),
    "b2c_exclusive_scan": ([c_void_p, c_void_p, c_int32, c_void_p, c_void_p], c_int32),
    "b2c_exclusive_scan_noalloc": ([c_void_p, c_void_p, c_int32, c_void_p], c_int32),
    "b2c_scan_noalloc_max_n": ([], c_int32),
    "b2c_body_predict": ([_P(Bodies), c_float, c_void_p], c_int32),
    "b2c_body_integrate": ([_P(Bodies), c_float, c_void_p], c_int32),
    "b2c_bead_world": ([_P(Bodies), _P(Beads), _P(Grid), c_void_p], c_int32),
    "b2c_grid_build": ([_P(Beads), _P(Grid), c_void_p], c_int32),
    "b2c_bead_contacts": ([_P(Beads), _P(Grid), _P(Contacts), c_void_p, c_void_p], c_int32),
    "b2c_jacobi_solve": ([_P(Bodies), _P(Contacts), c_void_p, c_void_p, _P(JacobiParams), c_float, c_void_p],
                         c_int32),
    "b2c_jacobi_substep": ([_P(Bodies), _P(Beads), _P(Grid), _P(Contacts), c_void_p, c_void_p, _P(JacobiParams),
                            c_float, c_void_p, c_void_p], c_int32),
    "b2c_bead_contacts_sorted": ([_P(Beads), _P(Grid), _P(Contacts), _P(Manifold), c_void_p, c_void_p], c_int32),
    "b2c_manifold_reduce": ([_P(Bodies), _P(Beads), _P(Contacts), _P(Manifold), _P(Contacts), c_void_p, _P(Pairs),
                             _P(Warm), c_void_p, _P(ColorParams), c_void_p], c_int32),
    "b2c_color_pairs": ([_P(Bodies), _P(Pairs), c_void_p, _P(ColorParams), c_void_p], c_int32),
    "b2c_color_solve": ([_P(Bodies), _P(Contacts), _P(Pairs), c_void_p, _P(ColorParams), c_float, c_void_p],
                        c_int32),
    "b2c_warm_store": ([_P(Contacts), c_void_p, _P(Warm), c_void_p, c_void_p], c_int32),
    "b2c_island_work_ints": ([c_int32, c_int32], ctypes.c_int64),
    "b2c_island_partition": ([c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_int32, c_void_p, c_void_p, c_void_p,
                              c_void_p, c_void_p, c_void_p], c_int32),
    "b2c_color_substep": ([_P(Bodies), _P(Beads), _P(Grid), _P(Contacts), _P(Manifold), _P(Contacts), c_void_p,
                           _P(Pairs), _P(Warm), c_void_p, _P(ColorParams), c_float, c_void_p, c_void_p], c_int32),
    "b2c_box_candidates": ([_P(Bodies), _P(Boxes), c_void_p, c_void_p], c_int32),
    "b2c_box_contacts": ([_P(Bodies), _P(Boxes), _P(Contacts), c_void_p, _P(Pairs), _P(Warm), c_void_p,
                          _P(ColorParams), c_void_p], c_int32),
    "b2c_box_substep": ([_P(Bodies), _P(Boxes), _P(Contacts), c_void_p, _P(Pairs), _P(Warm), c_void_p,
                         _P(ColorParams), c_float, c_void_p, c_void_p], c_int32),
    "b2c_ncp_setup": ([_P(NcpScene), _P(NcpState), c_int32, c_void_p], c_int32),
    "b2c_ncp_color": ([_P(NcpScene), _P(NcpState), _P(NcpParams), c_void_p], c_int32),
    "b2c_ncp_sweeps": ([_P(NcpScene), _P(NcpState), _P(NcpParams), c_int32, c_void_p], c_int32),
    "b2c_ncp_residual": ([_P(NcpScene), _P(NcpState), _P(NcpParams), c_void_p], c_int32),
    "b2c_world_contacts": ([_P(World), _P(Boxes), c_void_p, c_void_p], c_int32),
    "b2c_world_scene": ([_P(World), c_int32, _D, c_int32, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                         c_void_p, c_void_p, c_void_p], c_int32),
    "b2c_world_warm": ([_P(World), c_int32, c_void_p, c_void_p], c_int32),
    "b2c_world_warm_adjoint": ([_P(World), c_int32, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p], c_int32),
    "b2c_world_store": ([_P(World), c_int32, c_void_p, c_void_p], c_int32),
    "b2c_world_integrate": ([_P(World), c_void_p, _D, c_void_p], c_int32),
    "b2c_ncp_adjoint": ([_P(NcpScene), _P(NcpState), _P(NcpParams), c_int32, c_void_p, c_void_p, c_void_p, c_void_p,
                         c_void_p, c_void_p], c_int32),
    "b2c_ncp_trace_words": ([], c_int32),
    "b2c_ncp_sweeps_record": ([_P(NcpScene), _P(NcpState), _P(NcpParams), c_int32, c_void_p, ctypes.c_int64,
                               c_void_p], c_int32),
    "b2c_ncp_adjoint_unrolled": ([_P(NcpScene), _P(NcpState), _P(NcpParams), c_int32, c_void_p, ctypes.c_int64,
                                  c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                  c_void_p], c_int32),
    "b2c_world_adj_begin": ([_P(World), _P(NcpScene), c_void_p, _D, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                             c_void_p, c_void_p, c_void_p, c_void_p, c_void_p], c_int32),
    "b2c_world_adj_end": ([_P(World), _P(NcpScene), c_void_p, c_void_p, c_void_p, _D, c_void_p, c_void_p, c_void_p,
                           c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                           c_void_p], c_int32),
    "b2c_admm_smem_bytes": ([c_int32, c_int32], ctypes.c_int64),
    "b2c_admm_solve": ([_P(Admm), _P(AdmmParams), c_void_p], c_int32),
    "b2c_bncp_max_rows": ([], c_int32),
    "b2c_bncp_solve": ([_P(Bncp), c_int32, ctypes.c_double, c_int32, c_void_p], c_int32),
    "b2c_bncp_sensitivity": ([_P(Bncp), c_void_p, c_void_p, c_void_p], c_int32),
    "b2c_bncp_vjp": ([_P(Bncp), c_void_p, c_void_p, c_void_p, c_void_p], c_int32),
    "b2c_config_init": ([_P(Config)], None),
    "b2c_box_body_setup": ([c_int32, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p],
                           c_int32),
    "b2c_create": ([_P(Config), _P(c_void_p)], c_int32),
    "b2c_add_bodies": ([c_void_p, c_int32, c_void_p, c_void_p, c_void_p, c_void_p], c_int32),
    "b2c_set_body_mu": ([c_void_p, c_int32, c_int32, c_void_p], c_int32),
    "b2c_set_body_scene": ([c_void_p, c_int32, c_int32, c_void_p], c_int32),
    "b2c_body_count": ([c_void_p], c_int32),
    "b2c_set_kinematic": ([c_void_p, c_int32, c_void_p], c_int32),
    "b2c_step": ([c_void_p, _D, c_int32, c_void_p], c_int32),
    "b2c_sync_header": ([c_void_p, _P(StepHeader)], c_int32),
    "b2c_get_state": ([c_void_p, c_void_p, c_void_p, c_void_p, c_void_p], c_int32),
    "b2c_get_state_packed": ([c_void_p, c_void_p, c_void_p], c_int32),
    "b2c_set_state_packed": ([c_void_p, c_void_p, c_void_p], c_int32),
    "b2c_contact_forces": ([c_void_p, c_void_p], c_int32),
    "b2c_state_save": ([c_void_p, c_void_p, _P(ctypes.c_size_t)], c_int32),
    "b2c_state_load": ([c_void_p, c_void_p, ctypes.c_size_t], c_int32),
    "b2c_destroy": ([_P(c_void_p)], c_int32),
    "b2c_box_narrowphase_test": ([c_int32, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_float,
                                  c_void_p, c_void_p, c_void_p, c_void_p, c_void_p], c_int32),
}

_LIB = None


def exported_symbols():
    return sorted(_SIGS)


def load(build_if_missing: bool = True):
    """Load libb2c.so (building it first when it is missing or older than its sources)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = _build.LIB
    if build_if_missing:
        try:
            path = _build.build()
        except RuntimeError:
            if not os.path.exists(path):
                raise
    if not os.path.exists(path):
        raise RuntimeError(f"b2c: CUDA library {path} is missing; build it with build.py (nvcc, sm_100a)")
    L = ctypes.CDLL(path)
    for name, (args, res) in _SIGS.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _LIB = L
    return L


def check(rc: int, what: str) -> None:
    if rc != 0:
        msg = load().b2c_last_error().decode(errors="replace")
        raise RuntimeError(f"{what} failed with status {rc}: {msg}")
