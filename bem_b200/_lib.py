"""ctypes binding of include/spt_b200.h.

The structures below mirror the header field by field.  ``lib()`` loads
bem_b200/libspt_b200.so and raises if it is missing -- there is no CPU or
PyTorch fallback for any entry point.
"""

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libspt_b200.so")

SPT_OK, SPT_ERR_ARG, SPT_ERR_CUDA, SPT_ERR_CAPACITY = 0, 1, 2, 3
GEOM_FLAT, GEOM_TIP, GEOM_TIP_BEM, GEOM_WELL_BEM, GEOM_POST_BEM = 0, 1, 2, 3, 4
FORM_FP64, FORM_MIXED, FORM_SURROGATE = 0, 1, 2
FAR_REFERENCE, FAR_ADAPTIVE = 0, 1
FAR_RULES = {"reference": FAR_REFERENCE, "adaptive": FAR_ADAPTIVE}
GROUP_NEW, GROUP_RUNNING, GROUP_DONE, GROUP_NONFINITE, GROUP_TIMEOUT = 0, 1, 2, 3, 4
TEAM_AUTO, TEAM_CTA, TEAM_WARP = 0, 1, 2
COUNTERS = ("attempts", "accepted", "particle_steps", "stage_evals", "pair_evals", "ring_far", "ring_near",
            "near_pairs", "fp64_rounds", "fp64_targets", "live_steps", "cluster_evals")
N_COUNTERS = len(COUNTERS)
SEG_FIELDS = 11
BLOCK_SEGS = 32
RUN_NODES = 8

_d = ctypes.c_double
_i32 = ctypes.c_int32
_i64 = ctypes.c_int64
_p = ctypes.c_void_p


class SptGeometry(ctypes.Structure):
    _fields_ = [("kind", _i32), ("has_image", _i32), ("has_kill_below", _i32), ("has_z_max", _i32),
                ("E_gun", _d), ("R", _d), ("H", _d), ("L", _d), ("z0", _d), ("kill_z_below", _d),
                ("z_max", _d), ("z_handoff", _d), ("bottom_fillet", _d), ("rim_fillet", _d)]


class SptImage(ctypes.Structure):
    _fields_ = [("n_nodes", _i32), ("n_max", _i32), ("n_quad", _i32), ("mirror_symmetric", _i32),
                ("node", _p), ("seg", _p), ("quad", _p), ("a_inv", _p), ("rho_floor", _d), ("d_lo", _d),
                ("d_hi", _d)]


class SptBem(ctypes.Structure):
    _fields_ = [("n_seg", _i32), ("nodes_per_seg", _i32), ("seg_stride", _i64), ("node_stride", _i64),
                ("seg", _p), ("node", _p), ("gauss8_x", _d * 8), ("gauss8_w", _d * 8),
                ("far_rule", _i32), ("reserved", _i32), ("ratio4", _d), ("ratio2", _d), ("coarse", _p),
                ("coarse_stride", _i64), ("blk", _p), ("blk_stride", _i64), ("ratio_run", _d), ("run_nodes", _p),
                ("run_stride", _i64), ("clusters", _p), ("cluster_levels", _i32), ("cluster_terms", _i32),
                ("cluster_kappa", _d), ("image", SptImage)]


class SptState(ctypes.Structure):
    _fields_ = [("n_groups", _i32), ("max_group_size", _i32), ("n_particles", _i64),
                ("group_offset", _p), ("group_order", _p),
                ("x", _p), ("y", _p), ("z", _p), ("vx", _p), ("vy", _p), ("vz", _p),
                ("t_birth", _p), ("t_death", _p), ("charge", _p), ("mass", _p),
                ("t", _p), ("h", _p), ("status", _p), ("n_accepted", _p), ("n_rejected", _p), ("n_active", _p)]


class SptTraceParams(ctypes.Structure):
    _fields_ = [("t_max", _d), ("rtol", _d), ("atol", _d), ("plummer_radius", _d), ("charge_to_mass", _d),
                ("coulomb_constant", _d), ("safety", _d), ("min_factor", _d), ("max_factor", _d),
                ("initial_step_fraction", _d), ("max_attempts", _i64), ("form", _i32), ("log_capacity", _i32),
                ("log_h", _p), ("log_err", _p), ("counters", _p),
                ("n_screens", _i32), ("n_outputs", _i32), ("screens", _p), ("screen_rec", _p),
                ("screen_capacity", _i64), ("screen_count", _p), ("output_times", _p), ("output_rec", _p),
                ("output_flag", _p), ("sur_w", _p), ("sur_w16", _p), ("sur_s_start", _p), ("sur_log_scale", _p),
                ("sur_s_end", _d), ("sur_sig_floor", _d), ("sur_band", _d), ("sur_spot", _d), ("sur_d_min", _d),
                ("sur_d_max", _d), ("sur_stats", _p), ("round_points", _i32), ("cta_threads", _i32), ("kappa_max", _d),
                ("max_ctas", _i32), ("team", _i32)]


class SptAccelArgs(ctypes.Structure):
    _fields_ = [("n_groups", _i32), ("max_group_size", _i32), ("n_particles", _i64), ("group_offset", _p),
                ("x", _p), ("y", _p), ("z", _p), ("active", _p), ("charge", _p), ("mass", _p),
                ("charge_to_mass", _d), ("coulomb_constant", _d), ("plummer_radius", _d), ("form", _i32),
                ("ax", _p), ("ay", _p), ("az", _p)]


class SptGemmArgs(ctypes.Structure):
    _fields_ = [("M", _i32), ("N", _i32), ("K", _i32), ("a_mn", _i32), ("b_mn", _i32), ("epi", _i32),
                ("split_k", _i32), ("reserved", _i32), ("lda", _i64), ("ldb", _i64), ("ldc", _i64),
                ("split_stride", _i64), ("A", _p), ("B", _p), ("C", _p), ("bias", _p), ("Z", _p), ("H", _p),
                ("status", _p)]


IMAGE_MAX_MODES = 64
TRACE_IMAGE_MODES = 16
ABI_VERSION = 4
EPI_STORE, EPI_BIAS_SILU, EPI_DSILU = 0, 1, 2
_f = ctypes.c_float

# entry point -> (restype, argtypes)
SIGNATURES = {
    "spt_abi_version": (ctypes.c_int, []),
    "spt_last_error": (ctypes.c_int, [ctypes.c_char_p, _i32]),
    "spt_trace_workspace_bytes": (ctypes.c_int, [ctypes.POINTER(SptState), ctypes.POINTER(SptTraceParams),
                                                 ctypes.POINTER(SptGeometry), ctypes.POINTER(SptBem),
                                                 ctypes.POINTER(_i64)]),
    "spt_trace": (ctypes.c_int, [ctypes.POINTER(SptState), ctypes.POINTER(SptTraceParams),
                                 ctypes.POINTER(SptGeometry), ctypes.POINTER(SptBem), _p, _i64, _p]),
    "spt_accel": (ctypes.c_int, [ctypes.POINTER(SptAccelArgs), ctypes.POINTER(SptGeometry),
                                 ctypes.POINTER(SptBem), _p]),
    "spt_bem_field": (ctypes.c_int, [_p, _p, _p, _i64, ctypes.POINTER(SptBem), _i32, _p, _p, _p, _p]),
    "spt_surrogate_field": (ctypes.c_int, [_p, _p, _p, _i64, ctypes.POINTER(SptBem), ctypes.POINTER(SptTraceParams),
                                           _p, _p, _p, _p]),
    "spt_compact_groups": (ctypes.c_int, [_p, _i32, _p, _p, _p, _p]),
    "spt_ring_field": (ctypes.c_int, [_p, _p, _p, _i64, _i32, _p, _p, _p]),
    "spt_ellip_ke": (ctypes.c_int, [_p, _i64, _i32, _p, _p, _p]),
    "spt_bem_assemble": (ctypes.c_int, [_p, _p, _i32, _d, _i32, _p, _p, _p, _p]),
    "spt_mlp_gemm": (ctypes.c_int, [ctypes.POINTER(SptGemmArgs), _p]),
    "spt_mlp_first_layer": (ctypes.c_int, [_p, _i64, _p, _p, _p, _p, _p]),
    "spt_mlp_last_layer": (ctypes.c_int, [_p, _p, _i64, _p, _p, _p, _p, _f, _p, _p, _p, _p, _p]),
    "spt_mlp_colsum": (ctypes.c_int, [_p, _i64, _p, _p, _p, _p]),
    "spt_mlp_reduce_splits": (ctypes.c_int, [_p, _i32, _i64, _p, _p]),
    "spt_mlp_adam": (ctypes.c_int, [_p, _p, _p, _p, _i64, _f, _f, _f, _f, _i32, _p, _p, _p]),
    "spt_toroidal_q": (ctypes.c_int, [_p, _i64, _i32, _p, _p, _p]),
    "spt_image_assemble": (ctypes.c_int, [_p, _p, _i32, _i32, _d, _d, _i32, _p, _p, _p, _p]),
    "spt_image_force": (ctypes.c_int, [_p, _p, _p, _p, _p, _p, _i32, _i32, ctypes.POINTER(SptImage),
                                       ctypes.POINTER(SptGeometry), _d, _d, _p, _p, _p, _p]),
    "spt_trace_noalloc": (ctypes.c_int, [ctypes.POINTER(SptState), ctypes.POINTER(SptTraceParams),
                                         ctypes.POINTER(SptGeometry), ctypes.POINTER(SptBem), _p]),
}

_LIB = None


class SptError(RuntimeError):
    pass


def lib():
    """Load the CUDA library (once).  Raises if it has not been built."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise SptError(f"{LIB_PATH} is missing: build it with `python -m bem_b200.build`")
        h = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(h, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = h
    return _LIB


def last_error():
    buf = ctypes.create_string_buffer(512)
    lib().spt_last_error(buf, 512)
    return buf.value.decode(errors="replace")


def check(rc, what):
    if rc != SPT_OK:
        msg = last_error()
        if rc == SPT_ERR_ARG:
            raise ValueError(f"{what}: {msg}")
        raise SptError(f"{what} failed ({rc}): {msg}")


def ptr(t):
    """Device pointer of a torch tensor (None -> NULL)."""
    return None if t is None else ctypes.c_void_p(t.data_ptr())
