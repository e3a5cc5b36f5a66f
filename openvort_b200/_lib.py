"""ctypes binding of libov_gpu.so (include/openvort_b200.h).

The library is the only compute path: if it is missing or no sm_100a GPU is
present, calls raise OVError; nothing falls back to the CPU.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

from .tangle import TangleState, Vec3d

LIB_PATH = Path(__file__).resolve().parent / "libov_gpu.so"

OV_OK, OV_ERR_NO_DEVICE, OV_ERR_CUDA, OV_ERR_INVALID = 0, 1, 2, 3
OV_ERR_NONFINITE, OV_ERR_FLOW, OV_ERR_TREE_DEPTH, OV_ERR_TIMEOUT, OV_ERR_NOMEM = 4, 5, 6, 7, 8
OV_PREC_FP64, OV_PREC_MIXED = 0, 1
OV_FRAME_TEXT, OV_FRAME_BINARY = 0, 1
OV_FIELD_POS, OV_FIELD_VELS, OV_FIELD_VS = 1, 2, 4
OV_FIELD_TANGENTS, OV_FIELD_NORMALS, OV_FIELD_DXI, OV_FIELD_ALL = 8, 16, 32, 63

# every symbol include/openvort_b200.h declares
FUNCTIONS = [
    "shifted", "update_tangent_normal", "update_tangents_normals", "update_velocities",
    "update_velocity", "calculate_vs", "calculate_vs_shift", "octree_build", "octree_destroy",
    "octree_get_vs", "euler_step", "rk4_step", "ov_init", "ov_last_error",
    "ov_last_error_message", "ov_error_string", "ov_clear_error", "ov_set_precision",
    "ov_get_precision", "ov_set_rk4_classic", "ov_get_rk4_classic", "ov_get_last_stats",
    "ov_state_create", "ov_state_destroy", "ov_state_upload", "ov_state_download",
    "ov_state_update_tangle", "ov_state_rk4_step", "ov_state_run", "ov_state_eval_points",
    "ov_measure_fma_peak", "ov_state_get_stats", "ov_state_reset_stats", "ov_state_shard",
    "ov_state_shard_bytes", "ov_state_shard_begin", "ov_state_shard_end",
    "ov_set_mixed_near_factor", "ov_get_mixed_near_factor", "ov_set_colinear_cutoff",
    "ov_get_colinear_cutoff", "ov_direct_points_noalloc",
    "ov_batch_create", "ov_batch_destroy", "ov_batch_update", "ov_batch_run",
    "ov_batch_download", "ov_batch_set_tuning", "ov_batch_get_tuning", "ov_batch_autotune",
    "ov_batch_get_stats", "ov_adjoint_create", "ov_adjoint_destroy", "ov_adjoint_velocity",
    "ov_adjoint_velocity_vjp", "ov_adjoint_forward", "ov_adjoint_backward", "ov_adjoint_generation",
    "ov_reconnect_candidates", "ov_reconnect_vortices", "ov_reconnect_get_stats", "ov_remesh", "ov_enforce_boundaries", "ov_eliminate_small_loops",
    "ov_save_tangle", "ov_save_frame", "ov_state_save_frame", "ov_frame_wait", "ov_frame_info",
    "ov_load_frame", "ov_check_fast_math",
]
DATA = [
    "open_boundaries", "periodic_6", "periodic_18", "periodic_26", "periodic_z_open_xy",
    "wall_1_open", "wall_1_6", "wall_1_18", "wall_1_26", "wall_2_4", "wall_2_2", "wall_2_26",
    "channel_z", "vn_conf", "vs_conf", "vb_conf", "VORTEX_WIDTH", "KAPPA", "global_LIA_only",
    "global_alpha", "global_alpha_p", "global_dl_max", "global_num_threads",
    "global_use_mutual_friction", "global_use_BH", "global_BH_resolution", "global_BH_quadtree",
    "global_BH_grain", "global_hyperfriction", "global_max_curvature_scale", "global_hyperalpha",
    "global_small_loop_cutoff", "global_eliminate_origin_loops", "global_eliminate_loops_origin_cutoff",
    "global_eliminate_zaxis_loops", "global_eliminate_loops_zaxis_cutoff", "global_eliminate_outer_loops",
    "global_eliminate_outer_loops_cutoff",
]


class OVError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"libov_gpu error {code}: {msg}")
        self.code = code


class EvalStats(C.Structure):
    _fields_ = [("interactions", C.c_double), ("cell_interactions", C.c_double),
                ("cells", C.c_double), ("eval_ms", C.c_double), ("build_ms", C.c_double),
                ("total_ms", C.c_double)]


class RunStats(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("evals", "interactions", "cell_interactions",
                                          "bs_kernel_ms", "bs_launches", "build_ms",
                                          "last_run_ms", "launches", "n_targets", "n_segments",
                                          "warp_iterations")]


class BatchTuning(C.Structure):
    _fields_ = [("targets_per_block", C.c_int), ("sources_per_tile", C.c_int),
                ("blocks_per_sm", C.c_int), ("kernel_ms", C.c_double)]


class ReconnectStats(C.Structure):
    _fields_ = ([(n, C.c_int) for n in ("candidates", "tested", "nodes_summed", "fp64_rechecks",
                                        "reconnections")]
                + [(n, C.c_double) for n in ("search_s", "sums_s", "total_s")])


class BatchStats(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("evals", "interactions", "last_run_ms", "bs_kernel_ms",
                                          "kernels_per_step", "n_targets", "n_segments",
                                          "n_systems")]


_lib = None


def load(path: os.PathLike | str | None = None) -> C.CDLL:
    """Load libov_gpu.so (RTLD_LOCAL) and declare its prototypes."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise OVError(OV_ERR_NO_DEVICE, f"{p} is not built (run openvort_b200.build)")
    lib = C.CDLL(str(p))
    T = C.POINTER(TangleState)
    V = C.POINTER(Vec3d)
    sig = {
        "update_tangents_normals": (None, [T]),
        "update_tangent_normal": (None, [T, C.c_size_t]),
        "update_velocities": (None, [T, C.c_double, C.c_void_p]),
        "update_velocity": (None, [T, C.c_int, C.c_double, C.c_void_p]),
        "calculate_vs": (Vec3d, [T, Vec3d, C.c_int]),
        "calculate_vs_shift": (Vec3d, [T, Vec3d, C.c_int, V, C.POINTER(C.c_int), C.c_int]),
        "octree_build": (C.c_void_p, [T, C.c_int]),
        "octree_destroy": (None, [C.c_void_p]),
        "octree_get_vs": (None, [C.c_void_p, V, C.c_double, V, C.c_int]),
        "euler_step": (None, [T, C.c_double]),
        "rk4_step": (None, [T, C.c_double, C.c_double]),
        "ov_init": (C.c_int, [C.c_int]),
        "ov_last_error": (C.c_int, []),
        "ov_last_error_message": (C.c_char_p, []),
        "ov_error_string": (C.c_char_p, [C.c_int]),
        "ov_clear_error": (None, []),
        "ov_set_precision": (None, [C.c_int]),
        "ov_get_precision": (C.c_int, []),
        "ov_set_rk4_classic": (None, [C.c_int]),
        "ov_get_rk4_classic": (C.c_int, []),
        "ov_get_last_stats": (C.c_int, [C.POINTER(EvalStats)]),
        "ov_state_create": (C.c_void_p, []),
        "ov_state_destroy": (None, [C.c_void_p]),
        "ov_state_upload": (C.c_int, [C.c_void_p, T]),
        "ov_state_download": (C.c_int, [C.c_void_p, T, C.c_int]),
        "ov_state_update_tangle": (C.c_int, [C.c_void_p, C.c_double]),
        "ov_state_rk4_step": (C.c_int, [C.c_void_p, C.c_double, C.c_double]),
        "ov_state_run": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_int]),
        "ov_state_eval_points": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int,
                                           C.c_void_p]),
        "ov_measure_fma_peak": (C.c_int, [C.c_int, C.POINTER(C.c_double)]),
        "ov_check_fast_math": (C.c_int, [C.POINTER(C.c_double), C.POINTER(C.c_double)]),
        "ov_state_shard": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_size_t]),
        "ov_state_shard_bytes": (C.c_size_t, [C.c_void_p, C.c_int]),
        "ov_state_shard_begin": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_double]),
        "ov_state_shard_end": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_double]),
        "shifted": (Vec3d, [C.c_void_p, T, V]),
        "ov_state_get_stats": (C.c_int, [C.c_void_p, C.POINTER(RunStats)]),
        "ov_state_reset_stats": (None, [C.c_void_p]),
        "ov_set_mixed_near_factor": (None, [C.c_double]),
        "ov_get_mixed_near_factor": (C.c_double, []),
        "ov_direct_points_noalloc": (C.c_int, [T, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                               C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
        "ov_batch_create": (C.c_void_p, [T, C.c_int, C.c_void_p]),
        "ov_batch_destroy": (None, [C.c_void_p]),
        "ov_batch_update": (C.c_int, [C.c_void_p, C.c_double]),
        "ov_batch_run": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_int]),
        "ov_batch_download": (C.c_int, [C.c_void_p, T, C.c_int]),
        "ov_batch_set_tuning": (C.c_int, [C.c_void_p, C.POINTER(BatchTuning)]),
        "ov_batch_get_tuning": (C.c_int, [C.c_void_p, C.POINTER(BatchTuning)]),
        "ov_batch_autotune": (C.c_int, [C.c_void_p, C.POINTER(BatchTuning)]),
        "ov_batch_get_stats": (C.c_int, [C.c_void_p, C.POINTER(BatchStats)]),
        "ov_adjoint_create": (C.c_void_p, [T]),
        "ov_adjoint_destroy": (None, [C.c_void_p]),
        "ov_adjoint_velocity": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_void_p]),
        "ov_adjoint_velocity_vjp": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_void_p,
                                              C.c_void_p, C.c_void_p]),
        "ov_adjoint_forward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_double,
                                         C.c_int, C.c_int, C.c_void_p]),
        "ov_adjoint_backward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
        "ov_adjoint_generation": (C.c_ulonglong, [C.c_void_p]),
        "ov_reconnect_candidates": (C.c_int, [T, C.c_double, C.c_double, C.c_void_p, C.c_int]),
        "ov_reconnect_vortices": (C.c_int, [T, C.c_double, C.c_double, C.c_double]),
        "ov_reconnect_get_stats": (C.c_int, [C.POINTER(ReconnectStats)]),
        "ov_set_colinear_cutoff": (None, [C.c_double]),
        "ov_get_colinear_cutoff": (C.c_double, []),
        "ov_remesh": (C.c_int, [T, C.c_double, C.c_double, C.c_void_p]),
        "ov_enforce_boundaries": (C.c_int, [T]),
        "ov_eliminate_small_loops": (C.c_int, [T, C.c_int]),
        "ov_save_tangle": (C.c_int, [T, C.c_char_p]),
        "ov_save_frame": (C.c_int, [T, C.c_char_p, C.c_double, C.c_int]),
        "ov_state_save_frame": (C.c_int, [C.c_void_p, C.c_char_p, C.c_double, C.c_int]),
        "ov_frame_wait": (C.c_int, []),
        "ov_frame_info": (C.c_int, [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_double)]),
        "ov_load_frame": (C.c_int, [C.c_char_p, T, C.POINTER(C.c_double)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    if path is None:
        _lib = lib
    return lib


def check(lib: C.CDLL | None = None):
    """Raise OVError if the last call on this thread failed."""
    lib = lib or load()
    code = lib.ov_last_error()
    if code != OV_OK:
        msg = lib.ov_last_error_message().decode(errors="replace")
        lib.ov_clear_error()
        raise OVError(code, msg)


def stats(lib: C.CDLL | None = None) -> EvalStats:
    lib = lib or load()
    s = EvalStats()
    lib.ov_get_last_stats(C.byref(s))
    return s
