"""ctypes binding of libbaemm_cuda.so (include/baemm.h).

The library is loaded from this package directory only; there is no fallback:
if the shared object is missing or cannot be loaded, ``lib()`` raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbaemm_cuda.so")

BAEMM_OK = 0
STATUS_NAMES = {
    0: "BAEMM_OK", 1: "BAEMM_ERR_ARG", 2: "BAEMM_ERR_CUDA", 3: "BAEMM_ERR_ALLOC",
    4: "BAEMM_ERR_NOT_LOADED", 5: "BAEMM_ERR_NOT_CONVERGED", 6: "BAEMM_ERR_SIZE", 7: "BAEMM_ERR_TIMEOUT",
}
WAVE_PLANE = 201
WAVE_RADIAL = 202
APPLY_FP32 = 0
APPLY_TC = 1
APPLY_FP64 = 2
TUNE_DENSE_VARIANT = 1
TUNE_TC_SEGMENT = 2
TUNE_TC_CTAS = 3
TUNE_TC_STAGGER = 4
TUNE_TC_GEN_WARPS = 5
TUNE_TC_CHUNKS = 6
TUNE_TC_SHARE = 7

dp = C.POINTER(C.c_double)
fp = C.POINTER(C.c_float)
i32p = C.POINTER(C.c_int32)
i64p = C.POINTER(C.c_int64)
vp = C.c_void_p
REAL_OP = C.CFUNCTYPE(None, dp, dp, C.c_void_p)


class SolveStats(C.Structure):
    _fields_ = [
        ("gmres_iterations", C.c_int32),
        ("gmres_converged", C.c_int32),
        ("gmres_relative_residual", C.c_double),
        ("cg_iterations", C.c_int32),
        ("cg_converged", C.c_int32),
        ("refinement_steps", C.c_int32),
        ("seconds", C.c_double),
    ]


class TuneResult(C.Structure):
    _fields_ = [
        ("apply_mode", C.c_int32),
        ("dense_variant", C.c_int32),
        ("tc_segment", C.c_int32),
        ("tc_ctas", C.c_int32),
        ("tc_stagger", C.c_int32),
        ("candidates", C.c_int32),
        ("best_ms", C.c_double),
        ("before_ms", C.c_double),
        ("tc_gen_warps", C.c_int32),
        ("tc_chunks", C.c_int32),
        ("cached", C.c_int32),
        ("reserved", C.c_int32),
    ]


I, I64, D = C.c_int, C.c_int64, C.c_double
# name -> (restype, argtypes); every symbol declared in include/baemm.h
SIGNATURES = {
    "baemm_create": (I, [dp, I64, i64p, I64, dp, I64, I, I, C.POINTER(vp)]),
    "baemm_create_i32": (I, [dp, I64, i32p, I64, dp, I64, I, I, C.POINTER(vp)]),
    "baemm_destroy": (None, [vp]),
    "baemm_last_error": (C.c_char_p, [vp]),
    "baemm_device_info": (I, [vp, C.c_char_p, C.c_size_t]),
    "baemm_class_name": (C.c_char_p, []),
    "baemm_stream": (vp, [vp]),
    "baemm_set_stream": (I, [vp, vp]),
    "baemm_synchronize": (I, [vp]),
    "baemm_vertex_count": (I64, [vp]),
    "baemm_simplex_count": (I64, [vp]),
    "baemm_meas_count": (I64, [vp]),
    "baemm_get_wave_count": (I, [vp]),
    "baemm_get_wave_chunk_size": (I, [vp]),
    "baemm_set_wave_chunk_size": (I, [vp, I]),
    "baemm_get_block_size": (I, [vp]),
    "baemm_set_block_size": (I, [vp, I]),
    "baemm_use_diagonal": (I, [vp, I]),
    "baemm_set_gmres_params": (I, [vp, I, I]),
    "baemm_get_gmres_params": (I, [vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "baemm_set_apply_mode": (I, [vp, I]),
    "baemm_get_apply_mode": (I, [vp]),
    "baemm_set_tuning": (I, [vp, I, I]),
    "baemm_set_mesh": (I, [vp, dp, I64, i64p, I64]),
    "baemm_set_graphs": (I, [vp, I]),
    "baemm_graph_stats": (I, [vp, i64p, i64p]),
    "baemm_autotune": (I, [vp, I, I, C.POINTER(TuneResult)]),
    "baemm_get_tuning": (I, [vp, I]),
    "baemm_tc_entry_sharing": (I, [vp]),
    "baemm_set_refinement": (I, [vp, I, D]),
    "baemm_get_areas": (I, [vp, fp]),
    "baemm_get_triangle_normals": (I, [vp, fp]),
    "baemm_get_triangle_midpoints": (I, [vp, fp]),
    "baemm_get_single_layer_diagonal": (I, [vp, fp]),
    "baemm_get_mass_matrix": (I, [vp, i64p, i32p, fp, i64p]),
    "baemm_get_curl_operator": (I, [vp, i64p, i32p, fp, i64p]),
    "baemm_last_solve_stats": (I, [vp, C.POINTER(SolveStats)]),
    "baemm_load_parameters": (I, [vp, dp, dp, I, I, D]),
    "baemm_load_boundary_operators": (I, [vp, dp, dp, I, I]),
    "baemm_unload_boundary_operators": (I, [vp]),
    "baemm_apply_boundary_operators_z": (I, [vp, dp, dp, I64, dp, dp, I64]),
    "baemm_apply_boundary_operators_c": (I, [vp, fp, fp, I64, fp, fp, I64]),
    "baemm_apply_boundary_operators_dev_z": (I, [vp, dp, vp, I64, dp, vp, I64]),
    "baemm_apply_boundary_operators_dev_c": (I, [vp, fp, vp, I64, fp, vp, I64]),
    "baemm_apply_boundary_operators_noalloc_dev_c": (I, [vp, fp, vp, I64, fp, vp, I64]),
    "baemm_apply_boundary_operators_full_z": (I, [vp, dp, dp, I64, dp, dp, I64, dp, dp, I, I]),
    "baemm_apply_far_field_operators_z": (I, [vp, dp, dp, I64, dp, dp, I64, dp, dp, I, I]),
    "baemm_apply_far_field_operators_loaded_z": (I, [vp, dp, dp, I64, dp, dp, I64]),
    "baemm_apply_far_field_operators_dev_z": (I, [vp, dp, vp, I64, dp, vp, I64]),
    "baemm_apply_boundary_operators_rows_dev_z": (I, [vp, dp, vp, I64, dp, vp, I64, I64, I64, I]),
    "baemm_apply_boundary_operators_rows_dev_c": (I, [vp, fp, vp, I64, fp, vp, I64, I64, I64, I]),
    "baemm_boundary_operator_kernel_dev_c": (I, [vp, vp, vp, I64, I64]),
    "baemm_boundary_operator_kernel_dev_z": (I, [vp, vp, vp, I64, I64]),
    "baemm_apply_near_field_operators_z": (I, [vp, dp, dp, I64, dp, dp, I64, dp, I64]),
    "baemm_apply_near_field_operators_c": (I, [vp, fp, fp, I64, fp, fp, I64, fp, I64]),
    "baemm_apply_near_field_operators_full_z": (I, [vp, dp, dp, I64, dp, dp, I64, dp, dp, I, I, dp, I64]),
    "baemm_apply_near_field_operators_dev_z": (I, [vp, dp, vp, I64, dp, vp, I64, vp, I64]),
    "baemm_apply_near_field_operators_dev_c": (I, [vp, fp, vp, I64, fp, vp, I64, vp, I64]),
    "baemm_create_incident_wave_z": (I, [vp, dp, dp, I, dp, dp, I64, dp, dp, I, I, I]),
    "baemm_create_incident_wave_loaded_z": (I, [vp, dp, dp, dp, dp, I64, I]),
    "baemm_create_herglotz_wave_z": (I, [vp, dp, dp, I64, dp, dp, I64, dp, dp, I, I]),
    "baemm_create_herglotz_wave_loaded_z": (I, [vp, dp, dp, I64, dp, dp, I64]),
    "baemm_apply_mass_inverse_z": (I, [vp, dp, I64, dp, I64, I, D]),
    "baemm_apply_mass_inverse_d": (I, [vp, dp, I64, dp, I64, I, D]),
    "baemm_apply_lumped_mass_inverse_z": (I, [vp, dp, I64, dp, I64, I]),
    "baemm_apply_lumped_mass_inverse_d": (I, [vp, dp, I64, dp, I64, I]),
    "baemm_mass_dot_d": (I, [vp, D, dp, I64, D, dp, I64, I]),
    "baemm_far_field": (I, [vp, dp, I, dp, I, dp, I, D, D]),
    "baemm_far_field_parameters": (I, [vp, dp, I, dp, I, dp, I, dp, D, D]),
    "baemm_boundary_potential": (I, [vp, dp, dp, dp, dp, I, I, D, D]),
    "baemm_dirichlet_to_neumann": (I, [vp, dp, dp, dp, I, I, D, D]),
    "baemm_derivative_ff_helper": (I, [vp, dp, I, dp, I, dp, I, D, D]),
    "baemm_derivative_ff": (I, [vp, dp, I, dp, I, dp, dp, C.POINTER(dp), I, D, D]),
    "baemm_adjoint_derivative_ff": (I, [vp, dp, I, dp, I, dp, dp, C.POINTER(dp), I, D, D]),
    "baemm_gauss_newton_solve": (I, [vp, dp, I, dp, I, REAL_OP, vp, REAL_OP, vp, D, dp, I64, D, dp, I64,
                                     C.POINTER(dp), I, D, D, D, I, C.POINTER(C.c_int)]),
    "baemm_set_profiling": (I, [vp, I]),
    "baemm_profile_krylov": (I, [vp, I, I, I, dp]),
    "baemm_autotune_forget": (None, []),
    "baemm_packer_create": (vp, [I, I]),
    "baemm_packer_destroy": (None, [vp]),
    "baemm_set_packer": (I, [vp, vp]),
    "baemm_packer_stats": (I, [vp, i64p, i64p]),
    "baemm_selftest_bounded_wait": (I, [I, dp, i32p]),
    "baemm_profile_cg": (I, [vp, I, I, dp]),
    "baemm_last_apply_times": (I, [vp, fp]),
    "baemm_kernel_launch_count": (I64, []),
    "baemm_free": (None, [vp]),
}

_lib = None


def lib():
    """Load libbaemm_cuda.so (no fallback: raises if it is missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"libbaemm_cuda.so not found at {LIB_PATH}; build it with `python -m baemm_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class BaemmError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status
