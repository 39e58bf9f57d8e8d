"""ctypes binding of libregb200.so (the C ABI in include/regb200.h).

The library is the product: there is no fallback.  Loading fails loudly when the
.so is missing (build it with ``python -m tipl_b200.build``)."""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libregb200.so")

REGB_OK = 0
REGB_FALSE = 1
REGB_ERR_ARG = -1
REGB_ERR_CUDA = -2
REGB_ERR_NOMEM = -3
REGB_CANCELLED = -4
REGB_ERR_NOTFOUND = -5
REGB_PENDING = -6
REGB_ERR_BUDGET = -7

U8, F32, U16, BF16 = 0, 1, 2, 3
HOST, DEVICE = 0, 1


class Volume(C.Structure):
    _fields_ = [("ptr", C.c_void_p), ("dim", C.c_int * 3), ("dtype", C.c_int), ("location", C.c_int)]


class Field(C.Structure):
    _fields_ = [("ptr", C.c_void_p), ("dim", C.c_int * 3), ("location", C.c_int)]


class LinearParam(C.Structure):
    _fields_ = [("reg_type", C.c_int), ("cost_type", C.c_int), ("bound", C.c_int), ("search_count", C.c_uint),
                ("absolute_bound", C.c_int)]


class CdmParam(C.Structure):
    _fields_ = [("resolution", C.c_float), ("speed", C.c_float), ("smoothing", C.c_float),
                ("min_dimension", C.c_uint), ("gradient_type", C.c_int)]


class Stats(C.Structure):
    _fields_ = [("launches", C.c_longlong), ("mi_launches", C.c_longlong), ("mi_tasks", C.c_longlong),
                ("mi_voxels", C.c_double), ("mi_bytes", C.c_double), ("mi_ms", C.c_double),
                ("corr_launches", C.c_longlong), ("corr_tasks", C.c_longlong), ("corr_voxels", C.c_double),
                ("corr_bytes", C.c_double), ("corr_ms", C.c_double), ("mi_busy_ms", C.c_double),
                ("cdm_iterations", C.c_longlong), ("cdm_voxel_iterations", C.c_double),
                ("cdm_model_bytes", C.c_double)]


class RunnerState(C.Structure):
    _fields_ = [("arg_upper", C.c_float * 12), ("arg_lower", C.c_float * 12), ("reg_list", C.c_int * 8),
                ("n_reg", C.c_int), ("search_count", C.c_uint), ("multi_resolution", C.c_int),
                ("cost_type", C.c_int), ("precision", C.c_double), ("max_iterations", C.c_int)]


class EngineConfig(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_size_t), ("max_active", C.c_int), ("gather_us", C.c_int),
                ("cdm_iters_per_round", C.c_int), ("affine_workers", C.c_int)]


class NiftiInfo(C.Structure):
    _fields_ = [("dim", C.c_int * 3), ("vs", C.c_float * 3), ("srow", C.c_float * 12), ("file_dim", C.c_int * 8),
                ("datatype", C.c_int), ("bitpix", C.c_int), ("nvolumes", C.c_int), ("scl_slope", C.c_float),
                ("scl_inter", C.c_float), ("sform_code", C.c_int), ("is_mni", C.c_int), ("big_endian", C.c_int),
                ("nifti2", C.c_int), ("n_steps", C.c_int), ("steps", C.c_int * 8), ("descrip", C.c_char * 81)]


class Job(C.Structure):
    _fields_ = [("template_id", C.c_int), ("fixed", Volume), ("fixed_vs", C.c_float * 3), ("moving", Volume),
                ("moving_vs", C.c_float * 3), ("run_linear", C.c_int), ("linear", LinearParam),
                ("arg", C.c_float * 12), ("run_cdm", C.c_int), ("cdm", CdmParam), ("field_out", C.c_void_p),
                ("field_location", C.c_int), ("subject_pre", C.c_int), ("mm_reg", C.c_int),
                ("field_rev_out", C.c_void_p), ("mapping_out", C.c_void_p), ("inv_mapping_out", C.c_void_p),
                ("prev_field", C.c_void_p), ("prev_field_rev", C.c_void_p)]


class Result(C.Structure):
    _fields_ = [("status", C.c_int), ("linear_cost", C.c_float), ("arg", C.c_float * 12),
                ("cost_evals", C.c_longlong), ("cdm_ok", C.c_int), ("cdm_iterations", C.c_int),
                ("queued_ms", C.c_double), ("run_ms", C.c_double), ("cdm_rev_ok", C.c_int),
                ("r_linear", C.c_double), ("r_nonlinear", C.c_double)]


class EngineStats(C.Structure):
    _fields_ = [("queued", C.c_int), ("running", C.c_int), ("used_bytes", C.c_size_t),
                ("budget_bytes", C.c_size_t), ("affine_launches", C.c_longlong), ("affine_tasks", C.c_longlong),
                ("cdm_rounds", C.c_longlong), ("cdm_round_segments", C.c_longlong),
                ("cdm_round_ms", C.c_double), ("cdm_max_round_segments", C.c_int)]


class RegbError(RuntimeError):
    def __init__(self, status: int, what: str):
        super().__init__(f"regb status {status}: {what}")
        self.status = status


_lib = None

# name -> (restype, argtypes)
_SIGS = {
    "regb_version": (C.c_char_p, []),
    "regb_last_error": (C.c_char_p, []),
    "regb_device_info": (C.c_int, [C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_size_t),
                                   C.POINTER(C.c_size_t)]),
    "regb_release": (C.c_int, []),
    "regb_stats_reset": (C.c_int, [C.c_int]),
    "regb_stats_get": (C.c_int, [C.POINTER(Stats)]),
    "regb_linear_param_default": (None, [C.POINTER(LinearParam)]),
    "regb_cdm_param_default": (None, [C.POINTER(CdmParam)]),
    "regb_affine_to_matrix": (C.c_int, [C.c_void_p] * 6),
    "regb_affine_to_matrix_f64": (C.c_int, [C.c_void_p] * 6),
    "regb_matrix_inverse": (C.c_int, [C.c_void_p]),
    "regb_matrix_to_affine_param": (C.c_int, [C.c_void_p] * 6),
    "regb_has_mask": (C.c_int, [C.c_void_p, C.c_void_p]),
    "regb_normalize_to_u8": (C.c_int, [C.c_void_p, C.c_void_p, C.c_float, C.c_void_p]),
    "regb_widen_to_f32": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "regb_gaussian": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    "regb_displacement_to_mapping": (C.c_int, [C.c_void_p] * 4),
    "regb_inv_displacement_to_mapping": (C.c_int, [C.c_void_p] * 4),
    "regb_compose_mapping": (C.c_int, [C.c_void_p] * 4),
    "regb_match_fov": (C.c_int, [C.c_void_p] * 5),
    "regb_autotune": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "regb_tuning_get": (C.c_int, [C.c_void_p]),
    "regb_nifti_info_read": (C.c_int, [C.c_char_p, C.POINTER(NiftiInfo)]),
    "regb_nifti_load": (C.c_int, [C.c_char_p, C.c_int, C.POINTER(Volume), C.c_void_p, C.c_void_p]),
    "regb_nifti_save": (C.c_int, [C.c_char_p, C.POINTER(Volume), C.c_void_p, C.c_void_p, C.c_int, C.c_char_p]),
    "regb_correlation": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_double)]),
    "regb_subject_image_pre": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "regb_estimate_affine_param": (C.c_int, [C.c_void_p] * 5),
    "regb_resample": (C.c_int, [C.POINTER(Volume), C.POINTER(Volume), C.c_void_p, C.c_int, C.c_void_p]),
    "regb_mi_cost": (C.c_int, [C.POINTER(Volume), C.POINTER(Volume), C.c_void_p, C.c_int, C.c_void_p,
                               C.c_void_p, C.c_void_p]),
    "regb_mi32_cost": (C.c_int, [C.POINTER(Volume), C.POINTER(Volume), C.c_void_p, C.c_int, C.c_void_p,
                                 C.c_void_p, C.c_void_p]),
    "regb_mi_cost_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                       C.c_void_p, C.c_void_p]),
    "regb_corr_cost": (C.c_int, [C.POINTER(Volume), C.POINTER(Volume), C.c_void_p, C.c_int, C.c_void_p,
                                 C.c_void_p]),
    "regb_compose_displacement": (C.c_int, [C.POINTER(Volume), C.POINTER(Field), C.POINTER(Volume), C.c_void_p]),
    "regb_accumulate_displacement": (C.c_int, [C.POINTER(Field), C.POINTER(Field), C.c_void_p]),
    "regb_downsample": (C.c_int, [C.POINTER(Volume), C.POINTER(Volume), C.c_void_p]),
    "regb_upsample_field_x2": (C.c_int, [C.POINTER(Field), C.POINTER(Field), C.c_void_p]),
    "regb_cdm_gradient": (C.c_int, [C.POINTER(Volume), C.POINTER(Volume), C.POINTER(Field), C.c_int,
                                    C.POINTER(C.c_float), C.c_void_p]),
    "regb_cdm_poisson": (C.c_int, [C.POINTER(Field), C.c_void_p]),
    "regb_cdm_max_length": (C.c_int, [C.POINTER(Field), C.POINTER(C.c_float), C.c_void_p]),
    "regb_cdm_smooth": (C.c_int, [C.POINTER(Field), C.POINTER(Field), C.c_float, C.c_void_p]),
    "regb_cdm": (C.c_int, [C.POINTER(Volume), C.POINTER(Volume), C.POINTER(Field), C.POINTER(CdmParam),
                           C.c_void_p]),
    "regb_debug_fail_allocations": (C.c_int, [C.c_size_t, C.c_int]),
    "regb_autotune_buckets": (C.c_int, [C.c_char_p, C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int)]),
    "regb_tuning_get_buckets": (C.c_int, [C.c_void_p]),
    "regb_mm_reg_export_fields": (C.c_int, [C.c_char_p, C.POINTER(Field), C.POINTER(Field), C.c_void_p, C.c_void_p]),
    "regb_cdm_multi": (C.c_int, [C.POINTER(Volume), C.POINTER(Volume), C.c_int, C.POINTER(Field),
                                 C.POINTER(CdmParam), C.c_char_p, C.c_void_p]),
    "regb_cdm2d_multi": (C.c_int, [C.POINTER(Volume), C.POINTER(Volume), C.c_int, C.POINTER(Field),
                                   C.POINTER(CdmParam), C.c_char_p, C.c_void_p]),
    "regb_runner_state_from_param": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                               C.POINTER(LinearParam), C.POINTER(RunnerState)]),
    "regb_linear_run": (C.c_int, [C.POINTER(Volume), C.c_void_p, C.POINTER(Volume), C.c_void_p, C.c_void_p,
                                  C.POINTER(RunnerState), C.c_void_p, C.POINTER(C.c_float),
                                  C.POINTER(C.c_longlong)]),
    "regb_linear_run_multi": (C.c_int, [C.POINTER(Volume), C.c_void_p, C.POINTER(Volume), C.c_void_p, C.c_int,
                                        C.c_void_p, C.POINTER(RunnerState), C.c_void_p, C.POINTER(C.c_float),
                                        C.POINTER(C.c_longlong)]),
    "regb_engine_config_default": (None, [C.POINTER(EngineConfig)]),
    "regb_job_default": (None, [C.POINTER(Job)]),
    "regb_engine_create": (C.c_int, [C.POINTER(EngineConfig), C.POINTER(C.c_void_p)]),
    "regb_engine_destroy": (C.c_int, [C.c_void_p]),
    "regb_engine_add_template": (C.c_int, [C.c_void_p, C.POINTER(Volume), C.c_void_p, C.POINTER(C.c_int)]),
    "regb_engine_submit": (C.c_int, [C.c_void_p, C.POINTER(Job), C.POINTER(C.c_uint64)]),
    "regb_engine_poll": (C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(Result)]),
    "regb_engine_wait": (C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(Result)]),
    "regb_engine_cancel": (C.c_int, [C.c_void_p, C.c_uint64]),
    "regb_engine_release_job": (C.c_int, [C.c_void_p, C.c_uint64]),
    "regb_engine_get_stats": (C.c_int, [C.c_void_p, C.POINTER(EngineStats)]),
    "regb_linear": (C.c_int, [C.POINTER(Volume), C.c_void_p, C.POINTER(Volume), C.c_void_p, C.c_void_p,
                              C.POINTER(LinearParam), C.c_void_p, C.POINTER(C.c_float),
                              C.POINTER(C.c_longlong)]),
    "regb_linear_multi": (C.c_int, [C.POINTER(Volume), C.c_void_p, C.POINTER(Volume), C.c_void_p, C.c_int,
                                    C.c_void_p, C.POINTER(LinearParam), C.c_void_p, C.POINTER(C.c_float),
                                    C.POINTER(C.c_longlong)]),
}


def lib():
    """The loaded library (raises when it is absent)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m tipl_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def declared_symbols():
    return sorted(_SIGS)


def check(status: int, allow=(REGB_OK,)) -> int:
    if status in allow:
        return status
    msg = lib().regb_last_error()
    raise RegbError(status, msg.decode() if msg else "")
