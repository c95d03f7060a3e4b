"""ctypes declarations of include/sbr.h (the libsbr C ABI)."""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsbr.so")

SBR_OK = 0
STATUS_NAMES = {
    0: "SBR_OK", 1: "SBR_ERR_INVALID_ARG", 2: "SBR_ERR_EMPTY_MESH", 3: "SBR_ERR_BAD_INDEX",
    4: "SBR_ERR_NONFINITE", 5: "SBR_ERR_TOO_LARGE", 6: "SBR_ERR_CUDA", 7: "SBR_ERR_OOM",
    8: "SBR_ERR_NO_DEVICE", 9: "SBR_ERR_STACK", 10: "SBR_ERR_TIMEOUT", 11: "SBR_ERR_CANCELLED",
    12: "SBR_ERR_IO", 13: "SBR_ERR_PARSE", 14: "SBR_ERR_UNSUPPORTED",
}
MODE_BATCHED, MODE_PER_ANGLE = 0, 1
FIRST_HIT_AUTO, FIRST_HIT_RASTER, FIRST_HIT_TRAVERSE = 0, 1, 2
PREC_MIXED, PREC_FP32, PREC_FP64 = 0, 1, 2
POL_SCALAR, POL_HHVV = 0, 1
MAX_REC = 16


class BuildOpts(C.Structure):
    _fields_ = [
        ("model_scale", C.c_double),
        ("device", C.c_int32),
        ("leaf_size", C.c_int32),
        ("bin_count", C.c_int32),
        ("n_threads", C.c_int32),
        ("want_fp64", C.c_int32),
        ("gpu_build", C.c_int32),
        ("node_width", C.c_int32),
        ("reserved", C.c_int32 * 1),
    ]


class SceneInfo(C.Structure):
    _fields_ = [
        ("n_triangles", C.c_int64),
        ("n_nodes_bin", C.c_int64),
        ("n_nodes_gpu", C.c_int64),
        ("device_bytes", C.c_int64),
        ("aabb_lo", C.c_double * 3),
        ("aabb_hi", C.c_double * 3),
        ("build_ms", C.c_double),
        ("device", C.c_int32),
        ("bvh_depth", C.c_int32),
        ("sah_ms", C.c_double),
    ]


class Job(C.Structure):
    _fields_ = [
        ("theta_deg", C.c_void_p),
        ("phi_deg", C.c_void_p),
        ("n_angles", C.c_int64),
        ("freq_hz", C.c_void_p),
        ("n_freqs", C.c_int64),
        ("nx", C.c_int32),
        ("ny", C.c_int32),
        ("grid_size", C.c_double),
        ("max_bounces", C.c_int32),
        ("reflection_const", C.c_double),
    ]


class RunOpts(C.Structure):
    _fields_ = [
        ("mode", C.c_int32),
        ("precision", C.c_int32),
        ("polarization", C.c_int32),
        ("use_graph", C.c_int32),
        ("stream", C.c_void_p),
        ("ctas_per_sm", C.c_int32),
        ("first_hit", C.c_int32),
        ("blocks_per_item", C.c_int32),
        ("autotune", C.c_int32),
        ("node_width", C.c_int32),
        ("tile_cap", C.c_int32),
        ("reserved", C.c_int32 * 2),
    ]


class Result(C.Structure):
    _fields_ = [
        ("field", C.c_void_p),
        ("sigma_m2", C.c_void_p),
        ("rcs_dbsm", C.c_void_p),
        ("stats", C.c_void_p),
        ("device_ms", C.c_double),
    ]


class PlanInfo(C.Structure):
    _fields_ = [
        ("n_samples", C.c_int64),
        ("n_job_angles", C.c_int64),
        ("n_items", C.c_int64),
        ("n_rays_clipped", C.c_int64),
        ("n_rays_grid", C.c_int64),
        ("n_pol", C.c_int32),
        ("launches_per_execute", C.c_int32),
        ("device_bytes", C.c_int64),
        ("h2d_bytes", C.c_int64),
        ("d2h_bytes", C.c_int64),
        ("blocks_per_item", C.c_int32),
        ("ctas_per_sm", C.c_int32),
        ("node_width", C.c_int32),
        ("first_hit", C.c_int32),
    ]


class Config(C.Structure):
    _fields_ = [
        ("phi_start", C.c_double),
        ("phi_end", C.c_double),
        ("phi_samples", C.c_int32),
        ("theta_start", C.c_double),
        ("theta_end", C.c_double),
        ("theta_samples", C.c_int32),
        ("grid_size", C.c_double),
        ("nx", C.c_int32),
        ("ny", C.c_int32),
        ("tpb_x", C.c_int32),
        ("tpb_y", C.c_int32),
        ("max_bounces", C.c_int32),
        ("reflection_const", C.c_double),
        ("freq", C.c_double),
        ("show_info_gpu", C.c_int32),
        ("show_hit_stats", C.c_int32),
        ("model_scale", C.c_double),
        ("model_path", C.c_char * 4096),
        ("freq_source", C.c_int32),
        ("precision", C.c_int32),
        ("mode", C.c_int32),
        ("csv_digits", C.c_int32),
        ("error_bound", C.c_int32),
    ]


RAY_RECORD_FIELDS = [
    ("count", "i4"),
    ("flags", "i4"),
    ("dist", "f8"),
    ("normal", "f4", 3),
    ("lastdir", "f4", 3),
    ("tri", "i4", MAX_REC),
]

# Every function the header declares, with its ctypes signature.
_P, _I64, _I32, _SZ, _D = C.c_void_p, C.c_int64, C.c_int32, C.c_size_t, C.c_double
SIGNATURES = {
    "sbr_status_str": (C.c_char_p, [_I32]),
    "sbr_last_error": (C.c_char_p, []),
    "sbr_abi_version": (_I32, []),
    "sbr_scene_create": (_I32, [_P, _SZ, _P, _SZ, _P, _P]),
    "sbr_scene_destroy": (_I32, [_P]),
    "sbr_scene_info_get": (_I32, [_P, _P]),
    "sbr_scene_cancel": (_I32, [_P]),
    "sbr_scene_reset_cancel": (_I32, [_P]),
    "sbr_plan_create": (_I32, [_P, _P, _SZ, _P, _P]),
    "sbr_plan_execute": (_I32, [_P]),
    "sbr_plan_results": (_I32, [_P, _P]),
    "sbr_plan_device_results": (_I32, [_P, _P, _P]),
    "sbr_plan_info_get": (_I32, [_P, _P]),
    "sbr_plan_destroy": (_I32, [_P]),
    "sbr_run": (_I32, [_P, _P, _SZ, _P, _P]),
    "sbr_trace_records": (_I32, [_P, _P, _P, _P]),
    "sbr_trace_ray_list": (_I32, [_P, _P, _P, _P, _SZ, _P]),
    "sbr_error_bound": (_I32, [_P, _P, _SZ, _P, _P, _P, _P]),
    "sbr_run_noalloc": (_I32, [_P, _P, _P, _P, _P]),
    "sbr_adjoint": (_I32, [_P, _P, C.c_size_t, _P, _P, _P, _P]),
    "sbr_scene_update_vertices": (_I32, [_P, _P, _SZ]),
    "sbr_load_gltf": (_I32, [C.c_char_p, _P, _P, _P, _P]),
    "sbr_load_model": (_I32, [C.c_char_p, _P, _P, _P, _P]),
    "sbr_plan_create_multi": (_I32, [_P, _SZ, _P, _P, _SZ, _P, _P]),
    "sbr_config_load": (_I32, [C.c_char_p, C.c_int, _P, _P]),
    "sbr_config_angles": (_I32, [_P, _P, _P]),
    "sbr_load_obj": (_I32, [C.c_char_p, _P, _P, _P, _P]),
    "sbr_free": (None, [_P]),
    "sbr_write_csv": (_I32, [C.c_char_p, _P, _P, _P, _P, _P, _I64]),
    "sbr_write_csv_err": (_I32, [C.c_char_p, _P, _P, _P, _P, _P, _P, _I64]),
}

_lib = None


class SbrError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str = ""):
        self.status = status
        name = STATUS_NAMES.get(status, f"status {status}")
        super().__init__(f"{where}: {name}" + (f" ({detail})" if detail else ""))


def lib():
    """Loads libsbr.so.  There is no fallback: without the library nothing runs."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"libsbr.so is not built ({LIB_PATH}); run `make -C sagittasbr_b200/csrc` "
                "or __graft_entry__.build()")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(status: int, where: str) -> None:
    if status != SBR_OK:
        detail = lib().sbr_last_error()
        raise SbrError(status, where, detail.decode() if detail else "")
