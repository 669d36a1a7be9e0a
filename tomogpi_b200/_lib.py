"""ctypes binding of libtomogpi_b200.so (the C-ABI in include/tomogpi_b200.h).

The library is the only compute path: if it is missing or cannot be loaded, every
operator raises ``LibraryError``; nothing falls back to a CPU implementation.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("TOMOGPI_B200_LIB", str(HERE / "libtomogpi_b200.so")))

# enums (include/tomogpi_b200.h)
TOMO_OK = 0
STATUS = {0: "TOMO_OK", 1: "TOMO_ERR_INVALID", 2: "TOMO_ERR_CUDA", 3: "TOMO_ERR_NO_MEMORY",
          4: "TOMO_ERR_UNSUPPORTED", 5: "TOMO_ERR_TIMEOUT", 6: "TOMO_ERR_NUMERIC",
          7: "TOMO_ERR_IO"}
F32, BF16, F16 = 0, 1, 2
PROJ_RS, PROJ_RS_UM, PROJ_SIDDON_REF, PROJ_SIDDON = 0, 1, 2, 3
RS_LAYOUT_PLAIN, RS_LAYOUT_CELL8, RS_LAYOUT_TEX, RS_LAYOUT_HYBRID, RS_LAYOUT_MARCH = 0, 1, 2, 3, 4
BACK_VI, BACK_VI_UM, BACK_RS_ADJOINT, BACK_SIDDON_ADJOINT, BACK_RS_UM_ADJOINT, BACK_FDK = 0, 1, 2, 3, 4, 5

# Every exported entry point and its signature; tests check the library exports all of
# them and that each is declared in the header.
_vp = ctypes.c_void_p
_i32 = ctypes.c_int32


class TomoConfigCT(ctypes.Structure):
    _fields_ = [
        ("fod", ctypes.c_double), ("fdd", ctypes.c_double),
        ("num_start_angle", ctypes.c_double), ("den_start_angle", ctypes.c_double),
        ("num_stop_angle", ctypes.c_double), ("den_stop_angle", ctypes.c_double),
        ("projection_nb", _i32),
        ("u_detector_size", ctypes.c_float), ("v_detector_size", ctypes.c_float),
        ("u_detector_pixel_nb", _i32), ("v_detector_pixel_nb", _i32),
        ("x_volume_size", ctypes.c_float), ("y_volume_size", ctypes.c_float), ("z_volume_size", ctypes.c_float),
        ("x_volume_pixel_nb", _i32), ("y_volume_pixel_nb", _i32), ("z_volume_pixel_nb", _i32),
    ]


class TomoTuning(ctypes.Structure):
    _fields_ = [("rs_layout", _i32), ("vi_zc", _i32), ("vi_layout", _i32), ("rs_warp_u", _i32), ("rs_tile_u", _i32),
                ("reserved", _i32 * 3)]


class TomoTiffConfig(ctypes.Structure):
    _fields_ = [(n, _i32) for n in (
        "total_projection_nb", "used_projection_nb", "u_initial_nb", "v_initial_nb", "u_final_nb", "v_final_nb",
        "u_center_final", "v_center_final", "u_calibration_nb", "v_calibration_nb", "calibration_energy_nb",
        "digits")]


class TomoSolverStats(ctypes.Structure):
    _fields_ = [("proj_ms", ctypes.c_double), ("proj_launches", _i32), ("back_ms", ctypes.c_double),
                ("back_launches", _i32), ("kernel_launches", ctypes.c_int64)]


class TomoGradientParams(ctypes.Structure):
    _fields_ = [
        ("projector", ctypes.c_int), ("backprojector", ctypes.c_int), ("storage", ctypes.c_int),
        ("gradient_iteration_nb", _i32), ("optimal_step_iteration_nb", _i32),
        ("regularization_parameter", ctypes.c_double), ("positivity", _i32), ("real_sinogram_f32", _i32),
    ]


SIGNATURES = {
    "tomo_last_error": (ctypes.c_char_p, []),
    "tomo_version": (ctypes.c_char_p, []),
    "tomo_context_create": (ctypes.c_int, [ctypes.POINTER(TomoConfigCT), ctypes.c_int, ctypes.POINTER(_vp)]),
    "tomo_context_destroy": (ctypes.c_int, [_vp]),
    "tomo_context_geometry": (ctypes.c_int, [_vp, _vp, _vp, _vp]),
    "tomo_context_errors": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_uint), ctypes.c_int]),
    "tomo_context_get_tuning": (ctypes.c_int, [_vp, ctypes.POINTER(TomoTuning)]),
    "tomo_context_set_tuning": (ctypes.c_int, [_vp, ctypes.POINTER(TomoTuning)]),
    "tomo_context_test_stall": (ctypes.c_int, [_vp, ctypes.c_int]),
    "tomo_context_rs_layout": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(_i32)]),
    "tomo_project": (ctypes.c_int, [_vp, ctypes.c_int, _vp, ctypes.c_int, _vp, ctypes.c_int, _vp]),
    "tomo_backproject": (ctypes.c_int, [_vp, ctypes.c_int, _vp, ctypes.c_int, _vp, ctypes.c_int, _vp]),
    "tomo_project_host": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp]),
    "tomo_ramp_filter": (ctypes.c_int, [_vp, _vp, ctypes.c_int, _vp, _i32, ctypes.c_double, _vp]),
    "tomo_ramp_filter_host": (ctypes.c_int, [_vp, _vp, _vp, _i32, ctypes.c_double]),
    "tomo_solver_set_regularizer": (ctypes.c_int, [_vp, _i32, ctypes.c_double]),
    "tomo_solver_set_gg_beta": (ctypes.c_int, [_vp, ctypes.c_double]),
    "tomo_solver_set_weights": (ctypes.c_int, [_vp, _vp, _i32, _vp]),
    "tomo_context_create_views": (ctypes.c_int, [_vp, ctypes.c_int, _i32, _i32, _vp]),
    "tomo_solver_phase": (ctypes.c_int, [_vp, _vp, _vp, _i32, _i32, _vp]),
    "tomo_solver_buffers": (ctypes.c_int, [_vp, _vp, _vp]),
    "tomo_huber_regularization": (ctypes.c_int, [_vp, _vp, _i32, _i32, _i32, ctypes.c_double, ctypes.c_double, _i32,
                                                 _i32, _vp, _vp]),
    "tomo_laplacian_host": (ctypes.c_int, [ctypes.c_int, _vp, _vp, _i32, _i32, _i32]),
    "tomo_regularization_host": (ctypes.c_int, [ctypes.c_int, _i32, _vp, _vp, _i32, _i32, _i32, ctypes.c_double,
                                                ctypes.c_double, ctypes.c_double, _i32, _i32, _vp]),
    "tomo_gg_regularization": (ctypes.c_int, [_vp, _vp, _i32, _i32, _i32, ctypes.c_double, _i32, _i32, _vp, _vp]),
    "tomo_gg_regularization_beta": (ctypes.c_int, [_vp, _vp, _i32, _i32, _i32, ctypes.c_double, ctypes.c_double, _i32,
                                                   _i32, _vp, _vp]),
    "tomo_tiff_white_mean": (ctypes.c_int, [ctypes.c_char_p, _i32, _i32, _i32, _vp]),
    "tomo_tiff_negative_log_sinogram": (ctypes.c_int, [_vp, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, _vp]),
    "tomo_backproject_host": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp]),
    "tomo_project_noalloc": (ctypes.c_int, [ctypes.POINTER(TomoConfigCT), ctypes.c_int, ctypes.c_int, _vp, _vp, _vp]),
    "tomo_count_samples": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(ctypes.c_ulonglong), _vp]),
    "tomo_solver_create": (ctypes.c_int, [_vp, ctypes.POINTER(TomoGradientParams), ctypes.POINTER(_vp)]),
    "tomo_solver_destroy": (ctypes.c_int, [_vp]),
    "tomo_solver_iterate": (ctypes.c_int, [_vp, _vp, _vp, _i32, _i32, _vp]),
    "tomo_solver_iterate_host": (ctypes.c_int, [_vp, _vp, _vp, _i32, _i32, _vp]),
    "tomo_solver_set_timing": (ctypes.c_int, [_vp, ctypes.c_int]),
    "tomo_solver_get_stats": (ctypes.c_int, [_vp, ctypes.POINTER(TomoSolverStats), ctypes.c_int, _vp]),
    "tomo_solver_alphas": (ctypes.c_int, [_vp, _vp, _i32, ctypes.POINTER(_i32), _vp]),
    "tomo_solver_get_state": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(_i32), _vp]),
    "tomo_solver_set_state": (ctypes.c_int, [_vp, ctypes.c_double, _i32, _vp]),
    "tomo_batch_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(TomoGradientParams), ctypes.POINTER(_vp)]),
    "tomo_batch_destroy": (ctypes.c_int, [_vp]),
    "tomo_batch_footprint": (ctypes.c_int, [ctypes.POINTER(TomoConfigCT), ctypes.POINTER(TomoGradientParams),
                                            ctypes.POINTER(TomoTuning), ctypes.POINTER(ctypes.c_size_t)]),
    "tomo_batch_add": (ctypes.c_int, [_vp, ctypes.POINTER(TomoConfigCT), ctypes.POINTER(TomoTuning), _vp, _vp,
                                      ctypes.POINTER(_i32)]),
    "tomo_batch_remove": (ctypes.c_int, [_vp, _i32]),
    "tomo_batch_set_graph": (ctypes.c_int, [_vp, ctypes.c_int]),
    "tomo_batch_set_share": (ctypes.c_int, [_vp, ctypes.c_double]),
    "tomo_batch_set_priority": (ctypes.c_int, [_vp, _i32]),
    "tomo_batch_trim": (ctypes.c_int, [_vp, _vp]),
    "tomo_batch_host_times": (ctypes.c_int, [_vp, _vp]),
    "tomo_batch_iterate": (ctypes.c_int, [_vp, _i32, _vp]),
    "tomo_batch_job_status": (ctypes.c_int, [_vp, _i32, ctypes.POINTER(_i32), ctypes.POINTER(ctypes.c_double), _vp]),
    "tomo_batch_job_alphas": (ctypes.c_int, [_vp, _i32, _vp, _i32, ctypes.POINTER(_i32), _vp]),
    "tomo_batch_stats": (ctypes.c_int, [_vp, ctypes.POINTER(_i32), ctypes.POINTER(ctypes.c_int64),
                                        ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_int64)]),
    "tomo_laplacian": (ctypes.c_int, [_vp, _vp, _i32, _i32, _i32, _vp]),
    "tomo_sq_norm": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_size_t, _vp, _vp]),
    "tomo_convert": (ctypes.c_int, [_vp, ctypes.c_int, _vp, ctypes.c_int, ctypes.c_size_t, _vp]),
    "tomo_phantom": (ctypes.c_int, [_vp, _i32, _i32, _i32, _i32, _vp, _vp]),
}


class LibraryError(RuntimeError):
    pass


class TomoError(RuntimeError):
    def __init__(self, fn: str, status: int, msg: str):
        super().__init__(f"{fn} failed with {STATUS.get(status, status)}: {msg}")
        self.status = status


_lib = None


def load() -> ctypes.CDLL:
    """Load the CUDA library (once). Raises LibraryError if it is absent or broken."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise LibraryError(
            f"{LIB_PATH} not found: build it with `python -c 'import __graft_entry__ as g; g.build()'` "
            "(there is no CPU fallback)")
    try:
        lib = ctypes.CDLL(str(LIB_PATH))
    except OSError as exc:
        raise LibraryError(f"cannot load {LIB_PATH}: {exc}") from exc
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def call(name: str, *args) -> None:
    lib = load()
    st = getattr(lib, name)(*args)
    if st != TOMO_OK:
        raise TomoError(name, st, lib.tomo_last_error().decode(errors="replace"))


def config_struct(c) -> TomoConfigCT:
    return TomoConfigCT(*[getattr(c, name) for name, _ in TomoConfigCT._fields_])
