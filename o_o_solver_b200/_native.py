"""ctypes bindings of the library's C ABI (include/oos_gpu.h). The library is the only implementation: when it is
missing, loading fails with an error naming the build command (there is no CPU fallback)."""

from __future__ import annotations

import ctypes
import os

from . import build as _build

_i32p = ctypes.POINTER(ctypes.c_int32)
_i64p = ctypes.POINTER(ctypes.c_int64)
_f64p = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p


class FactorOptions(ctypes.Structure):
    _fields_ = [("max_ratio", ctypes.c_double), ("bailout", ctypes.c_int32), ("reference_diagonal", _f64p),
                ("pivoting", ctypes.c_int32), ("precision", ctypes.c_int32)]


class FactorInfo(ctypes.Structure):
    _fields_ = [
        ("positive", ctypes.c_int64),
        ("negative", ctypes.c_int64),
        ("zero", ctypes.c_int64),
        ("delayed", ctypes.c_int64),
        ("two_by_two", ctypes.c_int64),
        ("issue_count", ctypes.c_int64),
        ("equation_of_largest", ctypes.c_int32),
        ("zero_pivot_count", ctypes.c_int32),
        ("largest_ratio", ctypes.c_double),
        ("issues", ctypes.c_int32 * 16),
        ("zero_pivots", ctypes.c_int32 * 16),
        ("device_seconds", ctypes.c_double),
    ]


class RefineOptions(ctypes.Structure):
    _fields_ = [("tolerance", ctypes.c_double), ("max_steps", ctypes.c_int32), ("krylov", ctypes.c_int32)]


class RefineInfo(ctypes.Structure):
    _fields_ = [("steps", ctypes.c_int32), ("residual", ctypes.c_double), ("device_seconds", ctypes.c_double),
                ("backward_error", ctypes.c_double)]


class EigenRequest(ctypes.Structure):
    _fields_ = [("lower_bound", ctypes.c_double), ("upper_bound", ctypes.c_double), ("mode_count", ctypes.c_int64)]


class LanczosOptions(ctypes.Structure):
    _fields_ = [("block_size", ctypes.c_int64), ("modes_per_shift", ctypes.c_int64),
                ("convergence_tolerance", ctypes.c_double), ("maximum_shifts", ctypes.c_int64),
                ("maximum_restarts", ctypes.c_int64), ("seed", ctypes.c_uint64)]


# The exported symbols and their signatures: (name, restype, argtypes).
SIGNATURES = [
    ("oosgpu_last_error", ctypes.c_char_p, []),
    ("oosgpu_device_count", ctypes.c_int, []),
    ("oosgpu_release_cached_buffers", ctypes.c_int64, [ctypes.c_int]),
    ("oosgpu_symbolic_create", ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, _i32p, _i32p, _i64p, _i32p,
                                              ctypes.POINTER(_vp)]),
    ("oosgpu_symbolic_from_partition", ctypes.c_int, [ctypes.c_int32, _i64p, _i32p, _i32p, _i32p, ctypes.c_int32,
                                                      _i32p, _i32p, ctypes.POINTER(_vp)]),
    ("oosgpu_symbolic_sizes", ctypes.c_int, [_vp, _i64p, _f64p]),
    ("oosgpu_symbolic_solve_chains", ctypes.c_int, [_vp, _i64p]),
    ("oosgpu_symbolic_rows", ctypes.c_int, [_vp, _i64p, _i32p]),
    ("oosgpu_symbolic_destroy", None, [_vp]),
    ("oosgpu_factor_create", ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(_vp)]),
    ("oosgpu_factor_destroy", None, [_vp]),
    ("oosgpu_factor_stream", _vp, [_vp]),
    ("oosgpu_solve_prefetch", ctypes.c_int, [_vp, _f64p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int32]),
    ("oosgpu_factorise_partial", ctypes.c_int, [_vp, ctypes.c_int32, _i64p, _i32p, _f64p, ctypes.c_int32,
                                                 ctypes.POINTER(FactorOptions), _f64p, ctypes.POINTER(FactorInfo)]),
    ("oosgpu_partial_condense", ctypes.c_int, [_vp, _f64p, ctypes.c_int64, ctypes.c_int64, _f64p, ctypes.c_int64]),
    ("oosgpu_partial_recover", ctypes.c_int, [_vp, _f64p, ctypes.c_int64, ctypes.c_int64, _f64p, ctypes.c_int64]),
    ("oosgpu_factorise", ctypes.c_int, [_vp, ctypes.c_int32, _i64p, _i32p, _f64p, ctypes.POINTER(FactorOptions),
                                        ctypes.POINTER(FactorInfo)]),
    ("oosgpu_factorise_device", ctypes.c_int, [_vp, ctypes.c_int32, ctypes.c_int64, _vp, _vp, _vp,
                                               ctypes.POINTER(FactorOptions), ctypes.POINTER(FactorInfo)]),
    ("oosgpu_factor_panel", ctypes.c_int, [_vp, ctypes.c_int32, _i64p, _i64p, _f64p, _i32p, _f64p]),
    ("oosgpu_solve", ctypes.c_int, [_vp, _f64p, ctypes.c_int64, ctypes.c_int64]),
    ("oosgpu_solve_device", ctypes.c_int, [_vp, _vp, ctypes.c_int64, ctypes.c_int64]),
    ("oosgpu_last_solve_seconds", ctypes.c_double, [_vp]),
    ("oosgpu_solve_device_noalloc", ctypes.c_int, [_vp, _vp, ctypes.c_int64, ctypes.c_int64]),
    ("oosgpu_solve_refined", ctypes.c_int, [_vp, _f64p, ctypes.c_int64, _f64p, ctypes.c_int64, ctypes.c_int64,
                                            ctypes.POINTER(RefineOptions), ctypes.POINTER(RefineInfo)]),
    ("oosgpu_solve_refined_device", ctypes.c_int, [_vp, _vp, ctypes.c_int64, _vp, ctypes.c_int64, ctypes.c_int64,
                                                   ctypes.POINTER(RefineOptions), ctypes.POINTER(RefineInfo)]),
    ("oosgpu_factor_profile", ctypes.c_int, [_vp, ctypes.c_int32]),
    ("oosgpu_factor_launch_profile", ctypes.c_int, [_vp, ctypes.c_int32, ctypes.c_int64, _i32p, _i32p, _i32p,
                                                    _f64p, _i64p]),
    ("oosgpu_factor_kernel_stats", ctypes.c_int, [_vp, ctypes.c_int32, _f64p, _i64p, _f64p, _f64p]),
    ("oosgpu_factor_set_tuning", ctypes.c_int, [_vp, ctypes.c_int32]),
    ("oosgpu_factor_tuning_report", ctypes.c_int, [_vp, ctypes.c_int64, _i32p, _i32p, _i32p, _f64p, _f64p, _i32p,
                                                    ctypes.POINTER(ctypes.c_int64)]),
    ("oosgpu_factor_launch_counts", ctypes.c_int, [_vp, ctypes.c_int64, _i64p]),
    ("oosgpu_pencil_create", ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int32, _i64p, _i32p, _f64p, _f64p,
                                            ctypes.POINTER(_vp)]),
    ("oosgpu_pencil_create_buckling", ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int32, _i64p, _i32p, _f64p, _f64p,
                                                     ctypes.POINTER(_vp)]),
    ("oosgpu_pencil_destroy", None, [_vp]),
    ("oosgpu_pencil_stream", _vp, [_vp]),
    ("oosgpu_pencil_factorise", ctypes.c_int, [_vp, ctypes.c_double, ctypes.POINTER(FactorInfo)]),
    ("oosgpu_pencil_solve_device", ctypes.c_int, [_vp, _vp, ctypes.c_int64, ctypes.c_int64]),
    ("oosgpu_pencil_multiply_mass_device", ctypes.c_int, [_vp, _vp, ctypes.c_int64, _vp, ctypes.c_int64,
                                                          ctypes.c_int64]),
    ("oosgpu_pencil_properties", ctypes.c_int, [_vp, _f64p, _i32p, _i64p]),
    ("oosgpu_lanczos_defaults", None, [ctypes.POINTER(LanczosOptions)]),
    ("oosgpu_modes_solve", ctypes.c_int, [_vp, ctypes.POINTER(EigenRequest), ctypes.POINTER(LanczosOptions),
                                          ctypes.POINTER(_vp)]),
    ("oosgpu_modes_solve_start", ctypes.c_int, [_vp, ctypes.POINTER(EigenRequest), ctypes.POINTER(LanczosOptions),
                                                _vp, ctypes.c_int64, ctypes.c_int64, ctypes.POINTER(_vp)]),
    ("oosgpu_modes_summary", ctypes.c_int, [_vp, _i64p, _f64p]),
    ("oosgpu_modes_work", ctypes.c_int, [_vp, _i64p, _f64p]),
    ("oosgpu_modes_values", ctypes.c_int, [_vp, _f64p, _f64p]),
    ("oosgpu_modes_vectors", ctypes.c_int, [_vp, _f64p, ctypes.c_int64]),
    ("oosgpu_modes_vectors_device", _vp, [_vp]),
    ("oosgpu_modes_shifts", ctypes.c_int, [_vp, _f64p]),
    ("oosgpu_modes_destroy", None, [_vp]),
    ("oosgpu_symmetric_eigen", ctypes.c_int, [_f64p, ctypes.c_int64, ctypes.c_int64, _f64p, _f64p]),
    ("oosgpu_sturm_verify", ctypes.c_int, [ctypes.c_int64, _f64p, _i64p, ctypes.c_int64, _f64p, _f64p]),
    ("oosgpu_shift_next", ctypes.c_int, [ctypes.c_double, ctypes.c_double, ctypes.c_int64, ctypes.c_double, _f64p,
                                         ctypes.c_int64, _f64p, ctypes.c_int64, _f64p, ctypes.c_int64, _f64p,
                                         _f64p, _i32p]),
    ("oosgpu_model_plate", ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.c_double, ctypes.c_double,
                                          ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                          ctypes.POINTER(_vp)]),
    ("oosgpu_model_hex", ctypes.c_int, [ctypes.c_int32, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_double, ctypes.POINTER(_vp)]),
    ("oosgpu_mlp_create", ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_uint64, ctypes.c_int,
                                         ctypes.POINTER(_vp)]),
    ("oosgpu_mlp_destroy", None, [_vp]),
    ("oosgpu_mlp_parameter_count", ctypes.c_int64, [_vp]),
    ("oosgpu_mlp_get_parameters", ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_float)]),
    ("oosgpu_mlp_set_parameters", ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_float)]),
    ("oosgpu_mlp_predict", ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_float), ctypes.c_int32, ctypes.POINTER(ctypes.c_float)]),
    ("oosgpu_mlp_gradients", ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float), ctypes.c_int32, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)]),
    ("oosgpu_mlp_train", ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float), ctypes.c_int32, ctypes.c_int32, ctypes.c_float, ctypes.POINTER(ctypes.c_float)]),
    ("oosgpu_model_stiffened_panel", ctypes.c_int, [ctypes.c_int32, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                                    ctypes.c_double, ctypes.c_double, ctypes.c_int32, ctypes.c_double,
                                                    ctypes.c_double, ctypes.c_double, ctypes.POINTER(_vp)]),
    ("oosgpu_model_wing_box", ctypes.c_int, [ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                             ctypes.c_double, _f64p, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                             ctypes.c_double, ctypes.POINTER(_vp)]),
    ("oosgpu_model_destroy", None, [_vp]),
    ("oosgpu_model_sizes", ctypes.c_int, [_vp, _i64p]),
    ("oosgpu_model_graph", ctypes.c_int, [_vp, _i64p, _i32p, _f64p]),
    ("oosgpu_model_csc_terms", ctypes.c_int, [_vp, _i32p, _i64p]),
    ("oosgpu_model_csc", ctypes.c_int, [_vp, _i32p, ctypes.c_int32, _i64p, _i32p, _f64p]),
    ("oosgpu_model_csc_device", ctypes.c_int, [_vp, _i32p, ctypes.c_int32, ctypes.c_int32, _vp, _vp, _vp]),
    ("oosgpu_model_loads", ctypes.c_int, [_vp, _i32p, ctypes.c_int64, ctypes.c_uint64, ctypes.c_int32,
                                          ctypes.c_double, _f64p, ctypes.c_int64]),
]

_lib = None


def library_path() -> str:
    return _build.LIBRARY


def load(build_if_missing: bool = False):
    """The loaded library. build_if_missing compiles it first (nvcc); otherwise a missing library is an error."""
    global _lib
    if _lib is not None:
        return _lib
    path = _build.LIBRARY
    if build_if_missing:
        _build.build()
    if not os.path.exists(path):
        raise RuntimeError(f"the CUDA library is not built: {path} (python -m o_o_solver_b200.build)")
    lib = ctypes.CDLL(path)
    for name, restype, argtypes in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = restype
        fn.argtypes = argtypes
    _lib = lib
    return lib


class NativeError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


def check(status: int):
    if status != 0:
        raise NativeError(status, load().oosgpu_last_error().decode())


def ptr(array, kind):
    if array is None:
        return None
    return array.ctypes.data_as(kind)


i32p, i64p, f64p, vp = _i32p, _i64p, _f64p, _vp
