"""ctypes binding of libbubble_gw_c.so (the C ABI declared in include/).

The shared library is built in-tree (gw_fopt_b200/build.py).  Loading fails
loudly if it is missing; there is no Python or CPU fallback for the spectrum.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libbubble_gw_c.so")

# BgwStatus (include/bubble_gw.h)
OK, NULL_POINTER, INVALID_ARGUMENT, CALCULATION_ERROR, PANIC = 0, 1, 2, 3, 4
# BgwxKernel
KERNEL_FP64_DIRECT, KERNEL_FP64_FACTORED, KERNEL_MIXED, KERNEL_MIXED_SIMT = 0, 1, 2, 3
# BgwxLatticeKind / BgwxBoundaryCondition
LATTICE_PARALLELEPIPED, LATTICE_CARTESIAN, LATTICE_SPHERICAL, LATTICE_EMPTY = 0, 1, 2, 3
BC_PERIODIC, BC_REFLECTION, BC_NONE = 0, 1, 2


class BgwComplex64(C.Structure):
    _fields_ = [("re", C.c_double), ("im", C.c_double)]


class BgwTimeCutoffConfig(C.Structure):
    _fields_ = [("kind", C.c_int), ("smax", C.c_double), ("ratio_t_cut", C.c_double), ("ratio_t_0", C.c_double)]


class BgwxTimings(C.Structure):
    _fields_ = [("masks_ms", C.c_double), ("spectrum_ms", C.c_double), ("total_ms", C.c_double),
                ("h2d_bytes", C.c_double), ("d2h_bytes", C.c_double), ("launches", C.c_uint64),
                ("directions", C.c_uint64), ("fallbacks", C.c_uint64), ("beta_ms", C.c_double),
                ("gemm_ms", C.c_double), ("graph_replays", C.c_uint64)]


_dp = C.POINTER(C.c_double)
_szp = C.POINTER(C.c_size_t)
_hp = C.c_void_p

# name -> (restype, argtypes); every symbol declared in include/*.h
SIGNATURES = {
    "bgw_version": (C.c_char_p, []),
    "bgw_last_error_message": (C.c_char_p, []),
    "bgw_generalized_bulk_flow_empty_lattice_new": (C.c_int, [C.POINTER(_hp), _dp, C.c_size_t, _dp, C.c_size_t]),
    "bgw_generalized_bulk_flow_free": (None, [_hp]),
    "bgw_generalized_bulk_flow_set_num_threads": (C.c_int, [_hp, C.c_size_t]),
    "bgw_generalized_bulk_flow_set_resolution": (C.c_int, [_hp, C.c_size_t, C.c_size_t, C.c_bool]),
    "bgw_generalized_bulk_flow_set_gradient_scaling_params": (
        C.c_int, [_hp, _dp, _dp, C.c_size_t, C.c_size_t, C.c_double]),
    "bgw_generalized_bulk_flow_compute_c_integral": (
        C.c_int, [_hp, _dp, C.c_size_t, C.c_bool, C.c_double, C.c_double, C.c_size_t, _szp, C.c_size_t,
                  BgwTimeCutoffConfig, C.POINTER(BgwComplex64), C.c_size_t]),
    "bgwx_lattice_contains": (C.c_int, [C.c_int, _dp, _dp, C.c_size_t, C.POINTER(C.c_uint8), _szp]),
    "bgwx_lattice_exterior": (C.c_int, [C.c_int, _dp, C.c_int, _dp, C.c_size_t, _dp, C.c_size_t, _szp]),
    "bgwx_check_causality": (C.c_int, [_dp, C.c_size_t, _dp, C.c_size_t]),
    "bgwx_generalized_bulk_flow_new_unchecked": (C.c_int, [C.POINTER(_hp), _dp, C.c_size_t, _dp, C.c_size_t]),
    "bgwx_generalized_bulk_flow_set_kernel": (C.c_int, [_hp, C.c_int]),
    "bgwx_generalized_bulk_flow_set_launch_shape": (C.c_int, [_hp, C.c_size_t, C.c_size_t]),
    "bgwx_generalized_bulk_flow_set_autotune": (C.c_int, [_hp, C.c_bool]),
    "bgwx_generalized_bulk_flow_set_gemm_stages": (C.c_int, [_hp, C.c_size_t]),
    "bgwx_generalized_bulk_flow_last_gemm_stages": (C.c_int, [_hp, C.POINTER(C.c_size_t)]),
    "bgwx_generalized_bulk_flow_set_mask_chunking": (C.c_int, [_hp, C.c_size_t]),
    "bgwx_generalized_bulk_flow_set_keep_masks": (C.c_int, [_hp, C.c_bool]),
    "bgwx_generalized_bulk_flow_last_mask_chunking": (C.c_int, [_hp, C.POINTER(C.c_size_t)]),
    "bgwx_generalized_bulk_flow_last_launch_shape": (C.c_int, [_hp, C.POINTER(C.c_size_t),
                                                                C.POINTER(C.c_size_t)]),
    "bgwx_generalized_bulk_flow_first_colliding": (
        C.c_int, [_hp, C.c_size_t, C.c_size_t, C.POINTER(C.c_int32), _dp]),
    "bgwx_generalized_bulk_flow_compute_c_integral_khat": (
        C.c_int, [_hp, _dp, C.c_size_t, C.c_bool, C.c_double, C.c_double, C.c_size_t, _dp, C.c_size_t, _szp,
                  C.c_size_t, BgwTimeCutoffConfig, C.POINTER(BgwComplex64), C.c_size_t]),
    "bgwx_generalized_bulk_flow_compute_c_integral_khat_device": (
        C.c_int, [_hp, _dp, C.c_size_t, C.c_bool, C.c_double, C.c_double, C.c_size_t, _dp, C.c_size_t, _szp,
                  C.c_size_t, BgwTimeCutoffConfig, C.c_void_p, C.c_size_t]),
    "bgwx_generalized_bulk_flow_compute_ensemble_khat": (
        C.c_int, [_hp, _dp, _szp, _dp, _szp, C.c_size_t, C.c_bool, _dp, C.c_size_t, C.c_bool, C.c_double,
                  C.c_double, C.c_size_t, _dp, C.c_size_t, BgwTimeCutoffConfig, C.POINTER(BgwComplex64),
                  C.c_size_t]),
    "bgwx_generalized_bulk_flow_spectrum_vjp": (
        C.c_int, [_hp, _dp, C.c_size_t, C.c_bool, C.c_double, C.c_double, C.c_size_t, _dp, C.c_size_t,
                  BgwTimeCutoffConfig, C.POINTER(BgwComplex64), C.c_size_t, _dp, _dp, _dp]),
    "bgwx_generalized_bulk_flow_set_bubbles": (C.c_int, [_hp, _dp, C.c_size_t, _dp, C.c_size_t]),
    "bgwx_generalized_bulk_flow_compute_c_integrand": (
        C.c_int, [_hp, _dp, C.c_size_t, C.c_bool, C.c_double, C.c_double, C.c_size_t, _szp, C.c_size_t,
                  C.POINTER(BgwComplex64), C.c_size_t]),
    "bgwx_generalized_bulk_flow_power_spectrum": (
        C.c_int, [_hp, C.POINTER(BgwComplex64), C.c_size_t, C.c_size_t, _dp, C.c_size_t, _dp, _dp, _dp, _dp]),
    "bgwx_generalized_bulk_flow_power_spectrum_device": (
        C.c_int, [_hp, C.c_void_p, C.c_size_t, C.c_size_t, _dp, C.c_size_t, _dp, _dp, C.c_void_p, C.c_void_p]),
    "bgwx_generalized_bulk_flow_compute_c_tensor_khat": (
        C.c_int, [_hp, _dp, C.c_size_t, C.c_bool, C.c_double, C.c_double, C.c_size_t, _dp, C.c_size_t, _szp,
                  C.c_size_t, C.POINTER(BgwComplex64), C.c_size_t]),
    "bgwx_generalized_bulk_flow_compute_c_tensor_integrand": (
        C.c_int, [_hp, _dp, C.c_size_t, C.c_bool, C.c_double, C.c_double, C.c_size_t, _szp, C.c_size_t,
                  C.POINTER(BgwComplex64), C.c_size_t]),
    "bgwx_nucleate_exponential": (
        C.c_int, [C.POINTER(C.c_int64), _dp, C.POINTER(C.c_uint64), C.c_size_t, C.c_double, C.c_double, C.c_size_t,
                  _dp, C.c_size_t, _dp, C.c_size_t, C.POINTER(C.c_int32)]),
    "bgwx_generalized_bulk_flow_set_stream": (C.c_int, [_hp, C.c_void_p]),
    "bgwx_generalized_bulk_flow_drop_resident_inputs": (C.c_int, [_hp]),
    "bgwx_measure_compute_peaks": (C.c_int, [_dp, _dp, _dp]),
    "bgwx_first_colliding_noalloc": (
        C.c_int, [C.c_void_p, C.c_size_t, C.c_size_t, C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.c_void_p,
                  C.c_void_p, C.c_void_p]),
    "bgwx_rotation_for_khat": (None, [C.c_double, C.c_double, C.c_double, _dp]),
    "bgwx_generalized_bulk_flow_last_timings": (C.c_int, [_hp, C.POINTER(BgwxTimings)]),
    "bgwx_device_count": (C.c_int, []),
}

_lib = None


class NativeLibraryMissing(ImportError):
    pass


def lib():
    """Loads the in-tree C-ABI library (building it first if sources changed and nvcc exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        try:
            from . import build as _build
            _build.build()
        except Exception as exc:  # pragma: no cover - reported below
            raise NativeLibraryMissing(
                f"{LIB_PATH} is missing and could not be built ({exc}); the bulk-flow spectrum has no "
                "CPU fallback") from exc
    L = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


class BgwError(Exception):
    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status
        self.message = message


def check(status: int):
    if status != OK:
        raise BgwError(status, lib().bgw_last_error_message().decode())


def ptr(a):
    return a.ctypes.data_as(_dp) if a is not None and a.size else None
