"""ctypes front-end of the oracle (test infrastructure only).

The oracle is a CPU f64 restatement of gw_fopt's generalized bulk-flow path
(rust/bubble-gw/src/many_bubbles/generalized_bulk_flow.rs and
lattice_bubbles.rs).  Only tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg import this module; the product never does.

Parity status: unpinned against reference-produced numbers (the reference
crate cannot be built here and its only golden CSV is absent); pinned by the
known-answer tests in tests/test_oracle_kat.py.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

_dp = C.POINTER(C.c_double)
_i32p = C.POINTER(C.c_int32)
_szp = C.POINTER(C.c_size_t)


def build() -> str:
    """Compiles liboracle.so with the Makefile beside this file."""
    src = os.path.join(_HERE, "bgw_oracle.cpp")
    if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(_LIB_PATH)
        L.orc_last_error.restype = C.c_char_p
        L.orc_validate.argtypes = [_dp, C.c_size_t, _dp, C.c_size_t]
        L.orc_directions.argtypes = [C.c_size_t, C.c_size_t, _dp]
        L.orc_first_colliding.argtypes = [_dp, C.c_size_t, _dp, C.c_size_t, C.c_size_t, C.c_size_t,
                                          C.c_size_t, C.c_size_t, _i32p, _dp, C.c_int]
        L.orc_compute_c_integral.argtypes = [
            _dp, C.c_size_t, _dp, C.c_size_t, C.c_size_t, C.c_size_t, _dp, _dp, C.c_size_t, C.c_size_t,
            C.c_double, _dp, C.c_size_t, C.c_int, C.c_double, C.c_double, C.c_size_t, _szp, C.c_size_t,
            C.c_int, C.c_double, C.c_double, C.c_double, _dp, _dp, C.c_int]
        L.orc_compute_c_integral_khat.argtypes = [
            _dp, C.c_size_t, _dp, C.c_size_t, _dp, C.c_size_t, C.c_size_t, C.c_size_t, _dp, _dp, C.c_size_t,
            C.c_size_t, C.c_double, _dp, C.c_size_t, C.c_double, C.c_double, C.c_size_t, C.c_int, C.c_double,
            C.c_double, C.c_double, _dp, C.c_int]
        L.orc_compute_c_integrand.argtypes = [
            _dp, C.c_size_t, _dp, C.c_size_t, C.c_size_t, C.c_size_t, _dp, _dp, C.c_size_t, C.c_size_t,
            C.c_double, _dp, C.c_size_t, C.c_int, C.c_double, C.c_double, C.c_size_t, _szp, C.c_size_t, _dp, C.c_int]
        L.orc_compute_c_tensor.argtypes = [
            _dp, C.c_size_t, _dp, C.c_size_t, C.c_size_t, C.c_size_t, _dp, _dp, C.c_size_t, C.c_size_t,
            C.c_double, _dp, C.c_size_t, C.c_int, C.c_double, C.c_double, C.c_size_t, _szp, C.c_size_t, _dp, C.c_int]
        L.orc_rotation_for_khat.argtypes = [C.c_double, C.c_double, C.c_double, _dp]
        L.orc_rotate.argtypes = [_dp, _dp, C.c_size_t, _dp]
        L.orc_time_cutoff.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, _dp, C.c_size_t, _dp]
        L.orc_max_threads.restype = C.c_int
        _lib = L
    return _lib


def _d(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(_dp)


def _bubbles(a):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1, 4))
    return a, a.ctypes.data_as(_dp), a.shape[0]


class OracleError(RuntimeError):
    pass


def _check(rc):
    if rc != 0:
        raise OracleError(lib().orc_last_error().decode())


def max_threads() -> int:
    return int(lib().orc_max_threads())


def validate(interior, exterior=None):
    ai, pi, ni = _bubbles(interior)
    ae, pe, ne = _bubbles(np.zeros((0, 4)) if exterior is None else exterior)
    _check(lib().orc_validate(pi, ni, pe, ne))


def directions(n_cos, n_phi):
    out = np.empty((n_cos, n_phi, 3))
    lib().orc_directions(n_cos, n_phi, out.ctypes.data_as(_dp))
    return out


def first_colliding(interior, exterior, n_cos, n_phi, a_begin=0, a_end=None, threads=None, with_delta_tab=False):
    """(a_end-a_begin, n_cos, n_phi) int32 first-collider codes (-1 None, i, -(i+2))."""
    ai, pi, ni = _bubbles(interior)
    ae, pe, ne = _bubbles(np.zeros((0, 4)) if exterior is None else exterior)
    a_end = ni if a_end is None else a_end
    out = np.empty((a_end - a_begin, n_cos, n_phi), dtype=np.int32)
    dt = np.empty((a_end - a_begin, n_cos, n_phi)) if with_delta_tab else None
    _check(lib().orc_first_colliding(pi, ni, pe, ne, n_cos, n_phi, a_begin, a_end, out.ctypes.data_as(_i32p),
                                     dt.ctypes.data_as(_dp) if dt is not None else None,
                                     threads or max_threads()))
    return (out, dt) if with_delta_tab else out


def compute_c_integral(interior, exterior, n_cos, n_phi, w, t_end, n_t, t_begin=None, coefficients=((1.0,),),
                       powers=((3.0,),), damping=None, selected=None, cutoff=None, threads=None, want_abs=False):
    """(2, n_sets, n_w) complex128, the reference's compute_c_integral output."""
    ai, pi, ni = _bubbles(interior)
    ae, pe, ne = _bubbles(np.zeros((0, 4)) if exterior is None else exterior)
    co = np.ascontiguousarray(np.asarray(coefficients, dtype=np.float64))
    po = np.ascontiguousarray(np.asarray(powers, dtype=np.float64))
    S, M = co.shape
    w, pw = _d(np.asarray(w, dtype=np.float64).ravel())
    W = w.size
    out = np.zeros((2, S, W), dtype=np.complex128)
    absout = np.zeros((2, S, W)) if want_abs else None
    if selected is not None:
        sel = np.ascontiguousarray(np.asarray(selected, dtype=np.uint64).ravel())
        psel = sel.ctypes.data_as(_szp)
        nsel = sel.size
    else:
        psel, nsel = None, 0
    kind, smax, rc, r0 = 0, 0.0, np.nan, np.nan
    if cutoff is not None:
        kind, smax, rc, r0 = 1, cutoff[0], cutoff[1], cutoff[2]
    _check(lib().orc_compute_c_integral(
        pi, ni, pe, ne, n_cos, n_phi, co.ctypes.data_as(_dp), po.ctypes.data_as(_dp), S, M,
        np.nan if damping is None else float(damping), pw, W, 0 if t_begin is None else 1,
        0.0 if t_begin is None else float(t_begin), float(t_end), n_t, psel, nsel, kind, smax, rc, r0,
        out.ctypes.data_as(_dp), absout.ctypes.data_as(_dp) if want_abs else None, threads or max_threads()))
    return (out, absout) if want_abs else out


def compute_c_integrand(interior, exterior, n_cos, n_phi, w, t_end, n_t, t_begin=None, coefficients=((1.0,),),
                        powers=((3.0,),), damping=None, selected=None, threads=None):
    """(2, n_sets, n_w, n_t) complex128, the reference's compute_c_integrand output."""
    ai, pi, ni = _bubbles(interior)
    ae, pe, ne = _bubbles(np.zeros((0, 4)) if exterior is None else exterior)
    co = np.ascontiguousarray(np.asarray(coefficients, dtype=np.float64))
    po = np.ascontiguousarray(np.asarray(powers, dtype=np.float64))
    S, M = co.shape
    w, pw = _d(np.asarray(w, dtype=np.float64).ravel())
    out = np.zeros((2, S, w.size, n_t), dtype=np.complex128)
    if selected is not None:
        sel = np.ascontiguousarray(np.asarray(selected, dtype=np.uint64).ravel())
        psel, nsel = sel.ctypes.data_as(_szp), sel.size
    else:
        psel, nsel = None, 0
    _check(lib().orc_compute_c_integrand(
        pi, ni, pe, ne, n_cos, n_phi, co.ctypes.data_as(_dp), po.ctypes.data_as(_dp), S, M,
        np.nan if damping is None else float(damping), pw, w.size, 0 if t_begin is None else 1,
        0.0 if t_begin is None else float(t_begin), float(t_end), n_t, psel, nsel, out.ctypes.data_as(_dp),
        threads or max_threads()))
    return out


def rotation_for_khat(k):
    R = np.empty(9)
    lib().orc_rotation_for_khat(float(k[0]), float(k[1]), float(k[2]), R.ctypes.data_as(_dp))
    return R.reshape(3, 3)


def rotate(R, bubbles):
    R, pR = _d(np.asarray(R).ravel())
    b, pb, n = _bubbles(bubbles)
    out = np.empty_like(b)
    lib().orc_rotate(pR, pb, n, out.ctypes.data_as(_dp))
    return out


def compute_c_integral_khat(interior, exterior, khat, n_cos, n_phi, w, t_begin, t_end, n_t,
                            coefficients=((1.0,),), powers=((3.0,),), damping=None, cutoff=None, threads=None):
    """(K, 2, n_sets, n_w) complex128: one reference spectrum per rotated configuration."""
    ai, pi, ni = _bubbles(interior)
    ae, pe, ne = _bubbles(np.zeros((0, 4)) if exterior is None else exterior)
    kh, pk = _d(np.asarray(khat, dtype=np.float64).reshape(-1, 3))
    K = kh.shape[0]
    co = np.ascontiguousarray(np.asarray(coefficients, dtype=np.float64))
    po = np.ascontiguousarray(np.asarray(powers, dtype=np.float64))
    S, M = co.shape
    w, pw = _d(np.asarray(w, dtype=np.float64).ravel())
    W = w.size
    out = np.zeros((K, 2, S, W), dtype=np.complex128)
    kind, smax, rc, r0 = 0, 0.0, np.nan, np.nan
    if cutoff is not None:
        kind, smax, rc, r0 = 1, cutoff[0], cutoff[1], cutoff[2]
    _check(lib().orc_compute_c_integral_khat(
        pi, ni, pe, ne, pk, K, n_cos, n_phi, co.ctypes.data_as(_dp), po.ctypes.data_as(_dp), S, M,
        np.nan if damping is None else float(damping), pw, W, float(t_begin), float(t_end), n_t, kind, smax, rc,
        r0, out.ctypes.data_as(_dp), threads or max_threads()))
    return out


def time_cutoff(t, smax, ratio_t_cut=None, ratio_t_0=None):
    t, pt = _d(np.asarray(t, dtype=np.float64).ravel())
    out = np.empty_like(t)
    lib().orc_time_cutoff(1, float(smax), np.nan if ratio_t_cut is None else ratio_t_cut,
                          np.nan if ratio_t_0 is None else ratio_t_0, pt, t.size, out.ctypes.data_as(_dp))
    return out


def compute_c_tensor(interior, exterior, n_cos, n_phi, w, t_end, n_t, t_begin=None, coefficients=((1.0,),),
                     powers=((3.0,),), damping=None, selected=None, threads=None):
    """(6, n_sets, n_w) complex128 in the order xx, xy, xz, yy, yz, zz: the reference's
    NewGeneralizedBulkFlow.compute_c_tensor (new_generalized_bulk_flow.rs:1205-1275)."""
    ai, pi, ni = _bubbles(interior)
    ae, pe, ne = _bubbles(np.zeros((0, 4)) if exterior is None else exterior)
    co = np.ascontiguousarray(np.asarray(coefficients, dtype=np.float64))
    po = np.ascontiguousarray(np.asarray(powers, dtype=np.float64))
    S, M = co.shape
    w, pw = _d(np.asarray(w, dtype=np.float64).ravel())
    out = np.zeros((6, S, w.size), dtype=np.complex128)
    sel = None if selected is None else np.ascontiguousarray(selected, dtype=np.uintp)
    _check(lib().orc_compute_c_tensor(
        pi, ni, pe, ne, n_cos, n_phi, co.ctypes.data_as(_dp), po.ctypes.data_as(_dp), S, M,
        float("nan") if damping is None else float(damping), pw, w.size, 0 if t_begin is None else 1,
        0.0 if t_begin is None else float(t_begin), float(t_end), n_t,
        sel.ctypes.data_as(_szp) if sel is not None else None, 0 if sel is None else sel.size,
        out.ctypes.data_as(_dp), threads or max_threads()))
    return out


def compute_c_tensor_khat(interior, exterior, khat, n_cos, n_phi, w, t_end, n_t, t_begin=None,
                          coefficients=((1.0,),), powers=((3.0,),), damping=None, threads=None):
    """(K, 6, n_sets, n_w): compute_c_tensor on each k-hat's rotated configuration."""
    kh = np.asarray(khat, dtype=np.float64).reshape(-1, 3)
    outs = []
    for k in kh:
        R = rotation_for_khat(k)
        outs.append(compute_c_tensor(rotate(R, interior), rotate(R, np.zeros((0, 4)) if exterior is None else exterior),
                                     n_cos, n_phi, w, t_end, n_t, t_begin, coefficients, powers, damping,
                                     threads=threads))
    return np.stack(outs)
