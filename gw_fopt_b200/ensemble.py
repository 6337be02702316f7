"""Batched ensemble of nucleation realizations (B200 extension, separate from the drop-in surface).

The reference computes a Monte-Carlo ensemble by building one
``GeneralizedBulkFlow`` per realization and calling ``compute_c_integral`` on
each (rust/bubble-gw/src/many_bubbles/generalized_bulk_flow.rs:928-984).
:class:`BulkFlowEnsemble` runs every realization along the same k-hat
directions in one library call: the realizations go back to back on one CUDA
stream (largest first, so the device work arrays are sized once), each with
all of its k-hat frames batched into the same kernel launches, and the
(R, K, 2, S, W) result comes back in one copy.  Block r is bit-identical to
``GeneralizedBulkFlow.compute_c_integral_khat`` on realization r alone.
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Iterable, Optional

import numpy as np

from . import _lib as L
from .many_bubbles import ExponentialTimeCutoff, LatticeBubbles, _call, _cutoff_config

__all__ = ["BulkFlowEnsemble", "ensemble_mean_power"]


def _pair(item):
    if isinstance(item, LatticeBubbles):
        return item._interior, item._exterior
    interior, exterior = item
    i = np.ascontiguousarray(np.asarray(interior, dtype=np.float64).reshape(-1, 4))
    e = np.ascontiguousarray(np.asarray(exterior, dtype=np.float64).reshape(-1, 4)) if exterior is not None \
        else np.zeros((0, 4))
    return i, e


class BulkFlowEnsemble:
    """Spectra of many bubble configurations that share one resolution, scaling and frequency grid.

    ``realizations`` holds :class:`LatticeBubbles` objects or ``(interior, exterior)`` array pairs.
    With ``validate`` every realization must pass the causality check of ``LatticeBubbles``.
    """

    def __init__(self, realizations: Iterable, *, validate: bool = True):
        pairs = [_pair(r) for r in realizations]
        if not pairs:
            raise ValueError("an ensemble needs at least one realization")
        self._n_int = np.array([p[0].shape[0] for p in pairs], dtype=np.uintp)
        self._n_ext = np.array([p[1].shape[0] for p in pairs], dtype=np.uintp)
        self._int_off = np.concatenate([[0], np.cumsum(self._n_int)]).astype(np.uintp)
        self._ext_off = np.concatenate([[0], np.cumsum(self._n_ext)]).astype(np.uintp)
        self._interior = np.ascontiguousarray(np.concatenate([p[0] for p in pairs]).reshape(-1, 4))
        self._exterior = np.ascontiguousarray(np.concatenate([p[1] for p in pairs]).reshape(-1, 4))
        self._validate = bool(validate)
        # the settings handle holds no bubbles of its own
        h = C.c_void_p()
        _call(L.lib().bgwx_generalized_bulk_flow_new_unchecked(C.byref(h), None, 0, None, 0))
        self._h = h
        self._n_sets = 1
        self._n_res = None

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                L.lib().bgw_generalized_bulk_flow_free(h)
            except Exception:
                pass
            self._h = None

    def __len__(self):
        return int(self._n_int.size)

    @property
    def bubble_counts(self) -> np.ndarray:
        """Interior bubbles per realization."""
        return self._n_int.astype(np.int64)

    def set_resolution(self, n_cos_thetax: int, n_phix: int, precompute_first_bubbles: bool = True) -> None:
        _call(L.lib().bgw_generalized_bulk_flow_set_resolution(self._h, int(n_cos_thetax), int(n_phix),
                                                               bool(precompute_first_bubbles)))
        self._n_res = (int(n_cos_thetax), int(n_phix))

    def set_gradient_scaling_params(self, coefficients_sets, powers_sets, damping_factor=None) -> None:
        co = np.ascontiguousarray(np.asarray(coefficients_sets, dtype=np.float64))
        po = np.ascontiguousarray(np.asarray(powers_sets, dtype=np.float64))
        if co.ndim != 2 or co.shape != po.shape or co.shape[1] == 0:
            raise ValueError("Array shape mismatch: coefficients_sets and powers_sets must be (S, M) with M >= 1")
        _call(L.lib().bgw_generalized_bulk_flow_set_gradient_scaling_params(
            self._h, L.ptr(co), L.ptr(po), co.shape[0], co.shape[1],
            math.nan if damping_factor is None else float(damping_factor)))
        self._n_sets = co.shape[0]

    def set_kernel(self, kernel: str) -> None:
        """'fp64_direct', 'fp64_factored' or 'mixed'."""
        k = {"fp64_direct": L.KERNEL_FP64_DIRECT, "fp64_factored": L.KERNEL_FP64_FACTORED,
             "mixed": L.KERNEL_MIXED, "mixed_simt": L.KERNEL_MIXED_SIMT}[kernel]
        _call(L.lib().bgwx_generalized_bulk_flow_set_kernel(self._h, k))

    def compute_c_integral_khat(self, w_arr, khat, *, t_begin=None, t_end, n_t,
                                time_cutoff: Optional[ExponentialTimeCutoff] = None) -> np.ndarray:
        """(R, K, 2, n_sets, n_w) complex128: every realization's spectrum along every k-hat row."""
        w = np.ascontiguousarray(np.asarray(w_arr, dtype=np.float64).ravel())
        kh = np.ascontiguousarray(np.asarray(khat, dtype=np.float64).reshape(-1, 3))
        out = np.zeros((len(self), kh.shape[0], 2, self._n_sets, w.size), dtype=np.complex128)
        szp = C.POINTER(C.c_size_t)
        _call(L.lib().bgwx_generalized_bulk_flow_compute_ensemble_khat(
            self._h, L.ptr(self._interior), self._int_off.ctypes.data_as(szp), L.ptr(self._exterior),
            self._ext_off.ctypes.data_as(szp), len(self), self._validate, L.ptr(w), w.size, t_begin is not None,
            0.0 if t_begin is None else float(t_begin), float(t_end), int(n_t), L.ptr(kh), kh.shape[0],
            _cutoff_config(time_cutoff), out.ctypes.data_as(C.POINTER(L.BgwComplex64)), out.size))
        return out

    def last_timings(self) -> dict:
        t = L.BgwxTimings()
        _call(L.lib().bgwx_generalized_bulk_flow_last_timings(self._h, C.byref(t)))
        return {f: getattr(t, f) for f, _ in L.BgwxTimings._fields_}


def ensemble_mean_power(c: np.ndarray) -> np.ndarray:
    """Ensemble mean of |C|^2 over the realization axis of an (R, K, 2, S, W) array."""
    return np.mean(np.abs(c) ** 2, axis=0)
