"""Energy spectrum of the bulk-flow output, on the GPU.

The reference's consumer of compute_c_integral results
(src/gw_fopt/bubble_dynamics/utils/data_gw_bulkflow.py:26-190, DataGwBulkFlow)
combines the coefficient sets, forms 8 pi w^3 (|C_+|^2 + |C_x|^2) per k-hat
direction and integrates over cos(theta_k).  Here the same runs in one kernel
(gw_fopt_b200/csrc/postprocess.cu) on the (K, 2, S, W) array that
GeneralizedBulkFlow.compute_c_integral_khat returns, or on that array left in
device memory.  The DataFrame of the reference becomes arrays: one row per
k-hat direction.  Rows whose xi is None (the envelope spectrum, another
computation) are not produced by this library and are rejected.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L


def set_weights(xi_powers, xi_coefficients, powers_sets, check_sum=True):
    """Weights per coefficient set: xi_coefficients[j] added to the set whose power is
    xi_powers[j] + 3 (data_gw_bulkflow.py:51-106, the same checks and messages)."""
    if not isinstance(xi_powers, (list, np.ndarray)) or not isinstance(xi_coefficients, (list, np.ndarray)):
        raise ValueError("xi_powers and xi_coefficients must be lists or numpy arrays")
    xi_powers = np.asarray(xi_powers, dtype=object)
    xi_coefficients = np.asarray(xi_coefficients)
    if len(xi_powers) != len(xi_coefficients):
        raise ValueError("xi_powers and xi_coefficients must have the same length")
    if check_sum and not np.isclose(np.sum(xi_coefficients), 1.0):
        raise ValueError("xi_coefficients must sum to 1")
    if not all(p is None or isinstance(p, (int, float)) for p in xi_powers):
        raise ValueError("xi_powers must contain numbers or None")
    powers_available = list(np.asarray(powers_sets, dtype=np.float64).tolist())
    weights = np.zeros(len(powers_available))
    for p, coeff in zip(xi_powers, xi_coefficients):
        if p is None:
            raise ValueError("xi = None selects the envelope spectrum, which this library does not compute")
        power = p + 3
        if power not in powers_available:
            raise ValueError(f"Power {power} not in powers_sets_sample")
        weights[powers_available.index(power)] += float(coeff)
    return weights


def _check(flow, c, w, weights, cos_thetak):
    c = np.ascontiguousarray(c, dtype=np.complex128)
    if c.ndim != 4 or c.shape[1] != 2:
        raise ValueError(f"c must have shape (n_khat, 2, n_sets, n_w), got {c.shape}")
    w = np.ascontiguousarray(w, dtype=np.float64)
    weights = np.ascontiguousarray(weights, dtype=np.float64)
    ck = np.ascontiguousarray(cos_thetak, dtype=np.float64)
    K, _, S, W = c.shape
    if w.shape != (W,) or weights.shape != (S,) or ck.shape != (K,):
        raise ValueError(f"shape mismatch: c {c.shape}, w {w.shape}, weights {weights.shape}, cos_thetak {ck.shape}")
    return c, w, weights, ck


def power_spectrum(flow, c, w, weights, cos_thetak, per_direction=True):
    """(spectra (K, W) or None, de_dlogw (W,)) of c (K, 2, S, W) on flow's GPU:
    spectra = DataGwBulkFlow.de_dlogw_dcosthetak, de_dlogw = DataGwBulkFlow.de_dlogw."""
    c, w, weights, ck = _check(flow, c, w, weights, cos_thetak)
    K, _, S, W = c.shape
    de = np.empty(W)
    spec = np.empty((K, W)) if per_direction else None
    L.check(L.lib().bgwx_generalized_bulk_flow_power_spectrum(
        flow._h, c.ctypes.data_as(C.POINTER(L.BgwComplex64)), K, S, L.ptr(w), W, L.ptr(weights), L.ptr(ck),
        L.ptr(spec) if spec is not None else None, L.ptr(de)))
    return spec, de


def power_spectrum_device(flow, c_device, n_khat, n_sets, w, weights, cos_thetak, spectra_device, de_device):
    """The same on device pointers (integers, e.g. torch tensor data_ptr()): c (K, 2, S, W)
    complex128, spectra (K, W) float64 or 0, de (W,) float64."""
    w = np.ascontiguousarray(w, dtype=np.float64)
    weights = np.ascontiguousarray(weights, dtype=np.float64)
    ck = np.ascontiguousarray(cos_thetak, dtype=np.float64)
    L.check(L.lib().bgwx_generalized_bulk_flow_power_spectrum_device(
        flow._h, C.c_void_p(c_device), n_khat, n_sets, L.ptr(w), w.size, L.ptr(weights), L.ptr(ck),
        C.c_void_p(spectra_device) if spectra_device else None, C.c_void_p(de_device)))


def de_dlogw_dcosthetak(flow, c, w, cos_thetak, xi_powers, xi_coefficients, powers_sets, check_sum=True):
    """DataGwBulkFlow.de_dlogw_dcosthetak (data_gw_bulkflow.py:26-116) for rows c[k]."""
    return power_spectrum(flow, c, w, set_weights(xi_powers, xi_coefficients, powers_sets, check_sum),
                          cos_thetak)[0]


def de_dlogw(flow, c, w, cos_thetak, xi_powers, xi_coefficients, powers_sets, check_sum=True):
    """DataGwBulkFlow.de_dlogw (data_gw_bulkflow.py:118-146)."""
    return power_spectrum(flow, c, w, set_weights(xi_powers, xi_coefficients, powers_sets, check_sum),
                          cos_thetak, per_direction=False)[1]


def de_dlogw_interp(w, de, d, d0=1.0, rho_vacuum=1.0):
    """DataGwBulkFlow.de_dlogw_interp (data_gw_bulkflow.py:148-190): a cubic spline in w / d of
    (d / d0)^5 rho_vacuum^2 dE/dlnw (host, scipy)."""
    from scipy.interpolate import CubicSpline
    return CubicSpline(np.asarray(w) / d, (d / d0) ** 5 * rho_vacuum**2 * np.asarray(de))
