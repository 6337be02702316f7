"""CPU restatement of the spectrum post-processing (test infrastructure only).

Follows src/gw_fopt/bubble_dynamics/utils/data_gw_bulkflow.py:26-146 of the
reference (DataGwBulkFlow.de_dlogw_dcosthetak, de_dlogw) and :148-190
(de_dlogw_interp), with the DataFrame replaced by arrays: one row per k-hat
direction, c_rows (K, 2, n_sets, W) complex, cos_thetak (K,).  Only tests/
import this module; the product path is the CUDA kernel in
gw_fopt_b200/csrc/postprocess.cu.

Parity: pinned against golden vectors produced by running the reference's own
DataGwBulkFlow (tests/golden/make_postprocess_golden.py, fixture
tests/golden/postprocess_golden.npz).
"""
from __future__ import annotations

import numpy as np
from scipy.interpolate import CubicSpline


def de_dlogw_dcosthetak(c_rows, w, xi_powers, xi_coefficients, powers_sets):
    """data_gw_bulkflow.py:62-116: per row, C = sum coeff * c[:, index(p + 3), :],
    spectrum = 8 pi w^3 (|C_+|^2 + |C_x|^2).  Numbers only (no envelope rows)."""
    w = np.asarray(w, dtype=np.float64)
    powers_available = list(powers_sets)
    out = []
    for row in np.asarray(c_rows):
        cp = np.zeros_like(w, dtype=complex)
        cx = np.zeros_like(w, dtype=complex)
        for p, coeff in zip(xi_powers, xi_coefficients):
            idx = powers_available.index(p + 3)
            cp += coeff * row[0, idx, :]
            cx += coeff * row[1, idx, :]
        out.append(8 * np.pi * w**3 * (np.abs(cp) ** 2 + np.abs(cx) ** 2))
    return np.array(out)


def de_dlogw(c_rows, w, cos_thetak, xi_powers, xi_coefficients, powers_sets):
    """data_gw_bulkflow.py:118-146: 2 * trapezoid over x = sorted(cos_theta_k), rows in the order given."""
    spec = de_dlogw_dcosthetak(c_rows, w, xi_powers, xi_coefficients, powers_sets)
    return 2.0 * np.trapezoid(spec, x=np.sort(np.asarray(cos_thetak, dtype=np.float64)), axis=0)


def de_dlogw_interp(w, de, d, d0=1.0, rho_vacuum=1.0):
    """data_gw_bulkflow.py:148-190."""
    return CubicSpline(np.asarray(w) / d, (d / d0) ** 5 * rho_vacuum**2 * np.asarray(de))
