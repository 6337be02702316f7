"""Nucleation Monte Carlo on the GPU for ensembles.

bgwx_nucleate_exponential draws every realization's bubbles on the device, one
block per realization (gw_fopt_b200/csrc/nucleation.cu): exponential-rate
nucleation in a periodic box with rejection inside accepted bubbles and their
nearest periodic copies, random numbers from Philox4x32-10 keyed by the
realization's seed.  It removes the host-side generation from the batched
ensemble; the outputs feed BulkFlowEnsemble directly.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .workloads import EnsembleConfig, ensemble_config


def exponential_nucleation(n_bubbles, beta, seeds, L_box=1.0, gamma_scale=1.0, max_rejections=20000):
    """List of (interior (n, 4), exterior (6n, 4)) per realization, drawn on the GPU."""
    n = np.ascontiguousarray(np.atleast_1d(n_bubbles), dtype=np.int64)
    b = np.ascontiguousarray(np.atleast_1d(beta), dtype=np.float64)
    s = np.ascontiguousarray(np.atleast_1d(seeds), dtype=np.uint64)
    if not (n.shape == b.shape == s.shape) or n.ndim != 1:
        raise ValueError("n_bubbles, beta and seeds must be 1-D of one length")
    rows = int(np.clip(n, 0, None).sum())  # negative counts are rejected by the library
    interior = np.empty((rows, 4))
    exterior = np.empty((6 * rows, 4))
    attempts = np.empty(n.size, dtype=np.int32)
    L.check(L.lib().bgwx_nucleate_exponential(
        n.ctypes.data_as(C.POINTER(C.c_int64)), L.ptr(b), s.ctypes.data_as(C.POINTER(C.c_uint64)), n.size,
        float(L_box), float(gamma_scale), int(max_rejections), L.ptr(interior), interior.size, L.ptr(exterior),
        exterior.size, attempts.ctypes.data_as(C.POINTER(C.c_int32))))
    out, o = [], 0
    for k in n.tolist():
        out.append((interior[o:o + k], exterior[6 * o:6 * (o + k)]))
        o += k
    return out


def ensemble_draws(n_real=256, seed=4, n_min=50, n_max=800, beta_lo=5.0, beta_hi=15.0):
    """The per-realization (n, beta, seed) of the benchmark ensemble (the same draws as
    workloads.ensemble makes on the host)."""
    rng = np.random.default_rng(seed)
    ns = rng.integers(n_min, n_max + 1, n_real)
    betas = rng.uniform(beta_lo, beta_hi, n_real)
    seeds = rng.integers(0, 2 ** 31 - 1, n_real)
    return ns, betas, seeds


def ensemble_config_device(n_real=256, k_subset=None, max_rejections=20000) -> EnsembleConfig:
    """The batched-ensemble configuration with its realizations drawn on the GPU."""
    cfg = ensemble_config(n_real=0, k_subset=k_subset)
    cfg.name = cfg.name.replace("-0r-", f"-{n_real}r-") + "-device-nucleation"
    ns, betas, seeds = ensemble_draws(n_real)
    cfg.realizations = exponential_nucleation(ns, betas, seeds, max_rejections=max_rejections)
    return cfg
