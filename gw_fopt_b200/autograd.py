"""Differentiable bulk-flow spectrum for PyTorch (B200 extension, separate from the drop-in surface).

``BulkFlowSpectrum`` evaluates the (K, 2, S, W) spectrum of one bubble
configuration along K directions k-hat as a function of the gradient scaling
coefficients, their powers and the interior bubbles' nucleation events
(t, x, y, z), and differentiates it with the library's adjoint kernels
(bgwx_generalized_bulk_flow_spectrum_vjp, FP64, phases recomputed in the
backward pass).  Exterior bubbles are periodic images of the interior ones in
a cube of side ``box`` (the six face shifts of
rust/bubble-gw/src/many_bubbles/lattice/parallelepiped_lattice.rs:197-215), so
an image's gradient flows back to its source bubble; ``box=None`` means no
exterior bubbles.

``SurfaceTensionFit`` maps the fitted parameters of the post-collision
scaling onto one (coefficients, powers) set: with r = R_c/R = tau/dt,
    f(r) = alpha r^(xi + 3 + gamma) + delta r^(xi + 3),
the bulk-flow power law r^(xi + 3) (powers = xi + 3,
docs/generalized_bulkflow.md:46) times a surface-tension correction
alpha (R/R_c)^(-gamma) + delta (the form fitted by
src/gw_fopt/bubble_dynamics/utils/surface_tension_fitter.py:92-96).
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Optional

import numpy as np
import torch

from . import _lib as L
from .many_bubbles import _call, _cutoff_config

__all__ = ["BulkFlowSpectrum", "SurfaceTensionFit", "log_power_residual"]

_SHIFTS = np.array([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]], dtype=np.float64)


def _images(interior: np.ndarray, box: Optional[float]) -> np.ndarray:
    if box is None:
        return np.zeros((0, 4))
    out = np.repeat(interior, 6, axis=0)
    out[:, 1:4] = out[:, 1:4] + np.tile(_SHIFTS * box, (interior.shape[0], 1))
    return out


class _SpectrumFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, coefficients, powers, interior, model):
        c = coefficients.detach().cpu().numpy().astype(np.float64)
        p = powers.detach().cpu().numpy().astype(np.float64)
        x = interior.detach().cpu().numpy().astype(np.float64)
        out = model._forward(c, p, x)
        ctx.model = model
        ctx.save_for_backward(coefficients, powers, interior)
        real = np.ascontiguousarray(out).view(np.float64).reshape(out.shape + (2,))
        return torch.from_numpy(real.copy()).to(interior.device)

    @staticmethod
    def backward(ctx, grad):
        c, p, x = ctx.saved_tensors
        g = grad.detach().cpu().numpy().astype(np.float64)
        gc = np.ascontiguousarray(g[..., 0] + 1j * g[..., 1])
        dc, dp, dx = ctx.model._vjp(c.detach().cpu().numpy().astype(np.float64),
                                    p.detach().cpu().numpy().astype(np.float64),
                                    x.detach().cpu().numpy().astype(np.float64), gc)
        return (torch.from_numpy(dc).to(c.device, c.dtype) if ctx.needs_input_grad[0] else None,
                torch.from_numpy(dp).to(p.device, p.dtype) if ctx.needs_input_grad[1] else None,
                torch.from_numpy(dx).to(x.device, x.dtype) if ctx.needs_input_grad[2] else None,
                None)


class BulkFlowSpectrum:
    """C(coefficients, powers, interior): (K, 2, S, W, 2) float64 (real, imaginary last).

    ``kernel`` selects the forward kernel ('fp64_direct', 'fp64_factored' or
    'mixed'); the backward pass is the adjoint, FP64 with an FP64 kernel and with
    FP32 products folded into FP64 with a mixed one.  With ``keep_masks`` the
    forward keeps its collision masks on the device and a backward on the same
    bubbles reads them (the same gradients, one mask search fewer).
    """

    def __init__(self, *, n_cos: int, n_phi: int, w, khat, t_end: float, n_t: int, t_begin: float = 0.0,
                 box: Optional[float] = 1.0, time_cutoff=None, damping: Optional[float] = None,
                 kernel: str = "fp64_factored", keep_masks: bool = True):
        self.w = np.ascontiguousarray(np.asarray(w, dtype=np.float64).ravel())
        self.khat = np.ascontiguousarray(np.asarray(khat, dtype=np.float64).reshape(-1, 3))
        self.n_cos, self.n_phi = int(n_cos), int(n_phi)
        self.t_begin, self.t_end, self.n_t = float(t_begin), float(t_end), int(n_t)
        self.box = box
        self.damping = damping
        self._cut = _cutoff_config(time_cutoff)
        h = C.c_void_p()
        _call(L.lib().bgwx_generalized_bulk_flow_new_unchecked(C.byref(h), None, 0, None, 0))
        self._h = h
        _call(L.lib().bgw_generalized_bulk_flow_set_resolution(h, self.n_cos, self.n_phi, True))
        k = {"fp64_direct": L.KERNEL_FP64_DIRECT, "fp64_factored": L.KERNEL_FP64_FACTORED,
             "mixed": L.KERNEL_MIXED, "mixed_simt": L.KERNEL_MIXED_SIMT}[kernel]
        _call(L.lib().bgwx_generalized_bulk_flow_set_kernel(h, k))
        # the backward of a forward on the same bubbles reads the forward's masks instead of
        # searching again (when every frame's masks fit on the device)
        _call(L.lib().bgwx_generalized_bulk_flow_set_keep_masks(h, bool(keep_masks)))
        self.last_forward_ms = 0.0
        self.last_backward_ms = 0.0

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                L.lib().bgw_generalized_bulk_flow_free(h)
            except Exception:
                pass
            self._h = None

    def __call__(self, coefficients: torch.Tensor, powers: torch.Tensor, interior: torch.Tensor) -> torch.Tensor:
        return _SpectrumFn.apply(coefficients, powers, interior, self)

    # --- library calls ----------------------------------------------------------
    def _set(self, c, p, x):
        c = np.ascontiguousarray(np.asarray(c, dtype=np.float64).reshape(np.shape(c)[0], -1))
        p = np.ascontiguousarray(np.asarray(p, dtype=np.float64).reshape(c.shape))
        x = np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(-1, 4))
        ext = np.ascontiguousarray(_images(x, self.box))
        _call(L.lib().bgw_generalized_bulk_flow_set_gradient_scaling_params(
            self._h, L.ptr(c), L.ptr(p), c.shape[0], c.shape[1],
            math.nan if self.damping is None else float(self.damping)))
        _call(L.lib().bgwx_generalized_bulk_flow_set_bubbles(self._h, L.ptr(x), x.shape[0], L.ptr(ext),
                                                             ext.shape[0]))
        return c.shape

    def _timings(self):
        t = L.BgwxTimings()
        _call(L.lib().bgwx_generalized_bulk_flow_last_timings(self._h, C.byref(t)))
        return t

    def _forward(self, c, p, x):
        S, _ = self._set(c, p, x)
        out = np.zeros((self.khat.shape[0], 2, S, self.w.size), dtype=np.complex128)
        _call(L.lib().bgwx_generalized_bulk_flow_compute_c_integral_khat(
            self._h, L.ptr(self.w), self.w.size, True, self.t_begin, self.t_end, self.n_t, L.ptr(self.khat),
            self.khat.shape[0], None, 0, self._cut, out.ctypes.data_as(C.POINTER(L.BgwComplex64)), out.size))
        self.last_forward_ms = self._timings().total_ms
        return out

    def _vjp(self, c, p, x, gbar):
        (S, M) = self._set(c, p, x)
        n = x.reshape(-1, 4).shape[0]
        n_tot = n + (6 * n if self.box is not None else 0)
        gc = np.zeros((S, M))
        gp = np.zeros((S, M))
        gb = np.zeros((n_tot, 4))
        g = np.ascontiguousarray(gbar.reshape(-1).astype(np.complex128))
        _call(L.lib().bgwx_generalized_bulk_flow_spectrum_vjp(
            self._h, L.ptr(self.w), self.w.size, True, self.t_begin, self.t_end, self.n_t, L.ptr(self.khat),
            self.khat.shape[0], self._cut, g.ctypes.data_as(C.POINTER(L.BgwComplex64)), g.size, L.ptr(gc),
            L.ptr(gp), L.ptr(gb)))
        self.last_backward_ms = self._timings().total_ms
        gx = gb[:n].copy()
        if self.box is not None:
            gx += gb[n:].reshape(n, 6, 4).sum(axis=1)
        return gc, gp, gx.reshape(np.shape(x))

    def vjp(self, coefficients, powers, interior, gbar):
        """(d coefficients, d powers, d interior) of Re sum conj(gbar) C, without autograd."""
        return self._vjp(np.asarray(coefficients, dtype=np.float64), np.asarray(powers, dtype=np.float64),
                         np.asarray(interior, dtype=np.float64), np.asarray(gbar))


class SurfaceTensionFit(torch.nn.Module):
    """Learnable xi and the (alpha, gamma, delta) surface-tension correction, as one (1, 2) parameter set."""

    def __init__(self, xi: float = 1.5, alpha: float = 1.0, gamma: float = 0.0, delta: float = 0.0):
        super().__init__()
        self.xi = torch.nn.Parameter(torch.tensor(float(xi), dtype=torch.float64))
        self.alpha = torch.nn.Parameter(torch.tensor(float(alpha), dtype=torch.float64))
        self.gamma = torch.nn.Parameter(torch.tensor(float(gamma), dtype=torch.float64))
        self.delta = torch.nn.Parameter(torch.tensor(float(delta), dtype=torch.float64))

    def forward(self):
        coefficients = torch.stack([self.alpha, self.delta]).reshape(1, 2)
        powers = torch.stack([self.xi + 3.0 + self.gamma, self.xi + 3.0]).reshape(1, 2)
        return coefficients, powers


def log_power_residual(c: torch.Tensor, target_power: torch.Tensor) -> torch.Tensor:
    """Mean squared log-residual of P = |C_+|^2 + |C_x|^2 per (k-hat, set, w) against a target."""
    p = (c ** 2).sum(dim=-1).sum(dim=1)
    return ((torch.log(p) - torch.log(target_power)) ** 2).mean()
