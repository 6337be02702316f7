"""FP64 adjoint of the oracle spectrum, in numpy (test infrastructure only).

Differentiates the oracle's restatement of the bulk-flow spectrum
(rust/bubble-gw/src/many_bubbles/generalized_bulk_flow.rs:481-586 for B,
:588-664 for A, :775-873 for the time integral, :421-471 for the collision
delays tau) with respect to the scaling coefficients and powers
(:315-363, :549-567) and to every bubble row (t, x, y, z).  First-collider
codes and delays come from the oracle's exact search (oracle.first_colliding)
on each rotated frame.  Collision status and first-collider identity are
piecewise constant and carry no gradient.  Only tests import this module.

Notation per rotated frame (bubble a, row i, patch j, step k, dt = t_k - t_a > 0):
  C_{g,s}(w) = sum e^{i phi} T_{g,s},  phi = w ((t_k - z_a) - dt c_i),
  T_{g,s}    = pre_{i,k} dt^3 sum_j q_g(j) f_s,  pre = 1/2 (1 - c^2) dphi dc v_i u_k cut_k dt / (6 pi).
The loss enters through its cotangent G = dL/dRe C + i dL/dIm C.
"""
from __future__ import annotations

import math

import numpy as np

from . import oracle as O


def _grids(n_cos, n_phi, t_begin, t_end, n_t, cutoff):
    cos_t = np.array([-1.0 + (2.0 / (n_cos - 1)) * i for i in range(n_cos)])
    phi = np.array([(2.0 * math.pi / (n_phi - 1)) * j for j in range(n_phi)])
    t = np.array([t_begin + ((t_end - t_begin) / (n_t - 1)) * k for k in range(n_t)])
    cut = np.ones(n_t) if cutoff is None else O.time_cutoff(t, *cutoff)
    return cos_t, phi, t, cut


def spectrum_vjp(interior, exterior, khat, n_cos, n_phi, w, t_begin, t_end, n_t, gbar, coefficients=((1.0,),),
                 powers=((3.0,),), damping=None, cutoff=None):
    """Returns (d coefficients (S, M), d powers (S, M), d bubbles (n_int + n_ext, 4)) of
    L = Re sum conj(gbar) C for the (K, 2, S, W) spectrum along the khat rows."""
    interior = np.asarray(interior, dtype=np.float64).reshape(-1, 4)
    exterior = np.zeros((0, 4)) if exterior is None else np.asarray(exterior, dtype=np.float64).reshape(-1, 4)
    co = np.asarray(coefficients, dtype=np.float64)
    po = np.asarray(powers, dtype=np.float64)
    S, M = co.shape
    w = np.asarray(w, dtype=np.float64).ravel()
    kh = np.asarray(khat, dtype=np.float64).reshape(-1, 3)
    gbar = np.asarray(gbar, dtype=np.complex128).reshape(kh.shape[0], 2, S, w.size)
    n_int = interior.shape[0]
    allb = np.concatenate([interior, exterior])
    cos_t, phi, t, cut = _grids(n_cos, n_phi, t_begin, t_end, n_t, cutoff)
    dphi = 2.0 * math.pi / n_phi
    dc = 2.0 / (n_cos - 1)
    dt = t[1] - t[0]
    v = np.ones(n_cos)
    v[[0, -1]] = 0.5
    u = np.ones(n_t)
    u[[0, -1]] = 0.5
    wj = np.ones(n_phi)
    wj[[0, -1]] = 0.5
    q = np.stack([wj * np.cos(2.0 * phi), wj * np.sin(2.0 * phi)])  # (2, n_phi)
    pre = (0.5 * (1.0 - cos_t ** 2) * dphi * dc * v)[:, None] * (u * cut * dt / (6.0 * math.pi))[None, :]
    sth = np.abs(np.sqrt(1.0 - cos_t ** 2))
    nhat = np.stack([sth[:, None] * np.cos(phi)[None, :], sth[:, None] * np.sin(phi)[None, :],
                     np.broadcast_to(cos_t[:, None], (n_cos, n_phi))], axis=-1)  # (n_cos, n_phi, 3)
    invw = 0.0 if damping is None else 1.0 / damping

    g_co = np.zeros((S, M))
    g_po = np.zeros((S, M))
    g_b = np.zeros_like(allb)
    for f, k in enumerate(kh):
        R = O.rotation_for_khat(k)
        rb = O.rotate(R, allb)
        codes, tau = O.first_colliding(rb[:n_int], rb[n_int:], n_cos, n_phi, with_delta_tab=True)
        Gf = gbar[f]  # (2, S, W)
        for a in range(n_int):
            ta, za = rb[a, 0], rb[a, 3]
            dtk = t - ta
            ok = dtk > 0.0
            if not ok.any():
                continue
            ks = np.flatnonzero(ok)
            d = dtk[ks]  # (nk,)
            th = (t[ks][None, :] - za) - d[None, :] * cos_t[:, None]  # (n_cos, nk)
            e = np.exp(1j * w[:, None, None] * th[None])  # (W, n_cos, nk)
            P = np.einsum("gsw,wik->gsik", np.conj(Gf), e)
            Q = np.einsum("gsw,wik->gsik", np.conj(Gf) * w, e)
            bbar = P.real  # (2, S, n_cos, nk)
            imq = Q.imag
            tr = tau[a]  # (n_cos, n_phi)
            coll = (tr[:, :, None] > 0.0) & (d[None, None, :] >= tr[:, :, None])  # (n_cos, n_phi, nk)
            with np.errstate(divide="ignore", invalid="ignore"):
                r = np.where(coll, tr[:, :, None] / d[None, None, :], 1.0)
                lr = np.log(r)
                D = np.exp(-(d[None, None, :] - tr[:, :, None]) * invw) if damping is not None else np.ones_like(r)
                rp = np.exp(po[:, :, None, None, None] * lr[None, None]) * D[None, None]  # (S, M, c, p, k)
                rp = np.where(coll[None, None], rp, 0.0)
                fs = np.where(coll[None], np.einsum("sm,smcpk->scpk", co, rp), 1.0)  # (S, c, p, k)
                dfdt = np.einsum("sm,smcpk->scpk", co, rp * (-po[:, :, None, None, None] / d[None, None, None, None, :]
                                                            - invw))
                trs = np.where(tr > 0.0, tr, 1.0)
                dfdtau = np.einsum("sm,smcpk->scpk", co, rp * (po[:, :, None, None, None] / trs[None, None, :, :, None]
                                                              + invw))
            pk = pre[:, ks]  # (n_cos, nk)
            qf = np.einsum("gp,scpk->gsck", q, fs)  # sum_j q_g f_s
            qdf = np.einsum("gp,scpk->gsck", q, dfdt)
            T = pk[None, None] * d ** 3 * qf
            dTdd = pk[None, None] * (3.0 * d ** 2 * qf + d ** 3 * qdf)
            g_b[a, 0] += np.sum(-bbar * dTdd) + np.sum(-cos_t[None, None, :, None] * imq * T)
            gz = np.sum(imq * T)
            g_b[a, 1:4] += gz * R[2, :]
            wgt = bbar * pk[None, None] * d ** 3  # (g, s, c, k)
            g_co += np.einsum("gsck,gp,smcpk->sm", wgt, q, rp)
            g_po += np.einsum("gsck,gp,smcpk->sm", wgt, q, rp * co[:, :, None, None, None] * np.where(coll, lr, 0.0)[None, None])
            taubar = np.einsum("gsck,gp,scpk->cp", wgt, q, dfdtau)  # (n_cos, n_phi)
            for i in range(n_cos):
                for j in range(n_phi):
                    tb = taubar[i, j]
                    code = codes[a, i, j]
                    if tb == 0.0 or code == -1 or not tr[i, j] > 0.0:
                        continue
                    b = code if code >= 0 else n_int + (-code - 2)
                    Dl = rb[b] - rb[a]
                    nh = nhat[i, j]
                    dot = -Dl[0] + Dl[1:] @ nh
                    if abs(dot) < 1e-10:
                        continue
                    D2 = -Dl[0] ** 2 + Dl[1:] @ Dl[1:]
                    h = 0.5 * D2 / dot ** 2
                    gt = tb * (-Dl[0] / dot + h)
                    gx = tb * (Dl[1:] / dot - h * nh)
                    gxu = R.T @ gx
                    g_b[b, 0] += gt
                    g_b[b, 1:4] += gxu
                    g_b[a, 0] -= gt
                    g_b[a, 1:4] -= gxu
    return g_co, g_po, g_b
