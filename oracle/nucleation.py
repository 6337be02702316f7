"""CPU restatement of the device nucleation sampler (test infrastructure only).

Exponential-rate nucleation in a periodic box, as gw_fopt_b200/workloads.py's
exponential_nucleation draws it (a Poisson process with rate Gamma0 V e^{beta t};
a candidate is rejected when it lies inside an accepted bubble, nearest periodic
copy; the prefactor doubles and the draw restarts when the false vacuum runs out),
which follows the rejection of candidates inside existing bubbles and images in
rust/bubble-gw/src/many_bubbles/bubbles_nucleation/fixed_rate_nucleation.rs.
The random numbers come from the counter-based generator Philox4x32-10 (Salmon,
Moraes, Dror, Shaw, SC'11): candidate q of attempt a of a realization with seed s
uses the block philox(counter = (q, a, 0, 0), key = (s mod 2^32, s div 2^32)),
u_i = (x_i + 0.5) 2^-32.  Only tests/ import this module; the product path is
the CUDA kernel in gw_fopt_b200/csrc/nucleation.cu.
"""
from __future__ import annotations

import math

import numpy as np

M0, M1 = 0xD2511F53, 0xCD9E8D57
W0, W1 = 0x9E3779B9, 0xBB67AE85
MASK = 0xFFFFFFFF


def philox4x32(ctr, key, rounds=10):
    c0, c1, c2, c3 = (int(v) & MASK for v in ctr)
    k0, k1 = (int(v) & MASK for v in key)
    for _ in range(rounds):
        p0 = M0 * c0
        p1 = M1 * c2
        hi0, lo0 = p0 >> 32, p0 & MASK
        hi1, lo1 = p1 >> 32, p1 & MASK
        c0, c1, c2, c3 = (hi1 ^ c1 ^ k0) & MASK, lo1, (hi0 ^ c3 ^ k1) & MASK, lo0
        k0 = (k0 + W0) & MASK
        k1 = (k1 + W1) & MASK
    return c0, c1, c2, c3


def uniforms(q, attempt, seed):
    x = philox4x32((q, attempt, 0, 0), (seed & MASK, (seed >> 32) & MASK))
    return [(v + 0.5) * 2.0 ** -32 for v in x]


def exponential_nucleation(n, beta, seed, L=1.0, gamma_scale=1.0, max_rejections=20000, max_attempts=40):
    """(interior (n, 4) with min t = 0, exterior (6n, 4), attempts)."""
    V = L * L * L
    g0 = gamma_scale * n * beta / V
    for attempt in range(max_attempts):
        pos = np.empty((n, 3))
        tn = np.empty(n)
        k = rej = q = 0
        t = 0.0
        while k < n and rej < max_rejections:
            u = uniforms(q, attempt, seed)
            q += 1
            t = math.log(math.exp(beta * t) - beta * math.log(u[0]) / (g0 * V)) / beta
            x = (L * u[1], L * u[2], L * u[3])
            hit = False
            for j in range(k):
                dx, dy, dz = abs(x[0] - pos[j, 0]), abs(x[1] - pos[j, 1]), abs(x[2] - pos[j, 2])
                dx, dy, dz = min(dx, L - dx), min(dy, L - dy), min(dz, L - dz)
                r2 = (dx * dx + dy * dy) + dz * dz
                rad = t - tn[j]
                if r2 < rad * rad:
                    hit = True
                    break
            if hit:
                rej += 1
                continue
            pos[k] = x
            tn[k] = t
            k += 1
        if k == n:
            interior = np.empty((n, 4))
            interior[:, 0] = tn - tn[0] if n else tn
            interior[:, 1:4] = pos
            shifts = np.array([[L, 0, 0], [-L, 0, 0], [0, L, 0], [0, -L, 0], [0, 0, L], [0, 0, -L]])
            ext = np.repeat(interior, 6, axis=0)
            ext[:, 1:4] = ext[:, 1:4] + np.tile(shifts, (n, 1))
            return interior, ext, attempt + 1
        g0 *= 2.0
    raise RuntimeError("nucleation did not place all bubbles")
