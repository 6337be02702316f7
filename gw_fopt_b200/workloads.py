"""Seeded synthetic bubble configurations and spectrum grids.

No public dataset exists for this path; these generators stand in for the
reference's nucleation samplers with the same shapes and distributions:

* ``uniform_config``: N centres uniform in a cubic box, nucleation times
  uniform in [0, t_max]; the whole set is redrawn until every interior pair
  and every interior/periodic-image pair is causal (Minkowski interval >= 0),
  as LatticeBubbles::new requires (lattice_bubbles.rs:71-119).
* ``exponential_nucleation``: Monte Carlo of a nucleation rate
  Gamma(t) = Gamma0 exp(beta t) per unit volume: candidate events arrive as a
  Poisson process over the box and are rejected when they fall inside an
  already nucleated bubble or one of its periodic images (minimum-image
  distance), the rejection rule of
  rust/bubble-gw/src/many_bubbles/bubbles_nucleation/fixed_rate_nucleation.rs:188-275.
  Times are normalised so that the earliest bubble nucleates at t = 0
  (lattice_bubbles.rs:439-460).
* ``periodic_images``: the 6 face shifts of parallelepiped_lattice.rs:197-215.
* ``fibonacci_khat``: K directions z_i = 1-(2i+1)/K, phi_i = i*pi*(3-sqrt 5).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


def periodic_images(interior: np.ndarray, L: float = 1.0) -> np.ndarray:
    """(6N, 4): for each bubble the shifts +e1, -e1, +e2, -e2, +e3, -e3 of a cube of side L."""
    interior = np.asarray(interior, dtype=np.float64).reshape(-1, 4)
    shifts = np.array([[L, 0, 0], [-L, 0, 0], [0, L, 0], [0, -L, 0], [0, 0, L], [0, 0, -L]], dtype=np.float64)
    out = np.repeat(interior, 6, axis=0)
    out[:, 1:4] = out[:, 1:4] + np.tile(shifts, (interior.shape[0], 1))
    return out


def _causal(interior, exterior) -> bool:
    def ok(a, b):
        d = b[None, :, :] - a[:, None, :]
        s = (((-d[..., 0]) * d[..., 0] + d[..., 1] * d[..., 1]) + d[..., 2] * d[..., 2]) + d[..., 3] * d[..., 3]
        return s
    s_ii = ok(interior, interior)
    iu = np.triu_indices(interior.shape[0], 1)
    if np.any(s_ii[iu] < 0.0):
        return False
    if exterior.shape[0] and np.any(ok(interior, exterior) < 0.0):
        return False
    return True


def uniform_config(n: int, L: float = 1.0, t_max: float = 0.2, seed: int = 1, max_tries: int = 10000):
    """Uniform centres in [0, L)^3 and times in [0, t_max], redrawn until causal (with periodic images)."""
    rng = np.random.default_rng(seed)
    for _ in range(max_tries):
        b = np.empty((n, 4))
        b[:, 0] = rng.uniform(0.0, t_max, n)
        b[:, 1:4] = rng.uniform(0.0, L, (n, 3))
        ext = periodic_images(b, L)
        if _causal(b, ext):
            return b, ext
    raise RuntimeError("could not draw a causal configuration")


def exponential_nucleation(n: int, beta: float, L: float = 1.0, seed: int = 2, gamma_scale: float = 1.0,
                           max_rejections: int = 400000):
    """N bubbles from exponential-rate nucleation in a periodic box of side L.

    Returns (interior (N, 4), exterior (6N, 4)) with times normalised to min t = 0.
    The rate prefactor is chosen so that about N candidates arrive within one
    1/beta; it is doubled and the draw repeated if the false vacuum runs out
    before N bubbles are placed.
    """
    rng = np.random.default_rng(seed)
    V = L ** 3
    g0 = gamma_scale * n * beta / V  # Gamma0 V / beta = n * gamma_scale
    block = 256
    while True:
        pos = np.empty((n, 3))
        tn = np.empty(n)
        k = 0
        t = 0.0
        rejections = 0
        while k < n and rejections < max_rejections:
            # A block of candidates, drawn from the stream in the order of one
            # candidate at a time (u, then the three coordinates).  The arrival
            # times do not depend on acceptance, so the block is tested against
            # the bubbles accepted before it at once, and candidate by candidate
            # against those accepted inside it: the outcome is that of testing
            # one candidate at a time.
            state = rng.bit_generator.state
            r = rng.random((block, 4))
            tc = np.empty(block)
            for q in range(block):
                # next arrival of a Poisson process with rate g0 V e^{beta t}
                t = math.log(math.exp(beta * t) - beta * math.log(r[q, 0]) / (g0 * V)) / beta
                tc[q] = t
            xc = 0.0 + (L - 0.0) * r[:, 1:4]
            if k:
                d = np.abs(xc[:, None, :] - pos[None, :k, :])
                d = np.minimum(d, L - d)  # minimum image = nearest periodic copy
                r2 = np.einsum("bij,bij->bi", d, d)
                rad = tc[:, None] - tn[None, :k]
                hit = np.any(r2 < rad * rad, axis=1)
            else:
                hit = np.zeros(block, dtype=bool)
            k0 = k
            used = 0
            for q in range(block):
                if k >= n or rejections >= max_rejections:
                    break
                used += 1
                x = xc[q]
                if hit[q]:
                    rejections += 1
                    continue
                if k > k0:
                    d = np.abs(pos[k0:k] - x)
                    d = np.minimum(d, L - d)
                    r2 = np.einsum("ij,ij->i", d, d)
                    rad = tc[q] - tn[k0:k]
                    if np.any(r2 < rad * rad):
                        rejections += 1
                        continue
                pos[k] = x
                tn[k] = tc[q]
                k += 1
            if used < block:  # leave the stream where a one-at-a-time draw would have left it
                rng.bit_generator.state = state
                rng.random((used, 4))
        if k == n:
            break
        g0 *= 2.0
    interior = np.empty((n, 4))
    interior[:, 0] = tn - tn.min()
    interior[:, 1:4] = pos
    return interior, periodic_images(interior, L)


def fibonacci_khat(K: int) -> np.ndarray:
    """(K, 3) unit vectors on a Fibonacci sphere."""
    i = np.arange(K, dtype=np.float64)
    z = 1.0 - (2.0 * i + 1.0) / K
    phi = i * math.pi * (3.0 - math.sqrt(5.0))
    r = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    k = np.stack([r * np.cos(phi), r * np.sin(phi), z], axis=1)
    return k / np.linalg.norm(k, axis=1, keepdims=True)


@dataclass
class SpectrumConfig:
    """One synthetic workload: bubbles, angular/time grids, frequencies, directions, scaling."""
    name: str
    interior: np.ndarray
    exterior: np.ndarray
    n_cos: int
    n_phi: int
    n_t: int
    t_begin: float
    t_end: float
    w: np.ndarray
    khat: np.ndarray
    coefficients: np.ndarray = field(default_factory=lambda: np.array([[1.0]]))
    powers: np.ndarray = field(default_factory=lambda: np.array([[5.0]]))  # xi = 2 -> power xi + 3

    @property
    def n(self):
        return self.interior.shape[0]

    @property
    def pte(self) -> int:
        """Patch-time evaluations of one complete spectrum: K * N * n_cos * n_phi * n_t."""
        return self.khat.shape[0] * self.n * self.n_cos * self.n_phi * self.n_t

    @property
    def phase_terms(self) -> int:
        return self.khat.shape[0] * self.n * self.n_cos * self.n_t * self.w.size

    @property
    def phase_terms_t(self) -> int:
        return self.khat.shape[0] * self.n * self.n_t * self.w.size

    @property
    def counted_flops(self) -> float:
        """F = 6 PTE + 8 Phi + 20 Phi_t (declared counting convention)."""
        return 6.0 * self.pte + 8.0 * self.phase_terms + 20.0 * self.phase_terms_t


def config(idx: int, k_subset: int | None = None) -> SpectrumConfig:
    """The five synthetic configurations of the bulk-flow benchmark (1-based index)."""
    if idx == 1:
        b, e = uniform_config(8, 1.0, 0.2, seed=1)
        c = SpectrumConfig("plain-8b-32x32-T128-W32-K16", b, e, 32, 32, 128, 0.0, 1.5,
                           np.geomspace(1.0, 1000.0, 32), fibonacci_khat(16))
    elif idx == 2:
        b, e = exponential_nucleation(512, 8.0, seed=2)
        c = SpectrumConfig("fp64-512b-128x128-T512-W128-K64", b, e, 128, 128, 512, 0.0, 1.5,
                           np.geomspace(1.0, 3000.0, 128), fibonacci_khat(64))
    elif idx == 3:
        b, e = exponential_nucleation(4096, 20.0, seed=3)
        c = SpectrumConfig("mixed-4096b-192x192-T1024-W256-K128", b, e, 192, 192, 1024, 0.0, 1.5,
                           np.geomspace(1.0, 1e4, 256), fibonacci_khat(128))
    elif idx == 5:
        b, e = exponential_nucleation(256, 6.0, seed=5)
        c = SpectrumConfig("adjoint-256b-64x64-T256-W64-K32", b, e, 64, 64, 256, 0.0, 1.5,
                           np.geomspace(1.0, 1000.0, 64), fibonacci_khat(32))
    else:
        raise ValueError(f"no single-realization config {idx}")
    if k_subset is not None:
        c.khat = c.khat[:k_subset]
    return c


def ensemble(n_real: int = 256, seed: int = 4, n_min: int = 50, n_max: int = 800, beta_lo: float = 5.0,
             beta_hi: float = 15.0, max_rejections: int = 20000):
    """Realizations for the batched ensemble: N_r ~ U{n_min..n_max}, beta_r ~ U[beta_lo, beta_hi].

    At small beta L a box holds few bubbles before the false vacuum runs out, so
    placing hundreds needs a larger rate prefactor; the lower rejection limit
    makes the sampler move on to the doubled prefactor sooner."""
    rng = np.random.default_rng(seed)
    ns = rng.integers(n_min, n_max + 1, n_real)
    betas = rng.uniform(beta_lo, beta_hi, n_real)
    seeds = rng.integers(0, 2 ** 31 - 1, n_real)
    return [exponential_nucleation(int(n), float(bt), seed=int(s), max_rejections=max_rejections)
            for n, bt, s in zip(ns, betas, seeds)]


@dataclass
class EnsembleConfig:
    """The batched-ensemble workload: realizations plus the grids they share."""
    name: str
    realizations: list
    n_cos: int
    n_phi: int
    n_t: int
    t_begin: float
    t_end: float
    w: np.ndarray
    khat: np.ndarray
    coefficients: np.ndarray = field(default_factory=lambda: np.array([[1.0]]))
    powers: np.ndarray = field(default_factory=lambda: np.array([[5.0]]))

    @property
    def n_total(self) -> int:
        return int(sum(r[0].shape[0] for r in self.realizations))

    @property
    def pte(self) -> int:
        return self.khat.shape[0] * self.n_total * self.n_cos * self.n_phi * self.n_t

    @property
    def phase_terms(self) -> int:
        return self.khat.shape[0] * self.n_total * self.n_cos * self.n_t * self.w.size

    @property
    def phase_terms_t(self) -> int:
        return self.khat.shape[0] * self.n_total * self.n_t * self.w.size

    @property
    def counted_flops(self) -> float:
        return 6.0 * self.pte + 8.0 * self.phase_terms + 20.0 * self.phase_terms_t


def ensemble_config(n_real: int = 256, k_subset: int | None = None) -> EnsembleConfig:
    """Batched ensemble: 256 realizations, N_r ~ U{50..800}, beta_r L ~ U[5, 15] (seed 4), periodic;
    96x96 patches, 384 time steps on [0, 1.5], 128 w geomspace [1, 3000], 64 Fibonacci k-hat."""
    c = EnsembleConfig(f"ensemble-{n_real}r-96x96-T384-W128-K64", ensemble(n_real), 96, 96, 384, 0.0, 1.5,
                       np.geomspace(1.0, 3000.0, 128), fibonacci_khat(64))
    if k_subset is not None:
        c.khat = c.khat[:k_subset]
    return c
