"""One spectrum call of a synthetic workload, for profiling (ncu) and timing.

    python -m gw_fopt_b200.profile_case --config 3 --kernel mixed --khat 1 --bubbles 512 [--reps 1]

--bubbles restricts the radiating bubbles to the first B (all colliders stay
present), which keeps a profiler capture small while the per-bubble work and
the collision geometry are those of the full configuration.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import many_bubbles as mb
from . import workloads as W


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", type=int, default=3)
    ap.add_argument("--kernel", default="mixed", choices=["fp64_direct", "fp64_factored", "mixed"])
    ap.add_argument("--khat", type=int, default=1)
    ap.add_argument("--bubbles", type=int, default=0)
    ap.add_argument("--reps", type=int, default=1)
    a = ap.parse_args()
    c = W.config(a.config, k_subset=a.khat)
    g = mb.GeneralizedBulkFlow(mb.LatticeBubbles(mb.EmptyLattice(), c.interior, c.exterior))
    g.set_resolution(c.n_cos, c.n_phi)
    g.set_gradient_scaling_params(c.coefficients.tolist(), c.powers.tolist())
    g.set_kernel(a.kernel)
    sel = np.arange(a.bubbles) if a.bubbles else None
    for r in range(a.reps):
        t0 = time.perf_counter()
        out = g.compute_c_integral_khat(c.w, c.khat, t_begin=c.t_begin, t_end=c.t_end, n_t=c.n_t,
                                        selected_bubbles=sel)
        wall = time.perf_counter() - t0
        t = g.last_timings()
        n_rad = a.bubbles or c.n
        pte = c.khat.shape[0] * n_rad * c.n_cos * c.n_phi * c.n_t
        print(json.dumps({"rep": r, "config": c.name, "kernel": a.kernel, "khat": int(c.khat.shape[0]),
                          "radiating": int(n_rad), "wall_s": wall, "masks_ms": t["masks_ms"],
                          "spectrum_ms": t["spectrum_ms"], "total_ms": t["total_ms"], "fallbacks": t["fallbacks"],
                          "pte_per_s": pte / (t["total_ms"] * 1e-3), "checksum": float(np.abs(out).sum())}))


if __name__ == "__main__":
    main()
