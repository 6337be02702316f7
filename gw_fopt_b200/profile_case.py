"""One spectrum call of a synthetic workload, for profiling (ncu) and timing.

    python -m gw_fopt_b200.profile_case --config 3 --kernel mixed --khat 1 --bubbles 512 [--reps 1] [--n-t 256]
    python -m gw_fopt_b200.profile_case --config 4 --kernel mixed --khat 64 --realizations 256 [--compare 4]
    python -m gw_fopt_b200.profile_case --config 5 --kernel mixed --khat 32 --fit-steps 5

--bubbles restricts the radiating bubbles to the first B (all colliders stay
present), which keeps a profiler capture small while the per-bubble work and
the collision geometry are those of the full configuration.  Config 4 is the
batched ensemble; --realizations takes the first R of its 256 realizations and
--compare C also runs the first C realizations with the FP64 factored kernel
and reports the mixed kernel's error against it.  Config 5 is the adjoint
workload: forward and backward passes of the fit loss (mean squared log
residual of |C_+|^2 + |C_x|^2 against a target made at xi = 2 with perturbed
coefficients) and --fit-steps Adam steps on (xi, alpha, gamma, delta) and the
bubbles' nucleation events.
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
    ap.add_argument("--realizations", type=int, default=256)
    ap.add_argument("--compare", type=int, default=0)
    ap.add_argument("--device-nucleation", action="store_true",
                    help="config 4: draw the realizations on the GPU (gw_fopt_b200.nucleation)")
    ap.add_argument("--fit-steps", type=int, default=3)
    ap.add_argument("--n-t", type=int, default=0, help="override the configuration's time steps (smaller captures)")
    a = ap.parse_args()
    if a.config == 4:
        return run_ensemble(a)
    if a.config == 5:
        return run_adjoint(a)
    c = W.config(a.config, k_subset=a.khat)
    g = mb.GeneralizedBulkFlow(mb.LatticeBubbles(mb.EmptyLattice(), c.interior, c.exterior))
    g.set_resolution(c.n_cos, c.n_phi)
    g.set_gradient_scaling_params(c.coefficients.tolist(), c.powers.tolist())
    g.set_kernel(a.kernel)
    sel = np.arange(a.bubbles) if a.bubbles else None
    for r in range(a.reps):
        t0 = time.perf_counter()
        n_t = a.n_t or c.n_t
        out = g.compute_c_integral_khat(c.w, c.khat, t_begin=c.t_begin, t_end=c.t_end, n_t=n_t,
                                        selected_bubbles=sel)
        wall = time.perf_counter() - t0
        t = g.last_timings()
        n_rad = a.bubbles or c.n
        pte = c.khat.shape[0] * n_rad * c.n_cos * c.n_phi * n_t
        print(json.dumps({"rep": r, "config": c.name, "kernel": a.kernel, "khat": int(c.khat.shape[0]),
                          "radiating": int(n_rad), "wall_s": wall, "masks_ms": t["masks_ms"],
                          "spectrum_ms": t["spectrum_ms"], "total_ms": t["total_ms"], "fallbacks": t["fallbacks"],
                          "pte_per_s": pte / (t["total_ms"] * 1e-3), "checksum": float(np.abs(out).sum())}))


def run_ensemble(a):
    from .ensemble import BulkFlowEnsemble
    t0 = time.perf_counter()
    if a.device_nucleation:
        from .nucleation import ensemble_config_device
        c = ensemble_config_device(n_real=a.realizations, k_subset=a.khat)
    else:
        c = W.ensemble_config(k_subset=a.khat)
        c.realizations = c.realizations[:a.realizations]
    gen_s = time.perf_counter() - t0

    def make(kernel, reals):
        e = BulkFlowEnsemble(reals, validate=False)
        e.set_resolution(c.n_cos, c.n_phi)
        e.set_gradient_scaling_params(c.coefficients.tolist(), c.powers.tolist())
        e.set_kernel(kernel)
        return e

    ens = make(a.kernel, c.realizations)
    pte = c.pte
    for r in range(a.reps):
        t0 = time.perf_counter()
        out = ens.compute_c_integral_khat(c.w, c.khat, t_begin=c.t_begin, t_end=c.t_end, n_t=c.n_t)
        wall = time.perf_counter() - t0
        t = ens.last_timings()
        rec = {"rep": r, "config": c.name, "kernel": a.kernel, "realizations": len(c.realizations),
               "khat": int(c.khat.shape[0]), "bubbles": c.n_total, "generate_s": gen_s, "wall_s": wall,
               "total_ms": t["total_ms"], "launches": t["launches"], "pte": pte,
               "pte_per_s": pte / (t["total_ms"] * 1e-3), "checksum": float(np.abs(out).sum())}
        if a.compare and r == 0:
            n = min(a.compare, len(c.realizations))
            ref = make("fp64_factored", c.realizations[:n]).compute_c_integral_khat(
                c.w, c.khat, t_begin=c.t_begin, t_end=c.t_end, n_t=c.n_t)
            errs = []
            for q in range(n):
                g = out[q].reshape(-1, c.w.size)
                f = ref[q].reshape(-1, c.w.size)
                num = np.linalg.norm(g - f, axis=0)
                errs.append((float(np.linalg.norm(g - f) / np.linalg.norm(f)),
                             float(num.max() / np.linalg.norm(f, axis=0).max())))
            rec["compare_realizations"] = n
            rec["err_global_max"] = max(e[0] for e in errs)
            rec["err_peak_scaled_max"] = max(e[1] for e in errs)
            pm = np.mean(np.abs(out[:n]) ** 2, axis=0)
            pr = np.mean(np.abs(ref) ** 2, axis=0)
            rec["err_mean_power"] = float(np.linalg.norm(pm - pr) / np.linalg.norm(pr))
        print(json.dumps(rec))


def run_adjoint(a):
    import torch

    from .autograd import BulkFlowSpectrum, SurfaceTensionFit, log_power_residual
    c = W.config(5, k_subset=a.khat)
    model = BulkFlowSpectrum(n_cos=c.n_cos, n_phi=c.n_phi, w=c.w, khat=c.khat, t_end=c.t_end, n_t=c.n_t,
                             t_begin=c.t_begin, box=1.0, kernel=a.kernel)
    x = torch.tensor(c.interior, dtype=torch.float64, requires_grad=True)
    with torch.no_grad():
        co_t, po_t = SurfaceTensionFit(xi=2.0, alpha=1.1, gamma=0.4, delta=-0.1)()
        target = (model(co_t, po_t, x) ** 2).sum(-1).sum(1)
    fit = SurfaceTensionFit(xi=1.5, alpha=1.0, gamma=0.0, delta=0.0)
    opt = torch.optim.Adam(list(fit.parameters()) + [x], lr=1e-3)
    pte = c.khat.shape[0] * c.n * c.n_cos * c.n_phi * c.n_t
    for step in range(a.fit_steps):
        t0 = time.perf_counter()
        opt.zero_grad()
        co, po = fit()
        loss = log_power_residual(model(co, po, x), target)
        loss.backward()
        opt.step()
        wall = time.perf_counter() - t0
        print(json.dumps({"step": step, "config": c.name, "forward_kernel": a.kernel, "khat": int(c.khat.shape[0]),
                          "loss": float(loss), "xi": float(fit.xi), "alpha": float(fit.alpha),
                          "gamma": float(fit.gamma), "delta": float(fit.delta),
                          "forward_ms": model.last_forward_ms, "backward_ms": model.last_backward_ms,
                          "wall_s": wall, "pte": pte,
                          "pte_per_s_fwd_bwd": pte / ((model.last_forward_ms + model.last_backward_ms) * 1e-3)}))


if __name__ == "__main__":
    main()
