#!/usr/bin/env python
"""Benchmark of the generalized bulk-flow many-bubble GW spectrum on B200.

Metric: patch-time evaluations per second, PTE = K * N * n_cos * n_phi * n_t
for one complete spectrum (all k-hat directions, all bubbles, all t, all w),
masks included.  One step = one complete spectrum of the named synthetic
workload (seeded; no dataset exists for this path).

    python bench.py [--gpus N --steps K --warmup W] [--config 3] [--kernel mixed]
    python bench.py --impl reference ...   # the CPU restatement of the reference
    python bench.py --config 4 ...         # batched ensemble: one step = all realizations
    python bench.py --config 5 ...         # adjoint: one step = forward + backward of the fit loss
    python bench.py --once --config 3 --khat 1 --bubbles 512 [--n-t 256]   # one call, for ncu captures

value: device-resident inputs, result left in HBM (CUDA events on the
       launching stream, L2 flushed between steps by a 256 MiB write).
e2e:   the public Python API with host buffers, every input copied to the
       device and the result copied back each step.
Multi-GPU (torchrun): each rank computes its own k-hat directions of a
K*N-direction Fibonacci sphere (weak scaling, no data-path collective);
timing is the max over ranks.

--once runs one spectrum call of the chosen configuration restricted to its
first --khat directions, its first --bubbles radiating bubbles (every collider
stays present, so the per-bubble work and the collision geometry are those of
the full configuration) and optionally --n-t time steps, and prints the call's
device timings: the command that profiler captures run.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "patch-time evals/s: mixed-prec vs FP64 on one B200 at <=1e-6 rel err; CPU ref"
UNIT = "patch-time evals/s"
CPU_SAMPLE_BUBBLES = 64  # radiating bubbles of the CPU baseline, spread over nucleation order


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--config", type=int, default=3, choices=[1, 2, 3, 4, 5])
    ap.add_argument("--kernel", default="mixed", choices=["fp64_direct", "fp64_factored", "mixed", "mixed_simt"])
    ap.add_argument("--no-compare", action="store_true", help="skip the FP64 comparison measurements")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="automatic launch shape instead of the measured one")
    ap.add_argument("--once", action="store_true", help="one call of a sub-workload, for profiler captures")
    ap.add_argument("--khat", type=int, default=0, help="--once / config 4: first K k-hat directions")
    ap.add_argument("--bubbles", type=int, default=0, help="--once: first B radiating bubbles")
    ap.add_argument("--n-t", type=int, default=0, help="--once: override the time steps")
    ap.add_argument("--realizations", type=int, default=256, help="config 4: first R realizations")
    ap.add_argument("--compare-realizations", type=int, default=4, help="config 4: checked against FP64")
    return ap.parse_args()


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while running."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.path = tempfile.mktemp(suffix=".csv")
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait(timeout=10)
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                if int(f[0]) != self.index:
                    continue
                rows.append(f)
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = max(float(r[2]) for r in rows)
        load = [v for v in sm if v > 0.5 * mx] or sm
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[q] for r in rows for q in range(4) if r[5 + q].lower() == "active"})
        return {"sm_mhz": statistics.median(load), "sm_max_mhz": mx, "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------------------
def make_flow(cfg, kernel):
    from gw_fopt_b200 import many_bubbles as mb
    lb = mb.LatticeBubbles(mb.EmptyLattice(), cfg.interior, cfg.exterior)
    g = mb.GeneralizedBulkFlow(lb)
    g.set_resolution(cfg.n_cos, cfg.n_phi)
    g.set_gradient_scaling_params(cfg.coefficients.tolist(), cfg.powers.tolist())
    # the Python class hands the scaling parameters to the handle at its first compute call;
    # the device-output steps below call the C ABI directly, so they are handed over here
    g._push_params()
    g.set_kernel(kernel)
    return g


def cpu_sample(cfg):
    """The CPU baseline's fixed sample: CPU_SAMPLE_BUBBLES radiating bubbles spread evenly over
    nucleation order (the interior rows are sorted by nucleation time), every collider present
    (an exact partial sum of the first k-hat's spectrum), and the factor from its PTE to a full step."""
    n_s = min(CPU_SAMPLE_BUBBLES, cfg.n)
    sel = np.linspace(0, cfg.n - 1, n_s).round().astype(np.int64)
    pte_one = cfg.n_cos * cfg.n_phi * cfg.n_t  # one radiating bubble, one k-hat
    return sel, pte_one, cfg.pte / (n_s * pte_one)


def _oracle_run(cfg, sel, threads):
    from oracle import oracle as O
    R = O.rotation_for_khat(cfg.khat[0])
    ri, re = O.rotate(R, cfg.interior), O.rotate(R, cfg.exterior)
    t0 = time.perf_counter()
    O.compute_c_integral(ri, re, cfg.n_cos, cfg.n_phi, cfg.w, cfg.t_end, cfg.n_t, t_begin=cfg.t_begin,
                         coefficients=cfg.coefficients, powers=cfg.powers, selected=sel, threads=threads)
    return time.perf_counter() - t0


def cpu_baseline(cfg, threads: int | None = None):
    """The oracle (CPU f64 restatement, reference loop structure) on the fixed sample of cpu_sample."""
    from oracle import oracle as O
    threads = threads or O.max_threads()
    sel, pte_one, factor = cpu_sample(cfg)
    dt = _oracle_run(cfg, sel, threads)
    return {"value": sel.size * pte_one / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{sel.size} radiating bubbles spread over nucleation order x 1 k-hat of {cfg.name} "
                      f"(all {cfg.interior.shape[0] + cfg.exterior.shape[0]} colliders), {dt:.1f} s",
            "extrapolation_to_full_step": factor, "seconds": dt}


def compare_fp64(cfg, kernel, res, lib, L):
    """FP64 kernels on stated subsets of the same workload (directions are independent, and a
    subset of radiating bubbles with every collider present is an exact partial sum), plus the
    error of this run's spectrum against fp64_factored on the same directions."""
    from gw_fopt_b200 import workloads as W
    out = {}
    sub = min(16, cfg.khat.shape[0])
    g = make_flow(cfg, "fp64_factored")
    ref = g.compute_c_integral_khat(cfg.w, cfg.khat[:sub], t_begin=cfg.t_begin, t_end=cfg.t_end, n_t=cfg.n_t)
    t = g.last_timings()
    pte = sub * cfg.n * cfg.n_cos * cfg.n_phi * cfg.n_t
    out["fp64_factored"] = {"value": pte / (t["total_ms"] * 1e-3), "unit": UNIT, "sample": f"{sub} of {cfg.khat.shape[0]} k-hat"}
    if kernel.startswith("mixed"):
        got = res[:sub]
        d = (got - ref).reshape(-1, ref.shape[-1])
        r = ref.reshape(-1, ref.shape[-1])
        per_w = np.linalg.norm(d, axis=0) / np.linalg.norm(r, axis=0)
        out["mixed_error_vs_fp64"] = {"global": float(np.linalg.norm(d) / np.linalg.norm(r)),
                                      "peak_scaled": float(np.linalg.norm(d, axis=0).max() / np.linalg.norm(r, axis=0).max()),
                                      "per_w_median": float(np.median(per_w)), "per_w_max": float(per_w.max()),
                                      "sample": f"{sub} k-hat"}
    gd = make_flow(cfg, "fp64_direct")
    n_rad = min(cfg.n, 128)
    sel = np.arange(n_rad)
    gd.compute_c_integral_khat(cfg.w, cfg.khat[:1], t_begin=cfg.t_begin, t_end=cfg.t_end, n_t=cfg.n_t, selected_bubbles=sel)
    t = gd.last_timings()
    pte = n_rad * cfg.n_cos * cfg.n_phi * cfg.n_t
    out["fp64_direct"] = {"value": pte / (t["total_ms"] * 1e-3), "unit": UNIT,
                          "sample": f"{n_rad} radiating bubbles (all colliders) x 1 k-hat"}
    return out


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def run_b200(args):
    import torch
    from gw_fopt_b200 import _lib as L
    from gw_fopt_b200 import many_bubbles as mb
    from gw_fopt_b200 import workloads as W
    from gw_fopt_b200.sharding import khat_shard, max_over_ranks

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        pg = dist

    cfg = W.config(args.config)
    K = cfg.khat.shape[0]
    cfg.khat = khat_shard(K, rank, world)
    g = make_flow(cfg, args.kernel)
    if not args.no_autotune:
        g.set_autotune(True)  # the first warm-up step measures the launch shape
    lib = L.lib()
    S, Wn = cfg.coefficients.shape[0], cfg.w.size
    # a created stream: handle 0 (torch's legacy default stream) would mean "library's own stream"
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    assert stream.cuda_stream != 0
    L.check(lib.bgwx_generalized_bulk_flow_set_stream(g._h, C.c_void_p(stream.cuda_stream)))
    out_dev = torch.empty((K, 2, S, Wn), dtype=torch.complex128, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    w = np.ascontiguousarray(cfg.w)
    kh = np.ascontiguousarray(cfg.khat)
    cut = mb._UNIT_CUTOFF

    def step():
        L.check(lib.bgwx_generalized_bulk_flow_compute_c_integral_khat_device(
            g._h, L.ptr(w), Wn, True, cfg.t_begin, cfg.t_end, cfg.n_t, L.ptr(kh), K, None, 0, cut,
            C.c_void_p(out_dev.data_ptr()), out_dev.numel()))
        flush.zero_()  # L2 flush between timed iterations

    def barrier():
        if pg is not None:
            pg.barrier()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    barrier()
    torch.cuda.synchronize()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    evs[0].record(stream)
    for i in range(args.steps):
        step()
        evs[i + 1].record(stream)
    torch.cuda.synchronize()
    barrier()
    clocks = sampler.stop()
    e0, e1 = evs[0], evs[-1]
    step_ms = [evs[i].elapsed_time(evs[i + 1]) for i in range(args.steps)]
    launch_shape = g.last_launch_shape()
    gemm_stages = g.last_gemm_stages()
    ms = max_over_ranks(e0.elapsed_time(e1), device="cuda")
    ms_step = ms / args.steps
    pte_total = cfg.pte * world
    value = pte_total / (ms_step * 1e-3)

    # one synchronous call on the library's own stream for per-kernel timings
    L.check(lib.bgwx_generalized_bulk_flow_set_stream(g._h, None))
    res = g.compute_c_integral_khat(cfg.w, cfg.khat, t_begin=cfg.t_begin, t_end=cfg.t_end, n_t=cfg.n_t)
    tm = g.last_timings()
    # the timed device-output steps computed the same spectrum (same kernels and launch shape)
    assert np.array_equal(out_dev.cpu().numpy(), res), "device-output steps differ from the public call"
    launches_per_step = int(tm["launches"])

    # end to end through the public API with host buffers
    e2e = None
    if not args.no_e2e:
        L.check(lib.bgwx_generalized_bulk_flow_set_stream(g._h, C.c_void_p(stream.cuda_stream)))
        h2d = d2h = 0.0
        barrier()
        torch.cuda.synchronize()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        for _ in range(args.steps):
            L.check(lib.bgwx_generalized_bulk_flow_drop_resident_inputs(g._h))
            host_out = g.compute_c_integral_khat(cfg.w, cfg.khat, t_begin=cfg.t_begin, t_end=cfg.t_end,
                                                 n_t=cfg.n_t)
            t2 = g.last_timings()
            h2d, d2h = t2["h2d_bytes"], t2["d2h_bytes"]
        f1.record(stream)
        torch.cuda.synchronize()
        barrier()
        ms_e = max_over_ranks(f0.elapsed_time(f1), device="cuda")
        e2e = {"value": pte_total / (ms_e / args.steps * 1e-3), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "ms_per_step": ms_e / args.steps}
        assert np.array_equal(host_out, res)

    # roofline.  Counted work (declared convention) F = 6 PTE + 8 Phi + 20 Phi_t of the whole
    # spectrum stage, over the spectrum kernels' time; the dominant kernel's own executed
    # work (the time-phase GEMM: 2 * (2W) * n_t * columns * n_cos flops per frame) is reported
    # beside it against the same FMA peak.
    p64, p32, psfu = C.c_double(), C.c_double(), C.c_double()
    L.check(lib.bgwx_measure_compute_peaks(C.byref(p64), C.byref(p32), C.byref(psfu)))
    peaks = {"fp64_tflops": p64.value / 1e12, "fp32_tflops": p32.value / 1e12, "sfu_tops": psfu.value / 1e12}
    spec_s = tm["spectrum_ms"] * 1e-3
    counted = cfg.counted_flops / spec_s / 1e12 if spec_s > 0 else None
    # DRAM traffic of the dominant kernel per k-hat frame: from the committed ncu capture of the
    # same kernel on this workload's geometry (profiles/traffic.json says how it was scaled)
    traffic = traffic_note = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        try:
            tj = json.load(open(tpath))
            traffic = tj.get(f"config{args.config}:{args.kernel}")
            traffic_note = tj.get("_note")
        except Exception:
            traffic = None
    # the time-phase product: 2 (2W) n_t columns n_cos per frame for one real product
    gemm_flops = 2.0 * (2 * Wn) * cfg.n_t * (cfg.n * 2 * S) * cfg.n_cos * K
    stage = {"work": "counted F = 6 PTE + 8 Phi + 20 Phi_t per step", "achieved_counted_tflops": counted,
             "spectrum_ms": tm["spectrum_ms"], "masks_ms": tm["masks_ms"], "beta_ms": tm["beta_ms"],
             "gemm_ms": tm["gemm_ms"]}
    if args.kernel == "mixed" and tm["gemm_ms"] > 0:
        # k_gemm_i8: ten int8 digit-pair products per real product on the tensor cores (exact int32
        # accumulation); peak = dense int8, twice the measured bf16 dense rate on B200 (sustained:
        # the kernel runs inside a long step)
        mp = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        peak = 2.0 * mp["bf16_tflops_sustained"]
        achieved = 10.0 * gemm_flops / (tm["gemm_ms"] * 1e-3) / 1e12
        # one launch covers frames_per_launch frames: their beta digits stream once, the time-phase
        # digits are shared by the launch's frames
        fpl = int(launch_shape[0]) if launch_shape and launch_shape[0] else 1
        beta_bytes = 4.0 * cfg.n_cos * (cfg.n * 2 * S) * cfg.n_t
        atab_bytes = 4.0 * cfg.n_cos * (2 * Wn) * cfg.n_t
        roofline = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TOP/s (int8)",
                    "frac": achieved / peak, "traffic": traffic * fpl if traffic else None,
                    "traffic_unit": "DRAM bytes per k_gemm_i8 launch (per-frame ncu figure x frames per launch)",
                    "algorithmic_bytes_per_launch": fpl * beta_bytes + atab_bytes,
                    "traffic_source": traffic_note, "kernel": "k_gemm_i8",
                    "work": "10 digit-pair products x 2 x (2 n_w) x n_t x columns x n_cos int8 ops per frame",
                    "algorithmic_tflops": gemm_flops / (tm["gemm_ms"] * 1e-3) / 1e12,
                    "peak_source": "of measured: 2 x MEASURED_PEAKS.json bf16_tflops_sustained (dense int8)",
                    "spectrum_stage": stage, "peaks": peaks}
        # k_beta against HBM: it writes the four digit bytes of every beta value and reads every
        # patch's collision delay once (plus one FP64 scale per row); per frame
        beta_alg = 4.0 * cfg.n_cos * (cfg.n * 2 * S) * cfg.n_t + 8.0 * cfg.n * cfg.n_cos * cfg.n_phi \
            + 8.0 * cfg.n * cfg.n_cos
        btraffic = None
        try:
            btraffic = json.load(open(tpath)).get(f"config{args.config}:{args.kernel}:k_beta")
        except Exception:
            pass
        if tm["beta_ms"] > 0:
            b_ach = beta_alg * K / (tm["beta_ms"] * 1e-3) / 1e9
            beta_roof = {"bound": "hbm", "achieved": b_ach, "peak": mp["hbm_gbs"], "unit": "GB/s",
                         "frac": b_ach / mp["hbm_gbs"], "kernel": "k_beta",
                         "traffic": btraffic * fpl if btraffic else None,
                         "traffic_unit": "DRAM bytes per k_beta launch (per-frame ncu figure x frames per launch)",
                         "algorithmic_bytes_per_launch": fpl * beta_alg,
                         "work": "4 digit bytes per beta value written + 8 bytes per patch delay read + 8 bytes "
                                 "per row scale, per frame",
                         "peak_source": "of measured: MEASURED_PEAKS.json hbm_gbs",
                         "note": "issue-bound (about 60% issue active under ncu), not limited by HBM"}
            # the dominant kernel by device time heads the line; the other is kept beside it
            if tm["beta_ms"] > tm["gemm_ms"]:
                beta_roof.update({"spectrum_stage": stage, "peaks": peaks})
                gemm_roof = {k: v for k, v in roofline.items() if k not in ("spectrum_stage", "peaks")}
                roofline = dict(beta_roof, second_kernel=gemm_roof)
            else:
                roofline["second_kernel"] = beta_roof
    else:
        peak = (p32.value if args.kernel == "mixed_simt" else p64.value) / 1e12
        bound = "fp32" if args.kernel == "mixed_simt" else "fp64"
        if args.kernel != "fp64_direct" and tm["gemm_ms"] > 0:
            achieved = gemm_flops / (tm["gemm_ms"] * 1e-3) / 1e12
            kname = "k_gemm"
            work = "2 x (2 n_w) x n_t x columns x n_cos flops per frame"
        else:
            achieved = counted
            kname = "k_spec_direct + k_reduce"
            work = "counted F = 6 PTE + 8 Phi + 20 Phi_t per step"
        roofline = {"bound": bound, "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                    "frac": (achieved / peak) if achieved else None,
                    "traffic": traffic * (int(launch_shape[0]) if launch_shape and launch_shape[0] else 1)
                    if traffic else None, "traffic_unit": "DRAM bytes per launch",
                    "traffic_source": traffic_note, "kernel": kname,
                    "work": work, "peak_source": "of measured: bgwx_measure_compute_peaks (FMA chains on this GPU); "
                                                 "MEASURED_PEAKS.json holds HBM/bf16 only",
                    "spectrum_stage": stage, "peaks": peaks}

    compare = None
    if not args.no_compare and world == 1:
        compare = compare_fp64(cfg, args.kernel, res, lib, L)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "step_ms": [round(x, 2) for x in step_ms],
            "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if not args.kernel.startswith("mixed") else ("int8x4+f64" if args.kernel == "mixed" else "f32+f64"), "data": "synthetic",
            "config": {"workload": cfg.name, "bubbles": int(cfg.n), "colliders": int(cfg.n + cfg.exterior.shape[0]),
                       "n_cos": cfg.n_cos, "n_phi": cfg.n_phi, "n_t": cfg.n_t, "n_w": int(Wn),
                       "n_khat_per_gpu": int(K), "kernel": args.kernel, "pte_per_step": pte_total,
                       "l2": "flushed between steps (256 MiB write)", "parallelism": f"khat-shard x{world}",
                       "tables": "time-phase digits rebuilt in every call (inside the timed steps)",
                       "launch_shape": dict(zip(("frames_per_launch", "row_parts"), launch_shape),
                                            gemm_stages=gemm_stages, mask_chunking=g.last_mask_chunking(),
                                            autotuned=not args.no_autotune)},
            "roofline": roofline, "e2e": e2e, "gpu_launches": launches_per_step * args.steps, "clocks": clocks,
            "compare": compare}
    if compare:
        for k in ("fp64_factored", "fp64_direct"):
            if k in compare:
                compare[f"{args.kernel}_over_{k}"] = value / compare[k]["value"]
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(cfg)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()


def run_reference(args):
    """The reference's CPU path (the oracle restatement, all host threads) on the config's workload:
    each step runs a slice of the fixed CPU sample (cpu_sample), consecutive steps rotating through
    it, so that the timed steps cover every sampled bubble at least once; value = sampled PTE / time."""
    rank, world, local = dist_env()
    if rank != 0:
        return
    from gw_fopt_b200 import workloads as W
    from oracle import oracle as O
    cfg = W.config(args.config if args.config in (1, 2, 3) else 3)
    threads = O.max_threads()
    sel, pte_one, factor = cpu_sample(cfg)
    per = max(1, math.ceil(sel.size / max(args.steps, 1)))  # bubbles per step
    slices = [np.take(sel, np.arange(q * per, (q + 1) * per), mode="wrap") for q in range(args.steps + args.warmup)]
    for q in range(args.warmup):
        _oracle_run(cfg, slices[args.steps + q], threads)
    dt = 0.0
    for q in range(args.steps):
        dt += _oracle_run(cfg, slices[q], threads)
    v = args.steps * per * pte_one / dt
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": cfg.name, "bubbles": int(cfg.n), "n_cos": cfg.n_cos, "n_phi": cfg.n_phi,
                       "n_t": cfg.n_t, "n_w": int(cfg.w.size), "n_khat": int(cfg.khat.shape[0]),
                       "sample_radiating_bubbles": int(sel.size), "sample_bubbles_per_step": per, "sample_khat": 1,
                       "extrapolation_to_full_step": factor},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{sel.size} radiating bubbles spread over nucleation order x 1 k-hat, "
                                       f"{per} per step in rotation (all colliders present)"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_once(args):
    """One spectrum call of a sub-workload (for profiler captures), printing its device timings."""
    from gw_fopt_b200 import workloads as W
    if args.config == 4:
        return run_ensemble_bench(args, once=True)
    if args.config == 5:
        return run_adjoint_bench(args, once=True)
    c = W.config(args.config, k_subset=args.khat or None)
    g = make_flow(c, args.kernel)
    sel = np.arange(args.bubbles) if args.bubbles else None
    n_t = args.n_t or c.n_t
    out = g.compute_c_integral_khat(c.w, c.khat, t_begin=c.t_begin, t_end=c.t_end, n_t=n_t, selected_bubbles=sel)
    t = g.last_timings()
    n_rad = args.bubbles or c.n
    pte = c.khat.shape[0] * n_rad * c.n_cos * c.n_phi * n_t
    print(json.dumps({"config": c.name, "kernel": args.kernel, "khat": int(c.khat.shape[0]), "radiating": int(n_rad),
                      "n_t": n_t, "masks_ms": t["masks_ms"], "beta_ms": t["beta_ms"], "gemm_ms": t["gemm_ms"],
                      "spectrum_ms": t["spectrum_ms"], "total_ms": t["total_ms"], "fallbacks": t["fallbacks"],
                      "launches": t["launches"], "pte_per_s": pte / (t["total_ms"] * 1e-3),
                      "checksum": float(np.abs(out).sum())}), flush=True)


def run_ensemble_bench(args, once=False):
    """Config 4: one step = the spectra of every realization (first --realizations) along every
    k-hat (first --khat, default all 64) in one batched call through the public API."""
    from gw_fopt_b200 import workloads as W
    from gw_fopt_b200.ensemble import BulkFlowEnsemble
    c = W.ensemble_config(k_subset=args.khat or None)
    c.realizations = c.realizations[:args.realizations]

    def make(kernel, reals):
        e = BulkFlowEnsemble(reals, validate=False)
        e.set_resolution(c.n_cos, c.n_phi)
        e.set_gradient_scaling_params(c.coefficients.tolist(), c.powers.tolist())
        e.set_kernel(kernel)
        return e

    ens = make(args.kernel, c.realizations)
    pte = c.khat.shape[0] * sum(r[0].shape[0] for r in c.realizations) * c.n_cos * c.n_phi * c.n_t
    run = lambda: ens.compute_c_integral_khat(c.w, c.khat, t_begin=c.t_begin, t_end=c.t_end, n_t=c.n_t)
    if once:
        run()
        t = ens.last_timings()
        print(json.dumps({"config": c.name, "kernel": args.kernel, "total_ms": t["total_ms"],
                          "masks_ms": t["masks_ms"], "beta_ms": t["beta_ms"], "gemm_ms": t["gemm_ms"],
                          "launches": t["launches"], "pte_per_s": pte / (t["total_ms"] * 1e-3)}), flush=True)
        return
    for _ in range(args.warmup):
        out = run()
    dev_ms, wall_ms = [], []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        out = run()
        wall_ms.append((time.perf_counter() - t0) * 1e3)
        dev_ms.append(ens.last_timings()["total_ms"])
    t = ens.last_timings()
    line = {"metric": METRIC, "value": pte / (np.mean(dev_ms) * 1e-3), "unit": UNIT, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": float(np.mean(dev_ms)),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "int8x4+f64" if args.kernel == "mixed" else args.kernel, "data": "synthetic",
            "config": {"workload": c.name, "realizations": len(c.realizations), "n_khat": int(c.khat.shape[0]),
                       "bubbles": int(sum(r[0].shape[0] for r in c.realizations)), "kernel": args.kernel,
                       "pte_per_step": pte,
                       "stages_ms": {k: t[k] for k in ("masks_ms", "beta_ms", "gemm_ms")}},
            "e2e": {"value": pte / (np.mean(wall_ms) * 1e-3), "unit": UNIT, "h2d_bytes_per_step": int(t["h2d_bytes"]),
                    "d2h_bytes_per_step": int(t["d2h_bytes"]), "ms_per_step": float(np.mean(wall_ms)),
                    "timing": "host wall clock around the synchronous public call"},
            "gpu_launches": int(t["launches"]) * args.steps}
    if not args.no_compare and args.compare_realizations > 0:
        n = min(args.compare_realizations, len(c.realizations))
        ref = make("fp64_factored", c.realizations[:n]).compute_c_integral_khat(
            c.w, c.khat, t_begin=c.t_begin, t_end=c.t_end, n_t=c.n_t)
        per_w = []
        for q in range(n):
            d = (out[q] - ref[q]).reshape(-1, c.w.size)
            r = ref[q].reshape(-1, c.w.size)
            per_w.append(float((np.linalg.norm(d, axis=0) / np.linalg.norm(r, axis=0)).max()))
        line["compare"] = {"mixed_error_vs_fp64": {"per_w_max_over_realizations": max(per_w),
                                                   "sample": f"first {n} realizations"}}
    print(json.dumps(line), flush=True)


def run_adjoint_bench(args, once=False):
    """Config 5: one step = forward and backward of the fit loss (mean squared log residual of
    |C_+|^2 + |C_x|^2 against a target made at xi = 2 with perturbed coefficients) through the
    torch.autograd path, and one Adam step on (xi, alpha, gamma, delta) and the nucleation events."""
    import torch
    from gw_fopt_b200 import workloads as W
    from gw_fopt_b200.autograd import BulkFlowSpectrum, SurfaceTensionFit, log_power_residual
    c = W.config(5, k_subset=args.khat or None)
    model = BulkFlowSpectrum(n_cos=c.n_cos, n_phi=c.n_phi, w=c.w, khat=c.khat, t_end=c.t_end, n_t=c.n_t,
                             t_begin=c.t_begin, box=1.0, kernel=args.kernel)
    x = torch.tensor(c.interior, dtype=torch.float64, requires_grad=True)
    with torch.no_grad():
        co_t, po_t = SurfaceTensionFit(xi=2.0, alpha=1.1, gamma=0.4, delta=-0.1)()
        target = (model(co_t, po_t, x) ** 2).sum(-1).sum(1)
    fit = SurfaceTensionFit(xi=1.5, alpha=1.0, gamma=0.0, delta=0.0)
    opt = torch.optim.Adam(list(fit.parameters()) + [x], lr=1e-3)
    pte = c.khat.shape[0] * c.n * c.n_cos * c.n_phi * c.n_t

    def step():
        opt.zero_grad()
        co, po = fit()
        loss = log_power_residual(model(co, po, x), target)
        loss.backward()
        opt.step()
        return float(loss), model.last_forward_ms, model.last_backward_ms

    if once:
        loss, f, b = step()
        print(json.dumps({"config": c.name, "loss": loss, "forward_ms": f, "backward_ms": b}), flush=True)
        return
    for _ in range(args.warmup):
        step()
    fwd, bwd, wall = [], [], []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        loss, f, b = step()
        wall.append((time.perf_counter() - t0) * 1e3)
        fwd.append(f)
        bwd.append(b)
    ms = float(np.mean(fwd) + np.mean(bwd))
    line = {"metric": METRIC, "value": pte / (ms * 1e-3), "unit": UNIT + " (forward + backward)", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": args.kernel + " forward, f64 adjoint",
            "data": "synthetic",
            "config": {"workload": c.name, "bubbles": int(c.n), "n_khat": int(c.khat.shape[0]),
                       "forward_ms": float(np.mean(fwd)), "backward_ms": float(np.mean(bwd)), "loss": loss},
            "e2e": {"value": pte / (np.mean(wall) * 1e-3), "unit": UNIT, "ms_per_step": float(np.mean(wall)),
                    "timing": "host wall clock of the whole fit step"}}
    if not args.no_compare and args.kernel != "fp64_factored":
        # the forward spectrum of the fitted parameters against the FP64 factored kernel, per w
        ref_model = BulkFlowSpectrum(n_cos=c.n_cos, n_phi=c.n_phi, w=c.w, khat=c.khat, t_end=c.t_end, n_t=c.n_t,
                                     t_begin=c.t_begin, box=1.0, kernel="fp64_factored")
        with torch.no_grad():
            co, po = fit()
            got = model(co, po, x).numpy()
            ref = ref_model(co, po, x).numpy()
        d = (got - ref).reshape(-1, c.w.size, 2) if got.shape[-1] == 2 else (got - ref).reshape(-1, c.w.size)
        r = ref.reshape(d.shape)
        ax = tuple(q for q in range(d.ndim) if q != 1)
        per_w = np.sqrt((d ** 2).sum(axis=ax)) / np.sqrt((r ** 2).sum(axis=ax))
        line["compare"] = {"mixed_error_vs_fp64": {"per_w_max": float(per_w.max()),
                                                   "global": float(np.linalg.norm(d) / np.linalg.norm(r)),
                                                   "sample": "all k-hat, the fit step's parameters"}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.once:
        run_once(args)
    elif args.config == 4:
        run_ensemble_bench(args)
    elif args.config == 5:
        run_adjoint_bench(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
