#!/usr/bin/env python
"""Benchmark of the generalized bulk-flow many-bubble GW spectrum on B200.

Metric: patch-time evaluations per second, PTE = K * N * n_cos * n_phi * n_t
for one complete spectrum (all k-hat directions, all bubbles, all t, all w),
masks included.  One step = one complete spectrum of the named synthetic
workload (seeded; no dataset exists for this path).

    python bench.py [--gpus N --steps K --warmup W] [--config 3] [--kernel mixed]
    python bench.py --impl reference ...   # the CPU restatement of the reference

value: device-resident inputs, result left in HBM (CUDA events on the
       launching stream, L2 flushed between steps by a 256 MiB write).
e2e:   the public Python API with host buffers, every input copied to the
       device and the result copied back each step.
Multi-GPU (torchrun): each rank computes its own k-hat directions of a
K*N-direction Fibonacci sphere (weak scaling, no data-path collective);
timing is the max over ranks.
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


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--config", type=int, default=3)
    ap.add_argument("--kernel", default="mixed", choices=["fp64_direct", "fp64_factored", "mixed", "mixed_simt"])
    ap.add_argument("--no-compare", action="store_true", help="skip the FP64 comparison measurements")
    ap.add_argument("--cpu-seconds", type=float, default=10.0, help="CPU-baseline sample budget")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="automatic launch shape instead of the measured one")
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
    g.set_kernel(kernel)
    return g


def cpu_baseline(cfg, seconds: float, threads: int | None = None):
    """The oracle (CPU f64 restatement, reference loop structure) on a bounded sample:
    the first k-hat direction and as many radiating bubbles as fit in ~`seconds`."""
    from oracle import oracle as O
    threads = threads or O.max_threads()
    R = O.rotation_for_khat(cfg.khat[0])
    ri, re = O.rotate(R, cfg.interior), O.rotate(R, cfg.exterior)

    def run(sel):
        t0 = time.perf_counter()
        O.compute_c_integral(ri, re, cfg.n_cos, cfg.n_phi, cfg.w, cfg.t_end, cfg.n_t, t_begin=cfg.t_begin,
                             coefficients=cfg.coefficients, powers=cfg.powers, selected=sel, threads=threads)
        return time.perf_counter() - t0

    order = np.random.default_rng(0).permutation(cfg.n)
    t1 = run(order[:1])
    n_sel = int(max(1, min(cfg.n, seconds / max(t1, 1e-3))))
    sel = order[:n_sel]
    dt = run(sel)
    pte = n_sel * cfg.n_cos * cfg.n_phi * cfg.n_t
    return {"value": pte / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{n_sel} radiating bubbles x 1 k-hat of {cfg.name} (all {cfg.interior.shape[0] + cfg.exterior.shape[0]}"
                      f" colliders), {dt:.1f} s", "seconds": dt}


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
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clocks = sampler.stop()
    launch_shape = g.last_launch_shape()
    ms = max_over_ranks(e0.elapsed_time(e1), device="cuda")
    ms_step = ms / args.steps
    pte_total = cfg.pte * world
    value = pte_total / (ms_step * 1e-3)

    # one synchronous call on the library's own stream for per-kernel timings
    L.check(lib.bgwx_generalized_bulk_flow_set_stream(g._h, None))
    res = g.compute_c_integral_khat(cfg.w, cfg.khat, t_begin=cfg.t_begin, t_end=cfg.t_end, n_t=cfg.n_t)
    tm = g.last_timings()
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
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        try:
            traffic = json.load(open(tpath)).get(f"config{args.config}:{args.kernel}")
        except Exception:
            traffic = None
    # the time-phase product: 2 (2W) n_t columns n_cos flops per frame
    gemm_flops = 2.0 * (2 * Wn) * cfg.n_t * (cfg.n * 2 * S) * cfg.n_cos * K
    stage = {"work": "counted F = 6 PTE + 8 Phi + 20 Phi_t per step", "achieved_counted_tflops": counted,
             "spectrum_ms": tm["spectrum_ms"], "masks_ms": tm["masks_ms"], "beta_ms": tm["beta_ms"],
             "gemm_ms": tm["gemm_ms"]}
    if args.kernel == "mixed" and tm["gemm_ms"] > 0:
        # k_gemm_tc: three TF32 products per FP32 product on the tensor cores; peak = TF32 dense,
        # half of the measured bf16 dense figure (sustained: the kernel runs inside a long step)
        mp = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        peak = mp["bf16_tflops_sustained"] / 2.0
        achieved = 3.0 * gemm_flops / (tm["gemm_ms"] * 1e-3) / 1e12
        roofline = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                    "frac": achieved / peak, "traffic": traffic,
                    "traffic_unit": "DRAM bytes per k-hat frame (ncu, profiles/traffic.json)", "kernel": "k_gemm_tc",
                    "work": "3 x 2 x (2 n_w) x n_t x columns x n_cos TF32 flops per frame (FP32 split in three)",
                    "peak_source": "of measured: MEASURED_PEAKS.json bf16_tflops_sustained / 2 (TF32 dense)",
                    "spectrum_stage": stage, "peaks": peaks}
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
                    "frac": (achieved / peak) if achieved else None, "traffic": traffic, "kernel": kname,
                    "work": work, "peak_source": "of measured: bgwx_measure_compute_peaks (FMA chains on this GPU); "
                                                 "MEASURED_PEAKS.json holds HBM/bf16 only",
                    "spectrum_stage": stage, "peaks": peaks}

    compare = None
    if not args.no_compare and world == 1:
        compare = compare_fp64(cfg, args.kernel, res, lib, L)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if not args.kernel.startswith("mixed") else ("tf32x3+f64" if args.kernel == "mixed" else "f32+f64"), "data": "synthetic",
            "config": {"workload": cfg.name, "bubbles": int(cfg.n), "colliders": int(cfg.n + cfg.exterior.shape[0]),
                       "n_cos": cfg.n_cos, "n_phi": cfg.n_phi, "n_t": cfg.n_t, "n_w": int(Wn),
                       "n_khat_per_gpu": int(K), "kernel": args.kernel, "pte_per_step": pte_total,
                       "l2": "flushed between steps (256 MiB write)", "parallelism": f"khat-shard x{world}",
                       "launch_shape": dict(zip(("frames_per_launch", "row_parts"), launch_shape),
                                            autotuned=not args.no_autotune)},
            "roofline": roofline, "e2e": e2e, "gpu_launches": launches_per_step * args.steps, "clocks": clocks,
            "compare": compare}
    if compare:
        for k in ("fp64_factored", "fp64_direct"):
            if k in compare:
                compare[f"{args.kernel}_over_{k}"] = value / compare[k]["value"]
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(cfg, args.cpu_seconds)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()


def run_reference(args):
    rank, world, local = dist_env()
    if rank != 0:
        return
    from gw_fopt_b200 import workloads as W
    from oracle import oracle as O
    cfg = W.config(args.config)
    threads = O.max_threads()
    per_step = max(2.0, 40.0 / max(args.steps + args.warmup, 1))
    base = cpu_baseline(cfg, per_step, threads)
    n_sel = int(base["sample"].split()[0])
    R = O.rotation_for_khat(cfg.khat[0])
    ri, re = O.rotate(R, cfg.interior), O.rotate(R, cfg.exterior)
    sel = np.random.default_rng(0).permutation(cfg.n)[:n_sel]

    def step():
        O.compute_c_integral(ri, re, cfg.n_cos, cfg.n_phi, cfg.w, cfg.t_end, cfg.n_t, t_begin=cfg.t_begin,
                             coefficients=cfg.coefficients, powers=cfg.powers, selected=sel, threads=threads)

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = (time.perf_counter() - t0) / args.steps
    pte = n_sel * cfg.n_cos * cfg.n_phi * cfg.n_t
    v = pte / dt
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": cfg.name, "bubbles": int(cfg.n), "n_cos": cfg.n_cos, "n_phi": cfg.n_phi,
                       "n_t": cfg.n_t, "n_w": int(cfg.w.size), "n_khat": int(cfg.khat.shape[0]),
                       "sample_radiating_bubbles": n_sel, "sample_khat": 1},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{n_sel} radiating bubbles x 1 k-hat per step (all colliders present)"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
