"""Benchmark: stability-boundary points per second on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload ("sweep"): one milling setup -- 4 flutes, D 10 mm, helix 30 deg, 10 um runout,
Ktc 700 / Krc 210 / Kte 20 / Kre 30, 3 modes per axis (fn 600-3000 Hz, k 5e6-5e7 N/m,
zeta 0.01-0.05, seeded) -- swept over 4096 spindle speeds 3000-30000 rpm; each speed is a
10-iteration geometric bisection over [0.05, 15] mm whose trials run 60 revolutions with
40 slices and the reference's steps-per-tooth rule.  A step = the whole 4096-point sweep.

`value`  points/s with the inputs resident on the device: the prepared batch is a
         captured CUDA graph (mcs_plan_execute), timed with CUDA events on the library's
         stream, L2 flushed (a 256 MiB write) between timed steps.
`e2e`    the same through the public blocking call mcs_solve from page-locked host
         buffers: host preparation, H2D copies, the solve and the D2H of results per step.
Multi-GPU (torchrun): every rank solves its own seeded 4096-point sweep (weak scaling, no
collective on the data path); the time is the max over ranks.

--impl reference: the reference's CPU path on the host cores.  The reference is
JavaScript and no JS runtime exists on these machines, so this arm times the C++ FP64
restatement of it (oracle/) with one thread per core on a bounded sample of the sweep.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "machinig-sim_b200"))
sys.path.insert(0, str(ROOT / "oracle"))

WORKLOADS = {
    "sweep": "sweep: 4096 speeds 3000-30000 rpm, 4-flute D10 helix 30, 3+3 modes, 10 um "
             "runout, [0.05,15] x 10, 60 revs, 40 slices",
    "hetero": "hetero: 16384 seeded setups (D 3-20 mm, 2-6 flutes, helix 0-45, runout 0-20 um, "
              "1-3 modes per axis, process damping and size effect), [0.05,15] x 10, 60 revs, "
              "reference slice rule",
}
METRIC = "stability-boundary points/sec on 1 B200: surrogate-guided vs plain GPU vs Node CPU @<=2% depth err"
UNIT = "points/s"
FLOP_ENGAGED = 46.0   # FP32 flop per in-cut slice evaluation (force law, cutting.js:181-207)
FLOP_IDLE = 15.0      # per out-of-cut evaluation of the reference loop (angle, normal, store)
# DRAM bytes per point of one solve, from an ncu capture of a 3072-point sweep (FP32, 8
# buckets): dram__bytes.sum.per_second x gpu__time_duration of each bucket launch, summed,
# 4.63 MB per execution.  A point reads its parameters and writes its result once; the
# trial state lives in registers and shared memory, so the bytes scale with the points.
DRAM_BYTES_PER_POINT = {"sweep": 1508.0}


def env_rank():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def cpu_model() -> str:
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                return ln.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


def run_oracle_sample(wl, n_points: int, threads: int):
    """FP64 oracle over the first n_points of a seeded permutation of the workload."""
    import pyoracle as O
    from mcs import _abi as A

    perm = np.argsort(np.random.default_rng(7).random(wl.n))[:n_points]
    setups = [A.Setup.from_buffer_copy(r.tobytes()) for r in wl.setups]
    modals = [A.Modal.from_buffer_copy(r.tobytes()) for r in wl.modals]
    pts = wl.points[np.sort(perm)]
    P = (A.Point * len(pts)).from_buffer_copy(pts.tobytes())
    t = time.perf_counter()
    O.solve_batch(setups, modals, P, wl.opts, nthreads=threads)
    return len(pts), time.perf_counter() - t


def cpu_baseline(wl, target_s: float = 15.0) -> dict:
    cores = cpu_cores()
    n = min(wl.n, max(16, 2 * cores))
    npts, dt = run_oracle_sample(wl, n, cores)
    if dt < target_s / 3 and npts < wl.n:  # too short to be a stable figure: grow once
        n2 = min(wl.n, int(npts * target_s / max(dt, 1e-3) * 0.5))
        if n2 > npts:
            npts, dt = run_oracle_sample(wl, n2, cores)
    return {"value": npts / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{npts} of the {wl.n} {wl.name} points (seeded), C++ FP64 restatement of "
                      f"stabtd.js/cutting.js, {cores} threads on {cpu_model()}"}


def guided_serve(ctx, torch, stream, flush, device: int, no_cpu: bool) -> dict:
    """Surrogate-guided serving: 65536 seeded hetero queries (30 % of the setups outside the
    training seeds), the trained model's guided plan against the plain plan on the same
    queries, with agreement against the plain GPU bisection and, on a seeded 512-query
    subset, against the FP64 restatement of the reference on the host."""
    from mcs import _abi as A
    from mcs import surrogate as SG
    from mcs import workloads as W

    if not SG.DEFAULT_MODEL.exists():
        return {"unavailable": f"no trained model at {SG.DEFAULT_MODEL.name}"}
    sv = W.serve()
    sur = SG.load(ctx)
    rec = SG.record_of()

    def run(plan):
        plan.execute()  # warm-up (graph upload)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            flush.fill_(7)
        a.record(stream)
        plan.execute()
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b), plan.results()

    from mcs import tune as T

    sv.opts.max_buckets, tuned = T.autotune(ctx, sv.setups, sv.modals, sv.points, sv.opts,
                                            device_name=torch.cuda.get_device_name(device))
    with ClockSampler(device) as clk:
        pp = ctx.plan(sv.setups, sv.modals, sv.points, sv.opts)
        plain_ms, plain = run(pp)
        pp.close()
        gp = ctx.plan(sv.setups, sv.modals, sv.points, sv.opts, surrogate=sur)
        guided_ms, gres = run(gp)
        info = gp.guide_info()
        gp.close()
    sur.close()
    path = info["path"]
    both_open = (gres["open"] == 1) & (plain["open"] == 1)
    rel = np.where(both_open, 0.0, np.abs(gres["alim"] / plain["alim"] - 1))
    out = np.asarray(sv.meta["outside"])
    sub = np.asarray(sv.meta["fp64_subset"])
    # FP64 references on the subset: the GPU FP64 bisection and the host FP64 restatement
    o64 = A.make_opts(precision="fp64")
    for f in ("a_min", "a_max", "iters", "revs", "nonlinear", "honor_runout", "steps_per_tooth",
              "slices", "chatter_idx"):
        setattr(o64, f, getattr(sv.opts, f))
    g64 = ctx.solve(sv.setups, sv.modals, sv.points[sub], o64)

    def within(a, b):
        op = (a["open"] == 1) & (b["open"] == 1)
        return float(np.mean(op | (np.abs(a["alim"] / b["alim"] - 1) <= 0.02)))

    res = {
        "workload": f"serve: {sv.n} seeded hetero (setup, speed) queries, "
                    f"{float(out.mean()):.0%} outside the training seeds",
        "value": sv.n / (guided_ms / 1e3), "unit": UNIT,
        "plain_value": sv.n / (plain_ms / 1e3), "speedup_vs_plain": plain_ms / guided_ms,
        "trials_ratio": float(gres["trials"].sum() / plain["trials"].sum()),
        "paths": {A.PATH_NAMES[k]: float(np.mean(path == k)) for k in range(4)},
        "fallback_rate": float(np.mean(path == A.PATH_FALLBACK)),
        "within_2pct_of_plain": float(np.mean(rel <= 0.02)),
        "within_2pct_of_plain_outside_seeds": float(np.mean(rel[out] <= 0.02)),
        "median_rel_err_vs_plain_guided": float(np.median(rel[path == A.PATH_GUIDED]))
        if np.any(path == A.PATH_GUIDED) else None,
        "fp64_subset": len(sub),
        "within_2pct_of_gpu_fp64": within(gres[sub], g64),
        "plain_within_2pct_of_gpu_fp64": within(plain[sub], g64),
        "schedule": {"max_buckets": int(sv.opts.max_buckets), "tuning_ms": tuned["ms"],
                     "from_cache": bool(tuned["cached"])},
        "model": {"file": SG.DEFAULT_MODEL.name, "epochs": rec.get("epochs"),
                  "train_points": rec.get("train_points"),
                  "val_within_15pct": rec.get("val_within_15pct")},
        "clocks": clk.summary(),
    }
    if not no_cpu:
        import pyoracle as O

        setups = [A.Setup.from_buffer_copy(r.tobytes()) for r in sv.setups]
        modals = [A.Modal.from_buffer_copy(r.tobytes()) for r in sv.modals]
        pts = sv.points[sub]
        P = (A.Point * len(pts)).from_buffer_copy(pts.tobytes())
        r64, _ = O.solve_batch(setups, modals, P, sv.opts, nthreads=cpu_cores())
        res["within_2pct_of_cpu_fp64"] = within(gres[sub], r64)
        res["plain_within_2pct_of_cpu_fp64"] = within(plain[sub], r64)
    return res


def reference_arm(args) -> int:
    rank, world, _ = env_rank()
    if rank != 0:
        return 0
    from mcs import workloads as W

    wl = W.hetero(n=16384) if args.workload == "hetero" else W.sweep()
    cores = cpu_cores()
    n = min(wl.n, max(8, cores))
    for _ in range(args.warmup):
        run_oracle_sample(wl, n, cores)
    tot_p, tot_t = 0, 0.0
    for _ in range(args.steps):
        p, t = run_oracle_sample(wl, n, cores)
        tot_p += p
        tot_t += t
    v = tot_p / tot_t
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot_t / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded)",
        "config": {"workload": WORKLOADS[args.workload],
                   "sample_points_per_step": n},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{n} seeded {wl.name} points per step; the reference is "
                                   f"JavaScript with no JS runtime on this box, so its C++ "
                                   f"FP64 restatement runs, {cores} threads, {cpu_model()}"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def ours(args) -> int:
    import torch

    rank, world, local = env_rank()
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta

        dist.init_process_group("nccl" if torch.cuda.is_available() else "gloo",
                                timeout=timedelta(seconds=120))
    device = local if torch.cuda.is_available() else 0
    torch.cuda.set_device(device)
    import mcs
    from mcs import tune as T
    from mcs import workloads as W

    if args.workload == "hetero":  # 16384 seeded setups per rank (weak scaling)
        wl = W.hetero(n=16384, first_seed=16384 * rank)
    else:
        wl = W.sweep(seed=1 + rank)
    if args.points and args.points < wl.n:  # a smaller case of the same workload (profiling)
        wl = wl.subset(np.linspace(0, wl.n - 1, args.points).round().astype(int))
    if args.serial_trials:
        wl.opts.serial_trials = 1
    ctx = mcs.Context(device)
    stream = torch.cuda.ExternalStream(ctx.stream)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{device}")

    def barrier():
        if dist is not None:
            dist.barrier()

    def maxover(x: float) -> float:
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{device}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def timed(precision: str):
        """Device-resident plan of the sweep: per-step CUDA-event times, results, info."""
        opts = A.make_opts(precision=precision)
        for f in ("a_min", "a_max", "iters", "revs", "nonlinear", "honor_runout",
                  "steps_per_tooth", "slices", "chatter_idx", "serial_trials"):
            setattr(opts, f, getattr(wl.opts, f))
        # schedule (number of shared-memory size classes) from the autotuner, untimed
        if args.max_buckets:
            opts.max_buckets, tuned = args.max_buckets, {"ms": {}, "cached": False}
        else:
            opts.max_buckets, tuned = T.autotune(ctx, wl.setups, wl.modals, wl.points, opts,
                                                 device_name=torch.cuda.get_device_name(device))
        plan = ctx.plan(wl.setups, wl.modals, wl.points, opts)
        info = plan.info()
        info["schedule"] = {"max_buckets": int(opts.max_buckets), "tuning_ms": tuned["ms"],
                            "from_cache": bool(tuned["cached"])}
        for _ in range(args.warmup):
            plan.execute()
        res = plan.results()
        assert np.all((res["status"] == 0) | (res["status"] == 4)), np.unique(res["status"])
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        barrier()
        torch.cuda.synchronize()
        with ClockSampler(device) as clk:
            for i in range(args.steps):
                with torch.cuda.stream(stream):
                    flush.fill_(i & 0xFF)  # write 256 MiB (> 126 MB L2) between timed steps
                starts[i].record(stream)
                plan.execute()
                ends[i].record(stream)
            torch.cuda.synchronize()
        barrier()
        step_ms = [s_.elapsed_time(e_) for s_, e_ in zip(starts, ends)]
        res = plan.results()
        plan.close()
        return step_ms, res, info, clk.summary(), opts

    from mcs import _abi as A

    variants = {}
    for prec in (["fp32", "fp64"] if not args.fp32_only else [args.precision]):
        step_ms, res, info, clocks, opts = timed(prec)
        ms = maxover(float(np.sum(step_ms))) / args.steps
        variants[prec] = {"step_ms": step_ms, "ms": ms, "res": res, "info": info,
                          "clocks": clocks, "opts": opts}
    main = variants[args.precision]
    step_ms, ms, res, info, clocks = (main["step_ms"], main["ms"], main["res"], main["info"],
                                      main["clocks"])
    pts_total = wl.n * world
    value = pts_total / (ms / 1e3)

    # algorithmic work of one step (same inputs every step): the reference loop's
    # evaluations, in cut and out of cut
    evals = float(res["evals"].sum())
    engaged = float(res["engaged"].sum())
    flop = FLOP_ENGAGED * engaged + FLOP_IDLE * (evals - engaged)
    achieved_tflops = flop / (float(np.mean(step_ms)) / 1e3) / 1e12
    sms = torch.cuda.get_device_properties(device).multi_processor_count
    f_mhz = clocks["sm_mhz"] or 1965.0
    peak_tflops = sms * 128 * 2 * f_mhz * 1e6 / 1e12

    # ---- e2e: public blocking API from page-locked host buffers ----
    e2e = None
    def pinned(arr):
        t = torch.empty(arr.nbytes, dtype=torch.uint8, pin_memory=True)
        v = t.numpy().view(arr.dtype)
        v[:] = arr
        return t, v

    if not args.no_e2e:
        keep = []
        hs = [pinned(wl.setups), pinned(wl.modals), pinned(wl.points)]
        keep += hs
        out_t = torch.empty(len(wl.points) * A.RESULT_DTYPE.itemsize, dtype=torch.uint8,
                            pin_memory=True)
        out_v = out_t.numpy().view(A.RESULT_DTYPE)
        import ctypes as C

        L = ctx._L
        args_c = (ctx._h, C.c_void_p(hs[0][1].ctypes.data), len(wl.setups),
                  C.c_void_p(hs[1][1].ctypes.data), len(wl.modals),
                  C.c_void_p(hs[2][1].ctypes.data), len(wl.points), C.byref(main["opts"]),
                  C.c_void_p(out_v.ctypes.data))
        for _ in range(max(1, args.warmup // 2)):
            mcs._lib.check(L.mcs_solve(*args_c))
        e2e_steps = max(2, min(args.steps, 5))
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            mcs._lib.check(L.mcs_solve(*args_c))
        torch.cuda.synchronize()
        e2e_s = maxover(time.perf_counter() - t0) / e2e_steps
        barrier()
        assert np.array_equal(out_v["alim"], res["alim"]), "e2e and plan results differ"
        e2e = {"value": pts_total / e2e_s, "unit": UNIT,
               "h2d_bytes_per_step": int(info["h2d_bytes"]),
               "d2h_bytes_per_step": int(info["d2h_bytes"])}

    line = None
    if rank == 0:
        cpu = cpu_baseline(wl) if world == 1 and not args.no_cpu else None
        guided = (guided_serve(ctx, torch, stream, flush, device, args.no_cpu)
                  if world == 1 and not args.no_guided else None)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if args.precision == "fp32" else "f64",
            "data": "synthetic (seeded sweep; no public dataset exists for this path)",
            "config": {"workload": WORKLOADS[args.workload],
                       "points_per_gpu": wl.n,
                       "variant": f"plain GPU bisection, {args.precision} force law and "
                                  "modal integration, FP64 statistics and bracket",
                       "l2": "flushed between timed steps (256 MiB write)",
                       "kernels_per_step": info["kernels"], "graph": bool(info["graph"]),
                       "blocks": info["blocks"], "smem_per_warp_max": info["smem_per_warp"],
                       "schedule": info["schedule"]},
            "roofline": {"bound": "fp32", "achieved": achieved_tflops, "peak": peak_tflops,
                         "unit": "TFLOP/s", "frac": achieved_tflops / peak_tflops,
                         "traffic": (DRAM_BYTES_PER_POINT[args.workload] * wl.n
                                     if args.workload in DRAM_BYTES_PER_POINT
                                     and args.precision == "fp32" else None),
                         "traffic_unit": "bytes per step, scaled by points from an ncu "
                                         "capture of a 3072-point FP32 sweep",
                         "peak_source": f"derived: {sms} SMs x 128 FP32 lanes x 2 flop x "
                                        f"{f_mhz:.0f} MHz sampled SM clock (no FP32 figure "
                                        "in MEASURED_PEAKS.json)",
                         "work": f"{FLOP_ENGAGED:.0f} flop per in-cut and {FLOP_IDLE:.0f} per "
                                 f"out-of-cut reference evaluation; {evals:.3e} evaluations, "
                                 f"{engaged:.3e} in cut per step"},
            "cpu_baseline": cpu,
            "guided": guided,
            "e2e": e2e,
            "gpu_launches": int(info["kernels"]) * args.steps,
            "clocks": clocks,
            "results": {"open": int(res["open"].sum()), "alim_median": float(np.median(res["alim"]))},
            "variants": {k: {"value": pts_total / (v["ms"] / 1e3), "ms_per_step": v["ms"],
                             "kernels_per_step": v["info"]["kernels"],
                             "sm_mhz": v["clocks"]["sm_mhz"]} for k, v in variants.items()},
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline leg")
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"],
                    help="integration precision of the headline value")
    ap.add_argument("--fp32-only", action="store_true", help="time only the headline precision")
    ap.add_argument("--points", type=int, default=0,
                    help="solve an evenly spaced subset of the workload (profiling case)")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg")
    ap.add_argument("--no-guided", action="store_true",
                    help="skip the surrogate-guided serving leg")
    ap.add_argument("--workload", default="sweep", choices=["sweep", "hetero"],
                    help="sweep (the headline) or the heterogeneous batch")
    ap.add_argument("--max-buckets", type=int, default=0,
                    help="fixed schedule (shared-memory size classes); 0: autotune")
    ap.add_argument("--serial-trials", action="store_true",
                    help="one bisection trial per warp at a time (same results)")
    a = ap.parse_args(argv)
    if a.warmup < 3:
        a.warmup = 3
    if a.impl == "reference":
        return reference_arm(a)
    return ours(a)


if __name__ == "__main__":
    sys.exit(main())
