"""Benchmark: stability-boundary points per second on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Headline workload ("sweep", the plain method batched on the GPU): one milling setup -- 4
flutes, D 10 mm, helix 30 deg, 10 um runout, Ktc 700 / Krc 210 / Kte 20 / Kre 30, 3 modes
per axis (fn 600-3000 Hz, k 5e6-5e7 N/m, zeta 0.01-0.05, seeded) -- swept over 4096 spindle
speeds 3000-30000 rpm; each speed is a 10-iteration geometric bisection over [0.05, 15] mm
whose trials run 60 revolutions with 40 slices and the reference's steps-per-tooth rule.
A step = the whole 4096-point sweep.

`value`  points/s with the inputs resident on the device: the prepared batch is a
         captured CUDA graph (mcs_plan_execute), timed with CUDA events on the library's
         stream, L2 flushed (a 256 MiB write) between timed steps.
`e2e`    the same through the public blocking call mcs_solve from page-locked host
         buffers: host preparation, H2D copies, the solve and the D2H of results per step.
`accuracy`  the critical depths of the timed runs against the reference algorithm in FP64
         on the host (the CPU restatement of stabtd.js/cutting.js) on the workload's seeded
         256-point subset; that same host run is the `cpu_baseline` timing.
`workloads.hetero`  the heterogeneous batch (16384 seeded setups, process damping and size
         effect on, autotuned schedule, captured graph), measured the same way.
`guided`  surrogate-guided serving of 65536 queries against the plain plan, repeated.
`rows`   the playback engines (a batch of CuttingEngines, one dynBudget frame each), the
         chart's composite lobe diagram and the identification's unit-force runs, each
         beside the host restatement of the same runs and checked against it.
Multi-GPU (torchrun): every rank solves its own seeded sweep (weak scaling, no collective
on the data path); the time is the max over ranks.

--impl reference: the reference's CPU path on the host cores.  The reference is
JavaScript and no JS runtime exists on these machines (probed and recorded in the line),
so this arm times the C++ FP64 restatement of it (oracle/) with one thread per core on
seeded, cost-sorted samples of the same workload, a fresh sample every step.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
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
    "small": "small: 64 speeds 5000-20000 rpm, 4-flute D10 helix 30, 1 mode per axis, no "
             "runout, linear, [0.1,10] x 10, 60 revs, 200 steps per tooth, 40 slices",
}
METRIC = "stability-boundary points/sec on 1 B200: surrogate-guided vs plain GPU vs Node CPU @<=2% depth err"
UNIT = "points/s"
FLOP_ENGAGED = 46.0   # flop per in-cut slice evaluation (force law, cutting.js:181-207)
FLOP_IDLE = 15.0      # per out-of-cut evaluation of the reference loop (angle, normal, store)
SMEM_BYTES_ENGAGED = 8.0  # surface-ring load + store per in-cut evaluation (cutting.js:187-194)
# DRAM bytes per point of one solve, from an ncu capture of a 3072-point sweep (FP32, 8
# buckets): dram__bytes.sum.per_second x gpu__time_duration of each bucket launch, summed,
# 4.63 MB per execution.  A point reads its parameters and writes its result once; the
# trial state lives in registers and shared memory, so the bytes scale with the points.
DRAM_BYTES_PER_POINT = {("sweep", "fp32"): 1508.0}


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


def node_probe() -> dict:
    """Whether a JavaScript runtime exists here (the reference's own path needs one)."""
    found = {n: shutil.which(n) for n in ("node", "nodejs", "deno", "bun")}
    have = {k: v for k, v in found.items() if v}
    rec = {"runtimes_found": have or None}
    if not have:
        rec["reference_js"] = ("unavailable on this box: no JavaScript runtime (node, nodejs, "
                               "deno, bun) on PATH")
    else:
        rec["reference_js"] = ("unavailable on this box: a runtime exists but the reference's "
                               "JavaScript sources are not on this machine")
    return rec


def point_cost(wl, idx) -> np.ndarray:
    """Relative cost of each point (steps per trial x teeth x slices), for ordering host
    work largest first: the reference step rule max(48, ceil(T_tooth f_top 24))."""
    pts = wl.points[idx]
    st = wl.setups[pts["setup"]]
    md = wl.modals[pts["modal"]]
    N = st["tool"]["N"].astype(np.float64)
    fx = md["x"]["fn"].max(axis=1)
    fy = np.where(md["ny"] > 0, md["y"]["fn"].max(axis=1), fx)
    ftop = np.maximum(fx, fy)
    S = np.maximum(100.0, pts["S"])
    if wl.opts.steps_per_tooth:
        spt = np.full(len(pts), float(wl.opts.steps_per_tooth))
    else:
        spt = np.maximum(48.0, np.ceil(60.0 / (S * N) * ftop * 24))
    return spt * N * N


def run_oracle(wl, idx, threads: int):
    """The FP64 restatement of the reference over points idx (cost-sorted for the thread
    pool); returns (results in idx order, seconds)."""
    import pyoracle as O
    from mcs import _abi as A

    idx = np.asarray(idx)
    order = np.argsort(-point_cost(wl, idx), kind="stable")
    setups = [A.Setup.from_buffer_copy(r.tobytes()) for r in wl.setups]
    modals = [A.Modal.from_buffer_copy(r.tobytes()) for r in wl.modals]
    pts = wl.points[idx[order]]
    P = (A.Point * len(pts)).from_buffer_copy(pts.tobytes())
    t = time.perf_counter()
    res, _ = O.solve_batch(setups, modals, P, wl.opts, nthreads=threads)
    dt = time.perf_counter() - t
    out = np.empty_like(res)
    out[order] = res
    return out, dt


def fp64_subset(wl) -> np.ndarray:
    """The workload's seeded 256-point subset (the golden fixtures hold the same points);
    a workload of at most 256 points is its own subset."""
    from mcs import workloads as W

    if wl.n <= 256:
        return np.arange(wl.n)
    if "fp64_subset" in wl.meta:
        return np.asarray(wl.meta["fp64_subset"])
    return np.sort(np.argsort(W.uniform(np.arange(wl.n), 7, 0))[:256])


def within(a, b, tol=0.02) -> float:
    both_open = (a["open"] == 1) & (b["open"] == 1)
    rel = np.where(both_open, 0.0, np.abs(a["alim"] / b["alim"] - 1))
    return float(np.mean(rel <= tol))


def cpu_leg(wl) -> tuple[dict, np.ndarray, np.ndarray]:
    """cpu_baseline: the FP64 restatement on all host cores over the seeded 256-point
    subset; its results are also the accuracy reference of the GPU runs."""
    cores = cpu_cores()
    idx = fp64_subset(wl)
    res, dt = run_oracle(wl, idx, cores)
    rec = {"value": len(idx) / dt, "unit": UNIT, "cores": cores, "kind": "port",
           "sample": f"the seeded {len(idx)}-point subset of the {wl.n} {wl.name} points "
                     f"(cost-sorted), C++ FP64 restatement of stabtd.js/cutting.js, {cores} "
                     f"threads on {cpu_model()}, {dt:.1f} s"}
    return rec, idx, res


def pinned(torch, arr):
    t = torch.empty(max(1, arr.nbytes), dtype=torch.uint8, pin_memory=True)
    v = t.numpy()[: arr.nbytes].view(arr.dtype)
    v[:] = arr
    return t, v


def e2e_leg(ctx, torch, wl, opts, info, steps, warmup, maxover, barrier, pts_total, ref):
    """Points/s through the public blocking call mcs_solve from page-locked host buffers."""
    import ctypes as C

    import mcs
    from mcs import _abi as A

    hs = [pinned(torch, wl.setups), pinned(torch, wl.modals), pinned(torch, wl.points)]
    out_t = torch.empty(len(wl.points) * A.RESULT_DTYPE.itemsize, dtype=torch.uint8,
                        pin_memory=True)
    out_v = out_t.numpy().view(A.RESULT_DTYPE)
    L = ctx._L
    args_c = (ctx._h, C.c_void_p(hs[0][1].ctypes.data), len(wl.setups),
              C.c_void_p(hs[1][1].ctypes.data), len(wl.modals),
              C.c_void_p(hs[2][1].ctypes.data), len(wl.points), C.byref(opts),
              C.c_void_p(out_v.ctypes.data))
    for _ in range(max(1, warmup)):
        mcs._lib.check(L.mcs_solve(*args_c))
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        mcs._lib.check(L.mcs_solve(*args_c))
    torch.cuda.synchronize()
    e2e_s = maxover(time.perf_counter() - t0) / steps
    barrier()
    assert out_v.tobytes() == ref.tobytes(), "e2e and plan results differ"
    return {"value": pts_total / e2e_s, "unit": UNIT, "steps": steps,
            "h2d_bytes_per_step": int(info["h2d_bytes"]),
            "d2h_bytes_per_step": int(info["d2h_bytes"])}


def roofline(res, step_ms, precision, peaks, clocks, workload, n_points) -> dict:
    """The solve kernel's work against the measured FMA-issue peak of its precision."""
    evals = float(res["evals"].sum())
    engaged = float(res["engaged"].sum())
    flop = FLOP_ENGAGED * engaged + FLOP_IDLE * (evals - engaged)
    t = float(np.mean(step_ms)) / 1e3
    achieved = flop / t / 1e12
    key = "fp32_tflops" if precision == "fp32" else "fp64_tflops"
    peak = peaks[key]
    smem = SMEM_BYTES_ENGAGED * engaged / t / 1e12
    traffic = DRAM_BYTES_PER_POINT.get((workload, precision))
    return {"bound": precision, "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": achieved / peak,
            "traffic": traffic * n_points if traffic else None,
            "traffic_unit": "DRAM bytes per step, scaled by points from an ncu capture of a "
                            "3072-point FP32 sweep" if traffic else None,
            "peak_source": f"measured on this GPU (mcs_measure_peaks: {precision.upper()} FMA "
                           f"issue, every SM occupied, CUDA events), of measured",
            "smem": {"achieved_tbps": smem, "peak_tbps": peaks["smem_tbps"],
                     "frac": smem / peaks["smem_tbps"],
                     "note": "algorithmic surface-ring bytes: 8 B per in-cut evaluation"},
            "work": f"{FLOP_ENGAGED:.0f} flop per in-cut and {FLOP_IDLE:.0f} per out-of-cut "
                    f"reference evaluation; {evals:.3e} evaluations, {engaged:.3e} in cut "
                    f"per step",
            "clock_mhz": clocks["sm_mhz"]}


def guided_serve(ctx, torch, stream, flush, device: int, no_cpu: bool, repeats: int) -> dict:
    """Surrogate-guided serving: 65536 seeded hetero queries (30 % of the setups outside the
    training seeds), the trained model's guided plans against the plain plan on the same
    queries, each timed over `repeats` executions (median and spread), with agreement
    against the plain GPU bisection and, on a seeded 512-query subset, against the FP64
    restatement of the reference on the host.

    Guided methods: "speculate" (the default) runs the plain bisection's own trials for 8
    of its 10 levels, each round spending the warp's spare lanes on the tree nodes the
    prediction makes likely; "bracket" verifies a predicted +-15..50 % bracket at both ends,
    refines it and falls back to the full bisection.  The same speculative plan steered by
    an untrained network separates what the trained model gains from what the schedule
    and the 8 levels gain."""
    from mcs import Surrogate
    from mcs import _abi as A
    from mcs import surrogate as SG
    from mcs import tune as T
    from mcs import workloads as W
    from mcs._lib import default_guide_opts

    if not SG.DEFAULT_MODEL.exists():
        return {"unavailable": f"no trained model at {SG.DEFAULT_MODEL.name}"}
    sv = W.serve()
    sur = SG.load(ctx)
    untrained = Surrogate(ctx, 1)
    rec = SG.record_of()

    def run(plan):
        plan.execute()  # warm-up (graph upload)
        plan.execute()
        times = []
        for i in range(repeats):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            with torch.cuda.stream(stream):
                flush.fill_(i & 0xFF)
            a.record(stream)
            plan.execute()
            b.record(stream)
            torch.cuda.synchronize()
            times.append(a.elapsed_time(b))
        return times, plan.results()

    g_spec = default_guide_opts()
    g_skip = default_guide_opts()
    g_skip.skip_top = 1e-3  # skip the a_max trial where the model gives it < 0.1 %
    g_br = default_guide_opts()
    g_br.mode = A.GUIDE_BRACKET
    sv.opts.max_buckets, tuned = T.autotune(ctx, sv.setups, sv.modals, sv.points, sv.opts,
                                            device_name=torch.cuda.get_device_name(device))
    arms = {}
    with ClockSampler(device) as clk:
        pp = ctx.plan(sv.setups, sv.modals, sv.points, sv.opts)
        plain_t, plain = run(pp)
        pp.close()
        for name, model, g in (("speculate", sur, g_spec), ("bracket", sur, g_br),
                               ("speculate_untrained", untrained, g_spec),
                               ("speculate_skip_top", sur, g_skip)):
            gp = ctx.plan(sv.setups, sv.modals, sv.points, sv.opts, surrogate=model, guide=g)
            t, r = run(gp)
            arms[name] = (t, r, gp.guide_info())
            gp.close()
    out = np.asarray(sv.meta["outside"])
    sub = np.asarray(sv.meta["fp64_subset"])
    o64 = A.make_opts(precision="fp64")
    for f in ("a_min", "a_max", "iters", "revs", "nonlinear", "honor_runout", "steps_per_tooth",
              "slices", "chatter_idx"):
        setattr(o64, f, getattr(sv.opts, f))
    g64 = ctx.solve(sv.setups, sv.modals, sv.points[sub], o64)
    # the same serving in FP64 integration (the precision whose limits meet the 2 % bar), on
    # the first 16384 queries plus the FP64-checked ones, 3 executions per plan
    idx64 = np.union1d(np.arange(16384), sub)
    pos64 = np.searchsorted(idx64, sub)
    pts64 = sv.points[idx64]

    def run3(plan):
        plan.execute()
        times = []
        for i in range(3):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            with torch.cuda.stream(stream):
                flush.fill_(i & 0xFF)
            a.record(stream)
            plan.execute()
            b.record(stream)
            torch.cuda.synchronize()
            times.append(a.elapsed_time(b))
        return float(np.median(times)), plan.results()

    arms64 = {}
    for name, model, g in (("plain", None, None), ("speculate", sur, g_spec),
                           ("speculate_skip_top", sur, g_skip)):
        p64 = ctx.plan(sv.setups, sv.modals, pts64, o64, surrogate=model, guide=g)
        arms64[name] = run3(p64)
        p64.close()
    sur.close()
    untrained.close()
    plain_ms = float(np.median(plain_t))

    def arm_stats(t, r, info):
        ms = float(np.median(t))
        both_open = (r["open"] == 1) & (plain["open"] == 1)
        rel = np.where(both_open, 0.0, np.abs(r["alim"] / plain["alim"] - 1))
        ratios = np.array(plain_t) / np.array(t)
        path = info["path"]
        return {
            "value": sv.n / (ms / 1e3), "speedup_vs_plain": plain_ms / ms,
            "ms": {"median": ms, "min": min(t), "max": max(t)},
            "speedup_spread": [float(ratios.min()), float(ratios.max())],
            "trials_ratio": float(r["trials"].sum() / plain["trials"].sum()),
            "rounds_per_point": float(info["rounds"].mean()),
            "paths": {A.PATH_NAMES[k]: float(np.mean(path == k)) for k in range(4)},
            "fallback_rate": float(np.mean(path == A.PATH_FALLBACK)),
            "within_2pct_of_plain": float(np.mean(rel <= 0.02)),
            "within_2pct_of_plain_outside_seeds": float(np.mean(rel[out] <= 0.02)),
            "max_rel_err_vs_plain": float(rel.max()),
            "median_rel_err_vs_plain_guided": float(np.median(rel[path == A.PATH_GUIDED]))
            if np.any(path == A.PATH_GUIDED) else None,
            "within_2pct_of_gpu_fp64": within(r[sub], g64),
        }

    st = {k: arm_stats(*v) for k, v in arms.items()}
    main = st["speculate"]
    res = {
        "workload": f"serve: {sv.n} seeded hetero (setup, speed) queries, "
                    f"{float(out.mean()):.0%} outside the training seeds",
        "method": "speculate: the plain bisection's trials for 8 of its 10 levels (limits "
                  "within 1.12 % of the plain ones by construction), rounds steered by the "
                  "predicted N(mu, sigma)",
        "value": main["value"], "unit": UNIT,
        "plain_value": sv.n / (plain_ms / 1e3),
        "speedup_vs_plain": main["speedup_vs_plain"],
        "repeats": repeats,
        "plain_ms": {"median": plain_ms, "min": min(plain_t), "max": max(plain_t)},
        "guided_ms": main["ms"],
        "speedup_spread": main["speedup_spread"],
        "trials_ratio": main["trials_ratio"],
        "rounds_per_point": main["rounds_per_point"],
        "within_2pct_of_plain": main["within_2pct_of_plain"],
        "max_rel_err_vs_plain": main["max_rel_err_vs_plain"],
        "trained_vs_untrained_prior": main["value"] / st["speculate_untrained"]["value"],
        "untrained_prior": st["speculate_untrained"],
        "skip_top_1e-3": dict(st["speculate_skip_top"],
                              note="the a_max trial skipped where the predicted probability "
                                   "of a stable a_max is below 0.1 %; not exact where that "
                                   "prediction is wrong"),
        "bracket": st["bracket"],
        "fp64": {
            "queries": int(len(idx64)),
            "plain_value": len(idx64) / (arms64["plain"][0] / 1e3),
            **{k: {"value": len(idx64) / (arms64[k][0] / 1e3),
                   "speedup_vs_plain": arms64["plain"][0] / arms64[k][0],
                   "within_2pct_of_plain": within(arms64[k][1], arms64["plain"][1])}
               for k in ("speculate", "speculate_skip_top")}},
        "fp64_subset": len(sub),
        "within_2pct_of_gpu_fp64": main["within_2pct_of_gpu_fp64"],
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
        t_cpu = time.perf_counter()
        r64, _ = O.solve_batch(setups, modals, P, sv.opts, nthreads=cpu_cores())
        t_cpu = time.perf_counter() - t_cpu
        res["cpu_fp64"] = {"value": len(sub) / t_cpu, "unit": UNIT, "cores": cpu_cores(),
                           "sample": f"the {len(sub)} FP64-checked queries, C++ FP64 "
                                     "restatement, all host threads"}
        f64 = res["fp64"]
        f64["plain_within_2pct_of_cpu_fp64"] = within(arms64["plain"][1][pos64], r64)
        for k in ("speculate", "speculate_skip_top"):
            f64[k]["within_2pct_of_cpu_fp64"] = within(arms64[k][1][pos64], r64)
            f64[k]["vs_cpu"] = f64[k]["value"] / res["cpu_fp64"]["value"]
        res["within_2pct_of_cpu_fp64"] = within(arms["speculate"][1][sub], r64)
        res["bracket"]["within_2pct_of_cpu_fp64"] = within(arms["bracket"][1][sub], r64)
        res["skip_top_1e-3"]["within_2pct_of_cpu_fp64"] = within(
            arms["speculate_skip_top"][1][sub], r64)
        res["plain_within_2pct_of_cpu_fp64"] = within(plain[sub], r64)
    return res


def worker_latency(ctx, torch, precision: str, repeats: int = 3) -> dict:
    """Latency of the stability Worker's request (main.js:494-501): the 18 log-spaced lobe
    speeds of one setup, each with its own modes (the spindle model), through the blocking
    call mcs_solve, with and without several warps sharing each point's bisection."""
    from mcs import _abi as A
    from mcs import workloads as W

    wl = W.spindle_sweep()
    sel = wl.points["setup"] == 0
    pts = wl.points[sel]
    out = {"workload": f"{int(sel.sum())} lobe speeds 4000-30000 rpm with speed-dependent "
                       "modes, reference options ([0.05, 20] x 8, 120 revs)",
           "precision": precision}
    res = None
    for name, cw in (("one_warp", 1), ("multi_warp", 0)):
        o = A.Opts.from_buffer_copy(bytes(wl.opts))
        o.precision = A.precision_code(precision)
        o.coop_warps = cw
        ctx.solve(wl.setups, wl.modals, pts, o)  # warm-up
        ts = []
        for _ in range(repeats):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            r = ctx.solve(wl.setups, wl.modals, pts, o)
            ts.append(1e3 * (time.perf_counter() - t0))
        out[f"{name}_ms"] = float(np.median(ts))
        res = r if name == "one_warp" else res
        if name == "multi_warp":
            assert r.tobytes() == res.tobytes(), "multi-warp results differ"
    out["speedup"] = out["one_warp_ms"] / out["multi_warp_ms"]
    return out


# The Simulator's defaults (sim.js:44-50): D 10 mm, 3 flutes, helix 30, flute 25 mm, stickout
# 30 mm on a 50 kN/mm spindle, 5 um runout, modal zeta 0.04; A5052 (materials.js:25); a frame
# spends dynBudget = 220,000 slice-force evaluations (sim.js:50, "about 5 ms of JS").
SIM_TOOL = {"D": 10.0, "N": 3, "helixDeg": 30.0, "type": "flat", "fluteLen": 25.0,
            "stickout": 30.0, "kSpindle": 50000.0, "runout": 5.0}
A5052 = {"Ktc": 700.0, "Krc": 210.0, "Kac": 120.0, "Kte": 20.0, "Kre": 25.0, "Kae": 5.0,
         "mc": 0.10, "Ci": 2e4}
DYN_BUDGET = 220000


def _pool_map(fn, items, threads: int):
    """fn over items on `threads` host threads (the oracle's ctypes calls release the GIL)."""
    from concurrent.futures import ThreadPoolExecutor

    with ThreadPoolExecutor(max_workers=threads) as ex:
        return list(ex.map(fn, items))


def _event_ms(torch, stream, call) -> float:
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    call()
    b.record(stream)
    b.synchronize()
    return float(a.elapsed_time(b))


def playback_leg(ctx, torch, stream, no_cpu: bool, repeats: int = 5,
                 n: int = 148 * 8) -> dict:
    """The playback dynamics (CuttingEngine.run as Simulator.step drives it, sim.js:396-416):
    engines of the Simulator's default tool in a half-immersion down-milling cut with the
    thin wall engaged, each frame one dynBudget of slice-force evaluations.  `value` is a
    batch of 1184 engines (8 per SM) at spread speeds running frame after frame; `frame_ms`
    is one engine's frame, the interactive case.  The host restatement runs a sample of the
    same engines on every host thread, and its statistics check the GPU's."""
    import math

    from mcs import engine as E
    from mcs import spindle as SP

    tm = SP.tool_model(SIM_TOOL)
    modal = {"k": tm["k"], "fn": tm["fn"], "zeta": 0.04}
    tool = {k: SIM_TOOL[k] for k in ("N", "helixDeg", "type", "fluteLen", "runout")}
    tool["R"] = SIM_TOOL["D"] / 2
    ap, fz = 2.0, 0.05
    wall = {"k": 800.0, "m": 0.05, "zeta": 0.02, "nx": 0.0, "ny": 1.0}
    nz = math.ceil(ap / max(0.25, SIM_TOOL["fluteLen"] / 48))  # slices (cutting.js:63,103)
    cost = SIM_TOOL["N"] * nz                                   # sim.js:409
    steps = DYN_BUDGET // cost
    speeds = np.linspace(8000.0, 16000.0, n)
    cfgs = [E.config(tool, modal, A5052, s) for s in speeds]
    g = E.engagement(E.arc_map(math.pi / 2, math.pi), (1, 0), fz, -ap, ap, wall=wall)
    out = {"workload": f"{n} engines 8000-16000 rpm, Simulator default tool (D10, 3 flutes, "
                       f"stickout 30, 5 um runout), A5052, half-immersion down milling, "
                       f"ap {ap} mm ({nz} slices), fz {fz}, thin wall; a frame = "
                       f"{steps} steps = {steps * cost} slice-force evaluations (dynBudget)",
           "unit": "slice-force evaluations/s", "precision": "fp64"}
    eng = E.Engines(ctx, n)
    try:
        eng.configure(cfgs)
        eng.set_engagement([g] * n)
        arr = np.full(n, steps, dtype=np.int64)
        eng.run(arr)  # warm-up frame
        ts = [_event_ms(torch, stream, lambda: eng.run(arr)) for _ in range(repeats)]
        st = eng.take_stats()
    finally:
        eng.close()
    ms = float(np.median(ts))
    out["value"] = n * steps * cost / (ms / 1e3)
    out["batch_frame_ms"] = ms
    out["gpu_launches_per_frame"] = 1
    one = E.Engines(ctx, 1)
    try:
        one.configure([cfgs[n // 2]])
        one.set_engagement([g])
        a1 = np.array([steps], dtype=np.int64)
        one.run(a1)
        t1 = [_event_ms(torch, stream, lambda: one.run(a1)) for _ in range(repeats)]
        w1 = []
        for _ in range(repeats):
            t0 = time.perf_counter()
            one.run(a1)
            w1.append(1e3 * (time.perf_counter() - t0))
    finally:
        one.close()
    out["frame_ms"] = float(np.median(t1))
    out["frame_e2e_ms"] = float(np.median(w1))
    out["reference_frame_budget_ms"] = 5.0  # sim.js:50
    if no_cpu:
        return out
    import pyoracle as O

    cores = cpu_cores()
    sample = list(range(0, n, max(1, n // (4 * cores))))

    def host(i):
        e = O.Engine()
        e.configure_from(cfgs[i])
        e.engage(g)
        t = time.perf_counter()
        for _ in range(1 + repeats):
            e.run(steps)
        dt = time.perf_counter() - t
        return dt, e.take_stats_full()

    t = time.perf_counter()
    res = _pool_map(host, sample, cores)
    wall_s = time.perf_counter() - t
    evals = len(sample) * (1 + repeats) * steps * cost
    one_thread = float(np.median([r[0] for r in res])) / (1 + repeats)
    out["cpu_baseline"] = {"value": evals / wall_s, "unit": out["unit"], "cores": cores,
                           "kind": "port",
                           "sample": f"{len(sample)} of the engines, {1 + repeats} frames each, "
                                     "C++ FP64 restatement of cutting.js, all host threads",
                           "frame_ms_one_thread": 1e3 * one_thread}
    rel, steps_equal = 0.0, True
    for i, (_, ref) in zip(sample, res):
        for f in ("sumFx", "sumFy", "sumT", "sumF"):
            rel = max(rel, abs(float(st[i][f]) / float(ref[f]) - 1))
        steps_equal &= int(st[i]["n"]) == int(ref["n"])
    out["parity"] = {"engines_checked": len(sample), "max_rel_diff_force_sums": rel,
                     "step_counts_equal": bool(steps_equal)}
    out["vs_cpu"] = out["value"] / out["cpu_baseline"]["value"]
    return out


def composite_leg(ctx, no_cpu: bool, repeats: int = 5) -> dict:
    """The chart's speed-dependent lobe diagram (Simulator.lobes, sim.js:262-287): a
    diagram per 1000 rpm with the spindle model's modes at the node, read every 25 rpm,
    for the Simulator's default tool; one call of mcs.compositeLobes against the host
    restatement of the same loop, and the samples compared."""
    import math

    import mcs
    from mcs import spindle as SP

    sp = SP.Spindle.from_tool({k: SIM_TOOL[k] for k in ("D", "stickout", "kSpindle")},
                              {"auto": True, "k": 0, "fn": 0, "zeta": 0.04})
    base = {"N": 3, "Ktc": A5052["Ktc"], "Krc": A5052["Krc"], "phiSt": math.pi / 2,
            "phiEx": math.pi, "lobes": 30, "rpmMin": 2000, "rpmMax": 40000}
    got = mcs.compositeLobes(sp, base, ctx=ctx)[0]  # warm-up
    ts = []
    for _ in range(repeats):
        t0 = time.perf_counter()
        got = mcs.compositeLobes(sp, base, ctx=ctx)[0]
        ts.append(1e3 * (time.perf_counter() - t0))
    out = {"workload": f"Simulator default tool, 3 flutes, A5052, half immersion, 30 lobes, "
                       f"2000-40000 rpm: {len(got)} samples",
           "unit": "ms per diagram (e2e through mcs.compositeLobes)", "lower_is_better": True,
           "value": float(np.median(ts))}
    if no_cpu:
        return out
    import pyoracle as O

    t0 = time.perf_counter()
    ref = O.composite_lobes(sp.record, base, sp.frfs)[0]
    out["cpu_baseline"] = {"value": 1e3 * (time.perf_counter() - t0), "unit": "ms per diagram",
                           "cores": 1, "kind": "port",
                           "sample": "the same diagram, restatement of sim.js:262-287 and "
                                     "sld.js (Python node loop, C++ lobes), one thread"}
    g = np.array([p["alim"] for p in got])
    r = np.array([p["alim"] for p in ref])
    out["parity"] = {"samples": len(g), "max_rel_diff": float(np.max(np.abs(g / r - 1)))}
    out["vs_cpu"] = out["cpu_baseline"]["value"] / out["value"]
    return out


def identify_leg(ctx, no_cpu: bool, repeats: int = 5) -> dict:
    """The identification's unit-force runs (identify.js:26-40): per cutting test six
    rigid-tool engines, one per coefficient, two revolutions dropped and one averaged;
    256 seeded tests (1536 engines) in one mcs.identify.unit_forces call against the host
    restatement on every host thread, and the forces compared."""
    from mcs import engine as E
    from mcs import identify as I

    tool = {k: SIM_TOOL[k] for k in ("D", "N", "helixDeg", "fluteLen")}
    rng = np.random.default_rng(5)
    tests = [{"fz": float(rng.uniform(0.02, 0.1)), "ap": float(rng.uniform(0.5, 5.0)),
              "ae": float(rng.uniform(1.0, 10.0)), "mode": ("slot", "down", "up")[i % 3]}
             for i in range(256)]
    U = I.unit_forces(ctx, tool, tests)  # warm-up
    ts = []
    for _ in range(repeats):
        t0 = time.perf_counter()
        U = I.unit_forces(ctx, tool, tests)
        ts.append(1e3 * (time.perf_counter() - t0))
    ms = float(np.median(ts))
    out = {"workload": f"{len(tests)} seeded tests (slot/down/up, fz 0.02-0.1, ap 0.5-5, "
                       f"ae 1-10) of a D10 3-flute tool, 6 unit-force engines each",
           "unit": "tests/s (e2e through mcs.identify.unit_forces)", "value": len(tests) / ms * 1e3,
           "ms_per_call": ms}
    if no_cpu:
        return out
    import pyoracle as O

    cfgs, gs = [], []
    for t in tests:
        st, ex = I.immersion(t["mode"], t["ae"], tool["D"])
        for key in I.COEF_KEYS:
            mat = dict.fromkeys(I.COEF_KEYS, 0.0)
            mat.update({key: 1.0, "mc": 0.0, "Ci": 0.0})
            tl = I._engine_tool(tool, t["ap"], phase=0.0)
            tl["nonlinear"] = False
            cfgs.append(E.config(tl, E.RIGID, mat, 6000))
            gs.append(E.engagement(E.arc_map(st, ex), (1, 0), t["fz"], -t["ap"], t["ap"]))
    cores = cpu_cores()
    chunks = [list(range(k, len(tests), cores)) for k in range(cores)]

    def host(ch):
        sel = [6 * j + c for j in ch for c in range(6)]
        return ch, O.unit_forces_ref([cfgs[s] for s in sel], [gs[s] for s in sel])

    t0 = time.perf_counter()
    res = _pool_map(host, chunks, cores)
    dt = time.perf_counter() - t0
    ref = np.zeros_like(U)
    for ch, r in res:
        ref[ch] = r.reshape(len(ch), 6, 3)
    scale = np.maximum(np.abs(ref).max(axis=2, keepdims=True), 1e-300)
    out["cpu_baseline"] = {"value": len(tests) / dt, "unit": "tests/s", "cores": cores,
                           "kind": "port",
                           "sample": "the same tests, C++ FP64 restatement of identify.js "
                                     "unitForces, all host threads"}
    out["parity"] = {"tests": len(tests),
                     "max_rel_diff": float(np.max(np.abs(U - ref) / scale))}
    out["vs_cpu"] = out["value"] / out["cpu_baseline"]["value"]
    return out


def rows_leg(ctx, torch, stream, no_cpu: bool) -> dict:
    """The rows around the stability path, each beside its host restatement.  A leg that
    raises is recorded with its error; the headline line is printed regardless."""
    legs = {"playback": lambda: playback_leg(ctx, torch, stream, no_cpu),
            "composite_lobes": lambda: composite_leg(ctx, no_cpu),
            "identify": lambda: identify_leg(ctx, no_cpu)}
    out = {}
    for name, leg in legs.items():
        try:
            out[name] = leg()
        except Exception as e:  # noqa: BLE001  (recorded in the line, not swallowed)
            out[name] = {"error": f"{type(e).__name__}: {e}"}
    return out


def make_workload(name: str, rank: int, points: int = 0):
    from mcs import workloads as W

    if name == "hetero":  # 16384 seeded setups per rank (weak scaling)
        wl = W.hetero(n=16384, first_seed=16384 * rank)
    elif name == "small":  # the 64-speed reference case; the same on every rank
        wl = W.small()
    else:
        wl = W.sweep(seed=1 + rank)
    if points and points < wl.n:  # a smaller case of the same workload (profiling)
        wl = wl.subset(np.linspace(0, wl.n - 1, points).round().astype(int))
    return wl


def workload_config(name: str, wl) -> dict:
    """The workload a line measures; identical in both arms."""
    return {"workload": WORKLOADS[name], "points_per_gpu": int(wl.n)}


def reference_arm(args) -> int:
    rank, world, _ = env_rank()
    if rank != 0:
        return 0
    wl = make_workload(args.workload, 0, args.points)
    cores = cpu_cores()
    # seeded sample order over the whole workload; every step takes the next slice, so the
    # steps together cover the speed range instead of repeating one fixed sample
    perm = np.argsort(np.random.default_rng(7).random(wl.n))
    pos = 0

    def take(n):
        nonlocal pos
        idx = perm[np.arange(pos, pos + n) % wl.n]
        pos += n
        return idx

    # calibration (the first warm-up step): per-step sample sized so that the whole run
    # stays within a few minutes, and at least 8 points per thread (the pool's tail)
    steps_total = args.steps + args.warmup
    per_step_s = min(8.0, max(2.0, 150.0 / steps_total))
    _, dt0 = run_oracle(wl, take(2 * cores), cores)
    rate0 = 2 * cores / dt0
    n_step = int(min(wl.n, max(8 * cores, round(rate0 * per_step_s / cores) * cores)))
    for _ in range(args.warmup - 1):
        run_oracle(wl, take(n_step), cores)
    tot_p, tot_t = 0, 0.0
    for _ in range(args.steps):
        _, t = run_oracle(wl, take(n_step), cores)
        tot_p += n_step
        tot_t += t
    v = tot_p / tot_t
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot_t / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded)",
        "config": workload_config(args.workload, wl),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{n_step} seeded {wl.name} points per step (a fresh slice "
                                   f"of a seeded permutation each step, cost-sorted), the C++ "
                                   f"FP64 restatement of stabtd.js/cutting.js, {cores} "
                                   f"threads, {cpu_model()}"},
        "node_probe": node_probe(),
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
    from mcs import _abi as A
    from mcs import tune as T

    ctx = mcs.Context(device)
    stream = torch.cuda.ExternalStream(ctx.stream)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{device}")
    peaks = ctx.measure_peaks()  # roofline denominators, before any timed region

    def barrier():
        if dist is not None:
            dist.barrier()

    def maxover(x: float) -> float:
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{device}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def timed(wl, precision: str, steps: int, warmup: int):
        """Device-resident plan of a workload: per-step CUDA-event times, results, info."""
        opts = A.make_opts(precision=precision)
        for f in ("a_min", "a_max", "iters", "revs", "nonlinear", "honor_runout",
                  "steps_per_tooth", "slices", "chatter_idx", "serial_trials", "coop_warps",
                  "coop_points"):
            setattr(opts, f, getattr(wl.opts, f))
        if args.serial_trials:
            opts.serial_trials = 1
        if args.coop_warps >= 0:
            opts.coop_warps = args.coop_warps
        if args.coop_points >= 0:
            opts.coop_points = args.coop_points
        # schedule (number of shared-memory size classes) from the autotuner, untimed
        if args.max_buckets:
            opts.max_buckets, tuned = args.max_buckets, {"ms": {}, "cached": False}
        else:
            opts.max_buckets, tuned = T.autotune(ctx, wl.setups, wl.modals, wl.points, opts,
                                                 device_name=torch.cuda.get_device_name(device))
        plan = ctx.plan(wl.setups, wl.modals, wl.points, opts)
        info = plan.info()
        info["schedule"] = {"max_buckets": int(opts.max_buckets), "tuning_ms": tuned["ms"],
                            "from_cache": bool(tuned["cached"]),
                            "coop_warps": int(opts.coop_warps),
                            "coop_points_opt": int(opts.coop_points),
                            "coop_points": int(info["coop_points"])}
        for _ in range(warmup):
            plan.execute()
        res = plan.results()
        assert np.all((res["status"] == 0) | (res["status"] == 4)), np.unique(res["status"])
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        barrier()
        torch.cuda.synchronize()
        with ClockSampler(device) as clk:
            for i in range(steps):
                with torch.cuda.stream(stream):
                    flush.fill_(i & 0xFF)  # write 256 MiB (> 126 MB L2) between timed steps
                starts[i].record(stream)
                plan.execute()
                ends[i].record(stream)
            torch.cuda.synchronize()
        barrier()
        step_ms = [s_.elapsed_time(e_) for s_, e_ in zip(starts, ends)]
        res2 = plan.results()
        assert res2.tobytes() == res.tobytes(), "results changed between executions"
        plan.close()
        ms = maxover(float(np.sum(step_ms))) / steps
        return {"step_ms": step_ms, "ms": ms, "res": res, "info": info,
                "clocks": clk.summary(), "opts": opts}

    def measure(name: str, precisions, steps: int, warmup: int, e2e_steps: int, cpu: bool):
        """One workload: every precision timed as a plan, the headline precision also end
        to end; on rank 0 of a 1-GPU run the host FP64 baseline and the accuracy."""
        if args.strong and world > 1:  # one batch split by the library's cost-balanced shards
            from mcs import dist as D

            full = make_workload(name, 0, args.points)
            wl = full.subset(D.library_shards(full, world)[rank])
            pts_total = full.n
        else:  # every rank its own seeded batch (weak scaling)
            wl = make_workload(name, rank, args.points)
            pts_total = wl.n * world
        var = {p: timed(wl, p, steps, warmup) for p in precisions}
        head = var[precisions[0]]
        e2e = None
        if e2e_steps:
            e2e = e2e_leg(ctx, torch, wl, head["opts"], head["info"], e2e_steps,
                          max(1, warmup // 2), maxover, barrier, pts_total, head["res"])
        rec = {"wl": wl, "var": var, "e2e": e2e, "pts_total": pts_total, "cpu": None,
               "accuracy": None}
        if cpu and rank == 0 and world == 1:
            cpu_rec, idx, r64 = cpu_leg(wl)
            rec["cpu"] = cpu_rec
            rec["accuracy"] = {
                "reference": "FP64 restatement of the reference on the host, seeded "
                             f"{len(idx)}-point subset",
                **{f"within_2pct_of_cpu_fp64_{p}": within(v["res"][idx], r64)
                   for p, v in var.items()}}
            if wl.opts.honor_runout:
                rec["accuracy"]["runout_zero"] = runout_zero(wl, idx, r64, head["opts"])
        return rec

    def runout_zero(wl, idx, r64, opts) -> dict:
        """The reference's own chatterAt forces the runout to 0 (stabtd.js:16): the same
        subset solved that way on the GPU and by the FP64 restatement, and how far the
        runout the workload honours moves the limits."""
        import dataclasses

        o0 = A.Opts.from_buffer_copy(bytes(opts))
        o0.honor_runout = 0
        o0.precision = A.FP64
        g0 = ctx.solve(wl.setups, wl.modals, wl.points[idx], o0)
        h0, dt = run_oracle(dataclasses.replace(wl, opts=o0), idx, cpu_cores())
        both = (h0["open"] == 1) & (r64["open"] == 1)
        moved = np.where(both, 0.0, np.abs(h0["alim"] / r64["alim"] - 1))
        return {"points": len(idx), "within_2pct_of_cpu_fp64_fp64": within(g0, h0),
                "median_rel_change_by_runout": float(np.median(moved)),
                "changed_over_2pct_by_runout": float(np.mean(moved > 0.02)),
                "host_seconds": round(dt, 1)}

    def summarize(name: str, rec: dict, precision: str) -> dict:
        v = rec["var"][precision]
        return {
            "value": rec["pts_total"] / (v["ms"] / 1e3), "unit": UNIT, "ms_per_step": v["ms"],
            "config": workload_config(name, rec["wl"]),
            "roofline": roofline(v["res"], v["step_ms"], precision, peaks, v["clocks"], name,
                                 rec["wl"].n),
            "e2e": rec["e2e"], "cpu_baseline": rec["cpu"], "accuracy": rec["accuracy"],
            "launch": {"variant": f"plain GPU bisection, {precision} force law and modal "
                                  "integration, FP64 statistics and bracket",
                       "l2": "flushed between timed steps (256 MiB write)",
                       "kernels_per_step": v["info"]["kernels"],
                       "graph": bool(v["info"]["graph"]), "blocks": v["info"]["blocks"],
                       "smem_per_warp_max": v["info"]["smem_per_warp"],
                       "schedule": v["info"]["schedule"]},
            "variants": {p: {"value": rec["pts_total"] / (x["ms"] / 1e3),
                             "ms_per_step": x["ms"], "kernels_per_step": x["info"]["kernels"],
                             "sm_mhz": x["clocks"]["sm_mhz"],
                             "roofline_frac": roofline(x["res"], x["step_ms"], p, peaks,
                                                       x["clocks"], name, rec["wl"].n)["frac"]}
                         for p, x in rec["var"].items()},
            "clocks": v["clocks"],
        }

    precs = [args.precision] + ([] if args.headline_only else
                                [p for p in ("fp64", "fp32") if p != args.precision])
    main = measure(args.workload, precs, args.steps, args.warmup,
                   0 if args.no_e2e else max(2, min(args.steps, 5)), not args.no_cpu)
    hetero = small = None
    if not args.no_hetero and args.workload != "hetero":
        hetero = measure("hetero", precs, max(3, min(args.steps, 5)), 3,
                         0 if args.no_e2e else 2, not args.no_cpu)
    if not args.no_small and args.workload != "small":
        small = measure("small", precs, max(3, min(args.steps, 5)), 3,
                        0 if args.no_e2e else 2, not args.no_cpu)

    if rank == 0:
        head = summarize(args.workload, main, args.precision)
        v = main["var"][args.precision]
        guided = (guided_serve(ctx, torch, stream, flush, device, args.no_cpu,
                               args.guided_repeats)
                  if world == 1 and not args.no_guided else None)
        latency = (worker_latency(ctx, torch, args.precision)
                   if world == 1 and not args.no_latency else None)
        rows = (rows_leg(ctx, torch, stream, args.no_cpu)
                if world == 1 and not args.no_rows else None)
        line = {
            "metric": METRIC, "value": head["value"], "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": head["ms_per_step"],
            "higher_is_better": True,
            "scaling": "strong" if args.strong and world > 1 else "weak", "vs_baseline": None,
            "dtype": "f32" if args.precision == "fp32" else "f64",
            "data": "synthetic (seeded; no public dataset exists for this path)",
            "config": head["config"],
            "launch": head["launch"],
            "roofline": head["roofline"],
            "cpu_baseline": head["cpu_baseline"],
            "accuracy": head["accuracy"],
            "e2e": head["e2e"],
            "gpu_launches": int(v["info"]["kernels"]) * args.steps,
            "clocks": head["clocks"],
            "peaks": peaks,
            "results": {"open": int(v["res"]["open"].sum()),
                        "alim_median": float(np.median(v["res"]["alim"]))},
            "variants": head["variants"],
            "workloads": {**({"hetero": summarize("hetero", hetero, args.precision)}
                             if hetero else {}),
                          **({"small": summarize("small", small, args.precision)}
                             if small else {})} or None,
            "guided": guided,
            "worker_latency": latency,
            "rows": rows,
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
    ap.add_argument("--precision", default="fp64", choices=["fp32", "fp64"],
                    help="integration precision of the headline value (the other is a variant)")
    ap.add_argument("--headline-only", action="store_true",
                    help="time only the headline precision")
    ap.add_argument("--points", type=int, default=0,
                    help="solve an evenly spaced subset of the workload (profiling case)")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end legs")
    ap.add_argument("--no-guided", action="store_true",
                    help="skip the surrogate-guided serving leg")
    ap.add_argument("--no-hetero", action="store_true", help="skip the hetero workload leg")
    ap.add_argument("--no-small", action="store_true", help="skip the 64-speed reference case")
    ap.add_argument("--guided-repeats", type=int, default=5)
    ap.add_argument("--no-latency", action="store_true",
                    help="skip the latency of the Worker's 18-speed request")
    ap.add_argument("--no-rows", action="store_true",
                    help="skip the playback engines, composite lobes and identification legs")
    ap.add_argument("--workload", default="sweep", choices=["sweep", "hetero", "small"],
                    help="sweep (the headline), the heterogeneous batch or the 64-speed case")
    ap.add_argument("--max-buckets", type=int, default=0,
                    help="fixed schedule (shared-memory size classes); 0: autotune")
    ap.add_argument("--coop-warps", type=int, default=-1,
                    help="warps sharing each heaviest point's bisection (1: off; -1: default)")
    ap.add_argument("--coop-points", type=int, default=-1,
                    help="how many of the costliest points take that path (0: one per SM; "
                         "-1: default)")
    ap.add_argument("--strong", action="store_true",
                    help="N > 1: split one batch over the ranks (mcs_shard) instead of one "
                         "batch per rank")
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
