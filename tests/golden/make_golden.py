"""Generate the golden fixtures of the GPU parity tests from the CPU oracle.

    python tests/golden/make_golden.py [--threads N]

Writes, per workload, the oracle's timeDomainLimit results and the full trial trace
(every bisection depth with its chatter index parts and decision):

  small.npz    all 64 speeds of the small sweep
  sweep.npz    the 256-speed FP64 subset of the 4096-speed sweep
  hetero.npz   256 seeded setups of the heterogeneous batch
  edge.npz     edge cases: slot / up milling / ball end / 1 and 8 flutes / > 32 slices
  self_agreement.npz  the reference's own sweep and hetero limits under 1e-6 / 1e-5 feed
               changes (how well it agrees with itself)
  spindle.npz  the 18-speed lobe curve with speed-dependent modes (spindle.js), 3 cases

The oracle is a restatement of the reference (src/stabtd.js, src/cutting.js) pinned by the
reference's own known answers (tests/test_oracle_pins.py); these files freeze its output
so the GPU tests need no long CPU runs.
"""
from __future__ import annotations

import argparse
import math
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(ROOT / "machinig-sim_b200"))

import pyoracle as O  # noqa: E402
from mcs import _abi as A  # noqa: E402
from mcs import workloads as W  # noqa: E402


def as_ctypes(wl: W.Workload, idx):
    setups = [A.Setup.from_buffer_copy(r.tobytes()) for r in wl.setups]
    modals = [A.Modal.from_buffer_copy(r.tobytes()) for r in wl.modals]
    pts = wl.points[idx]
    P = (A.Point * len(pts)).from_buffer_copy(pts.tobytes())
    return setups, modals, P, pts


def compact(wl: W.Workload, idx) -> W.Workload:
    """Only the setups and modals the chosen points use, indices remapped."""
    pts = wl.points[idx].copy()
    su, si = np.unique(pts["setup"], return_inverse=True)
    mu, mi = np.unique(pts["modal"], return_inverse=True)
    pts["setup"] = si
    pts["modal"] = mi
    return W.Workload(wl.name, wl.setups[su], wl.modals[mu], pts, wl.opts, wl.meta)


def run(wl: W.Workload, idx, threads: int, out: Path):
    wl = compact(wl, idx)
    idx_orig, idx = np.asarray(idx), np.arange(len(idx))
    setups, modals, P, pts = as_ctypes(wl, idx)
    t = time.time()
    res, tr = O.solve_batch(setups, modals, P, wl.opts, nthreads=threads, traces=True)
    sens = [sensitivity(wl, pts, res, tr, threads, eps) for eps in SENS_LEVELS]
    dt = time.time() - t
    np.savez_compressed(out, setups=wl.setups, modals=wl.modals, points=pts,
                        index=idx_orig, opts=A.opts_record(wl.opts), results=res,
                        traces=tr, sens_levels=np.array(SENS_LEVELS),
                        sens_index=np.stack([s[0] for s in sens]),
                        sens_flip=np.stack([s[1] for s in sens]))
    flips = ", ".join(f"{int(s[1].sum())} at {e:g}" for e, s in zip(SENS_LEVELS, sens))
    print(f"{out.name}: {len(idx)} points in {dt:.1f} s; of {int((tr['ap'] > 0).sum())} "
          f"traced trials these flip under a feed perturbation: {flips}", flush=True)


# relative feed perturbations probed: one FP32 rounding (1e-7) up to what an FP32
# trajectory of ~1e5 steps accumulates (1e-5)
SENS_LEVELS = [1e-7, 1e-6, 3e-6, 1e-5]


def sensitivity(wl, pts, res, tr, threads, eps):
    """How the FP64 reference's own decision at each traced depth reacts to feeds scaled by
    (1 +- eps): the largest index change and whether the decision flips.  A trial whose
    decision flips under a rounding-sized input change (1e-7: one FP32 rounding; 1e-6: the
    error an FP32 trajectory accumulates) is ill-conditioned: no integration in another
    precision or operation order can be expected to reproduce it."""
    per = tr.shape[1]
    rows = [(p, j) for p in range(len(res)) for j in range(int(res["trials"][p]))]
    trials = np.zeros(len(rows), dtype=A.TRIAL_DTYPE)
    for i, (p, j) in enumerate(rows):
        trials[i] = (p, 0, tr[p, j]["ap"])
    T = (A.Trial * len(rows)).from_buffer_copy(trials.tobytes())
    P = (A.Point * len(pts)).from_buffer_copy(pts.tobytes())
    modals = [A.Modal.from_buffer_copy(r.tobytes()) for r in wl.modals]
    dmax = np.zeros((len(res), per))
    flip = np.zeros((len(res), per), dtype=bool)
    for sgn in (+1, -1):
        st = wl.setups.copy()
        st["fz"] *= 1 + sgn * eps
        setups = [A.Setup.from_buffer_copy(r.tobytes()) for r in st]
        out = O.chatter_batch(setups, modals, P, T, wl.opts, nthreads=threads)
        for i, (p, j) in enumerate(rows):
            a, b = tr[p, j]["index"], out["index"][i]
            d = abs(b - a) if np.isfinite(a) and np.isfinite(b) else np.inf
            dmax[p, j] = max(dmax[p, j], d)
            flip[p, j] |= bool(out["chatter"][i]) != bool(tr[p, j]["chatter"])
    return dmax, flip


# relative feed changes of the self-agreement fixture: the FP64 reference's own limits
# under an input change of the size an FP32 trajectory's rounding amounts to
SELF_LEVELS = [1e-6, -1e-6, 1e-5]


def self_agreement(out: Path, threads: int):
    """self_agreement.npz: for the sweep and hetero subsets, the FP64 reference's
    timeDomainLimit with the feed scaled by (1 + eps) for each eps of SELF_LEVELS.  Where a
    1e-6 change of an input moves the reference's own limit by more than 2 %, no
    integration in another precision can be expected to land within 2 % of it either; the
    GPU parity tests compare their FP32 agreement with this one."""
    rec = {"levels": np.array(SELF_LEVELS)}
    for name, wl, idx in (("sweep", W.sweep(), np.array(W.sweep().meta["fp64_subset"])),
                          ("hetero", W.hetero(),
                           np.sort(np.argsort(W.uniform(np.arange(16384), 7, 0))[:256]))):
        wl = compact(wl, idx)
        modals = [A.Modal.from_buffer_copy(r.tobytes()) for r in wl.modals]
        P = (A.Point * len(wl.points)).from_buffer_copy(wl.points.tobytes())
        alim, opn = [], []
        t = time.time()
        for eps in SELF_LEVELS:
            st = wl.setups.copy()
            st["fz"] *= 1 + eps
            setups = [A.Setup.from_buffer_copy(r.tobytes()) for r in st]
            res, _ = O.solve_batch(setups, modals, P, wl.opts, nthreads=threads)
            alim.append(res["alim"])
            opn.append(res["open"])
        rec[f"{name}_alim"] = np.stack(alim)
        rec[f"{name}_open"] = np.stack(opn)
        print(f"{out.name}: {name} {len(idx)} points x {len(SELF_LEVELS)} feeds in "
              f"{time.time() - t:.1f} s", flush=True)
    np.savez_compressed(out, **rec)


def spindle_workload() -> W.Workload:
    """The speed-dependent sweep of mcs.workloads.spindle_sweep with every modal set from
    the oracle's own restatement of modesAt (src/spindle.js:64-85), not the library's."""
    from mcs import spindle as SP

    wl = W.spindle_sweep()
    speeds = wl.meta["speeds"]
    modals = []
    for name in wl.meta["cases"]:
        case = W.SPINDLE_CASES[name]
        sp = SP.Spindle.from_tool(case["tool"], case["modal"],
                                  spindle_mode=case.get("spindle_mode"))
        frfs = A.array_of(A.SpeedFrf, sp.frfs)
        modals.append(O.modes_at(sp.record, speeds, list(frfs)[: len(sp.frfs)]))
    wl.modals = np.concatenate(modals)
    return wl


def edge_workload() -> W.Workload:
    """Cases off the benchmark grid: slot, up milling, ball end, N = 1 and 8, 48 slices,
    helix 0 (every slice in phase), a multi-mode asymmetric tool and an empty arc."""
    base = W._base_setup(1)[0]
    cases = []

    def add(mod, modal, S):
        s = base.copy()
        for k, v in mod.items():
            if k in ("N", "type", "R", "helix_deg", "flute_len", "runout", "runout_phase"):
                s["tool"][k] = v
            elif k in ("Ktc", "Krc", "Kte", "Kre", "mc", "Ci"):
                s["mat"][k] = v
            else:
                s[k] = v
        cases.append((s, modal, S))

    one = np.zeros(1, dtype=A.MODAL_DTYPE)[0]
    one["nx"] = 1
    one["x"][0] = (1e4, 1000.0, 0.02)
    two = np.zeros(1, dtype=A.MODAL_DTYPE)[0]
    two["nx"], two["ny"] = 2, 2
    two["x"][0], two["x"][1] = (18000.0, 1150.0, 0.05), (11000.0, 2250.0, 0.035)
    two["y"][0], two["y"][1] = (22000.0, 1250.0, 0.05), (13000.0, 2400.0, 0.03)
    four = np.zeros(1, dtype=A.MODAL_DTYPE)[0]
    four["nx"] = 4
    for j, (k, f, z) in enumerate([(2e4, 900.0, 0.03), (3e4, 1500.0, 0.02),
                                   (5e4, 2600.0, 0.02), (8e4, 3900.0, 0.01)]):
        four["x"][j] = (k, f, z)
    add({"arc_st": 0.0, "arc_ex": math.pi}, one, 9000.0)                     # slot
    add({"arc_st": 0.0, "arc_ex": math.acos(1 - 2 * 0.3)}, one, 11000.0)    # up 30 %
    add({"type": A.TOOL_BALL, "R": 4.0}, one, 14000.0)                     # ball end
    add({"N": 1}, one, 17000.0)
    add({"N": 8, "R": 8.0}, one, 6000.0)
    add({"helix_deg": 0.0, "N": 2, "arc_st": 0.0, "arc_ex": math.pi}, one, 12000.0)
    add({"mc": 0.25, "Ci": 1.5e5, "Ktc": 2100.0, "Krc": 850.0, "Kte": 35.0, "Kre": 45.0},
        one, 4000.0)                                                       # S50C-like, PD
    add({"runout": 0.008, "runout_phase": 1.0}, two, 10000.0)              # 2+2 modes
    add({"helix_deg": 45.0, "R": 1.5, "fz": 0.02}, four, 20000.0)          # long helix lag
    add({"arc_st": 3.5, "arc_ex": 4.0}, one, 8000.0)                       # arc past pi: empty
    add({"arc_st": math.pi / 2, "arc_ex": math.pi, "fz": 0.15}, one, 1500.0)  # thick chips
    setups = np.array([c[0] for c in cases], dtype=A.SETUP_DTYPE)
    modals = np.array([c[1] for c in cases], dtype=A.MODAL_DTYPE)
    pts = np.zeros(len(cases), dtype=A.POINT_DTYPE)
    pts["setup"] = np.arange(len(cases))
    pts["modal"] = np.arange(len(cases))
    pts["S"] = [c[2] for c in cases]
    # reference slice rule with aMax 24 -> up to 48 slices (two per lane); 30 revolutions
    opts = A.make_opts(aMin=0.05, aMax=24.0, iters=8, revs=30, nonlinear=True,
                       honorRunout=True)
    return W.Workload("edge", setups, modals, pts, opts, {})


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--only", default="")
    a = ap.parse_args(argv)
    th = a.threads or O.cpu_count()
    todo = (a.only.split(",") if a.only else
            ["small", "edge", "sweep", "hetero", "self", "spindle"])
    if "small" in todo:
        w = W.small()
        run(w, np.arange(w.n), th, HERE / "small.npz")
    if "edge" in todo:
        w = edge_workload()
        run(w, np.arange(w.n), th, HERE / "edge.npz")
    if "sweep" in todo:
        w = W.sweep()
        run(w, np.array(w.meta["fp64_subset"]), th, HERE / "sweep.npz")
    if "hetero" in todo:
        w = W.hetero()
        idx = np.sort(np.argsort(W.uniform(np.arange(w.n), 7, 0))[:256])
        run(w, idx, th, HERE / "hetero.npz")
    if "self" in todo:
        self_agreement(HERE / "self_agreement.npz", th)
    if "spindle" in todo:
        w = spindle_workload()
        run(w, np.arange(w.n), th, HERE / "spindle.npz")
    return 0


if __name__ == "__main__":
    sys.exit(main())
