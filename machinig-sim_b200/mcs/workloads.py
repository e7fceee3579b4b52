"""Seeded synthetic workloads of the stability benchmark.

There is no public dataset for this path: the reference's own tests use hand-set cases.
These generators build batches with the shapes, sizes and value ranges of the five
benchmark configurations.  Every random draw is a SplitMix64 hash of (seed, field), so a
setup is a pure function of its seed and any subset can be regenerated on its own.

  small       64 speeds, one deterministic setup, FP64-CPU-runnable
  sweep       4096 speeds over 3000-30000 rpm, 3 modes per axis, 10 um runout
  hetero      16384 seeded setups, process damping and size effect on
  train       262144 (setup, speed) points for surrogate labels, 90/10 split by seed
  serve       65536 queries, 30 % from seeds outside the training range
  spindle     the Worker's 18-speed lobe curve with each speed's own modes (spindle.js)

Fixed choices the benchmark leaves open: flute length 25 mm (the Simulator default,
src/sim.js:45); Kac = Kae = 0 (they act only on Fz); Kre = Kte * U(1.1, 1.5) and
Ci log-uniform 2e4-3e5 N/m (the spans of src/materials.js:25-32); runout phase
U(0, 2 pi); 60 revolutions per trial; 40 equal slices for "small"/"sweep", the
reference slice rule otherwise.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import _abi as A

MASK64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64(x: np.ndarray) -> np.ndarray:
    """SplitMix64 finaliser over a uint64 array (wrapping arithmetic)."""
    with np.errstate(over="ignore"):
        z = x.astype(np.uint64) + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def uniform(seed, stream: int, fld: int) -> np.ndarray:
    """U[0, 1) per seed for (stream, field): a pure function of its arguments."""
    s = np.asarray(seed, dtype=np.uint64)
    with np.errstate(over="ignore"):
        h = splitmix64(s ^ (np.uint64(stream) << np.uint64(40)))
        h = splitmix64(h + np.uint64(fld) * np.uint64(0x632BE59BD9B4E019))
    return (h >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def _u(seed, stream, fld, lo, hi):
    return lo + (hi - lo) * uniform(seed, stream, fld)


def _logu(seed, stream, fld, lo, hi):
    return np.exp(_u(seed, stream, fld, math.log(lo), math.log(hi)))


@dataclass
class Workload:
    name: str
    setups: np.ndarray          # SETUP_DTYPE records
    modals: np.ndarray          # MODAL_DTYPE records
    points: np.ndarray          # POINT_DTYPE records
    opts: A.Opts
    meta: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return len(self.points)

    def subset(self, idx) -> "Workload":
        idx = np.asarray(idx)
        return Workload(f"{self.name}[{len(idx)}]", self.setups, self.modals, self.points[idx],
                        self.opts, dict(self.meta, subset=len(idx)))


def immersion_arc(down: np.ndarray, r: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """identify.js immersion(): down [pi - pe, pi], up [0, pe], slot [0, pi] for r >= 1."""
    pe = np.arccos(np.clip(1 - 2 * r, -1.0, 1.0))
    st = np.where(r >= 1, 0.0, np.where(down, math.pi - pe, 0.0))
    ex = np.where(r >= 1, math.pi, np.where(down, math.pi, pe))
    return st, ex


def _base_setup(n: int) -> np.ndarray:
    s = np.zeros(n, dtype=A.SETUP_DTYPE)
    s["tool"]["N"] = 4
    s["tool"]["type"] = A.TOOL_FLAT
    s["tool"]["R"] = 5.0
    s["tool"]["helix_deg"] = 30.0
    s["tool"]["flute_len"] = 25.0
    s["mat"]["Ktc"] = 700.0
    s["mat"]["Krc"] = 210.0
    s["mat"]["Kte"] = 20.0
    s["mat"]["Kre"] = 30.0
    s["arc_st"] = math.pi - math.acos(1 - 2 * 0.5)  # 50 % down milling
    s["arc_ex"] = math.pi
    s["fz"] = 0.05
    return s


def small() -> Workload:
    """64 speeds 5000-20000 rpm; 4 flutes D10 helix 30; Ktc 700 Krc 210 Kte 20 Kre 30, no
    size effect or process damping; one mode per axis fn 1000 Hz, k 1e7 N/m, zeta 0.02;
    50 % down milling, fz 0.05; 40 slices, 200 steps per tooth, 60 revolutions;
    bisection [0.1, 10] x 10."""
    setups = _base_setup(1)
    modals = np.zeros(1, dtype=A.MODAL_DTYPE)
    modals["nx"] = 1
    modals["x"][0, 0] = (1e4, 1000.0, 0.02)
    points = np.zeros(64, dtype=A.POINT_DTYPE)
    points["S"] = np.linspace(5000.0, 20000.0, 64)
    opts = A.make_opts(aMin=0.1, aMax=10.0, iters=10, revs=60, nonlinear=False,
                       stepsPerTooth=200, slices=40)
    return Workload("small", setups, modals, points, opts,
                    {"speeds": 64, "rpm": [5000, 20000], "bisection": [0.1, 10, 10]})


def sweep(seed: int = 1, n_speeds: int = 4096) -> Workload:
    """One setup (small's tool and material, 10 um runout, seeded phase), 3 modes per axis
    fn U(600, 3000) Hz, k log-U(5e6, 5e7) N/m, zeta U(0.01, 0.05); n_speeds speeds over
    3000-30000 rpm with the reference step rule; 40 slices; [0.05, 15] x 10."""
    setups = _base_setup(1)
    setups["tool"]["runout"] = 0.010
    setups["tool"]["runout_phase"] = _u(seed, 1, 0, 0.0, 2 * math.pi)
    modals = np.zeros(1, dtype=A.MODAL_DTYPE)
    modals["nx"] = 3
    modals["ny"] = 3
    for a, ax in enumerate(("x", "y")):
        for j in range(3):
            f = 10 + 3 * (3 * a + j)
            modals[ax][0, j] = (_logu(seed, 1, f, 5e3, 5e4), _u(seed, 1, f + 1, 600.0, 3000.0),
                                _u(seed, 1, f + 2, 0.01, 0.05))
    points = np.zeros(n_speeds, dtype=A.POINT_DTYPE)
    points["S"] = np.linspace(3000.0, 30000.0, n_speeds)
    opts = A.make_opts(aMin=0.05, aMax=15.0, iters=10, revs=60, nonlinear=False,
                       honorRunout=True, slices=40)
    perm = np.argsort(uniform(np.arange(n_speeds), 2, seed))
    return Workload("sweep", setups, modals, points, opts,
                    {"speeds": n_speeds, "rpm": [3000, 30000], "bisection": [0.05, 15, 10],
                     "fp64_subset": np.sort(perm[:256]).tolist()})


def hetero_setups(seeds: np.ndarray) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Seeded setups of the heterogeneous batch: (setups, modals, per-setup speed)."""
    s = np.asarray(seeds, dtype=np.uint64)
    n = len(s)
    st = np.zeros(n, dtype=A.SETUP_DTYPE)
    D = _u(s, 3, 0, 3.0, 20.0)
    st["tool"]["N"] = 2 + np.minimum(4, (uniform(s, 3, 1) * 5).astype(np.int32))
    st["tool"]["type"] = A.TOOL_FLAT
    st["tool"]["R"] = D / 2
    st["tool"]["helix_deg"] = _u(s, 3, 2, 0.0, 45.0)
    st["tool"]["flute_len"] = 25.0
    st["tool"]["runout"] = _u(s, 3, 3, 0.0, 0.020)
    st["tool"]["runout_phase"] = _u(s, 3, 4, 0.0, 2 * math.pi)
    ktc = _u(s, 3, 5, 500.0, 2500.0)
    kte = _u(s, 3, 7, 10.0, 40.0)
    st["mat"]["Ktc"] = ktc
    st["mat"]["Krc"] = ktc * _u(s, 3, 6, 0.2, 0.5)
    st["mat"]["Kte"] = kte
    st["mat"]["Kre"] = kte * _u(s, 3, 8, 1.1, 1.5)
    st["mat"]["mc"] = _u(s, 3, 9, 0.2, 0.3)
    st["mat"]["Ci"] = _logu(s, 3, 10, 2e4, 3e5)
    r = _u(s, 3, 11, 0.05, 1.0)
    down = uniform(s, 3, 12) < 0.5
    st["arc_st"], st["arc_ex"] = immersion_arc(down, r)
    st["fz"] = _u(s, 3, 13, 0.02, 0.15)
    md = np.zeros(n, dtype=A.MODAL_DTYPE)
    md["nx"] = 1 + np.minimum(2, (uniform(s, 3, 14) * 3).astype(np.int32))
    md["ny"] = 1 + np.minimum(2, (uniform(s, 3, 15) * 3).astype(np.int32))
    for a, ax in enumerate(("x", "y")):
        for j in range(3):
            f = 20 + 3 * (3 * a + j)
            md[ax]["k"][:, j] = _logu(s, 3, f, 1e3, 1e5)
            md[ax]["fn"][:, j] = _u(s, 3, f + 1, 500.0, 4000.0)
            md[ax]["zeta"][:, j] = _u(s, 3, f + 2, 0.005, 0.05)
    # clear the unused mode slots so the records are canonical
    for ax, cnt in (("x", md["nx"]), ("y", md["ny"])):
        for j in range(3):
            off = cnt <= j
            md[ax]["k"][off, j] = 0
            md[ax]["fn"][off, j] = 0
            md[ax]["zeta"][off, j] = 0
    speed = _u(s, 3, 40, 3000.0, 30000.0)
    return st, md, speed


# the heterogeneous batches run FP32 integration: the surrogate's labels are FP32 limits and
# guided serving is compared with the plain FP32 bisection
HETERO_OPTS = dict(aMin=0.05, aMax=15.0, iters=10, revs=60, nonlinear=True, honorRunout=True,
                   precision="fp32")


def hetero(n: int = 16384, first_seed: int = 0) -> Workload:
    """n seeded setups, one point each: D U(3, 20), N in 2..6, helix U(0, 45), runout
    U(0, 20) um, Ktc U(500, 2500), Krc/Ktc U(0.2, 0.5), Kte U(10, 40), mc U(0.2, 0.3),
    1-3 modes per axis fn U(500, 4000) Hz, k log-U(1e6, 1e8) N/m, zeta U(0.005, 0.05),
    immersion U(0.05, 1) up or down, fz U(0.02, 0.15), S U(3000, 30000); process damping
    and size effect on; [0.05, 15] x 10."""
    seeds = np.arange(first_seed, first_seed + n, dtype=np.uint64)
    st, md, speed = hetero_setups(seeds)
    pts = np.zeros(n, dtype=A.POINT_DTYPE)
    pts["setup"] = np.arange(n)
    pts["modal"] = np.arange(n)
    pts["S"] = speed
    return Workload("hetero", st, md, pts, A.make_opts(HETERO_OPTS),
                    {"setups": n, "first_seed": first_seed})


def train(n_setups: int = 16384, speeds_per_setup: int = 16) -> Workload:
    """Surrogate labels: n_setups hetero setups x speeds_per_setup seeded speeds; the
    validation tenth is chosen by setup seed (meta["val_setup"])."""
    seeds = np.arange(n_setups, dtype=np.uint64)
    st, md, _ = hetero_setups(seeds)
    n = n_setups * speeds_per_setup
    pts = np.zeros(n, dtype=A.POINT_DTYPE)
    sidx = np.repeat(np.arange(n_setups), speeds_per_setup)
    j = np.tile(np.arange(speeds_per_setup), n_setups)
    pts["setup"] = sidx
    pts["modal"] = sidx
    pts["S"] = _u(sidx.astype(np.uint64) * np.uint64(64) + j.astype(np.uint64), 4, 0,
                  3000.0, 30000.0)
    val = uniform(seeds, 5, 0) < 0.1
    return Workload("train", st, md, pts, A.make_opts(HETERO_OPTS),
                    {"setups": n_setups, "speeds_per_setup": speeds_per_setup,
                     "val_setup": val})


def serve(n: int = 65536, train_setups: int = 16384, outside: float = 0.3) -> Workload:
    """Surrogate-guided serving queries: a fraction `outside` of the setups come from
    seeds past the training range, the rest from training seeds at fresh speeds."""
    q = np.arange(n, dtype=np.uint64)
    out = uniform(q, 6, 0) < outside
    seed = np.where(out, np.uint64(train_setups) + q,
                    (uniform(q, 6, 1) * train_setups).astype(np.uint64))
    st, md, _ = hetero_setups(seed)
    pts = np.zeros(n, dtype=A.POINT_DTYPE)
    pts["setup"] = np.arange(n)
    pts["modal"] = np.arange(n)
    pts["S"] = _u(q, 6, 2, 3000.0, 30000.0)
    perm = np.argsort(uniform(q, 6, 3))
    return Workload("serve", st, md, pts, A.make_opts(HETERO_OPTS),
                    {"queries": n, "outside": out, "fp64_subset": np.sort(perm[:512]).tolist()})


# Speed-dependent modes (src/spindle.js): the cases of the reference's spindle tests
# (test/spindle.test.mjs:47-49, 82-88, 98-103) on the Simulator's defaults (sim.js:44-46):
# a 3-flute D10 tool with a short stickout on a 50 kN/mm spindle that loses 25 % bearing
# stiffness at 30000 rpm; the same tool with a spindle/holder mode; and FRFs measured at
# 0 and 30000 rpm, interpolated between.
SPINDLE_CASES = {
    "chain": {"tool": {"D": 10.0, "stickout": 15.0, "kSpindle": 50000.0},
              "modal": {"auto": True, "k": 0.0, "fn": 0.0, "zeta": 0.04}},
    "spindle_mode": {"tool": {"D": 10.0, "stickout": 15.0, "kSpindle": 50000.0},
                     "modal": {"auto": True, "k": 0.0, "fn": 0.0, "zeta": 0.04},
                     "spindle_mode": {"on": True, "fn": 1200.0, "zeta": 0.05}},
    "measured": {"tool": {"D": 10.0, "stickout": 30.0, "kSpindle": 50000.0},
                 "modal": {"k": 10000.0, "fn": 3000.0, "zeta": 0.03, "speedFrfs": [
                     {"S": 0.0, "modesX": [{"k": 12000.0, "fn": 3000.0, "zeta": 0.03}]},
                     {"S": 30000.0, "modesX": [{"k": 9000.0, "fn": 2400.0, "zeta": 0.04}]}]}},
}


def spindle_sweep(speeds=None) -> Workload:
    """The Worker's lobe curve with speed-dependent modes (main.js:494-501): for each case
    of SPINDLE_CASES the 18 log-spaced speeds over 4000-30000 rpm, each point with the modal
    set sim.modalNow(S) gives (mcs.spindle); half-immersion down milling with the
    Simulator's A5052 (materials.js:25), fz 0.05 mm, 3 flutes, helix 30, flute length 12 mm
    (the 7.4 kHz tool mode of the two-mass case needs 888 steps per tooth at 4000 rpm, and
    a slot's surface window would not fit in shared memory); the reference's
    timeDomainLimit options ([0.05, 20] x 8, 120 revolutions, size effect and process
    damping)."""
    from . import spindle as SP

    speeds = SP.lobe_speeds() if speeds is None else list(speeds)
    names = list(SPINDLE_CASES)
    st = np.zeros(len(names), dtype=A.SETUP_DTYPE)
    st["tool"]["N"] = 3
    st["tool"]["type"] = A.TOOL_FLAT
    st["tool"]["R"] = 5.0
    st["tool"]["helix_deg"] = 30.0
    st["tool"]["flute_len"] = 12.0
    st["mat"]["Ktc"], st["mat"]["Krc"] = 700.0, 210.0
    st["mat"]["Kte"], st["mat"]["Kre"] = 20.0, 25.0
    st["mat"]["mc"], st["mat"]["Ci"] = 0.10, 2e4
    st["arc_st"], st["arc_ex"] = math.pi / 2, math.pi
    st["fz"] = 0.05
    modals, pts = [], []
    for c, name in enumerate(names):
        case = SPINDLE_CASES[name]
        sp = SP.Spindle.from_tool(case["tool"], case["modal"],
                                  spindle_mode=case.get("spindle_mode"))
        for j, r in enumerate(sp.modes_at(speeds)):
            pts.append((c, len(modals), speeds[j]))
            modals.append(r)
    points = np.zeros(len(pts), dtype=A.POINT_DTYPE)
    points["setup"] = [p[0] for p in pts]
    points["modal"] = [p[1] for p in pts]
    points["S"] = [p[2] for p in pts]
    return Workload("spindle", st, np.array(modals, dtype=A.MODAL_DTYPE), points,
                    A.make_opts(), {"cases": names, "speeds": speeds})


CONFIGS = {"small": small, "sweep": sweep, "hetero": hetero, "train": train, "serve": serve}
