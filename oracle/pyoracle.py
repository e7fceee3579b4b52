"""ctypes wrapper of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and the cpu_baseline leg of
bench.py use it as the checker.  The oracle restates the reference's JavaScript hot path
in FP64 (see oracle/oracle.h for the file:line map); the product never calls it.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess
import sys
from pathlib import Path
from typing import Sequence

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
sys.path.insert(0, str(ROOT / "machinig-sim_b200"))

from mcs import _abi as A  # noqa: E402  (struct layouts of include/mcs.h)

_LIB = None


class Stats(C.Structure):
    _fields_ = [(n, C.c_double) for n in
                ("n", "sumF", "maxF", "sumFx", "sumFy", "sumX", "sumY", "engTeeth")]


class EngineInfo(C.Structure):
    _fields_ = [("steps_per_tooth", C.c_int32), ("steps_per_rev", C.c_int32),
                ("nz", C.c_int32), ("decim", C.c_int32), ("max_slices", C.c_int32),
                ("pad", C.c_int32), ("dt", C.c_double), ("omega", C.c_double),
                ("dz", C.c_double)]


class TraceEntry(C.Structure):
    _fields_ = [("ap", C.c_double), ("index", C.c_double), ("once", C.c_double),
                ("amp", C.c_double), ("chatter", C.c_int32), ("pad", C.c_int32)]


class SdmParams(C.Structure):
    _fields_ = [("m", C.c_double), ("k", C.c_double), ("zeta", C.c_double),
                ("Kt", C.c_double), ("Kn", C.c_double), ("N", C.c_int32),
                ("steps", C.c_int32), ("phi_st", C.c_double), ("phi_ex", C.c_double),
                ("rpm", C.c_double)]


TRACE_DTYPE = np.dtype([("ap", "<f8"), ("index", "<f8"), ("once", "<f8"), ("amp", "<f8"),
                        ("chatter", "<i4"), ("pad", "<i4")])


def build() -> Path:
    """Compile liboracle.so with its Makefile (g++)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return HERE / "liboracle.so"


def lib():
    global _LIB
    if _LIB is not None:
        return _LIB
    path = HERE / "liboracle.so"
    if not path.exists():
        build()
    L = C.CDLL(str(path))
    P = C.POINTER
    L.or_engine_new.restype = C.c_void_p
    L.or_engine_free.argtypes = [C.c_void_p]
    L.or_engine_configure.argtypes = [C.c_void_p, P(A.Tool), C.c_int, P(A.Modal), P(A.Material),
                                      C.c_double, C.c_double, C.c_int, C.c_int]
    L.or_engine_hb.restype = P(C.c_float)
    L.or_engine_hb.argtypes = [C.c_void_p]
    L.or_engine_set_engagement.argtypes = [C.c_void_p] + [C.c_double] * 5
    L.or_engine_set_state.argtypes = [C.c_void_p] + [C.c_double] * 4
    L.or_engine_run.argtypes = [C.c_void_p, C.c_int64]
    L.or_engine_chatter_index.argtypes = [C.c_void_p, P(C.c_double)]
    L.or_engine_take_stats.argtypes = [C.c_void_p, P(Stats)]
    L.or_engine_chip_vols.argtypes = [C.c_void_p, P(C.c_double), C.c_int]
    L.or_engine_chip_vols.restype = C.c_int
    L.or_engine_get_info.argtypes = [C.c_void_p, P(EngineInfo)]
    L.or_chatter_at.argtypes = [P(A.Setup), P(A.Modal), C.c_double, C.c_double, P(A.Opts),
                                P(A.TrialResult)]
    L.or_time_domain_limit.argtypes = [P(A.Setup), P(A.Modal), C.c_double, P(A.Opts),
                                       P(A.Result), C.c_void_p]
    L.or_solve_batch.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, P(A.Opts),
                                 C.c_void_p, C.c_void_p, C.c_int]
    L.or_chatter_batch.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t,
                                   P(A.Opts), C.c_void_p, C.c_int]
    L.or_frf.argtypes = [P(A.Mode), C.c_int, C.c_double, P(C.c_double)]
    L.or_static_k.argtypes = [P(A.Mode), C.c_int]
    L.or_static_k.restype = C.c_double
    L.or_dominant.argtypes = [P(A.Mode), C.c_int]
    L.or_dominant.restype = C.c_int
    L.or_directional_coeffs.argtypes = [C.c_double] * 3 + [P(C.c_double)]
    L.or_stability_lobes.argtypes = [P(A.LobeQuery), P(A.Modal), P(C.c_double), P(C.c_double),
                                     P(C.c_int32), C.c_int]
    L.or_stability_lobes.restype = C.c_int
    L.or_lobes_alim.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, P(C.c_double), C.c_size_t,
                                P(C.c_double)]
    L.or_fit_modes.argtypes = [P(C.c_double)] * 3 + [C.c_int, C.c_int, P(A.Mode)]
    L.or_fit_modes.restype = C.c_int
    L.or_sdm_rho.argtypes = [P(SdmParams), C.c_double]
    L.or_sdm_rho.restype = C.c_double
    L.or_sdm_limit.argtypes = [P(SdmParams), C.c_double]
    L.or_sdm_limit.restype = C.c_double
    L.or_tool_model.argtypes = [C.c_double] * 4 + [P(C.c_double)]
    L.or_immersion.argtypes = [C.c_int, C.c_double, C.c_double, P(C.c_double)]
    L.or_engine_set_axial.argtypes = [C.c_void_p, C.c_double, C.c_double]
    L.or_engine_set_wear.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double]
    L.or_engine_eb.restype = P(C.c_float)
    L.or_engine_eb.argtypes = [C.c_void_p]
    L.or_engine_set_end.argtypes = [C.c_void_p, C.c_double, C.c_double] + [P(C.c_double)] * 3
    L.or_engine_set_work.argtypes = [C.c_void_p] + [C.c_double] * 5
    L.or_engine_set_engagement_profile.argtypes = [C.c_void_p] + [C.c_double] * 5 + [
        P(C.c_double)] * 2
    L.or_engine_take_stats_full.argtypes = [C.c_void_p, C.c_void_p]
    L.or_engine_history.argtypes = [C.c_void_p, C.c_void_p, P(C.c_int32), P(C.c_int64)]
    L.or_engine_reset_history.argtypes = [C.c_void_p]
    L.or_engine_set_decim.argtypes = [C.c_void_p, C.c_int]
    L.or_modes_at.argtypes = [P(A.Spindle), C.c_void_p, C.c_size_t, P(C.c_double), C.c_size_t,
                              C.c_void_p]
    L.or_modes_at.restype = None
    _LIB = L
    return L


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


# ---------------------------------------------------------------- engine
class Engine:
    """CuttingEngine restatement driven the way the reference tests drive it."""

    def __init__(self):
        self._L = lib()
        self._h = C.c_void_p(self._L.or_engine_new())

    def __del__(self):
        try:
            self._L.or_engine_free(self._h)
        except Exception:
            pass

    def configure(self, tool: dict, modal: dict, mat: dict, S: float, fn_max: float = 0.0,
                  steps_per_tooth: int = 0, slices: int = 0):
        """tool: engine units (runout in mm, cutting.js:43); nonlinear read from the tool."""
        t = A.Tool()
        t.N = int(tool["N"])
        t.type = A.TOOL_BALL if tool.get("type", "flat") == "ball" else A.TOOL_FLAT
        t.R = float(tool["R"])
        t.helix_deg = float(tool.get("helixDeg", 0.0))
        t.flute_len = float(tool["fluteLen"])
        t.runout = float(tool.get("runout", 0.0) or 0.0)
        t.runout_phase = float(tool.get("runoutPhase", 0.0) or 0.0)
        nl = 0 if tool.get("nonlinear", True) is False else 1
        self._L.or_engine_configure(self._h, C.byref(t), nl, C.byref(A.make_modal(modal)),
                                    C.byref(A.make_material(mat)), float(S), float(fn_max),
                                    int(steps_per_tooth), int(slices))

    @property
    def Hb(self) -> np.ndarray:
        p = self._L.or_engine_hb(self._h)
        return np.ctypeslib.as_array(p, shape=(A.BINS,))

    def set_engagement(self, u, fz, tipZ, ap):
        self._L.or_engine_set_engagement(self._h, float(u[0]), float(u[1]), float(fz),
                                         float(tipZ), float(ap))

    def set_state(self, x=0.0, y=0.0, vx=0.0, vy=0.0):
        self._L.or_engine_set_state(self._h, x, y, vx, vy)

    def run(self, n: int):
        self._L.or_engine_run(self._h, int(n))

    def chatter_index(self) -> dict:
        out = (C.c_double * 3)()
        self._L.or_engine_chatter_index(self._h, out)
        return {"index": out[0], "amp": out[1], "once": out[2]}

    def take_stats(self) -> dict:
        s = Stats()
        self._L.or_engine_take_stats(self._h, C.byref(s))
        return {n: getattr(s, n) for n, _ in Stats._fields_}

    def chip_vols(self) -> list[float]:
        n = self._L.or_engine_chip_vols(self._h, None, 0)
        buf = (C.c_double * max(1, n))()
        self._L.or_engine_chip_vols(self._h, buf, n)
        return list(buf[:n])

    def info(self) -> dict:
        i = EngineInfo()
        self._L.or_engine_get_info(self._h, C.byref(i))
        return {n: getattr(i, n) for n, _ in EngineInfo._fields_}

    # the playback / identification terms, driven by the library's record types
    def configure_from(self, c: A.EngineConfig):
        """configure() from an mcs_engine_config record (the same inputs the GPU engine
        gets), the axial coefficients and the decimation with it."""
        mat = A.Material(c.Ktc, c.Krc, c.Kte, c.Kre, c.mc, c.Ci)
        self._L.or_engine_configure(self._h, C.byref(c.tool), int(c.nonlinear),
                                    C.byref(c.modal), C.byref(mat), c.S, c.fn_max, 0, 0)
        self._L.or_engine_set_axial(self._h, c.Kac, c.Kae)
        if c.decim > 0:
            self._L.or_engine_set_decim(self._h, int(c.decim))

    def engage(self, g: A.Engagement):
        """setEngagement, setEndEngagement, setWork and setWear from an mcs_engagement."""
        self.Hb[:] = np.frombuffer(bytes(g.Hb), dtype=np.float32)
        r = np.frombuffer(bytes(g.slice_r), dtype=np.float64).copy()
        k = np.frombuffer(bytes(g.slice_kap), dtype=np.float64).copy()
        if g.profile:
            self._L.or_engine_set_engagement_profile(self._h, g.ux, g.uy, g.fz, g.tip_z, g.ap,
                                                     _dptr(r), _dptr(k))
        else:
            self.set_engagement((g.ux, g.uy), g.fz, g.tip_z, g.ap)
        eb = np.ctypeslib.as_array(self._L.or_engine_eb(self._h), shape=(36 * 6,))
        eb[:] = np.frombuffer(bytes(g.Eb), dtype=np.float32)
        rz = [np.frombuffer(bytes(a), dtype=np.float64).copy() for a in (g.ring_z, g.ring_zo,
                                                                          g.ring_zi)]
        self._L.or_engine_set_end(self._h, g.fza, g.end_r, *[_dptr(a) for a in rz])
        self._L.or_engine_set_work(self._h, g.wall_k, g.wall_m, g.wall_zeta, g.wall_nx,
                                   g.wall_ny)
        self._L.or_engine_set_wear(self._h, int(g.wear), g.Kte, g.Kre)

    def take_stats_full(self) -> np.ndarray:
        out = np.zeros(1, dtype=A.ENGINE_STATS_DTYPE)
        self._L.or_engine_take_stats_full(self._h, C.c_void_p(out.ctypes.data))
        return out[0]

    def history(self):
        out = np.zeros((5, A.ENGINE_HIST), dtype=np.float32)
        head, count = C.c_int32(), C.c_int64()
        self._L.or_engine_history(self._h, C.c_void_p(out.ctypes.data), C.byref(head),
                                  C.byref(count))
        return out, head.value, count.value

    def reset_history(self):
        self._L.or_engine_reset_history(self._h)


# ---------------------------------------------------------------- stabtd.js
def chatter_at(setup: A.Setup, modal: A.Modal, S: float, ap: float, opts: A.Opts) -> dict:
    r = A.TrialResult()
    lib().or_chatter_at(C.byref(setup), C.byref(modal), S, ap, C.byref(opts), C.byref(r))
    return {"index": r.index, "once": r.once, "amp": r.amp, "chatter": bool(r.chatter)}


def time_domain_limit(setup: A.Setup, modal: A.Modal, S: float, opts: A.Opts,
                      trace: bool = False):
    r = A.Result()
    tr = (TraceEntry * (opts.iters + 1))() if trace else None
    lib().or_time_domain_limit(C.byref(setup), C.byref(modal), S, C.byref(opts), C.byref(r),
                               C.cast(tr, C.c_void_p) if trace else None)
    res = A.result_dict({"alim": r.alim, "lo": r.lo, "hi": r.hi, "open": r.open})
    if trace:
        res["trace"] = np.frombuffer(tr, dtype=TRACE_DTYPE, count=r.trials).copy()
    return res


def timeDomainLimit(tool, modal, mat, S, arc, fz, opts=None):
    """Same call shape as src/stabtd.js:24 (tool.runout in um)."""
    o = A.make_opts(opts)
    return time_domain_limit(A.make_setup(tool, mat, arc, fz), A.make_modal(modal), S, o)


def solve_batch(setups: Sequence[A.Setup], modals: Sequence[A.Modal], points, opts: A.Opts,
                nthreads: int = 0, traces: bool = False):
    """Thread-pool batch; returns (results ndarray, traces ndarray[n, iters+1] or None)."""
    S = A.array_of(A.Setup, setups)
    M = A.array_of(A.Modal, modals)
    n = len(points) if not isinstance(points, C.Array) else len(points)
    out = (A.Result * max(1, n))()
    per = opts.iters + 1
    tr = (TraceEntry * max(1, n * per))() if traces else None
    lib().or_solve_batch(C.cast(S, C.c_void_p), C.cast(M, C.c_void_p), C.cast(points, C.c_void_p),
                         n, C.byref(opts), C.cast(out, C.c_void_p),
                         C.cast(tr, C.c_void_p) if traces else None, int(nthreads))
    res = A.result_view(out, n).copy()
    trv = np.frombuffer(tr, dtype=TRACE_DTYPE, count=n * per).reshape(n, per).copy() if traces else None
    return res, trv


def chatter_batch(setups, modals, points, trials, opts: A.Opts, nthreads: int = 0):
    S = A.array_of(A.Setup, setups)
    M = A.array_of(A.Modal, modals)
    n = len(trials)
    out = (A.TrialResult * max(1, n))()
    lib().or_chatter_batch(C.cast(S, C.c_void_p), C.cast(M, C.c_void_p), C.cast(points, C.c_void_p),
                           C.cast(trials, C.c_void_p), n, C.byref(opts), C.cast(out, C.c_void_p),
                           int(nthreads))
    return A.trial_result_view(out, n).copy()


# ---------------------------------------------------------------- frf.js / sld.js
def frf(modes, f):
    arr = A.array_of(A.Mode, [A.Mode(m["k"], m["fn"], m["zeta"]) for m in modes])
    out = (C.c_double * 2)()
    lib().or_frf(arr, len(modes), float(f), out)
    return [out[0], out[1]]


def directional_coeffs(Kr, phiSt, phiEx):
    out = (C.c_double * 4)()
    lib().or_directional_coeffs(Kr, phiSt, phiEx, out)
    return dict(zip(("xx", "xy", "yx", "yy"), out))


def lobe_query(N, Ktc, Krc, phiSt, phiEx, lobes=8, rpmMin=1000, rpmMax=40000, modal=0):
    return A.LobeQuery(int(N), int(lobes), float(Ktc), float(Krc), float(phiSt), float(phiEx),
                       float(rpmMin), float(rpmMax), int(modal), 0)


def stabilityLobes(params: dict):
    """stabilityLobes(params) of src/sld.js:23 -> list of lobes [[{rpm, alim}]]."""
    p = dict(params)
    q = lobe_query(p["N"], p["Ktc"], p["Krc"], p["phiSt"], p["phiEx"], p.get("lobes", 8),
                   p.get("rpmMin", 1000), p.get("rpmMax", 40000))
    modal = A.make_modal(p)
    cap = 400 * 4 * 2 * max(1, q.lobes)
    rpm = (C.c_double * cap)()
    alim = (C.c_double * cap)()
    lens = (C.c_int32 * max(1, q.lobes))()
    n = lib().or_stability_lobes(C.byref(q), C.byref(modal), rpm, alim, lens, cap)
    out, pos = [], 0
    for j in range(n):
        out.append([{"rpm": rpm[pos + i], "alim": alim[pos + i]} for i in range(lens[j])])
        pos += lens[j]
    return out


def alimAt(lobes, rpm):
    """alimAt of src/sld.js:64 over the lobe lists stabilityLobes returns."""
    best = math.inf
    for lobe in lobes:
        for i in range(1, len(lobe)):
            a, b = lobe[i - 1], lobe[i]
            if a["rpm"] <= rpm <= b["rpm"]:
                span = b["rpm"] - a["rpm"]
                t = (rpm - a["rpm"]) / (span if span != 0 else 1)
                best = min(best, a["alim"] + (b["alim"] - a["alim"]) * t)
    return best


def lobes_alim(modals, queries, rpms):
    M = A.array_of(A.Modal, modals)
    Q = A.array_of(A.LobeQuery, queries)
    r = np.ascontiguousarray(rpms, dtype=np.float64)
    out = np.zeros(len(queries) * len(r))
    lib().or_lobes_alim(C.cast(M, C.c_void_p), C.cast(Q, C.c_void_p), len(queries), _dptr(r),
                        len(r), _dptr(out))
    return out.reshape(len(queries), len(r))


def fit_modes(f, G, max_modes=4):
    f = np.ascontiguousarray(f, dtype=np.float64)
    re = np.ascontiguousarray([g[0] for g in G], dtype=np.float64)
    im = np.ascontiguousarray([g[1] for g in G], dtype=np.float64)
    out = (A.Mode * max_modes)()
    n = lib().or_fit_modes(_dptr(f), _dptr(re), _dptr(im), len(f), max_modes, out)
    return [{"k": out[i].k, "fn": out[i].fn, "zeta": out[i].zeta} for i in range(n)]


# ---------------------------------------------------------------- sdm / tool
def sdm_limit(m, k, zeta, Kt, Kn, N, phiSt, phiEx, rpm, steps=40, a_max=0.02):
    p = SdmParams(m, k, zeta, Kt, Kn, N, steps, phiSt, phiEx, rpm)
    return lib().or_sdm_limit(C.byref(p), a_max)


def sdm_rho(m, k, zeta, Kt, Kn, N, phiSt, phiEx, rpm, a, steps=40):
    p = SdmParams(m, k, zeta, Kt, Kn, N, steps, phiSt, phiEx, rpm)
    return lib().or_sdm_rho(C.byref(p), a)


def tool_model(D, stickout, kSpindle, mHolder=0.05):
    out = (C.c_double * 4)()
    lib().or_tool_model(D, stickout, kSpindle, mHolder, out)
    return {"k": out[0], "fn": out[1], "kTool": out[2], "mEff": out[3]}


def immersion(mode: str, ae: float, D: float):
    out = (C.c_double * 2)()
    lib().or_immersion({"slot": 0, "down": 1, "up": 2}[mode], ae, D, out)
    return [out[0], out[1]]


def cpu_count() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


# ---------------------------------------------------------------- spindle.js
def modes_at(spindle: A.Spindle, speeds, frfs=()) -> np.ndarray:
    """modesAt (src/spindle.js:64-85) at each speed: MODAL_DTYPE records."""
    S = np.ascontiguousarray(speeds, dtype=np.float64)
    F = A.array_of(A.SpeedFrf, list(frfs))
    out = np.zeros(max(1, len(S)), dtype=A.MODAL_DTYPE)
    lib().or_modes_at(C.byref(spindle), C.cast(F, C.c_void_p), len(frfs), _dptr(S), len(S),
                      C.c_void_p(out.ctypes.data))
    return out[: len(S)]


LOBE_NODE, LOBE_STEP = 1000, 25  # src/sim.js:37


def composite_lobes(spindle: A.Spindle, params: dict, frfs=()):
    """Simulator.lobes for speed-dependent dynamics (src/sim.js:269-285): a diagram per
    LOBE_NODE with the modes at the node's centre, each read every LOBE_STEP across its own
    node, Infinity read as 1e3; returns [curve]."""
    base = {"lobes": 30, "rpmMin": 2000, "rpmMax": 40000, **params}
    curve = []
    lo, hi = base["rpmMin"] * 0.8, base["rpmMax"] * 1.1
    S0 = lo
    while S0 < hi:
        m = modes_at(spindle, [S0 + LOBE_NODE / 2], frfs)[0]
        own = {**base, "rpmMin": S0, "rpmMax": S0 + LOBE_NODE, "k": 0, "fn": 0, "zeta": 0,
               "modesX": [{"k": x["k"], "fn": x["fn"], "zeta": x["zeta"]} for x in m["x"][: m["nx"]]],
               "modesY": [{"k": y["k"], "fn": y["fn"], "zeta": y["zeta"]} for y in m["y"][: m["ny"]]]}
        lob = stabilityLobes(own)
        S = S0
        while S < min(hi, S0 + LOBE_NODE):
            a = alimAt(lob, S)
            curve.append({"rpm": S, "alim": 1e3 if a == math.inf else a})
            S += LOBE_STEP
        S0 += LOBE_NODE
    return [curve]


# ---------------------------------------------------------------- identify.js / validate.js
def _rigid_engine(cfg, g):
    e = Engine()
    e.configure_from(cfg)
    e.engage(g)
    return e


def unit_forces_ref(cfgs, gs):
    """unitForces (src/identify.js:26-40) per prepared (config, engagement) pair: two
    revolutions, takeStats, one revolution; the mean force on the workpiece (-sum/n)."""
    out = []
    for c, g in zip(cfgs, gs):
        e = _rigid_engine(c, g)
        spr = e.info()["steps_per_rev"]
        e.run(2 * spr)
        e.take_stats_full()
        e.run(spr)
        s = e.take_stats_full()
        out.append([-s["sumFx"] / s["n"], -s["sumFy"] / s["n"], -s["sumFz"] / s["n"]])
    return np.array(out)


def sim_revolution_ref(cfg, g, nb=360):
    """simRevolution (src/validate.js:76-100) for a prepared (config, engagement) pair whose
    config samples every step: two revolutions, the history emptied, one revolution, then
    the history interpolated onto nb angle bins (force on the workpiece)."""
    e = _rigid_engine(cfg, g)
    n = e.info()["steps_per_rev"]
    e.run(2 * n)
    e.reset_history()
    e.run(n)
    h, _, _ = e.history()
    out = np.zeros((3, nb))
    for c in range(3):
        for b in range(nb):
            x = (b + 0.5) / nb * n - 0.5
            i0 = math.floor(x)
            f = x - i0
            a, cc = float(h[c][(i0 + n) % n]), float(h[c][(i0 + 1) % n])
            out[c][b] = -(a + (cc - a) * f)
    return out
