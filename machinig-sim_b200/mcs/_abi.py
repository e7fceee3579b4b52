"""ctypes mirror of include/mcs.h and conversion from the reference's argument objects.

The reference passes plain JavaScript objects (src/stabtd.js:12-14, src/stabworker.js:6-14):

* ``tool``  ``{N, R, helixDeg, type, fluteLen, runout [um], runoutPhase}``
* ``modal`` ``{k [N/mm], fn [Hz], zeta, modesX?, modesY?}`` (src/frf.js:6-11)
* ``mat``   ``{Ktc, Krc, Kte, Kre, mc, Ci}`` (src/materials.js)
* ``arc``   ``[phiSt, phiEx]`` and ``fz`` [mm]

The helpers here turn such dicts into the C structs.  Units follow the engine
(src/cutting.js:37-43): the tool's runout arrives in micrometres as in the
Simulator's tool objects and is handed to the engine in millimetres.
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Any, Iterable, Mapping, Sequence

import numpy as np

MAX_MODES = 4
MAX_TEETH = 8
BINS = 180

MCS_OK = 0
MCS_ERR_ARG = 1
MCS_ERR_CUDA = 2
MCS_ERR_TIMEOUT = 3
MCS_ERR_DIVERGED = 4
MCS_ERR_CANCELLED = 5
MCS_ERR_NOMEM = 6
MCS_ERR_UNSUPPORTED = 7
MCS_ERR_STATE = 8

STATUS_NAMES = {
    MCS_OK: "MCS_OK",
    MCS_ERR_ARG: "MCS_ERR_ARG",
    MCS_ERR_CUDA: "MCS_ERR_CUDA",
    MCS_ERR_TIMEOUT: "MCS_ERR_TIMEOUT",
    MCS_ERR_DIVERGED: "MCS_ERR_DIVERGED",
    MCS_ERR_CANCELLED: "MCS_ERR_CANCELLED",
    MCS_ERR_NOMEM: "MCS_ERR_NOMEM",
    MCS_ERR_UNSUPPORTED: "MCS_ERR_UNSUPPORTED",
    MCS_ERR_STATE: "MCS_ERR_STATE",
}

TOOL_FLAT = 0
TOOL_BALL = 1


class Mode(C.Structure):
    _fields_ = [("k", C.c_double), ("fn", C.c_double), ("zeta", C.c_double)]


class Modal(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32),
                ("x", Mode * MAX_MODES), ("y", Mode * MAX_MODES)]


class Tool(C.Structure):
    _fields_ = [("N", C.c_int32), ("type", C.c_int32), ("R", C.c_double),
                ("helix_deg", C.c_double), ("flute_len", C.c_double),
                ("runout", C.c_double), ("runout_phase", C.c_double)]


class Material(C.Structure):
    _fields_ = [("Ktc", C.c_double), ("Krc", C.c_double), ("Kte", C.c_double),
                ("Kre", C.c_double), ("mc", C.c_double), ("Ci", C.c_double)]


class Setup(C.Structure):
    _fields_ = [("tool", Tool), ("mat", Material), ("arc_st", C.c_double),
                ("arc_ex", C.c_double), ("fz", C.c_double)]


class Point(C.Structure):
    _fields_ = [("setup", C.c_uint32), ("modal", C.c_uint32), ("S", C.c_double)]


class Opts(C.Structure):
    _fields_ = [("a_min", C.c_double), ("a_max", C.c_double), ("iters", C.c_int32),
                ("revs", C.c_int32), ("nonlinear", C.c_int32), ("honor_runout", C.c_int32),
                ("steps_per_tooth", C.c_int32), ("slices", C.c_int32),
                ("chatter_idx", C.c_double), ("precision", C.c_int32),
                ("max_buckets", C.c_int32), ("serial_trials", C.c_int32), ("coop_warps", C.c_int32),
                ("coop_points", C.c_int32), ("pad", C.c_int32)]


class Result(C.Structure):
    _fields_ = [("alim", C.c_double), ("lo", C.c_double), ("hi", C.c_double),
                ("open", C.c_int32), ("status", C.c_int32), ("trials", C.c_int32),
                ("steps_per_tooth", C.c_int32), ("evals", C.c_uint64),
                ("engaged", C.c_uint64)]


class Trial(C.Structure):
    _fields_ = [("point", C.c_uint32), ("pad", C.c_uint32), ("ap", C.c_double)]


class TrialResult(C.Structure):
    _fields_ = [("index", C.c_double), ("once", C.c_double), ("amp", C.c_double),
                ("chatter", C.c_int32), ("status", C.c_int32)]


class LobeQuery(C.Structure):
    _fields_ = [("N", C.c_int32), ("lobes", C.c_int32), ("Ktc", C.c_double),
                ("Krc", C.c_double), ("phi_st", C.c_double), ("phi_ex", C.c_double),
                ("rpm_min", C.c_double), ("rpm_max", C.c_double), ("modal", C.c_uint32),
                ("pad", C.c_uint32)]


class PlanInfo(C.Structure):
    _fields_ = [("blocks", C.c_int32), ("warps_per_sm", C.c_int32),
                ("smem_per_warp", C.c_int32), ("slots", C.c_int32), ("modes", C.c_int32),
                ("graph", C.c_int32), ("kernels", C.c_int32), ("coop_points", C.c_int32),
                ("n_points", C.c_uint64), ("h2d_bytes", C.c_uint64), ("d2h_bytes", C.c_uint64)]


class SpeedFrf(C.Structure):
    _fields_ = [("S", C.c_double), ("modes", Modal)]


class Spindle(C.Structure):
    _fields_ = [("rest", Modal), ("drop", C.c_double), ("s_ref", C.c_double),
                ("k_tool", C.c_double), ("k_sp", C.c_double), ("two_dof", C.c_int32),
                ("pad", C.c_int32), ("m_tool", C.c_double), ("m_sp", C.c_double),
                ("z_tool", C.c_double), ("z_sp", C.c_double)]


END_BINS, END_RINGS, MAX_SLICES = 36, 6, 64
ENGINE_HIST, ENGINE_TS = 4096, 64


class EngineConfig(C.Structure):
    _fields_ = [("tool", Tool), ("modal", Modal)] + [
        (n, C.c_double) for n in ("Ktc", "Krc", "Kac", "Kte", "Kre", "Kae", "mc", "Ci", "S",
                                  "fn_max")] + [("nonlinear", C.c_int32), ("decim", C.c_int32)]


class Engagement(C.Structure):
    _fields_ = [("Hb", C.c_float * 180), ("ux", C.c_double), ("uy", C.c_double),
                ("fz", C.c_double), ("tip_z", C.c_double), ("ap", C.c_double),
                ("profile", C.c_int32), ("wear", C.c_int32), ("Kte", C.c_double),
                ("Kre", C.c_double), ("slice_r", C.c_double * MAX_SLICES),
                ("slice_kap", C.c_double * MAX_SLICES),
                ("Eb", C.c_float * (END_BINS * END_RINGS)), ("fza", C.c_double),
                ("end_r", C.c_double), ("ring_z", C.c_double * END_RINGS),
                ("ring_zo", C.c_double * END_RINGS), ("ring_zi", C.c_double * END_RINGS),
                ("wall_k", C.c_double), ("wall_m", C.c_double), ("wall_zeta", C.c_double),
                ("wall_nx", C.c_double), ("wall_ny", C.c_double)]


ENGINE_STATS_FIELDS = ("n", "sumF", "maxF", "sumFx", "sumFy", "sumFz", "maxFz", "sumT",
                       "maxT", "sumX", "sumY", "minX", "maxX", "minY", "maxY", "sumZc", "wZc",
                       "sumW", "maxW", "sumHb", "sumB", "sumRb", "engTeeth")
ENGINE_STATS_DTYPE = np.dtype([(n, "<f8") for n in ENGINE_STATS_FIELDS])


class EngineState(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("x", "y", "vx", "vy", "t", "w", "wv", "dt",
                                          "run_mean_w")] + [
        (n, C.c_int32) for n in ("pr", "nz", "steps_per_tooth", "steps_per_rev", "max_slices",
                                 "decim")] + [("step_count", C.c_uint64)]


class Peaks(C.Structure):
    _fields_ = [("fp32_tflops", C.c_double), ("fp64_tflops", C.c_double),
                ("smem_tbps", C.c_double)]


# numpy views of the record arrays (same layout as the ctypes structs)
RESULT_DTYPE = np.dtype([("alim", "<f8"), ("lo", "<f8"), ("hi", "<f8"), ("open", "<i4"),
                         ("status", "<i4"), ("trials", "<i4"), ("steps_per_tooth", "<i4"),
                         ("evals", "<u8"), ("engaged", "<u8")])
TRIAL_RESULT_DTYPE = np.dtype([("index", "<f8"), ("once", "<f8"), ("amp", "<f8"),
                               ("chatter", "<i4"), ("status", "<i4")])
assert RESULT_DTYPE.itemsize == C.sizeof(Result)
assert TRIAL_RESULT_DTYPE.itemsize == C.sizeof(TrialResult)

DEFAULTS = {"aMin": 0.05, "aMax": 20.0, "iters": 8, "revs": 120, "nonlinear": True}
CHATTER_IDX = 0.45


def _modes(lst: Iterable[Mapping[str, float]] | None) -> list[tuple[float, float, float]]:
    if not lst:
        return []
    return [(float(m["k"]), float(m["fn"]), float(m["zeta"])) for m in lst]


def make_modal(modal: Mapping[str, Any]) -> Modal:
    """modeSet (src/frf.js:6-11): x = modesX or the single {k, fn, zeta}; y = modesY or x."""
    xs = _modes(modal.get("modesX"))
    if not xs:
        xs = [(float(modal["k"]), float(modal["fn"]), float(modal["zeta"]))]
    ys = _modes(modal.get("modesY"))
    if len(xs) > MAX_MODES or len(ys) > MAX_MODES:
        raise ValueError(f"at most {MAX_MODES} modes per axis")
    out = Modal()
    out.nx = len(xs)
    out.ny = len(ys)
    for i, (k, fn, z) in enumerate(xs):
        out.x[i] = Mode(k, fn, z)
    for i, (k, fn, z) in enumerate(ys):
        out.y[i] = Mode(k, fn, z)
    return out


def make_tool(tool: Mapping[str, Any]) -> Tool:
    t = Tool()
    t.N = int(tool["N"])
    t.type = TOOL_BALL if tool.get("type", "flat") == "ball" else TOOL_FLAT
    t.R = float(tool["R"]) if "R" in tool else float(tool["D"]) / 2
    t.helix_deg = float(tool.get("helixDeg", 30.0))
    t.flute_len = float(tool.get("fluteLen", 25.0))
    t.runout = float(tool.get("runout", 0.0) or 0.0) / 1000.0   # um -> mm
    t.runout_phase = float(tool.get("runoutPhase", 0.0) or 0.0)
    return t


def make_material(mat: Mapping[str, Any]) -> Material:
    return Material(float(mat["Ktc"]), float(mat["Krc"]), float(mat.get("Kte", 0.0)),
                    float(mat.get("Kre", 0.0)), float(mat.get("mc", 0.0) or 0.0),
                    float(mat.get("Ci", 0.0) or 0.0))


def make_setup(tool, mat, arc: Sequence[float], fz: float) -> Setup:
    return Setup(make_tool(tool), make_material(mat), float(arc[0]), float(arc[1]), float(fz))


def make_opts(o: Mapping[str, Any] | None = None, **kw) -> Opts:
    """timeDomainLimit/chatterAt options (src/stabtd.js:14,24) with the reference defaults,
    plus the explicit extensions honorRunout, stepsPerTooth, slices, chatterIdx,
    precision ("fp64", the default: FP64 force law and modal integration; "fp32"), maxBuckets
    (the schedule; 0 = the library's default, see mcs.tune), coopWarps (warps sharing the
    bisection of each of the heaviest points; 0 = the library's default, 1 = off),
    coopPoints (how many of the costliest points do so; 0 = one per SM) and serialTrials
    (True: one bisection trial at a time instead of speculative lane groups; same
    results)."""
    d = dict(DEFAULTS)
    if o:
        d.update(o)
    d.update(kw)
    return Opts(float(d["aMin"]), float(d["aMax"]), int(d["iters"]), int(d["revs"]),
                1 if d.get("nonlinear", True) is not False else 0,
                1 if d.get("honorRunout", False) else 0,
                int(d.get("stepsPerTooth", 0) or 0), int(d.get("slices", 0) or 0),
                float(d.get("chatterIdx", CHATTER_IDX)), precision_code(d.get("precision")),
                int(d.get("maxBuckets", 0) or 0), 1 if d.get("serialTrials", False) else 0,
                int(d.get("coopWarps", 0) or 0), int(d.get("coopPoints", 0) or 0), 0)


FP32 = 0
FP64 = 1
MAX_BUCKETS = 32


def precision_code(p) -> int:
    """None (the default) is FP64, the reference's own arithmetic: the mode whose limits
    meet the 2 % bar against it; FP32 integration is the faster variant."""
    if p in ("fp32", "f32", 0):
        return FP32
    if p is None or p in ("fp64", "f64", 1):
        return FP64
    raise ValueError(f"precision must be 'fp32' or 'fp64', not {p!r}")


def array_of(ctype, items: Sequence) -> C.Array:
    arr = (ctype * max(1, len(items)))()
    for i, it in enumerate(items):
        arr[i] = it
    return arr


def points_array(setup_idx, modal_idx, speeds) -> C.Array:
    """Point records from three equally long sequences (numpy-friendly)."""
    s = np.asarray(setup_idx, dtype=np.uint32)
    m = np.asarray(modal_idx, dtype=np.uint32)
    v = np.asarray(speeds, dtype=np.float64)
    n = len(v)
    arr = (Point * max(1, n))()
    rec = np.dtype([("setup", "<u4"), ("modal", "<u4"), ("S", "<f8")])
    view = np.frombuffer(arr, dtype=rec, count=n)
    view["setup"] = s
    view["modal"] = m
    view["S"] = v
    return arr


def result_view(arr, n: int) -> np.ndarray:
    return np.frombuffer(arr, dtype=RESULT_DTYPE, count=n)


def trial_result_view(arr, n: int) -> np.ndarray:
    return np.frombuffer(arr, dtype=TRIAL_RESULT_DTYPE, count=n)


def result_dict(r) -> dict:
    """The {alim, bracket} object timeDomainLimit returns (src/stabtd.js:25,31)."""
    hi = math.inf if r["open"] else float(r["hi"])
    return {"alim": float(r["alim"]), "bracket": [float(r["lo"]), hi]}


# numpy record layouts of the input structs (for building large batches without Python
# loops); checked against the ctypes mirror at import
MODE_DTYPE = np.dtype([("k", "<f8"), ("fn", "<f8"), ("zeta", "<f8")])
MODAL_DTYPE = np.dtype([("nx", "<i4"), ("ny", "<i4"), ("x", MODE_DTYPE, (MAX_MODES,)),
                        ("y", MODE_DTYPE, (MAX_MODES,))])
TOOL_DTYPE = np.dtype([("N", "<i4"), ("type", "<i4"), ("R", "<f8"), ("helix_deg", "<f8"),
                       ("flute_len", "<f8"), ("runout", "<f8"), ("runout_phase", "<f8")])
MATERIAL_DTYPE = np.dtype([("Ktc", "<f8"), ("Krc", "<f8"), ("Kte", "<f8"), ("Kre", "<f8"),
                           ("mc", "<f8"), ("Ci", "<f8")])
SETUP_DTYPE = np.dtype([("tool", TOOL_DTYPE), ("mat", MATERIAL_DTYPE), ("arc_st", "<f8"),
                        ("arc_ex", "<f8"), ("fz", "<f8")])
POINT_DTYPE = np.dtype([("setup", "<u4"), ("modal", "<u4"), ("S", "<f8")])
TRIAL_DTYPE = np.dtype([("point", "<u4"), ("pad", "<u4"), ("ap", "<f8")])
OPTS_DTYPE = np.dtype([("a_min", "<f8"), ("a_max", "<f8"), ("iters", "<i4"), ("revs", "<i4"),
                       ("nonlinear", "<i4"), ("honor_runout", "<i4"),
                       ("steps_per_tooth", "<i4"), ("slices", "<i4"), ("chatter_idx", "<f8"),
                       ("precision", "<i4"), ("max_buckets", "<i4"),
                       ("serial_trials", "<i4"), ("coop_warps", "<i4"),
                       ("coop_points", "<i4"), ("pad", "<i4")])
for _d, _c in ((MODAL_DTYPE, Modal), (SETUP_DTYPE, Setup), (POINT_DTYPE, Point),
               (TRIAL_DTYPE, Trial), (OPTS_DTYPE, Opts)):
    assert _d.itemsize == C.sizeof(_c), (_d, _c)


def as_records(items, dtype) -> np.ndarray:
    """ctypes struct array / list of structs / record ndarray -> contiguous record ndarray."""
    if isinstance(items, np.ndarray):
        if items.dtype != dtype:
            raise TypeError(f"expected records of {dtype}, got {items.dtype}")
        return np.ascontiguousarray(items)
    if isinstance(items, C.Array):
        return np.frombuffer(items, dtype=dtype).copy()
    out = np.zeros(len(items), dtype=dtype)
    raw = out.view(np.uint8).reshape(len(items), dtype.itemsize) if len(items) else None
    for i, it in enumerate(items):
        raw[i] = np.frombuffer(bytes(it), dtype=np.uint8)
    return out


def opts_record(o: Opts) -> np.ndarray:
    return np.frombuffer(bytes(o), dtype=OPTS_DTYPE).copy()


def opts_from_record(rec) -> Opts:
    """Opts from a stored record; records written before fields were added end early and
    the missing trailing fields read as 0 (their defaults)."""
    raw = np.asarray(rec).tobytes()
    return Opts.from_buffer_copy(raw + bytes(max(0, C.sizeof(Opts) - len(raw))))


# ---------------------------------------------------------------- surrogate
FEATURES = 20
PATH_GUIDED, PATH_FALLBACK, PATH_DIRECT, PATH_OPEN = 0, 1, 2, 3
PATH_NAMES = {PATH_GUIDED: "guided", PATH_FALLBACK: "fallback", PATH_DIRECT: "direct",
              PATH_OPEN: "open"}


class TrainOpts(C.Structure):
    _fields_ = [("epochs", C.c_int32), ("batch", C.c_int32), ("lr", C.c_float),
                ("beta1", C.c_float), ("beta2", C.c_float), ("eps", C.c_float),
                ("seed", C.c_uint64), ("warm", C.c_int32), ("keep_best", C.c_int32)]


class GuideOpts(C.Structure):
    _fields_ = [("z", C.c_float), ("hw_min", C.c_float), ("hw_max", C.c_float),
                ("hw_direct", C.c_float), ("refine", C.c_int32), ("mode", C.c_int32),
                ("levels", C.c_int32), ("skip_top", C.c_float)]


GUIDE_SPECULATE = 0
GUIDE_BRACKET = 1


class GuideInfo(C.Structure):
    _fields_ = [("mu", C.c_float), ("sigma", C.c_float), ("path", C.c_int32),
                ("rounds", C.c_int32)]


GUIDE_INFO_DTYPE = np.dtype([("mu", "<f4"), ("sigma", "<f4"), ("path", "<i4"),
                             ("rounds", "<i4")])
assert GUIDE_INFO_DTYPE.itemsize == C.sizeof(GuideInfo)
