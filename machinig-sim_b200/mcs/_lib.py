"""ctypes binding of libmcs.so (include/mcs.h) and the Context that owns a device.

The library is the only compute path: if libmcs.so is missing or no CUDA device is
present, every call raises -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import threading
import weakref
from pathlib import Path
from typing import Sequence

import numpy as np

from . import _abi as A

PKG = Path(__file__).resolve().parent.parent
LIB_PATH = PKG / "libmcs.so"

# every symbol include/mcs.h declares
EXPORTS = (
    "mcs_default_opts", "mcs_last_error", "mcs_create", "mcs_destroy", "mcs_stream",
    "mcs_solve", "mcs_chatter_at", "mcs_plan_create", "mcs_plan_execute", "mcs_plan_results",
    "mcs_plan_info_get", "mcs_plan_destroy", "mcs_solve_async", "mcs_job_poll",
    "mcs_job_cancel", "mcs_job_wait", "mcs_job_free", "mcs_lobes_alim", "mcs_solve_noalloc",
    "mcs_default_train_opts", "mcs_default_guide_opts", "mcs_features", "mcs_surrogate_create",
    "mcs_surrogate_destroy", "mcs_surrogate_train", "mcs_surrogate_predict", "mcs_surrogate_grad",
    "mcs_surrogate_get_params", "mcs_surrogate_set_params", "mcs_solve_guided",
    "mcs_plan_create_guided", "mcs_plan_guide_info", "mcs_tune", "mcs_measure_peaks",
    "mcs_modes_at", "mcs_lobes_composite", "mcs_curve_alim", "mcs_solve_multi", "mcs_shard",
    "mcs_engine_create", "mcs_engine_destroy", "mcs_engine_configure", "mcs_engine_set_engagement",
    "mcs_engine_set_state", "mcs_engine_run", "mcs_engine_take_stats", "mcs_engine_get_state",
    "mcs_engine_history", "mcs_engine_reset_history", "mcs_engine_chatter_index",
)
_VOID = ("mcs_default_opts", "mcs_last_error", "mcs_stream", "mcs_job_free",
         "mcs_default_train_opts", "mcs_default_guide_opts")

_LIB = None
_LOCK = threading.Lock()


class MCSError(RuntimeError):
    """A non-OK mcs_status, with mcs_last_error()'s message."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{A.STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def load(path: Path | str | None = None):
    """Load libmcs.so and declare its prototypes (raises if it is not built)."""
    global _LIB
    with _LOCK:
        if _LIB is not None and path is None:
            return _LIB
        p = Path(path) if path else LIB_PATH
        if not p.exists():
            raise ImportError(f"{p} is not built: run `python machinig-sim_b200/build.py`")
        L = C.CDLL(str(p))
        P = C.POINTER
        vp = C.c_void_p
        L.mcs_default_opts.argtypes = [P(A.Opts)]
        L.mcs_default_opts.restype = None
        L.mcs_last_error.restype = C.c_char_p
        L.mcs_create.argtypes = [P(vp), C.c_int]
        L.mcs_destroy.argtypes = [vp]
        L.mcs_stream.argtypes = [vp]
        L.mcs_stream.restype = vp
        batch = [vp, vp, C.c_size_t, vp, C.c_size_t, vp, C.c_size_t, P(A.Opts)]
        L.mcs_solve.argtypes = batch + [vp]
        L.mcs_chatter_at.argtypes = [vp, vp, C.c_size_t, vp, C.c_size_t, vp, C.c_size_t, vp,
                                     C.c_size_t, P(A.Opts), vp]
        L.mcs_plan_create.argtypes = batch + [P(vp)]
        L.mcs_plan_execute.argtypes = [vp]
        L.mcs_plan_results.argtypes = [vp, vp]
        L.mcs_plan_info_get.argtypes = [vp, P(A.PlanInfo)]
        L.mcs_plan_destroy.argtypes = [vp]
        L.mcs_solve_async.argtypes = batch + [vp, P(vp)]
        L.mcs_job_poll.argtypes = [vp, P(C.c_size_t), P(C.c_int)]
        L.mcs_job_cancel.argtypes = [vp]
        L.mcs_job_wait.argtypes = [vp]
        L.mcs_job_free.argtypes = [vp]
        L.mcs_job_free.restype = None
        L.mcs_lobes_alim.argtypes = [vp, vp, C.c_size_t, vp, C.c_size_t, vp, C.c_size_t, vp]
        L.mcs_tune.argtypes = batch + [vp, C.c_size_t, vp, P(C.c_int32)]
        L.mcs_solve_noalloc.argtypes = batch + [vp]
        L.mcs_default_train_opts.argtypes = [P(A.TrainOpts)]
        L.mcs_default_train_opts.restype = None
        L.mcs_default_guide_opts.argtypes = [P(A.GuideOpts)]
        L.mcs_default_guide_opts.restype = None
        L.mcs_features.argtypes = batch[1:] + [vp]
        L.mcs_surrogate_create.argtypes = [vp, C.c_uint64, P(vp)]
        L.mcs_surrogate_destroy.argtypes = [vp]
        L.mcs_surrogate_train.argtypes = [vp, vp, vp, C.c_size_t, vp, vp, C.c_size_t,
                                          P(A.TrainOpts), vp, vp]
        L.mcs_surrogate_predict.argtypes = [vp, vp, C.c_size_t, vp, vp]
        L.mcs_surrogate_grad.argtypes = [vp, vp, vp, C.c_size_t, vp, vp]
        L.mcs_surrogate_get_params.argtypes = [vp, vp, P(C.c_size_t)]
        L.mcs_surrogate_set_params.argtypes = [vp, vp, C.c_size_t]
        L.mcs_solve_guided.argtypes = [vp, vp] + batch[1:] + [P(A.GuideOpts), vp, vp]
        L.mcs_plan_create_guided.argtypes = [vp, vp] + batch[1:] + [P(A.GuideOpts), P(vp)]
        L.mcs_plan_guide_info.argtypes = [vp, vp]
        L.mcs_measure_peaks.argtypes = [vp, P(A.Peaks)]
        L.mcs_modes_at.argtypes = [P(A.Spindle), vp, C.c_size_t, vp, C.c_size_t, vp]
        L.mcs_lobes_composite.argtypes = [vp, P(A.Spindle), vp, C.c_size_t, P(A.LobeQuery), vp,
                                          vp, C.c_size_t, P(C.c_size_t)]
        L.mcs_curve_alim.argtypes = [vp, vp, C.c_size_t, vp, C.c_size_t, vp]
        L.mcs_solve_multi.argtypes = [vp, C.c_size_t] + batch[1:] + [vp]
        L.mcs_shard.argtypes = batch[1:] + [C.c_size_t, vp, vp]
        L.mcs_engine_create.argtypes = [vp, C.c_size_t, P(vp)]
        for f in ("destroy", "reset_history"):
            getattr(L, f"mcs_engine_{f}").argtypes = [vp]
        for f in ("configure", "set_engagement", "set_state", "run", "take_stats", "get_state",
                  "chatter_index"):
            getattr(L, f"mcs_engine_{f}").argtypes = [vp, vp]
        L.mcs_engine_history.argtypes = [vp, vp, vp, vp]
        for name in EXPORTS:
            if name not in _VOID:
                getattr(L, name).restype = C.c_int
        if path is None:
            _LIB = L
        return L


def last_error() -> str:
    return (load().mcs_last_error() or b"").decode(errors="replace")


def check(status: int) -> None:
    if status != A.MCS_OK:
        raise MCSError(status, last_error())


def default_opts() -> A.Opts:
    o = A.Opts()
    load().mcs_default_opts(C.byref(o))
    return o


def _ptr(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data) if a.size else C.c_void_p(0)


class Batch:
    """Inputs of a solve as contiguous record arrays (setups, modals, points)."""

    def __init__(self, setups, modals, points):
        self.setups = A.as_records(setups, A.SETUP_DTYPE)
        self.modals = A.as_records(modals, A.MODAL_DTYPE)
        self.points = A.as_records(points, A.POINT_DTYPE)

    def args(self):
        return (_ptr(self.setups), len(self.setups), _ptr(self.modals), len(self.modals),
                _ptr(self.points), len(self.points))


class Plan:
    """Device-resident solve batch launched as a captured CUDA graph (optionally guided by
    a surrogate, which must outlive the plan)."""

    def __init__(self, ctx: "Context", batch: Batch, opts: A.Opts, surrogate=None,
                 guide: A.GuideOpts | None = None):
        self.ctx = ctx
        self.batch = batch
        self.n = len(batch.points)
        self.surrogate = surrogate
        h = C.c_void_p()
        if surrogate is None:
            check(ctx._L.mcs_plan_create(ctx._h, *batch.args(), C.byref(opts), C.byref(h)))
        else:
            g = guide if guide is not None else default_guide_opts()
            check(ctx._L.mcs_plan_create_guided(ctx._h, surrogate._h, *batch.args(),
                                                C.byref(opts), C.byref(g), C.byref(h)))
        self._h = h
        ctx._adopt(self)

    def guide_info(self) -> np.ndarray:
        out = np.zeros(max(1, self.n), dtype=A.GUIDE_INFO_DTYPE)
        check(self.ctx._L.mcs_plan_guide_info(self._h, _ptr(out)))
        return out[: self.n]

    def execute(self) -> None:
        check(self.ctx._L.mcs_plan_execute(self._h))

    def results(self) -> np.ndarray:
        out = np.zeros(self.n, dtype=A.RESULT_DTYPE)
        check(self.ctx._L.mcs_plan_results(self._h, _ptr(out)))
        return out

    def info(self) -> dict:
        i = A.PlanInfo()
        check(self.ctx._L.mcs_plan_info_get(self._h, C.byref(i)))
        return {n: getattr(i, n) for n, _ in A.PlanInfo._fields_}

    def close(self) -> None:
        if getattr(self, "_h", None):
            self.ctx._L.mcs_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Job:
    """Asynchronous solve (the Worker protocol): poll, cancel, wait."""

    def __init__(self, ctx: "Context", batch: Batch, opts: A.Opts):
        self.ctx = ctx
        self.batch = batch
        self.n = len(batch.points)
        self.out = np.zeros(max(1, self.n), dtype=A.RESULT_DTYPE)
        h = C.c_void_p()
        check(ctx._L.mcs_solve_async(ctx._h, *batch.args(), C.byref(opts), _ptr(self.out),
                                     C.byref(h)))
        self._h = h
        ctx._adopt(self)

    def poll(self) -> tuple[int, bool]:
        done = C.c_size_t()
        fin = C.c_int()
        check(self.ctx._L.mcs_job_poll(self._h, C.byref(done), C.byref(fin)))
        return int(done.value), bool(fin.value)

    def cancel(self) -> None:
        check(self.ctx._L.mcs_job_cancel(self._h))

    def wait(self) -> np.ndarray:
        """Results; raises MCSError(MCS_ERR_CANCELLED) after a cancel (results still set)."""
        st = self.ctx._L.mcs_job_wait(self._h)
        if st not in (A.MCS_OK, A.MCS_ERR_CANCELLED):
            check(st)
        self.cancelled = st == A.MCS_ERR_CANCELLED
        return self.out[: self.n]

    def close(self) -> None:
        if getattr(self, "_h", None):
            self.ctx._L.mcs_job_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Context:
    """One CUDA device (mcs_create).  Thread-safe: the library serialises calls."""

    def __init__(self, device: int = 0):
        self._L = load()
        h = C.c_void_p()
        check(self._L.mcs_create(C.byref(h), int(device)))
        self._h = h
        self.device = device
        self._children = weakref.WeakSet()

    def _adopt(self, obj) -> None:
        """Plans, jobs and surrogates of this context are closed before it."""
        self._children.add(obj)

    @property
    def stream(self) -> int:
        return int(self._L.mcs_stream(self._h) or 0)

    def solve(self, setups, modals, points, opts: A.Opts) -> np.ndarray:
        b = Batch(setups, modals, points)
        out = np.zeros(max(1, len(b.points)), dtype=A.RESULT_DTYPE)
        check(self._L.mcs_solve(self._h, *b.args(), C.byref(opts), _ptr(out)))
        return out[: len(b.points)]

    def chatter_at(self, setups, modals, points, trials, opts: A.Opts) -> np.ndarray:
        b = Batch(setups, modals, points)
        t = A.as_records(trials, A.TRIAL_DTYPE)
        out = np.zeros(max(1, len(t)), dtype=A.TRIAL_RESULT_DTYPE)
        check(self._L.mcs_chatter_at(self._h, *b.args(), _ptr(t), len(t), C.byref(opts),
                                     _ptr(out)))
        return out[: len(t)]

    def plan(self, setups, modals, points, opts: A.Opts, surrogate=None,
             guide: A.GuideOpts | None = None) -> Plan:
        return Plan(self, Batch(setups, modals, points), opts, surrogate, guide)

    def features(self, setups, modals, points, opts: A.Opts) -> np.ndarray:
        b = Batch(setups, modals, points)
        out = np.zeros((max(1, len(b.points)), A.FEATURES), dtype=np.float32)
        check(self._L.mcs_features(*b.args(), C.byref(opts), _ptr(out)))
        return out[: len(b.points)]

    def solve_guided(self, surrogate, setups, modals, points, opts: A.Opts,
                     guide: A.GuideOpts | None = None):
        """(results, guide info) of the surrogate-guided solve.

        guide.mode GUIDE_SPECULATE (the default) runs the plain bisection's own trials for
        guide.levels levels, steered by the prediction (the bracket is the plain one after
        those levels); GUIDE_BRACKET verifies and refines a predicted bracket."""
        b = Batch(setups, modals, points)
        n = len(b.points)
        out = np.zeros(max(1, n), dtype=A.RESULT_DTYPE)
        info = np.zeros(max(1, n), dtype=A.GUIDE_INFO_DTYPE)
        g = guide if guide is not None else default_guide_opts()
        check(self._L.mcs_solve_guided(self._h, surrogate._h, *b.args(), C.byref(opts),
                                       C.byref(g), _ptr(out), _ptr(info)))
        return out[:n], info[:n]

    def tune(self, setups, modals, points, opts: A.Opts, candidates=(4, 8, 16, 32)):
        """(best max_buckets, {candidate: ms}) from one timed execution per candidate."""
        b = Batch(setups, modals, points)
        cand = np.ascontiguousarray(candidates, dtype=np.int32)
        ms = np.zeros(len(cand), dtype=np.float64)
        best = C.c_int32()
        check(self._L.mcs_tune(self._h, *b.args(), C.byref(opts), _ptr(cand), len(cand),
                               _ptr(ms), C.byref(best)))
        return int(best.value), {int(c): float(t) for c, t in zip(cand, ms)}

    def solve_async(self, setups, modals, points, opts: A.Opts) -> Job:
        return Job(self, Batch(setups, modals, points), opts)

    def lobes_alim(self, modals, queries: Sequence[A.LobeQuery], rpm) -> np.ndarray:
        m = A.as_records(modals, A.MODAL_DTYPE)
        q = A.array_of(A.LobeQuery, list(queries))
        r = np.ascontiguousarray(rpm, dtype=np.float64)
        out = np.zeros((len(queries), len(r)), dtype=np.float64)
        check(self._L.mcs_lobes_alim(self._h, _ptr(m), len(m), C.cast(q, C.c_void_p),
                                     len(queries), _ptr(r), len(r), _ptr(out)))
        return out

    def lobes_composite(self, spindle, base: A.LobeQuery):
        """(rpm, alim) of the speed-dependent composite diagram (mcs_lobes_composite)."""
        n = C.c_size_t()
        F = A.array_of(A.SpeedFrf, spindle.frfs)
        args = (self._h, C.byref(spindle.record), C.cast(F, C.c_void_p), len(spindle.frfs),
                C.byref(base))
        check(self._L.mcs_lobes_composite(*args, None, None, 0, C.byref(n)))
        rpm = np.zeros(max(1, n.value))
        alim = np.zeros(max(1, n.value))
        check(self._L.mcs_lobes_composite(*args, _ptr(rpm), _ptr(alim), n.value, C.byref(n)))
        return rpm[: n.value], alim[: n.value]

    def measure_peaks(self) -> dict:
        """Measured FP32/FP64 FMA rates [TFLOP/s] and shared-memory bandwidth [TB/s] of this
        device (mcs_measure_peaks): the solve kernels' roofline denominators."""
        p = A.Peaks()
        check(self._L.mcs_measure_peaks(self._h, C.byref(p)))
        return {"fp32_tflops": p.fp32_tflops, "fp64_tflops": p.fp64_tflops,
                "smem_tbps": p.smem_tbps}

    def close(self) -> None:
        if getattr(self, "_h", None):
            kids = list(getattr(self, "_children", ()))
            # plans and jobs first: a guided plan holds its surrogate
            for k in sorted(kids, key=lambda o: isinstance(o, Surrogate)):
                k.close()
            self._L.mcs_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def default_train_opts() -> A.TrainOpts:
    o = A.TrainOpts()
    load().mcs_default_train_opts(C.byref(o))
    return o


def default_guide_opts() -> A.GuideOpts:
    o = A.GuideOpts()
    load().mcs_default_guide_opts(C.byref(o))
    return o


class Surrogate:
    """The MLP surrogate on a context's device (mcs_surrogate_*)."""

    def __init__(self, ctx: Context, seed: int = 1):
        self.ctx = ctx
        self._L = ctx._L
        h = C.c_void_p()
        check(self._L.mcs_surrogate_create(ctx._h, int(seed), C.byref(h)))
        self._h = h
        ctx._adopt(self)

    def train(self, X, y, Xv=None, yv=None, opts: A.TrainOpts | None = None):
        """Returns (train_loss[epochs], val_loss[epochs])."""
        o = opts if opts is not None else default_train_opts()
        X = np.ascontiguousarray(X, dtype=np.float32)
        y = np.ascontiguousarray(y, dtype=np.float32)
        nv = 0 if Xv is None else len(Xv)
        Xv = np.ascontiguousarray(Xv if nv else np.zeros((1, A.FEATURES)), dtype=np.float32)
        yv = np.ascontiguousarray(yv if nv else np.zeros(1), dtype=np.float32)
        tl = np.zeros(o.epochs, dtype=np.float32)
        vl = np.zeros(o.epochs, dtype=np.float32)
        check(self._L.mcs_surrogate_train(self._h, _ptr(X), _ptr(y), len(X), _ptr(Xv), _ptr(yv),
                                          nv, C.byref(o), _ptr(tl), _ptr(vl)))
        return tl, vl

    def predict(self, X):
        X = np.ascontiguousarray(X, dtype=np.float32)
        mu = np.zeros(max(1, len(X)), dtype=np.float32)
        sg = np.zeros(max(1, len(X)), dtype=np.float32)
        check(self._L.mcs_surrogate_predict(self._h, _ptr(X), len(X), _ptr(mu), _ptr(sg)))
        return mu[: len(X)], sg[: len(X)]

    def grad(self, X, y):
        X = np.ascontiguousarray(X, dtype=np.float32)
        y = np.ascontiguousarray(y, dtype=np.float32)
        n = C.c_size_t()
        check(self._L.mcs_surrogate_get_params(self._h, None, C.byref(n)))
        g = np.zeros(n.value, dtype=np.float32)
        loss = C.c_float()
        check(self._L.mcs_surrogate_grad(self._h, _ptr(X), _ptr(y), len(X), C.byref(loss),
                                         _ptr(g)))
        return float(loss.value), g

    def get_params(self) -> np.ndarray:
        n = C.c_size_t()
        check(self._L.mcs_surrogate_get_params(self._h, None, C.byref(n)))
        out = np.zeros(n.value, dtype=np.float32)
        check(self._L.mcs_surrogate_get_params(self._h, _ptr(out), C.byref(n)))
        return out

    def set_params(self, p) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        check(self._L.mcs_surrogate_set_params(self._h, _ptr(p), len(p)))

    def close(self) -> None:
        """Raises MCSError (MCS_ERR_STATE) while a guided plan still uses the surrogate."""
        if getattr(self, "_h", None):
            check(self._L.mcs_surrogate_destroy(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_DEFAULT: dict[int, Context] = {}


def default_context(device: int = 0) -> Context:
    """A process-wide context per device, created on first use."""
    with _LOCK:
        ctx = _DEFAULT.get(device)
    if ctx is None:
        ctx = Context(device)
        with _LOCK:
            _DEFAULT.setdefault(device, ctx)
            ctx = _DEFAULT[device]
    return ctx


def shard(setups, modals, points, opts: A.Opts, n_shards: int):
    """(shard of each point, cost of each point) of mcs_shard: the split mcs_solve_multi
    uses (host arithmetic, no device)."""
    b = Batch(setups, modals, points)
    n = len(b.points)
    of = np.zeros(max(1, n), dtype=np.int32)
    cost = np.zeros(max(1, n), dtype=np.float64)
    check(load().mcs_shard(*b.args(), C.byref(opts), int(n_shards), _ptr(of), _ptr(cost)))
    return of[:n], cost[:n]


def solve_multi(contexts: Sequence["Context"], setups, modals, points, opts: A.Opts):
    """mcs_solve over several contexts at once (mcs_solve_multi), results in input order."""
    b = Batch(setups, modals, points)
    n = len(b.points)
    hs = (C.c_void_p * len(contexts))(*[c._h.value for c in contexts])
    out = np.zeros(max(1, n), dtype=A.RESULT_DTYPE)
    check(load().mcs_solve_multi(C.cast(hs, C.c_void_p), len(contexts), *b.args(),
                                 C.byref(opts), _ptr(out)))
    return out[:n]
