"""A batch of time-domain cutting engines on the GPU: the reference's CuttingEngine
(src/cutting.js:21-321) with its state kept on the device between runs (mcs_engine_*).

    eng = Engines(ctx, n)
    eng.configure([config(tool, modal, mat, S) ...])       # configure() of each engine
    eng.set_engagement([engagement(Hb, u, fz, tipZ, ap) ...])
    eng.run([steps ...])                                   # run(n) of every engine at once
    eng.take_stats()   # takeStats(): structured array of the reference's fields

The Simulator's playback drives one engine substep by substep (Simulator.step,
sim.js:351-420); identification and validation (mcs.identify) run many rigid-tool engines
in one launch.  tool/modal/mat are the reference's objects (runout in um as the Simulator's
tool holds it, converted to mm as ensureEngine does, sim.js:255).
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Any, Callable, Mapping, Sequence

import numpy as np

from . import _abi as A
from ._lib import Context, _ptr, check

RIGID = {"k": 1e9, "fn": 1000.0, "zeta": 0.5}  # identify.js:15, validate.js:14


def config(tool: Mapping[str, Any], modal: Mapping[str, Any], mat: Mapping[str, Any], S: float,
           fn_max: float = 0.0, decim: int = 0) -> A.EngineConfig:
    """configure(tool, modal, mat, S, fnMax) arguments (cutting.js:39): tool {N, R or D,
    helixDeg, type, fluteLen, runout [um], runoutPhase, nonlinear}, mat {Ktc, Krc, Kac, Kte,
    Kre, Kae, mc, Ci}."""
    c = A.EngineConfig()
    c.tool = A.make_tool(tool)
    c.tool.runout_phase = float(tool.get("runoutPhase", 0.0) or 0.0)
    c.modal = A.make_modal(modal)
    for k in ("Ktc", "Krc", "Kac", "Kte", "Kre", "Kae", "mc", "Ci"):
        setattr(c, k, float(mat.get(k, 0.0) or 0.0))
    c.S = float(S)
    c.fn_max = float(fn_max)
    c.nonlinear = 0 if tool.get("nonlinear", True) is False else 1
    c.decim = int(decim)
    return c


def _fill_f32(dst, values) -> None:
    """Copy values, as float32 and flattened, into the ctypes float array dst (same length)."""
    a = np.ascontiguousarray(np.asarray(values, dtype=np.float32).ravel())
    if a.size != len(dst):
        raise ValueError(f"{a.size} values for {len(dst)} entries")
    C.memmove(C.addressof(dst), a.ctypes.data, a.nbytes)


def engagement(Hb, u=(1.0, 0.0), fz: float = 0.0, tipZ: float = 0.0, ap: float = 0.0, *,
               rAt: Callable[[float], float] | None = None, dz: float | None = None,
               Eb=None, fza: float = 0.0, rOut: float = 0.0,
               zAt: Callable[[float], float] | None = None, wall: Mapping[str, Any] | None = None,
               wear: Mapping[str, float] | None = None) -> A.Engagement:
    """One substep's engagement: setEngagement(u, fz, tipZ, ap) with the map Hb[180] (and a
    general edge profile rAt: pass the engine's slice pitch dz, cutting.js:63, so that the
    slice radii and edge angles are taken as setEngagement takes them), setEndEngagement
    (fza, rOut, zAt) with the end-face map Eb[36 * 6], setWork(wall {k, m, zeta, nx, ny})
    and setWear({Kte, Kre})."""
    g = A.Engagement()
    _fill_f32(g.Hb, Hb)
    g.ux, g.uy = float(u[0]), float(u[1])
    g.fz, g.tip_z, g.ap = float(fz), float(tipZ), float(ap)
    if rAt is not None:
        if dz is None:
            raise ValueError("a profile needs the engine's slice pitch dz")
        nz = 0 if ap <= 0 else int(math.ceil(ap / dz))
        for k in range(min(nz, A.MAX_SLICES)):
            b = min(dz, ap - k * dz)
            zr = k * dz + 0.5 * b
            r = max(1e-3, rAt(zr))
            dr = (rAt(zr + 0.05) - rAt(max(0.0, zr - 0.05))) / (0.05 + zr if zr < 0.05 else 0.1)
            g.slice_r[k] = r
            g.slice_kap[k] = 1 / math.sqrt(1 + dr * dr)
        g.profile = 1
    if Eb is not None:
        _fill_f32(g.Eb, Eb)
    g.fza, g.end_r = float(fza), float(rOut)
    if fza > 0:
        za = zAt or (lambda r: 0.0)
        dr = rOut / A.END_RINGS
        for j in range(A.END_RINGS):
            r = (j + 0.5) * dr
            g.ring_z[j] = za(r)
            g.ring_zo[j] = za(min(rOut, r + 0.25 * dr))
            g.ring_zi[j] = za(max(0.0, r - 0.25 * dr))
    if wall:
        g.wall_k, g.wall_m, g.wall_zeta = float(wall["k"]), float(wall["m"]), float(wall["zeta"])
        g.wall_nx, g.wall_ny = float(wall["nx"]), float(wall["ny"])
    if wear:
        g.wear = 1
        g.Kte, g.Kre = float(wear["Kte"]), float(wear["Kre"])
    return g


def arc_map(st: float, ex: float, inside: float = 0.0, outside: float = -1e3) -> np.ndarray:
    """The static map chatterAt and the identification runs build (stabtd.js:17,
    identify.js:33): bins whose centre lies in [st, ex] hold `inside`, the rest `outside`."""
    phi = (np.arange(A.BINS) + 0.5) / A.BINS * 2 * math.pi
    return np.where((phi >= st) & (phi <= ex), inside, outside).astype(np.float32)


class Engines:
    """n CuttingEngine objects on the context's device."""

    def __init__(self, ctx: Context, n: int):
        self.ctx = ctx
        self.n = int(n)
        h = C.c_void_p()
        check(ctx._L.mcs_engine_create(ctx._h, self.n, C.byref(h)))
        self._h = h
        ctx._adopt(self)

    def _array(self, ctype, items):
        items = list(items)
        if len(items) != self.n:
            raise ValueError(f"{len(items)} records for {self.n} engines")
        return A.array_of(ctype, items)

    def configure(self, cfgs: Sequence[A.EngineConfig]) -> None:
        check(self.ctx._L.mcs_engine_configure(self._h, C.cast(self._array(A.EngineConfig, cfgs),
                                                               C.c_void_p)))

    def set_engagement(self, gs: Sequence[A.Engagement]) -> None:
        check(self.ctx._L.mcs_engine_set_engagement(
            self._h, C.cast(self._array(A.Engagement, gs), C.c_void_p)))

    def set_state(self, xv) -> None:
        a = np.ascontiguousarray(np.broadcast_to(np.asarray(xv, dtype=np.float64),
                                                 (self.n, 4)))
        check(self.ctx._L.mcs_engine_set_state(self._h, _ptr(a)))

    def run(self, steps) -> None:
        a = np.ascontiguousarray(np.broadcast_to(np.asarray(steps, dtype=np.int64), (self.n,)))
        check(self.ctx._L.mcs_engine_run(self._h, _ptr(a)))

    def take_stats(self) -> np.ndarray:
        out = np.zeros(self.n, dtype=A.ENGINE_STATS_DTYPE)
        check(self.ctx._L.mcs_engine_take_stats(self._h, _ptr(out)))
        return out

    def state(self) -> list[dict]:
        s = (A.EngineState * self.n)()
        check(self.ctx._L.mcs_engine_get_state(self._h, C.cast(s, C.c_void_p)))
        return [{f: getattr(x, f) for f, _ in A.EngineState._fields_} for x in s]

    def history(self):
        """(out[n, 5, 4096] = Fx, Fy, Fz [N], x, y [um]; head[n]; count[n])."""
        out = np.zeros((self.n, 5, A.ENGINE_HIST), dtype=np.float32)
        head = np.zeros(self.n, dtype=np.int32)
        count = np.zeros(self.n, dtype=np.int64)
        check(self.ctx._L.mcs_engine_history(self._h, _ptr(out), _ptr(head), _ptr(count)))
        return out, head, count

    def reset_history(self) -> None:
        check(self.ctx._L.mcs_engine_reset_history(self._h))

    def chatter_index(self) -> np.ndarray:
        out = np.zeros((self.n, 3), dtype=np.float64)
        check(self.ctx._L.mcs_engine_chatter_index(self._h, _ptr(out)))
        return out

    def close(self) -> None:
        if getattr(self, "_h", None):
            self.ctx._L.mcs_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
