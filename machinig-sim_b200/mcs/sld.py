"""Zero-order stability lobes on the GPU: stabilityLobes + alimAt of src/sld.js:23-76
evaluated at given spindle speeds in one call (mcs_lobes_alim).

    lim = lobeLimit({**modal, "N": 3, "Ktc": 2100, "Krc": 850, "phiSt": a, "phiEx": b,
                     "lobes": 30, "rpmMin": 2000, "rpmMax": 40000}, rpms)

equals ``[alimAt(stabilityLobes(params), s) for s in rpms]`` of the reference.

With speed-dependent dynamics the chart's diagram is a composite (Simulator.lobes,
sim.js:262-287): compositeLobes builds it from one GPU diagram per 1000 rpm with that
speed's modes, and alimAt reads any lobe list per pixel (charts.js:170-185).
"""
from __future__ import annotations

from typing import Any, Mapping, Sequence

import numpy as np

from . import _abi as A
from ._lib import Context, _ptr, check, default_context, load


def lobe_query(params: Mapping[str, Any], modal_index: int = 0) -> A.LobeQuery:
    return A.LobeQuery(int(params["N"]), int(params.get("lobes", 8)), float(params["Ktc"]),
                       float(params["Krc"]), float(params["phiSt"]), float(params["phiEx"]),
                       float(params.get("rpmMin", 1000)), float(params.get("rpmMax", 40000)),
                       int(modal_index), 0)


def lobeLimit(params: Mapping[str, Any], rpm, *, ctx: Context | None = None) -> np.ndarray:
    """alimAt(stabilityLobes(params), rpm) for each speed in rpm (inf where uncovered)."""
    c = ctx if ctx is not None else default_context()
    out = c.lobes_alim([A.make_modal(params)], [lobe_query(params)], np.atleast_1d(rpm))
    return out[0]


def lobeLimits(params_list: Sequence[Mapping[str, Any]], rpm, *,
               ctx: Context | None = None) -> np.ndarray:
    """Many lobe diagrams at once: out[q, r] for query q at speed rpm[r]."""
    c = ctx if ctx is not None else default_context()
    modals = [A.make_modal(p) for p in params_list]
    qs = [lobe_query(p, i) for i, p in enumerate(params_list)]
    return c.lobes_alim(modals, qs, np.atleast_1d(rpm))


def compositeLobes(spindle, params: Mapping[str, Any], *, ctx: Context | None = None):
    """The chart's speed-dependent diagram [[{rpm, alim}]] (sim.js:269-285): params gives N,
    Ktc, Krc, phiSt, phiEx, lobes (30) and rpmMin/rpmMax (2000/40000); the modes come from
    the spindle model (mcs.spindle.Spindle) at each node's centre."""
    c = ctx if ctx is not None else default_context()
    p = {"lobes": 30, "rpmMin": 2000, "rpmMax": 40000, **dict(params)}
    rpm, alim = c.lobes_composite(spindle, lobe_query(p))
    return [[{"rpm": float(r), "alim": float(a)} for r, a in zip(rpm, alim)]]


def alimAt(lobes, rpm):
    """alimAt (sld.js:64-76) of lobe lists [[{rpm, alim}]] at each speed in rpm: the minimum
    over the lobes of the interpolation on the segments covering the speed (mcs_curve_alim,
    host arithmetic); inf where none does.  A scalar speed gives a float."""
    r = np.ascontiguousarray(np.atleast_1d(rpm), dtype=np.float64)
    best = np.full(len(r), np.inf)
    out = np.zeros(max(1, len(r)))
    for lobe in lobes:
        cr = np.ascontiguousarray([pt["rpm"] for pt in lobe], dtype=np.float64)
        ca = np.ascontiguousarray([pt["alim"] for pt in lobe], dtype=np.float64)
        check(load().mcs_curve_alim(_ptr(cr), _ptr(ca), len(cr), _ptr(r), len(r), _ptr(out)))
        best = np.minimum(best, out[: len(r)])
    return float(best[0]) if np.ndim(rpm) == 0 else best
