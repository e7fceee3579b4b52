"""The reference's stability-search API on the GPU: chatterAt and timeDomainLimit of
src/stabtd.js:14-32, with the same arguments and return shapes, plus a batched form.

    r = timeDomainLimit(tool, modal, mat, S, arc, fz, {"nonlinear": True})
    r["alim"], r["bracket"]          # bracket[1] == inf when stable at aMax

Arguments are the reference's plain objects (see mcs._abi).  opts takes the reference
keys aMin, aMax, iters, revs, nonlinear and the explicit extensions honorRunout
(chatterAt forces runout to 0, stabtd.js:16), stepsPerTooth, slices and chatterIdx.
"""
from __future__ import annotations

from typing import Any, Mapping, Sequence

import numpy as np

from . import _abi as A
from ._lib import Context, MCSError, default_context


def _ctx(ctx: Context | None) -> Context:
    return ctx if ctx is not None else default_context()


def _one(tool, modal, mat, S, arc, fz):
    setups = [A.make_setup(tool, mat, arc, fz)]
    modals = [A.make_modal(modal)]
    points = A.points_array([0], [0], [float(S)])
    return setups, modals, points


def chatterAt(tool, modal, mat, S, arc, fz, ap, opts: Mapping[str, Any] | None = None, *,
              ctx: Context | None = None) -> bool:
    """One time-domain trial at depth ap: True when the chatter index exceeds 0.45."""
    setups, modals, points = _one(tool, modal, mat, S, arc, fz)
    trials = np.array([(0, 0, float(ap))], dtype=A.TRIAL_DTYPE)
    r = _ctx(ctx).chatter_at(setups, modals, points, trials, A.make_opts(opts))
    if r["status"][0] not in (A.MCS_OK, A.MCS_ERR_DIVERGED):
        raise MCSError(int(r["status"][0]), "trial did not complete")
    return bool(r["chatter"][0])


def chatterIndex(tool, modal, mat, S, arc, fz, ap, opts=None, *, ctx=None) -> dict:
    """The chatterIndex() parts of one trial: {index, amp, once} (cutting.js:299-318)."""
    setups, modals, points = _one(tool, modal, mat, S, arc, fz)
    trials = np.array([(0, 0, float(ap))], dtype=A.TRIAL_DTYPE)
    r = _ctx(ctx).chatter_at(setups, modals, points, trials, A.make_opts(opts))[0]
    return {"index": float(r["index"]), "amp": float(r["amp"]), "once": float(r["once"])}


def timeDomainLimit(tool, modal, mat, S, arc, fz, opts: Mapping[str, Any] | None = None, *,
                    ctx: Context | None = None) -> dict:
    """Critical depth by bisection: {alim, bracket: [stable, chatter]} (stabtd.js:24-32)."""
    setups, modals, points = _one(tool, modal, mat, S, arc, fz)
    r = _ctx(ctx).solve(setups, modals, points, A.make_opts(opts))[0]
    # a run-away trial (MCS_ERR_DIVERGED) decides "stable" as the reference's NaN > 0.45
    # does; the result is returned like the reference's
    if r["status"] not in (A.MCS_OK, A.MCS_ERR_DIVERGED):
        raise MCSError(int(r["status"]), "point did not complete")
    return A.result_dict(r)


def timeDomainLimits(tool, mat, arc, fz, points: Sequence[Mapping[str, Any]],
                     opts: Mapping[str, Any] | None = None, *, ctx: Context | None = None,
                     spindle=None):
    """The Worker's sweep in one call: points = [{S, modal}] (stabworker.js:8-13).
    With a spindle model (mcs.spindle.Spindle) a point may leave out its modal: it gets
    the modes at its own speed, as sim.modalNow(S) gives them (main.js:495-496).
    Returns [{S, alim, open}] in point order."""
    setups = [A.make_setup(tool, mat, arc, fz)]
    need = [i for i, p in enumerate(points) if p.get("modal") is None]
    if need and spindle is None:
        raise ValueError("points without a modal need a spindle model")
    at = spindle.modes_at([float(points[i]["S"]) for i in need]) if need else []
    own = dict(zip(need, at))
    modals = [A.Modal.from_buffer_copy(own[i].tobytes()) if i in own
              else A.make_modal(p["modal"]) for i, p in enumerate(points)]
    pts = A.points_array(np.zeros(len(points)), np.arange(len(points)),
                         [float(p["S"]) for p in points])
    res = _ctx(ctx).solve(setups, modals, pts, A.make_opts(opts))
    return [{"S": float(p["S"]), "alim": float(r["alim"]), "open": bool(r["open"])}
            for p, r in zip(points, res)]
