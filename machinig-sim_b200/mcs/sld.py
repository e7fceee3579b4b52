"""Zero-order stability lobes on the GPU: stabilityLobes + alimAt of src/sld.js:23-76
evaluated at given spindle speeds in one call (mcs_lobes_alim).

    lim = lobeLimit({**modal, "N": 3, "Ktc": 2100, "Krc": 850, "phiSt": a, "phiEx": b,
                     "lobes": 30, "rpmMin": 2000, "rpmMax": 40000}, rpms)

equals ``[alimAt(stabilityLobes(params), s) for s in rpms]`` of the reference.
"""
from __future__ import annotations

from typing import Any, Mapping, Sequence

import numpy as np

from . import _abi as A
from ._lib import Context, default_context


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
