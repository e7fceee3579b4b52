"""The Worker's lobe curve with speed-dependent modes on the GPU: timeDomainLimits with a
spindle model gives each point the modes at its own speed (sim.modalNow(S), main.js:496),
and its limits equal a solve of the same points with those modal sets given explicitly;
against the oracle they are held by the parity tests (test_gpu_parity, fixture spindle)."""
from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def test_time_domain_limits_with_a_spindle_model(ctx):
    import mcs
    from mcs import _abi as A
    from mcs import spindle as SP
    from mcs import workloads as W

    g = load_golden("spindle")
    case = W.SPINDLE_CASES["chain"]
    sp = SP.Spindle.from_tool(case["tool"], case["modal"])
    tool = {"N": 3, "R": 5.0, "helixDeg": 30.0, "type": "flat", "fluteLen": 12.0}
    mat = {"Ktc": 700.0, "Krc": 210.0, "Kte": 20.0, "Kre": 25.0, "mc": 0.10, "Ci": 2e4}
    speeds = SP.lobe_speeds()
    got = mcs.timeDomainLimits(tool, mat, [math.pi / 2, math.pi], 0.05,
                               [{"S": s} for s in speeds], {"revs": 120}, ctx=ctx,
                               spindle=sp)
    sel = g["points"]["setup"] == 0
    ref = ctx.solve(g["setups"], g["modals"], g["points"][sel], A.opts_from_record(g["opts"]))
    assert [r["S"] for r in got] == speeds
    assert np.array_equal([r["alim"] for r in got], ref["alim"])
    # the explicit modal objects of sweep_points give the same limits
    pts = SP.sweep_points(sp, speeds)
    again = mcs.timeDomainLimits(tool, mat, [math.pi / 2, math.pi], 0.05, pts, {"revs": 120},
                                 ctx=ctx)
    assert [r["alim"] for r in again] == [r["alim"] for r in got]
