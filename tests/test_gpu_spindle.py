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


@pytest.mark.parametrize("case", ["chain", "spindle_mode", "measured"])
def test_composite_lobes_match_the_oracle(ctx, oracle, case):
    """The chart's speed-dependent diagram (Simulator.lobes, sim.js:269-285): every 25-rpm
    sample of every 1000-rpm node against the oracle's restatement (FP64 both)."""
    import mcs
    from mcs import spindle as SP
    from mcs import workloads as W

    c = W.SPINDLE_CASES[case]
    sp = SP.Spindle.from_tool(c["tool"], c["modal"], spindle_mode=c.get("spindle_mode"))
    base = {"N": 3, "Ktc": 700.0, "Krc": 210.0, "phiSt": 0.0, "phiEx": math.pi, "lobes": 30,
            "rpmMin": 2000, "rpmMax": 40000}
    got = mcs.compositeLobes(sp, base, ctx=ctx)[0]
    ref = oracle.composite_lobes(sp.record, base, sp.frfs)[0]
    assert [p["rpm"] for p in got] == [p["rpm"] for p in ref]
    g = np.array([p["alim"] for p in got])
    r = np.array([p["alim"] for p in ref])
    rel = np.abs(g / r - 1)
    print(f"{case}: {len(g)} samples, max rel diff {rel.max():.2e}")
    assert rel.max() < 1e-9


def test_composite_follows_each_speeds_own_diagram(ctx):
    """spindle.test.mjs:36-45: the composite diagram agrees with each speed's own diagram
    (its own FRF) within 1 % from 4000 to 38000 rpm."""
    import mcs
    from mcs import spindle as SP

    sp = SP.Spindle.from_tool({"D": 10.0, "stickout": 30.0, "kSpindle": 50000.0},
                              {"auto": True, "k": 0, "fn": 0, "zeta": 0.04})
    base = {"N": 3, "Ktc": 700.0, "Krc": 210.0, "phiSt": 0.0, "phiEx": math.pi, "lobes": 30,
            "rpmMin": 2000, "rpmMax": 40000}
    dep = mcs.compositeLobes(sp, base, ctx=ctx)
    worst = 0.0
    for S in range(4000, 38001, 1700):
        own = mcs.lobeLimit({**sp.modal_now(S), **base}, [float(S)], ctx=ctx)[0]
        worst = max(worst, abs(mcs.alimAt(dep, float(S)) / own - 1))
    print(f"composite vs per-speed diagrams: worst {worst * 100:.2f} %")
    assert worst < 0.01
