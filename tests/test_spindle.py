"""Speed-dependent tool-tip modes (src/spindle.js): the library's mcs_modes_at (host code,
no device needed) against the reference's own assertions (test/spindle.test.mjs) and, bit
for bit, against the oracle's independent restatement of modesAt."""
from __future__ import annotations

import math

import numpy as np
import pytest


def _sp(modal, **kw):
    from mcs import spindle as SP

    return SP.Spindle(modal, **kw)


def _fn(m, i=0):
    return float(m["x"][i]["fn"])


def test_bearing_model_and_tip_factor():
    """spindle.test.mjs:11-21: 1 at rest, the stated loss at S_ref, falling with speed; a
    slender tool changes less than a stubby one on the same spindle."""
    rest = {"k": 1.0, "fn": 1.0, "zeta": 0.03}
    # a spindle-only chain (tool infinitely stiff) shows the bearing factor itself
    b = _sp(rest, kTool=1e30, kSp=5e4).modes_at([0.0, 10000.0, 20000.0, 30000.0])["x"][:, 0]["k"]
    assert b[0] == 1.0 and abs(b[3] - 0.75) < 1e-12 and b[1] > b[2]
    assert _sp(rest, kTool=1e30, kSp=5e4, soft={"drop": 0.0}).modes_at([30000.0])["x"][0, 0]["k"] == 1.0
    slender = _sp(rest, kTool=13000, kSp=50000).modes_at([30000.0])["x"][0, 0]["k"]
    stubby = _sp(rest, kTool=200000, kSp=50000).modes_at([30000.0])["x"][0, 0]["k"]
    assert slender > stubby and stubby < 0.85 and slender > 0.9


def test_simulator_defaults_soften_with_speed():
    """spindle.test.mjs:27-33: the default tool's tip mode at rest is the hammer-test value
    (the tool model's fn, rounded) and drops with speed."""
    from mcs import spindle as SP

    tool = {"D": 10.0, "stickout": 30.0, "kSpindle": 50000.0}
    sp = SP.Spindle.from_tool(tool, {"auto": True, "k": 0, "fn": 0, "zeta": 0.04})
    m = sp.modes_at([0.0, 15000.0, 30000.0])
    assert _fn(m[0]) == math.floor(SP.tool_model(tool)["fn"] + 0.5)
    assert _fn(m[0]) > _fn(m[1]) > _fn(m[2])


def test_measured_frfs_interpolate():
    """spindle.test.mjs:92-103: FRFs measured at several speeds replace the model."""
    frfs = [{"S": 0.0, "modesX": [{"k": 12000.0, "fn": 3000.0, "zeta": 0.03}]},
            {"S": 30000.0, "modesX": [{"k": 9000.0, "fn": 2400.0, "zeta": 0.04}]}]
    sp = _sp({"k": 10000, "fn": 3000, "zeta": 0.03}, kTool=1e4, kSp=5e4, speed_frfs=frfs)
    m = sp.modes_at([15000.0, 40000.0])
    assert abs(_fn(m[0]) - 2700) < 1e-9 and abs(float(m[0]["x"][0]["k"]) - 10500) < 1e-9
    assert _fn(m[1]) == 2400.0, "held beyond the measured range"
    assert float(m[0]["y"][0]["fn"]) == float(m[0]["x"][0]["fn"]), "Y follows X"


def test_two_mass_spindle_mode():
    """spindle.test.mjs:107-118: two tip modes whose compliances add up to the static chain,
    the spindle mode below the tool's; a rigid spindle leaves the tool's mode alone."""
    kT = 10600.0
    mT = kT * 1e3 / (2 * math.pi * 2400) ** 2
    kS = 50000.0
    mS = kS * 1e3 / (2 * math.pi * 1200) ** 2
    two = {"mTool": mT, "mSp": mS, "zTool": 0.03, "zSp": 0.05}
    rest = {"k": 1.0, "fn": 1.0, "zeta": 0.03}
    m = _sp(rest, kTool=kT, kSp=kS, soft={"drop": 0.0}, two_dof=two).modes_at([0.0])[0]
    ks = m["x"]["k"][:2]
    assert m["nx"] == 2 and abs(1 / np.sum(1 / ks) - 1 / (1 / kT + 1 / kS)) < 1e-6 * kT
    assert _fn(m, 0) < 1200 and _fn(m, 1) > 2400 and float(m["x"][0]["zeta"]) == 0.05
    st = _sp(rest, kTool=kT, kSp=1e9, soft={"drop": 0.0}, two_dof=two).modes_at([0.0])[0]
    assert abs(_fn(st, 0) / 2400 - 1) < 1e-3 and float(st["x"][0]["zeta"]) == 0.03
    assert float(st["x"][1]["k"]) > 1e6
    # the bearing softening lowers the spindle mode most
    soft = _sp(rest, kTool=kT, kSp=kS, two_dof=two).modes_at([0.0, 30000.0])
    r0, r1 = _fn(soft[1], 0) / _fn(soft[0], 0), _fn(soft[1], 1) / _fn(soft[0], 1)
    assert r0 < r1 and _fn(soft[1], 0) < _fn(soft[0], 0)


def test_library_matches_the_oracle_bit_for_bit(oracle):
    """Every branch of modesAt, on seeded inputs: the library and the oracle's restatement
    give the same doubles."""
    from mcs import _abi as A
    from mcs import workloads as W

    rng = np.random.default_rng(5)
    S = np.concatenate([[0.0, -5.0, 30000.0, 45000.0], rng.uniform(0, 40000, 60)])
    cases = []
    for k in range(6):
        modal = {"k": float(rng.uniform(5e3, 5e4)), "fn": float(rng.uniform(500, 4000)),
                 "zeta": float(rng.uniform(0.01, 0.05)),
                 "modesX": [{"k": float(rng.uniform(5e3, 5e4)), "fn": float(rng.uniform(500, 4000)),
                             "zeta": 0.02} for _ in range(1 + k % 3)]}
        if k % 2:
            modal["modesY"] = [{"k": 2e4, "fn": 1800.0, "zeta": 0.03}]
        soft = {"drop": float(rng.uniform(0, 0.95)), "Sref": float(rng.uniform(1e4, 4e4))}
        cases.append(_sp(modal, kTool=float(rng.uniform(5e3, 3e5)), kSp=5e4, soft=soft))
    cases.append(_sp({"k": 1e4, "fn": 2000, "zeta": 0.04}, kTool=2e4, kSp=5e4,
                     two_dof={"mTool": 0.1, "mSp": 0.9, "zTool": 0.04, "zSp": 0.05}))
    frfs = [{"S": 20000.0, "modesX": [{"k": 9e3, "fn": 2500.0, "zeta": 0.04}]},
            {"S": 0.0, "modesX": [{"k": 1.2e4, "fn": 3000.0, "zeta": 0.03}],
             "modesY": [{"k": 1.1e4, "fn": 2900.0, "zeta": 0.03}]},
            {"S": 35000.0, "modesX": [{"k": 8e3, "fn": 2300.0, "zeta": 0.05},
                                      {"k": 3e4, "fn": 5000.0, "zeta": 0.02}]}]
    cases.append(_sp({"k": 1e4, "fn": 3000, "zeta": 0.03}, speed_frfs=frfs))
    for sp in cases:
        got = sp.modes_at(S)
        ref = oracle.modes_at(sp.record, S, sp.frfs)
        assert got.tobytes() == ref.tobytes()
    # the speed-dependent sweep fixture's modal sets are the oracle's: the library's agree
    from conftest import load_golden

    g = load_golden("spindle")
    assert W.spindle_sweep().modals.tobytes() == g["modals"].tobytes()


def test_bad_spindle_models_are_rejected():
    from mcs import MCSError

    with pytest.raises(MCSError):
        _sp({"k": 1e4, "fn": 2000, "zeta": 0.04}, kTool=2e4, kSp=5e4,
            two_dof={"mTool": 0.0, "mSp": 1.0}).modes_at([1000.0])
    with pytest.raises(MCSError):
        _sp({"k": 1e4, "fn": 2000, "zeta": 0.04}).modes_at([float("nan")])


def test_curve_alim_matches_the_reference_read_out(oracle):
    """mcs_curve_alim (the chart's per-pixel alimAt, charts.js:170-185) against the oracle's
    alimAt on lobes of its own stabilityLobes, ascending and with an unsorted polyline."""
    import mcs

    params = {"N": 3, "Ktc": 2100, "Krc": 850, "phiSt": math.pi / 2, "phiEx": math.pi,
              "lobes": 12, "rpmMin": 2000, "rpmMax": 40000, "k": 1.1e4, "fn": 1900,
              "zeta": 0.03}
    lobes = oracle.stabilityLobes(params)
    rpm = np.concatenate([np.linspace(1500, 42000, 400), [lobes[0][0]["rpm"]]])
    got = mcs.alimAt(lobes, rpm)
    ref = np.array([oracle.alimAt(lobes, r) for r in rpm])
    assert np.array_equal(np.isfinite(got), np.isfinite(ref))
    assert np.array_equal(got[np.isfinite(ref)], ref[np.isfinite(ref)])
    odd = [[{"rpm": 3.0, "alim": 1.0}, {"rpm": 1.0, "alim": 2.0}, {"rpm": 2.0, "alim": 3.0},
            {"rpm": 4.0, "alim": 5.0}]]
    for r in (0.5, 1.0, 1.5, 2.0, 2.5, 3.5, 4.0, 5.0):
        a, b = mcs.alimAt(odd, r), oracle.alimAt(odd, r)
        assert (a == b) or (math.isinf(a) and math.isinf(b)), (r, a, b)
