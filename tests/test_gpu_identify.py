"""Coefficient identification and validation on batched GPU engines (mcs.identify) against
the oracle's restatement of the same runs and against the reference's own assertions
(test/identify.test.mjs, test/validate.test.mjs): the slot unit forces equal Altintas'
closed form, noisy mean forces at four feeds give the coefficients back, one feed holds
the edge terms, and a synthetic force record gives its coefficients and runout back."""
from __future__ import annotations

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

S50C = {"Ktc": 2100, "Krc": 850, "Kac": 400, "Kte": 35, "Kre": 45, "Kae": 10, "mc": 0.14,
        "Ci": 1.5e5}
A5052 = {"Ktc": 700, "Krc": 210, "Kac": 120, "Kte": 20, "Kre": 25, "Kae": 5, "mc": 0.10,
         "Ci": 2e4}


def _prepared(tool, test, mat, decim=0, S=6000):
    from mcs import engine as E
    from mcs import identify as I

    st, ex = I.immersion(test["mode"], test["ae"], tool["D"])
    tl = I._engine_tool(tool, test["ap"])
    tl["nonlinear"] = (mat.get("mc") or 0) > 0
    c = E.config(tl, E.RIGID, mat, S, decim=decim)
    g = E.engagement(E.arc_map(st, ex), (1, 0), test["fz"], -test["ap"], test["ap"])
    return c, g


def test_unit_forces_match_the_oracle_and_the_closed_form(ctx, oracle):
    """identify.test.mjs:8-16: slot, no runout, linear model -> Altintas' closed form
    within 1 %; every component against the oracle's run of the same engines."""
    from mcs import identify as I

    tool = {"D": 10, "N": 3, "helixDeg": 30, "fluteLen": 25}
    N, c = 3, 0.05
    for ap in (2.0, 1.3):
        t = {"fz": c, "ap": ap, "ae": 10, "mode": "slot"}
        U = I.unit_forces(ctx, tool, [t])[0]
        want = {"Ktc": [0, -N * ap * c / 4, 0], "Krc": [N * ap * c / 4, 0, 0],
                "Kac": [0, 0, N * ap * c / math.pi], "Kte": [0, -N * ap / math.pi, 0],
                "Kre": [N * ap / math.pi, 0, 0], "Kae": [0, 0, N * ap / 2]}
        for j, k in enumerate(I.COEF_KEYS):
            mag = max(abs(v) for v in want[k])
            for i in range(3):
                assert abs(U[j][i] - want[k][i]) < 0.01 * mag, (k, i, U[j][i], want[k][i])
        prep = []
        for key in I.COEF_KEYS:
            mat = dict.fromkeys(I.COEF_KEYS, 0.0)
            mat.update({key: 1.0, "mc": 0.0, "Ci": 0.0})
            prep.append(_prepared(tool, t, mat))
        ref = oracle.unit_forces_ref([p[0] for p in prep], [p[1] for p in prep])
        scale = np.abs(ref).max(axis=1, keepdims=True)
        assert np.all(np.abs(U - ref) <= 1e-9 * scale)


def _synth(ctx, tool, m, mode, ae, mc, noise):
    """synth() of identify.test.mjs:19-27: mean forces at four feeds with noise."""
    from mcs import identify as I

    seed = [3]

    def rnd():
        seed[0] = (seed[0] * 16807) % 2147483647
        return seed[0] / 2147483647 - 0.5

    tests = [{"fz": fz, "ap": 2, "ae": ae, "mode": mode} for fz in (0.02, 0.04, 0.06, 0.08)]
    U = I.unit_forces(ctx, tool, tests, mc)
    for i, t in enumerate(tests):
        F = [sum(m[k] * U[i][j][c] for j, k in enumerate(I.COEF_KEYS)) * (1 + noise * rnd())
             for c in range(3)]
        t["Fx"], t["Fy"], t["Fz"] = F
    return tests


@pytest.mark.parametrize("name,mode,ae,runout,mc", [
    ("slot", "slot", 10, 0, 0.0), ("down 3 mm, runout 5 um, size effect", "down", 3, 5, 0.14),
    ("up 5 mm", "up", 5, 0, 0.0)])
def test_identify_recovers_the_coefficients(ctx, name, mode, ae, runout, mc):
    """identify.test.mjs:28-35."""
    from mcs import identify as I

    tool = {"D": 10, "N": 3, "helixDeg": 30, "fluteLen": 25, "runout": runout}
    tests = _synth(ctx, tool, S50C, mode, ae, mc, 0.02)
    cur = {**S50C, "Ktc": 1000, "Krc": 300, "Kac": 100, "Kte": 10, "Kre": 10, "Kae": 1}
    r = I.identify(ctx, tool, tests, cur, mc)
    print(name, {k: round(v, 1) for k, v in r["coefs"].items()}, "R2", r["r2"])
    for k in ("Ktc", "Krc", "Kte"):
        assert abs(r["coefs"][k] / S50C[k] - 1) < 0.1, k
    assert abs(r["coefs"]["Kac"] / S50C["Kac"] - 1) < 0.15
    assert r["r2"] > 0.999 and not r["edgeFixed"]


def test_one_feed_holds_the_edge_terms(ctx):
    """identify.test.mjs:38-42."""
    from mcs import identify as I

    tool = {"D": 10, "N": 3, "helixDeg": 30, "fluteLen": 25}
    tests = _synth(ctx, tool, A5052, "slot", 10, 0.0, 0.0)[1:2]
    r = I.identify(ctx, tool, tests, A5052, 0.0)
    assert r["edgeFixed"] and r["coefs"]["Kte"] == A5052["Kte"]
    assert abs(r["coefs"]["Ktc"] / A5052["Ktc"] - 1) < 1e-3


def test_sim_revolution_matches_the_oracle(ctx, oracle):
    from mcs import identify as I

    tool = {"D": 10, "N": 3, "helixDeg": 30, "type": "flat", "fluteLen": 25, "runout": 7,
            "runoutPhase": 1.1}
    test = {"S": 6000, "fz": 0.05, "ap": 2, "ae": 3, "mode": "down"}
    got = I.sim_revolution(ctx, tool, A5052, test)
    c, g = _prepared(tool, test, {"Ci": 0.0, **A5052}, decim=1, S=6000)
    ref = oracle.sim_revolution_ref(c, g)
    pp = np.ptp(ref, axis=1, keepdims=True)
    assert np.all(np.abs(got - ref) <= 1e-6 * pp)


def test_fit_record_recovers_coefficients_and_runout(ctx):
    """validate.test.mjs:6-10, 19-27, 39-46: a noisy synthetic record with a ringing,
    averaged over its revolutions, equals the clean revolution; the fit gives the
    coefficients within 4 % and the runout (7 um, between the grid's sizes) within 0.5 um."""
    from mcs import identify as I

    m = A5052
    tool = {"D": 10, "N": 3, "helixDeg": 30, "type": "flat", "fluteLen": 25}
    test = {"S": 6000, "fz": 0.05, "ap": 2, "ae": 3, "mode": "down"}
    truth = {**m, "Ktc": m["Ktc"] * 1.15, "Krc": m["Krc"] * 0.85, "Kte": m["Kte"] * 1.4}
    t_tool = {**tool, "runout": 7, "runoutPhase": 1.1}
    noisy = I.parse_record(I.synthetic_record(ctx, t_tool, truth, test, noise=0.05, ring=0.05,
                                              ringHz=2317, revs=30))
    sa = I.sync_average(noisy["t"], noisy["F"], test["S"])
    clean = I.sim_revolution(ctx, t_tool, truth, test)
    cmp = I.compare(sa["avg"], I.shifted(clean, I.align(sa["avg"], clean)))
    assert all(c["r"] > 0.99 and c["rmsPct"] < 4 for c in cmp), cmp
    assert abs(sa["revs"] - 30) < 0.1
    pk = I.async_peak(noisy["t"], noisy["F"], test["S"], tool["N"], sa["avg"])
    assert abs(pk["f"] - 2317) < 15 and pk["share"] > 0.1
    f = I.fit_record(ctx, tool, m, test, sa["avg"])
    print("fit", {k: round(v, 2) for k, v in f["coefs"].items()}, "runout", f["runout"])
    for k in ("Ktc", "Krc", "Kac", "Kte", "Kre"):
        assert abs(f["coefs"][k] / truth[k] - 1) < 0.04, (k, f["coefs"][k], truth[k])
    assert abs(f["runout"] - 7) <= 0.5
    assert all(c["rmsPct"] < 4 for c in f["cmp"])
