"""Host parts of identification and validation (mcs.identify): the table and record
parsers, the least squares on given unit forces, the synchronous average and the
asynchronous peak, against the reference's own assertions (test/identify.test.mjs,
test/validate.test.mjs) where they need no simulation."""
from __future__ import annotations

import math

import numpy as np


def test_parse_tests():
    """identify.test.mjs:44-48."""
    from mcs import identify as I

    r = I.parse_tests("# fz ap ae Fx Fy Fz\n0.05, 2, 10, 150, -230, 70\nfz ap\n"
                      "0.04\t2\t10\t140\t-200\t60\n1 2 x 4 5 6", "down")
    assert len(r["tests"]) == 2 and r["tests"][1]["Fy"] == -200
    assert r["tests"][0]["mode"] == "down" and r["bad"] == [5]


def test_parse_record():
    """validate.test.mjs:13-17."""
    from mcs import identify as I

    r = I.parse_record("# S=3000 fz=0.05 ap=2 ae=3 mode=DOWN D=8 N=4 helix=35\nt,Fx,Fy,Fz\n"
                       "0,1,2,3\n0.001;4;5;6\n0.002 7 8\nx\n1,2\n")
    assert r["test"] == {"S": 3000, "fz": 0.05, "ap": 2, "ae": 3, "mode": "down", "D": 8,
                         "N": 4, "helix": 35}
    assert r["t"] == [0, 0.001, 0.002] and r["F"][1] == [2, 5, 8] and len(r["bad"]) == 1


def test_least_squares_recovers_exact_coefficients():
    """With exact mean forces of a known coefficient set the least squares returns it; with
    one feed the edge terms stay at the current values (identify.test.mjs:36-41)."""
    from mcs import identify as I

    rng = np.random.default_rng(2)
    U = rng.normal(size=(4, 6, 3)) * np.array([1, 1, 1, 20, 20, 20])[None, :, None]
    truth = dict(zip(I.COEF_KEYS, (2100.0, 850.0, 400.0, 35.0, 45.0, 10.0)))
    tests = []
    for i, fz in enumerate((0.02, 0.04, 0.06, 0.08)):
        F = [sum(truth[k] * U[i][j][c] for j, k in enumerate(I.COEF_KEYS)) for c in range(3)]
        tests.append({"fz": fz, "ap": 2, "ae": 10, "mode": "slot", "Fx": F[0], "Fy": F[1],
                      "Fz": F[2]})
    cur = dict(zip(I.COEF_KEYS, (1000.0, 300.0, 100.0, 10.0, 10.0, 1.0)))
    r = I.identify_from_units(U, tests, cur)
    assert not r["edgeFixed"] and r["r2"] > 0.999999
    for k in I.COEF_KEYS:
        assert abs(r["coefs"][k] / truth[k] - 1) < 1e-9, k
    one = I.identify_from_units(U[1:2], tests[1:2], {**truth, "Ktc": 1.0})
    assert one["edgeFixed"] and one["coefs"]["Kte"] == truth["Kte"]


def test_sync_average_fills_empty_bins_and_finds_a_ringing():
    """validate.test.mjs:45-49 and 31-38 on a record made here: a waveform locked to the
    spindle plus a ringing at 2317 Hz, sampled too coarsely to hit every bin."""
    from mcs import identify as I

    S, fs, revs = 6000.0, 20000.0, 30
    t = np.arange(int(revs * 60 / S * fs)) / fs
    ang = 2 * math.pi * S / 60 * t
    ring = 5.0 * np.sin(2 * math.pi * 2317 * t)
    F = [100 * np.sin(3 * ang) + ring, 80 * np.cos(3 * ang) + ring, 20 * np.sin(ang)]
    sa = I.sync_average(t, F, S)
    assert abs(sa["revs"] - revs) < 0.1
    pk = I.async_peak(t, F, S, 3, sa["avg"])
    assert abs(pk["f"] - 2317) < 15 and pk["share"] > 0.1
    coarse = np.arange(int(5 * 60 / S * 3000)) / 3000.0
    a = I.sync_average(coarse, [np.sin(2 * math.pi * S / 60 * coarse)] * 3, S)
    assert np.all(np.isfinite(a["avg"])) and np.any(a["cnt"] == 0) and a["avg"].shape == (3, 360)
