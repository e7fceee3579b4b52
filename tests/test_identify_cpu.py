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


def test_engagement_records_and_unit_force_inputs():
    """The engine records the host builds: a map of the wrong length is rejected, the map
    and end-face arrays land in the record as float32 (infinities kept), and the unit-force
    runs hand the library one configuration per coefficient with the test's engagement."""
    import ctypes as C

    import pytest

    from mcs import _abi as A
    from mcs import engine as E
    from mcs import identify as I

    with pytest.raises(ValueError):
        E.engagement(np.zeros(A.BINS - 1), (1, 0), 0.05, -1.0, 1.0)
    hb = np.where(np.arange(A.BINS) % 3 == 0, -np.inf, np.linspace(-1, 2, A.BINS))
    eb = np.linspace(0, 0.3, A.END_BINS * A.END_RINGS).reshape(A.END_BINS, A.END_RINGS)
    g = E.engagement(hb, (1, 0), 0.05, -1.0, 1.0, Eb=eb, fza=0.02, rOut=4.0)
    assert np.array_equal(np.frombuffer(bytes(g.Hb), dtype=np.float32),
                          hb.astype(np.float32))
    assert np.array_equal(np.frombuffer(bytes(g.Eb), dtype=np.float32),
                          eb.astype(np.float32).ravel())

    seen = {}

    class Recorder:  # stands in for the device engines
        def __init__(self, ctx, n):
            self.n = n

        def configure(self, cfgs):
            seen["cfg"] = [bytes(c) for c in cfgs]

        def set_engagement(self, gs):
            seen["eng"] = [bytes(x) for x in gs]

        def run(self, steps):
            seen.setdefault("steps", []).append(np.asarray(steps).copy())

        def take_stats(self):
            out = np.zeros(self.n, dtype=A.ENGINE_STATS_DTYPE)
            out["n"] = 1
            return out

        def close(self):
            pass

    real = E.Engines
    E.Engines = Recorder
    try:
        tool = {"D": 10.0, "N": 3, "helixDeg": 30.0, "fluteLen": 25.0}
        tests = [{"fz": 0.05, "ap": 2.0, "ae": 10.0, "mode": "slot"},
                 {"fz": 0.08, "ap": 1.0, "ae": 3.0, "mode": "down"}]
        U = I.unit_forces(None, tool, tests)
    finally:
        E.Engines = real
    assert U.shape == (2, 6, 3)
    # one configuration per coefficient; both tests use the same tool (flute length
    # max(25, ap + 1) = 25), so their six configurations agree
    assert len(seen["cfg"]) == 12 and len(set(seen["cfg"][:6])) == 6
    assert seen["cfg"][:6] == seen["cfg"][6:]
    for t, test in enumerate(tests):
        st, ex = I.immersion(test["mode"], test["ae"], tool["D"])
        want = bytes(E.engagement(E.arc_map(st, ex), (1, 0), test["fz"], -test["ap"],
                                  test["ap"]))
        assert seen["eng"][6 * t: 6 * t + 6] == [want] * 6
    # two revolutions, statistics dropped, one revolution
    assert np.array_equal(seen["steps"][0], 2 * seen["steps"][1])
    assert C.sizeof(A.Engagement) == len(seen["eng"][0])
