"""The GPU cutting engines (mcs_engine_*) against the oracle's CuttingEngine: the same
configure / engagement / run sequence on both, compared on every statistic takeStats()
returns, the history ring, the chatter index and the carried state.

The cases are stable cuts, where the FP64 trajectories of the two implementations stay
within rounding of each other (the GPU sums a step's slice forces in a warp butterfly, the
reference slice by slice): a stability trial with process damping, size effect and runout;
a rigid-tool unit-force run (identify.js:26-40) with the axial coefficients; a plunge on
the end edges with a ball-nose tip profile; a thin wall with flank wear and a stock-like
height map; a tapered edge profile (rAt)."""
from __future__ import annotations

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 1e-9  # relative, on sums over thousands of steps of FP64 arithmetic


def _cases():
    from mcs import engine as E

    rng = np.random.default_rng(11)
    S50C = {"Ktc": 2100, "Krc": 850, "Kac": 400, "Kte": 35, "Kre": 45, "Kae": 10, "mc": 0.14,
            "Ci": 1.5e5}
    cases = []
    # 1. a stability trial at a small depth: half-immersion down milling, 2 + 1 modes
    tool = {"N": 3, "R": 5.0, "helixDeg": 30, "fluteLen": 25, "runout": 5.0, "runoutPhase": 0.7}
    modal = {"k": 0, "fn": 0, "zeta": 0,
             "modesX": [{"k": 1.2e4, "fn": 1900.0, "zeta": 0.03},
                        {"k": 4e4, "fn": 3400.0, "zeta": 0.02}],
             "modesY": [{"k": 1.5e4, "fn": 2100.0, "zeta": 0.03}]}
    c = E.config(tool, modal, S50C, 8000)
    g = [E.engagement(E.arc_map(math.pi / 2, math.pi), (1, 0), 0.05, -0.4, 0.4)]
    cases.append(("trial", c, g, [(0, 3000)], (0.0, 0.0, 0.01, 0.0)))
    # 2. a rigid-tool unit-force run: Kac alone, slot, size effect
    mat = dict.fromkeys(("Ktc", "Krc", "Kac", "Kte", "Kre", "Kae"), 0.0)
    mat.update(Kac=1.0, mc=0.2, Ci=0.0)
    c = E.config({"N": 4, "R": 4.0, "helixDeg": 35, "fluteLen": 6.0, "runout": 8.0},
                 E.RIGID, mat, 6000)
    g = [E.engagement(E.arc_map(0, math.pi), (1, 0), 0.04, -5.0, 5.0)]
    cases.append(("unit", c, g, [(0, 2 * 4 * 0 + 1000)], None))
    # 3. a plunge: end edges only (no side engagement), ball-nose tip profile
    R = 4.0
    c = E.config({"N": 2, "R": R, "helixDeg": 30, "fluteLen": 20, "type": "ball"},
                 {"k": 2e4, "fn": 2500.0, "zeta": 0.04}, S50C, 5000)
    zat = lambda r: R - math.sqrt(max(0.0, R * R - r * r))
    eb = (rng.uniform(0.0, 0.3, (36, 6)) * (rng.uniform(size=(36, 6)) > 0.2)).astype(np.float32)
    g = [E.engagement(np.full(180, -np.inf, dtype=np.float32), (1, 0), 0.0, -1.0, 0.0, Eb=eb,
                      fza=0.02, rOut=R * 0.95, zAt=zat)]
    cases.append(("plunge", c, g, [(0, 1500)], None))
    # 4. a thin wall, flank wear, a stock-like map; two substeps with a new engagement
    c = E.config({"N": 3, "R": 5.0, "helixDeg": 40, "fluteLen": 15},
                 {"k": 2.5e4, "fn": 2200.0, "zeta": 0.04}, S50C, 9000, fn_max=3000)
    hb = np.where(np.sin((np.arange(180) + 0.5) / 180 * 2 * math.pi) > 0.02,
                  rng.uniform(-0.5, 2.0, 180), -np.inf).astype(np.float32)
    wall = {"k": 800.0, "m": 0.05, "zeta": 0.02, "nx": 0.0, "ny": 1.0}
    g1 = E.engagement(hb, (1, 0), 0.06, -2.0, 3.5, wall=wall, wear={"Kte": 50.0, "Kre": 60.0})
    g2 = E.engagement(np.roll(hb, 7), (0.8, 0.6), 0.05, -2.0, 3.0, wall=wall)
    cases.append(("wall", c, [g1, g2], [(0, 1200), (1, 900)], None))
    # 5. a tapered edge: the radius grows 0.2 mm per mm up the flute
    taper = lambda z: 2.0 + 0.2 * z
    c = E.config({"N": 4, "R": 2.0, "helixDeg": 30, "fluteLen": 12},
                 {"k": 8e3, "fn": 1800.0, "zeta": 0.03}, S50C, 12000)
    dz = max(0.25, 12 / 48)
    g = [E.engagement(E.arc_map(0.0, 1.2), (1, 0), 0.03, -3.0, 3.0, rAt=taper, dz=dz)]
    cases.append(("taper", c, g, [(0, 1600)], None))
    return cases


def _oracle_run(oracle, cfg, gs, seq, kick):
    e = oracle.Engine()
    e.configure_from(cfg)
    stats = []
    for i, (gi, n) in enumerate(seq):
        e.engage(gs[gi])
        if kick is not None and i == 0:
            e.set_state(*kick)
        e.run(n)
    return e


def test_engines_match_the_oracle(ctx, oracle):
    from mcs import _abi as A
    from mcs import engine as E

    cases = _cases()
    n = len(cases)
    eng = E.Engines(ctx, n)
    eng.configure([c[1] for c in cases])
    n_sub = max(len(c[3]) for c in cases)
    for sub in range(n_sub):
        gs = [c[2][c[3][min(sub, len(c[3]) - 1)][0]] for c in cases]
        eng.set_engagement(gs)
        if sub == 0:
            eng.set_state([c[4] if c[4] is not None else (0, 0, 0, 0) for c in cases])
        eng.run([c[3][sub][1] if sub < len(c[3]) else 0 for c in cases])
    got = eng.take_stats()
    hist, head, count = eng.history()
    ci = eng.chatter_index()
    st = eng.state()
    again = eng.take_stats()  # takeStats resets
    assert np.all(again["n"] == 0) and np.all(np.isinf(again["minX"]))
    for k, (name, cfg, gs, seq, kick) in enumerate(cases):
        o = _oracle_run(oracle, cfg, gs, seq, kick)
        ref = o.take_stats_full()
        for f in A.ENGINE_STATS_FIELDS:
            a, b = float(got[k][f]), float(ref[f])
            tol = RTOL * max(abs(b), 1e-300) + (1e-300 if b == 0 else 0)
            if f in ("minX", "maxX", "minY", "maxY", "sumX", "sumY", "sumW", "maxW"):
                tol = RTOL * max(abs(b), 1e-12)  # positions near zero: absolute floor
            assert abs(a - b) <= tol or (a == b), (name, f, a, b)
        oh, ohead, ocount = o.history()
        assert head[k] == ohead and count[k] == ocount, name
        m = min(int(count[k]), A.ENGINE_HIST)
        idx = (ohead - 1 - np.arange(m)) % A.ENGINE_HIST
        scale = np.maximum(np.abs(oh[:, idx]).max(axis=1, keepdims=True), 1e-30)
        assert np.all(np.abs(hist[k][:, idx] - oh[:, idx]) <= 1e-6 * scale), name
        oc = o.chatter_index()
        assert abs(ci[k][0] - oc["index"]) <= 1e-6 * max(1.0, abs(oc["index"])), name
        info = o.info()
        assert st[k]["steps_per_tooth"] == info["steps_per_tooth"], name
        assert st[k]["pr"] == sum(n for _, n in seq) % info["steps_per_rev"], name
        print(f"{name}: n {int(got[k]['n'])}, sumFx {got[k]['sumFx']:.6e}, "
              f"sumFz {got[k]['sumFz']:.6e}, sumT {got[k]['sumT']:.6e}")
    eng.close()


def test_engine_rejects_misuse(ctx):
    from mcs import MCSError
    from mcs import engine as E

    eng = E.Engines(ctx, 2)
    with pytest.raises(MCSError):  # run before configure
        eng.run([10, 10])
    c = E.config({"N": 2, "R": 3.0, "fluteLen": 10}, {"k": 1e4, "fn": 2000, "zeta": 0.03},
                 {"Ktc": 700, "Krc": 210}, 6000)
    eng.configure([c, c])
    with pytest.raises(MCSError):  # no engagement yet
        eng.run([10, 0])
    eng.set_engagement([E.engagement(E.arc_map(0, math.pi), (1, 0), 0.05, -1, 1)] * 2)
    eng.run([10, 0])  # an idle engine is fine
    s = eng.take_stats()
    assert s["n"][0] == 10 and s["n"][1] == 0
    with pytest.raises(MCSError):
        eng.run([-1, 0])
    eng.close()
