"""CPU test of bench.py's legs for the playback engines, the composite lobe diagram and the
unit-force identification: the GPU calls are replaced by the oracle's restatement of the
same runs, so the legs' workloads, host baselines, timings and parity records are checked
without a device (the figures themselves come from the B200 runs)."""
from __future__ import annotations

import time
import types

import numpy as np


class _OracleEngines:
    """mcs.engine.Engines with every engine an oracle CuttingEngine."""

    def __init__(self, ctx, n):
        import pyoracle as O

        self.n = n
        self.es = [O.Engine() for _ in range(n)]

    def configure(self, cfgs):
        for e, c in zip(self.es, cfgs):
            e.configure_from(c)

    def set_engagement(self, gs):
        for e, g in zip(self.es, gs):
            e.engage(g)

    def run(self, steps):
        for e, s in zip(self.es, np.broadcast_to(np.asarray(steps), (self.n,))):
            e.run(int(s))

    def take_stats(self):
        from mcs import _abi as A

        return np.array([e.take_stats_full() for e in self.es], dtype=A.ENGINE_STATS_DTYPE)

    def close(self):
        pass


class _HostEvent:
    def __init__(self, **_):
        self.t = 0.0

    def record(self, stream):
        self.t = time.perf_counter()

    def synchronize(self):
        pass

    def elapsed_time(self, other):
        return 1e3 * (other.t - self.t)


def _stand_ins(monkeypatch, oracle):
    import mcs
    from mcs import engine as E
    from mcs import identify as I

    monkeypatch.setattr(E, "Engines", _OracleEngines)

    def unit_forces(ctx, tool, tests, mc=0.0):
        cfgs, gs = [], []
        for t in tests:
            st, ex = I.immersion(t["mode"], t["ae"], tool["D"])
            for key in I.COEF_KEYS:
                mat = dict.fromkeys(I.COEF_KEYS, 0.0)
                mat.update({key: 1.0, "mc": mc, "Ci": 0.0})
                tl = I._engine_tool(tool, t["ap"], phase=0.0)
                tl["nonlinear"] = mc > 0
                cfgs.append(E.config(tl, E.RIGID, mat, 6000))
                gs.append(E.engagement(E.arc_map(st, ex), (1, 0), t["fz"], -t["ap"], t["ap"]))
        return oracle.unit_forces_ref(cfgs, gs).reshape(len(tests), 6, 3)

    monkeypatch.setattr(I, "unit_forces", unit_forces)

    def composite(sp, base, ctx=None):
        p = {"lobes": 30, "rpmMin": 2000, "rpmMax": 40000, **base}
        return oracle.composite_lobes(sp.record, p, sp.frfs)

    monkeypatch.setattr(mcs, "compositeLobes", composite)
    return types.SimpleNamespace(cuda=types.SimpleNamespace(Event=_HostEvent))


def test_rows_legs_on_host_stand_ins(monkeypatch, oracle):
    import bench

    torch = _stand_ins(monkeypatch, oracle)
    lob = bench.composite_leg(None, False, repeats=1)
    assert lob["parity"]["samples"] > 1000 and lob["parity"]["max_rel_diff"] == 0.0
    assert lob["value"] > 0 and lob["cpu_baseline"]["value"] > 0
    ident = bench.identify_leg(None, False, repeats=1)
    assert ident["parity"]["tests"] == 256 and ident["parity"]["max_rel_diff"] == 0.0
    assert ident["cpu_baseline"]["cores"] >= 1
    play = bench.playback_leg(None, torch, None, False, repeats=1, n=4)
    # one frame is the Simulator's budget of slice-force evaluations
    assert 0.9 * bench.DYN_BUDGET <= play["value"] * play["batch_frame_ms"] / 1e3 / 4 \
        <= bench.DYN_BUDGET
    assert play["parity"]["engines_checked"] == 4
    assert play["parity"]["max_rel_diff_force_sums"] == 0.0
    assert play["parity"]["step_counts_equal"]


def test_rows_leg_records_a_failing_leg(monkeypatch):
    import bench

    def broken(*a, **k):
        raise RuntimeError("no device")

    monkeypatch.setattr(bench, "playback_leg", broken)
    monkeypatch.setattr(bench, "composite_leg", lambda ctx, no_cpu: {"value": 1.0})
    monkeypatch.setattr(bench, "identify_leg", lambda ctx, no_cpu: {"value": 2.0})
    out = bench.rows_leg(None, None, None, True)
    assert out["playback"] == {"error": "RuntimeError: no device"}
    assert out["composite_lobes"]["value"] == 1.0 and out["identify"]["value"] == 2.0
