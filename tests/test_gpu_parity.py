"""GPU parity: the CUDA path (through the C ABI) against the FP64 oracle on the same
seeded inputs, via the committed golden fixtures.

Bars (the FP32 integration against the FP64 reference, decision at index > 0.45):
  * decision replay: the GPU's chatterAt at every depth the oracle's bisection visited
    returns the oracle's decision; trials whose oracle index lies within DECISION_BAND of
    the threshold are near-ties that FP32 rounding may legitimately flip;
  * critical depth: |alim_gpu / alim_fp64 - 1| <= 2 % on at least 99 % of points;
  * chatter index value: within INDEX_RTOL relative (+ INDEX_ATOL) of the oracle for
    trials that stay stable (chatter trials grow chaotically and are compared by decision).
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

DECISION_BAND = 0.02   # |index - 0.45| below this: a near-tie
DEPTH_RTOL = 0.02      # critical-depth tolerance (north star: 2 %)
DEPTH_QUANTILE = 0.99  # ... on at least 99 % of points
INDEX_RTOL = 2e-3
INDEX_ATOL = 1e-4


def opts_of(g):
    from mcs import _abi as A

    return A.Opts.from_buffer_copy(g["opts"].tobytes())


def replay(ctx, g):
    """GPU chatterAt at every traced oracle depth -> (oracle trace rows, gpu results)."""
    from mcs import _abi as A

    tr = g["traces"]
    res = g["results"]
    rows = []
    for p in range(len(res)):
        for j in range(int(res["trials"][p])):
            rows.append((p, j))
    trials = np.zeros(len(rows), dtype=A.TRIAL_DTYPE)
    ref = np.zeros(len(rows), dtype=tr.dtype)
    for i, (p, j) in enumerate(rows):
        trials[i] = (p, 0, tr[p, j]["ap"])
        ref[i] = tr[p, j]
    out = ctx.chatter_at(g["setups"], g["modals"], g["points"], trials, opts_of(g))
    return ref, out


def check_replay(name, ref, out, min_agree=1.0):
    assert np.all(out["status"] == 0), f"{name}: trial status {np.unique(out['status'])}"
    agree = out["chatter"] == ref["chatter"]
    near = np.abs(ref["index"] - 0.45) < DECISION_BAND
    rate = agree.mean()
    far_bad = np.flatnonzero(~agree & ~near)
    print(f"{name}: decision agreement {agree.sum()}/{len(agree)} = {rate:.4f}; "
          f"disagreements outside the near-tie band: {len(far_bad)}")
    assert len(far_bad) == 0, (
        f"{name}: decisions differ away from the threshold at rows {far_bad[:10]}: "
        f"oracle idx {ref['index'][far_bad[:10]]}, gpu idx {out['index'][far_bad[:10]]}")
    assert rate >= min_agree
    return rate


def check_depths(name, ref, got):
    assert np.all(got["status"] == 0), f"{name}: status {np.unique(got['status'])}"
    both_open = (ref["open"] == 1) & (got["open"] == 1)
    rel = np.abs(got["alim"] / ref["alim"] - 1)
    rel[both_open] = 0.0
    ok = rel <= DEPTH_RTOL
    print(f"{name}: depth within {DEPTH_RTOL:.0%} on {ok.sum()}/{len(ok)}; "
          f"median rel err {np.median(rel):.2e}, worst {rel.max():.3f}")
    assert ok.mean() >= DEPTH_QUANTILE, f"{name}: worst points {np.argsort(-rel)[:5]}"


@pytest.mark.parametrize("name", ["small", "edge", "sweep", "hetero"])
def test_decision_replay(ctx, name):
    g = load_golden(name)
    ref, out = replay(ctx, g)
    check_replay(name, ref, out, min_agree=0.97)


@pytest.mark.parametrize("name", ["small", "edge", "sweep", "hetero"])
def test_bisection_depths(ctx, name):
    g = load_golden(name)
    got = ctx.solve(g["setups"], g["modals"], g["points"], opts_of(g))
    check_depths(name, g["results"], got)
    # the device counts the reference loop's evaluations exactly (steps * N * nz per trial)
    assert np.all(got["evals"] > 0)
    assert np.all(got["engaged"] <= got["evals"])


def test_index_values_stable_trials(ctx):
    """Stable trials are smooth functions of the inputs: the FP32 index tracks FP64."""
    g = load_golden("small")
    ref, out = replay(ctx, g)
    stable = (ref["index"] < 0.3) & (out["index"] < 0.3)
    d = np.abs(out["index"] - ref["index"])
    tol = INDEX_ATOL + INDEX_RTOL * np.abs(ref["index"])
    frac = (d[stable] <= tol[stable]).mean()
    print(f"stable trials: {stable.sum()}, index within tol: {frac:.4f}, "
          f"max abs diff {d[stable].max():.2e}")
    assert frac >= 0.95


def test_deterministic(ctx):
    g = load_golden("small")
    a = ctx.solve(g["setups"], g["modals"], g["points"], opts_of(g))
    b = ctx.solve(g["setups"], g["modals"], g["points"], opts_of(g))
    assert a.tobytes() == b.tobytes()


def test_plan_matches_solve(ctx):
    g = load_golden("small")
    a = ctx.solve(g["setups"], g["modals"], g["points"], opts_of(g))
    plan = ctx.plan(g["setups"], g["modals"], g["points"], opts_of(g))
    for _ in range(2):
        plan.execute()
        b = plan.results()
        assert a.tobytes() == b.tobytes()
    info = plan.info()
    assert info["graph"] == 1 and info["kernels"] >= 1
    plan.close()


def test_lobes_match_oracle(ctx, oracle):
    from mcs import _abi as A

    g = load_golden("small")
    sweep = load_golden("sweep")
    modals = np.concatenate([g["modals"], sweep["modals"]])
    qs = [oracle.lobe_query(4, 700, 210, math.pi / 2, math.pi, 30, 2000, 40000, 0),
          oracle.lobe_query(4, 700, 210, 0.0, math.pi, 12, 3000, 30000, 1),
          oracle.lobe_query(3, 2100, 850, math.pi / 2, math.pi, 30, 2000, 40000, 1)]
    rpm = np.linspace(2500.0, 39000.0, 777)
    got = ctx.lobes_alim(modals, qs, rpm)
    cm = [A.Modal.from_buffer_copy(m.tobytes()) for m in modals]
    ref = oracle.lobes_alim(cm, qs, rpm)
    fin = np.isfinite(ref)
    assert np.array_equal(fin, np.isfinite(got))
    rel = np.abs(got[fin] / ref[fin] - 1)
    print(f"lobes: {fin.sum()} finite values, max rel diff {rel.max():.2e}")
    assert rel.max() < 1e-9
