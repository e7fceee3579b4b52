"""The schedule autotuner on the GPU: results do not depend on the schedule, the tuner
times every candidate and picks one of them, and a cached choice is reused."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_results_identical_for_every_schedule(ctx):
    # the direct call forks one stream per bucket; the plan's graph chains the buckets as
    # programmatic dependent launches: both launch paths, at up to 32 buckets
    from mcs import _abi as A
    from mcs import workloads as W

    wl = W.hetero(n=1536, first_seed=777)
    ref = None
    for nb in (1, 3, 16, 32):
        o = A.make_opts(dict(W.HETERO_OPTS), maxBuckets=nb)
        r = ctx.solve(wl.setups, wl.modals, wl.points, o)
        plan = ctx.plan(wl.setups, wl.modals, wl.points, o)
        plan.execute()
        assert plan.results().tobytes() == r.tobytes()
        info = plan.info()
        # the size classes, plus one multi-warp bucket per block width in use (at most 3)
        assert info["kernels"] <= nb + (3 if info["coop_points"] else 0), info
        plan.close()
        if ref is None:
            ref = r
        assert r.tobytes() == ref.tobytes(), nb


def test_tune_times_every_candidate(ctx):
    from mcs import workloads as W

    wl = W.sweep(n_speeds=512)
    best, ms = ctx.tune(wl.setups, wl.modals, wl.points, wl.opts, (2, 8, 16))
    assert best in (2, 8, 16)
    assert set(ms) == {2, 8, 16} and all(v > 0 for v in ms.values())
    assert ms[best] == min(ms.values())


def test_tune_rejects_bad_schedules(ctx):
    from mcs import MCSError, _abi as A
    from mcs import workloads as W

    wl = W.sweep(n_speeds=64)
    for bad in ((0,), (33,), ()):
        with pytest.raises(MCSError):
            ctx.tune(wl.setups, wl.modals, wl.points, wl.opts, bad)
    o = A.make_opts(maxBuckets=A.MAX_BUCKETS + 1)
    with pytest.raises(MCSError):
        ctx.solve(wl.setups, wl.modals, wl.points, o)


def test_autotune_caches_its_choice(ctx, tmp_path):
    from mcs import tune as T
    from mcs import workloads as W

    wl = W.hetero(n=1024, first_seed=4242)
    path = tmp_path / "tune.json"
    best, rec = T.autotune(ctx, wl.setups, wl.modals, wl.points, wl.opts, candidates=(4, 16),
                           sample=512, cache=path)
    assert not rec["cached"] and rec["sample_points"] == 512 and best in (4, 16)
    best2, rec2 = T.autotune(ctx, wl.setups, wl.modals, wl.points, wl.opts,
                             candidates=(4, 16), cache=path)
    assert rec2["cached"] and best2 == best


def test_lane_group_trials_match_serial_trials(ctx):
    """Speculative bisection levels run in lane groups give byte-identical results to one
    trial at a time (plain solve, plan and guided solve; the same counters too)."""
    from mcs import _abi as A
    from mcs import surrogate as SG
    from mcs import workloads as W
    from mcs._lib import default_guide_opts

    wl = W.hetero(n=1024, first_seed=31337)
    serial = A.Opts.from_buffer_copy(bytes(wl.opts))
    serial.serial_trials = 1
    a = ctx.solve(wl.setups, wl.modals, wl.points, serial)
    b = ctx.solve(wl.setups, wl.modals, wl.points, wl.opts)
    assert a.tobytes() == b.tobytes()
    plan = ctx.plan(wl.setups, wl.modals, wl.points, wl.opts)
    plan.execute()
    assert plan.results().tobytes() == a.tobytes()
    plan.close()
    s = SG.load(ctx)
    for mode in (A.GUIDE_SPECULATE, A.GUIDE_BRACKET):
        g = default_guide_opts()
        g.mode = mode
        ga, ia = ctx.solve_guided(s, wl.setups, wl.modals, wl.points, serial, g)
        gb, ib = ctx.solve_guided(s, wl.setups, wl.modals, wl.points, wl.opts, g)
        assert ga.tobytes() == gb.tobytes()
        for f in ("mu", "sigma", "path"):
            assert np.array_equal(ia[f], ib[f]), f
        # one trial per round serially; lane groups take fewer rounds, never more
        assert np.array_equal(ia["rounds"], ga["trials"])
        assert np.all(ib["rounds"] <= ia["rounds"])
        assert ib["rounds"].sum() < ia["rounds"].sum()
    s.close()
    with pytest.raises(Exception):
        bad = A.Opts.from_buffer_copy(bytes(wl.opts))
        bad.serial_trials = 2
        ctx.solve(wl.setups, wl.modals, wl.points, bad)


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_lane_groups_with_fixed_slice_count(ctx, precision):
    """A fixed slice count of 16 or fewer also packs trials into lane groups; the results
    equal one trial at a time in both precisions."""
    from mcs import _abi as A
    from mcs import workloads as W

    wl = W.hetero(n=256, first_seed=2024)
    o = A.make_opts(dict(W.HETERO_OPTS), slices=8, revs=20, precision=precision)
    s = A.Opts.from_buffer_copy(bytes(o))
    s.serial_trials = 1
    a = ctx.solve(wl.setups, wl.modals, wl.points, s)
    b = ctx.solve(wl.setups, wl.modals, wl.points, o)
    assert a.tobytes() == b.tobytes()
    assert np.all(a["trials"] >= 1)
