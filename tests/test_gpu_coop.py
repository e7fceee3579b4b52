"""Multi-warp bisection: the heaviest points of a plain solve share their bisection among
several warps of one block, each running one trial of the next levels speculatively
(mcs_opts.coop_warps).  The midpoints are the serial bisection's own square roots and only
the trials on the decision path count, so every width gives byte-identical results to one
trial at a time, in both precisions, through plans and direct calls, with cancellation."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _opts(wl, **kw):
    from mcs import _abi as A

    o = A.Opts.from_buffer_copy(bytes(wl.opts))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_every_width_gives_the_serial_results(ctx, precision):
    from mcs import _abi as A
    from mcs import workloads as W

    wl = W.sweep(n_speeds=384)
    p = A.precision_code(precision)
    ref = ctx.solve(wl.setups, wl.modals, wl.points, _opts(wl, revs=20, precision=p,
                                                           coop_warps=1))
    for w in (0, 3, 4, 8):
        o = _opts(wl, revs=20, precision=p, coop_warps=w)
        got = ctx.solve(wl.setups, wl.modals, wl.points, o)
        assert got.tobytes() == ref.tobytes(), w
        plan = ctx.plan(wl.setups, wl.modals, wl.points, o)
        info = plan.info()
        # the heaviest points take the multi-warp path: one per SM for an explicit width,
        # up to two per SM under the library's rule (a batch of 2.6 points per SM)
        assert 0 < info["coop_points"] <= (2 * 148 if w == 0 else 148), info
        plan.execute()
        assert plan.results().tobytes() == ref.tobytes(), w
        plan.close()
    off = ctx.plan(wl.setups, wl.modals, wl.points, _opts(wl, revs=20, precision=p,
                                                          coop_warps=1))
    assert off.info()["coop_points"] == 0
    off.close()


def test_library_rule_follows_the_tail(ctx):
    """The library's rule gives the multi-warp path to the points that would outlast the
    rest of their batch: none in the 4096-speed sweep (bound by its total work), the slow
    low-speed points of a 768-speed sweep, and every point of an 18-point request."""
    from mcs import workloads as W

    def heads(wl):
        plan = ctx.plan(wl.setups, wl.modals, wl.points, wl.opts)
        n = plan.info()["coop_points"]
        plan.close()
        return n

    assert heads(W.sweep()) == 0
    n768 = heads(W.sweep(n_speeds=768))
    assert 100 <= n768 <= 2 * 148, n768
    assert heads(W.sweep(n_speeds=18)) == 18


def test_small_batch_runs_every_point_on_several_warps(ctx):
    """A Worker-sized request (fewer points than SMs) puts every point on the multi-warp
    path; its limits still replay the oracle's bisection of the reference case."""
    from conftest import load_golden

    from mcs import _abi as A

    g = load_golden("small")
    o = A.opts_from_record(g["opts"])
    o.precision = A.FP64
    plan = ctx.plan(g["setups"], g["modals"], g["points"], o)
    assert plan.info()["coop_points"] == len(g["points"])
    plan.execute()
    got = plan.results()
    plan.close()
    o.coop_warps = 1
    ref = ctx.solve(g["setups"], g["modals"], g["points"], o)
    assert got.tobytes() == ref.tobytes()
    rel = np.abs(got["alim"] / g["results"]["alim"] - 1)
    assert np.all(rel <= 0.02), rel.max()


def test_serial_trial_points_and_nonlinear_cuts(ctx):
    """Hetero points without lane groups (serial_trials) have process damping, size effect
    and the reference slice rule; the multi-warp path covers them too."""
    from mcs import workloads as W

    wl = W.hetero(n=512, first_seed=9001)
    ref = ctx.solve(wl.setups, wl.modals, wl.points, _opts(wl, serial_trials=1, coop_warps=1,
                                                           revs=20))
    o = _opts(wl, serial_trials=1, coop_warps=8, revs=20)
    got = ctx.solve(wl.setups, wl.modals, wl.points, o)
    assert got.tobytes() == ref.tobytes()
    plan = ctx.plan(wl.setups, wl.modals, wl.points, o)
    assert plan.info()["coop_points"] > 0
    plan.close()


def test_cancelled_job_on_the_multi_warp_path(ctx):
    """A cancelled job stops its multi-warp points at a round boundary and reports them as
    cancelled; finished points keep the serial results."""
    from mcs import _abi as A
    from mcs import workloads as W

    wl = W.sweep(n_speeds=96)
    o = _opts(wl, revs=60, coop_warps=4)
    ref = ctx.solve(wl.setups, wl.modals, wl.points, _opts(wl, revs=60, coop_warps=1))
    job = ctx.solve_async(wl.setups, wl.modals, wl.points, o)
    job.cancel()
    res = job.wait()
    job.close()
    st = res["status"]
    assert np.all((st == A.MCS_OK) | (st == A.MCS_ERR_CANCELLED))
    done = st == A.MCS_OK
    assert res[done].tobytes() == ref[done].tobytes()


def test_bad_width_is_rejected(ctx):
    from mcs import MCSError
    from mcs import workloads as W

    wl = W.sweep(n_speeds=16)
    for bad in (-1, 9):
        with pytest.raises(MCSError):
            ctx.solve(wl.setups, wl.modals, wl.points, _opts(wl, coop_warps=bad))
