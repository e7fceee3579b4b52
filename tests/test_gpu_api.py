"""The host API on the GPU: the reference-shaped functions (stabtd.js / stabworker.js /
sld.js), asynchronous jobs with cancellation, and error reporting through the C ABI."""
from __future__ import annotations

import math
import threading
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

S50C = dict(Ktc=2100, Krc=850, Kte=35, Kre=45, mc=0.14, Ci=1.5e5)
TOOL = dict(N=3, R=5, helixDeg=30, type="flat", fluteLen=25)
ARC = [math.pi / 2, math.pi]


@pytest.fixture(scope="module")
def modal(oracle):
    tm = oracle.tool_model(10, 30, 50000)
    return {"k": tm["k"], "fn": tm["fn"], "zeta": 0.04}


def test_time_domain_limit_matches_reference_numbers(ctx, modal, oracle):
    """The reference's own case (stabtd.test.mjs:9-17) at its defaults, FP64 integration:
    the published 0.94 mm @ 8000 rpm and 0.92 mm @ 2500 rpm without process damping."""
    import mcs

    hi = mcs.timeDomainLimit(TOOL, modal, S50C, 8000, ARC, 0.05, {"precision": "fp64"}, ctx=ctx)
    lin = mcs.timeDomainLimit(TOOL, modal, S50C, 2500, ARC, 0.05,
                              {"nonlinear": False, "precision": "fp64"}, ctx=ctx)
    pd = mcs.timeDomainLimit(TOOL, modal, S50C, 2500, ARC, 0.05, {"precision": "fp64"}, ctx=ctx)
    assert f"{hi['alim']:.2f}" == "0.94"
    assert f"{lin['alim']:.2f}" == "0.92"
    assert f"{pd['alim']:.1f}" == "8.3"
    assert hi["bracket"][0] < hi["alim"] < hi["bracket"][1]
    ref = oracle.timeDomainLimit(TOOL, modal, S50C, 8000, ARC, 0.05)
    assert hi["alim"] == pytest.approx(ref["alim"], rel=1e-12)


def test_open_bracket_like_the_reference(ctx, modal):
    """Stable at aMax: {alim: aMax, bracket: [aMax, Infinity]} (stabtd.js:25)."""
    import mcs

    r = mcs.timeDomainLimit(TOOL, modal, S50C, 8000, ARC, 0.05, {"aMax": 0.3, "revs": 30},
                            ctx=ctx)
    assert r["alim"] == 0.3 and r["bracket"] == [0.3, math.inf]


def test_chatter_at(ctx, modal, oracle):
    import mcs

    for ap, want in ((0.3, False), (3.0, True)):
        assert mcs.chatterAt(TOOL, modal, S50C, 8000, ARC, 0.05, ap, {"revs": 60}, ctx=ctx) is want
    ci = mcs.chatterIndex(TOOL, modal, S50C, 8000, ARC, 0.05, 0.3, {"revs": 60,
                                                                    "precision": "fp64"}, ctx=ctx)
    from mcs import _abi as A

    o = A.make_opts({"revs": 60})
    ref = oracle.chatter_at(A.make_setup(TOOL, S50C, ARC, 0.05), A.make_modal(modal), 8000.0,
                            0.3, o)
    assert ci["index"] == pytest.approx(ref["index"], rel=1e-9, abs=1e-12)


def test_worker_sweep_matches_per_point(ctx, modal):
    """timeDomainLimits over the Worker's 18 log-spaced speeds (main.js:495-501)."""
    import mcs

    r0, r1 = 4000, 30000
    pts = [{"S": round(r0 * (r1 / r0) ** (i / 17)), "modal": modal} for i in range(18)]
    opts = {"revs": 30, "iters": 5}
    batch = mcs.timeDomainLimits(TOOL, S50C, ARC, 0.05, pts, opts, ctx=ctx)
    assert [b["S"] for b in batch] == [p["S"] for p in pts]
    for p, b in list(zip(pts, batch))[::6]:
        one = mcs.timeDomainLimit(TOOL, modal, S50C, p["S"], ARC, 0.05, opts, ctx=ctx)
        assert one["alim"] == b["alim"]


def test_stab_worker_protocol_and_supersession(ctx, modal):
    """A newer message replaces an older one: only the newer posts, then done."""
    import mcs

    got = []
    done = threading.Event()

    def onmessage(m):
        got.append(m)
        if m.get("done"):
            done.set()

    w = mcs.StabWorker(onmessage, ctx=ctx)
    slow = [{"S": 3000 + 10 * i, "modal": modal} for i in range(2000)]
    fast = [{"S": 8000, "modal": modal}, {"S": 12000, "modal": modal}]
    base = {"tool": TOOL, "mat": S50C, "arc": ARC, "fz": 0.05, "nonlinear": True}
    w.postMessage(dict(base, key="old", points=slow))
    w.postMessage(dict(base, key="new", points=fast))
    assert done.wait(120)
    w.join(60)
    assert not w.errors
    assert all(m["key"] == "new" for m in got)
    assert [m["S"] for m in got if not m.get("done")] == [8000, 12000]
    assert got[-1] == {"key": "new", "done": True}


def test_async_job_cancel(ctx):
    from mcs import workloads as W

    wl = W.sweep()
    wl.opts.revs = 120
    job = ctx.solve_async(wl.setups, wl.modals, wl.points, wl.opts)
    time.sleep(0.02)
    job.cancel()
    res = job.wait()
    assert job.cancelled
    st = res["status"]
    assert set(np.unique(st)) <= {0, 5}
    assert (st == 5).sum() > 0
    done, fin = job.poll()
    assert fin and done == wl.n
    job.close()


def test_async_job_completes(ctx):
    from mcs import workloads as W

    wl = W.small()
    wl.opts.revs = 10
    job = ctx.solve_async(wl.setups, wl.modals, wl.points, wl.opts)
    res = job.wait()
    assert not job.cancelled and np.all(res["status"] == 0)
    ref = ctx.solve(wl.setups, wl.modals, wl.points, wl.opts)
    assert res.tobytes() == ref.tobytes()
    job.close()


def test_argument_errors(ctx):
    import mcs
    from mcs import _abi as A
    from mcs import workloads as W

    wl = W.small()
    bad = wl.points.copy()
    bad["setup"][3] = 7
    with pytest.raises(mcs.MCSError) as e:
        ctx.solve(wl.setups, wl.modals, bad, wl.opts)
    assert e.value.status == A.MCS_ERR_ARG and "setup index" in str(e.value)
    o = A.make_opts(aMin=1.0, aMax=0.5)
    with pytest.raises(mcs.MCSError):
        ctx.solve(wl.setups, wl.modals, wl.points, o)
    nan = wl.points.copy()
    nan["S"][0] = float("nan")
    with pytest.raises(mcs.MCSError):
        ctx.solve(wl.setups, wl.modals, nan, wl.opts)
    with pytest.raises(mcs.MCSError) as e:
        ctx.solve(wl.setups, wl.modals, wl.points, A.make_opts(slices=65))
    assert e.value.status == A.MCS_ERR_UNSUPPORTED
    # the context stays usable after errors
    assert len(ctx.solve(wl.setups, wl.modals, wl.points[:2], A.make_opts(revs=5, iters=1))) == 2


def test_empty_batch(ctx):
    from mcs import _abi as A
    from mcs import workloads as W

    wl = W.small()
    out = ctx.solve(wl.setups, wl.modals, wl.points[:0], wl.opts)
    assert len(out) == 0
    lim = ctx.lobes_alim(wl.modals, [], np.array([1000.0]))
    assert lim.shape == (0, 1)


def test_lobe_limit_mirror(ctx, oracle, modal):
    import mcs

    p = dict(modal, N=3, Ktc=2100, Krc=850, phiSt=ARC[0], phiEx=ARC[1], lobes=30,
             rpmMin=2000, rpmMax=40000)
    rpm = np.array([2500.0, 8000.0, 12345.0, 39000.0])
    got = mcs.lobeLimit(p, rpm, ctx=ctx)
    lobes = oracle.stabilityLobes(p)
    want = [oracle.alimAt(lobes, r) for r in rpm]
    assert np.allclose(got, want, rtol=1e-10)


def test_solve_multi_equals_solve(ctx):
    """mcs_solve_multi over one context, and over two contexts on the same device (one host
    thread each), gives mcs_solve's records in input order."""
    import mcs
    from mcs import workloads as W

    wl = W.hetero(n=300, first_seed=55)
    wl.opts.revs = 20
    ref = ctx.solve(wl.setups, wl.modals, wl.points, wl.opts)
    one = mcs.solve_multi([ctx], wl.setups, wl.modals, wl.points, wl.opts)
    assert one.tobytes() == ref.tobytes()
    c2 = mcs.Context(0)
    try:
        two = mcs.solve_multi([ctx, c2], wl.setups, wl.modals, wl.points, wl.opts)
    finally:
        c2.close()
    assert two.tobytes() == ref.tobytes()
