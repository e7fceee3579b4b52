"""The surrogate on the GPU: BF16 forward and backward kernels against the FP64 reference
MLP (oracle/mlp_ref.py), training, and the guided solve against the plain bisection."""
from __future__ import annotations

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def params():
    from test_surrogate_cpu import random_params

    return random_params(np.random.default_rng(11), scale=1.0)


@pytest.fixture(scope="module")
def feats(ctx):
    from mcs import workloads as W

    wl = W.hetero(n=2048, first_seed=50000)
    return wl, ctx.features(wl.setups, wl.modals, wl.points, wl.opts)


def test_forward_matches_fp64_reference(ctx, params, feats):
    import mlp_ref as R
    from mcs import Surrogate

    _, X = feats
    s = Surrogate(ctx, 1)
    s.set_params(params.astype(np.float32))
    mu, sg = s.predict(X)
    mu_r, sg_r = R.predict(params.astype(np.float32).astype(np.float64), X.astype(np.float64))
    err_mu = np.abs(mu - mu_r)
    print(f"forward: |mu| rms {np.sqrt(np.mean(mu_r ** 2)):.3f}, max |d mu| {err_mu.max():.4f}, "
          f"max rel d sigma {np.max(np.abs(sg / sg_r - 1)):.4f}")
    # BF16 weights and activations: ~0.4 % per layer
    assert np.all(err_mu <= 0.03 * (1 + np.abs(mu_r)))
    assert np.all(np.abs(sg / sg_r - 1) <= 0.06)
    s.close()


def test_tensor_core_inference_many_tiles(ctx, params, feats):
    """Inference runs on the tcgen05 kernel (128-row tiles, persistent CTAs).  39963 rows
    need several tiles per CTA and end in a ragged tile; the outputs match the FP64
    reference MLP and give the same NLL as the training forward (the GEMM kernel)."""
    import mlp_ref as R
    from mcs import Surrogate

    _, X = feats
    rng = np.random.default_rng(2)
    n = 40000 - 37
    Xb = (np.concatenate([X] * 20)[:n]
          * (1 + 0.01 * rng.standard_normal((n, X.shape[1])))).astype(np.float32)
    p32 = params.astype(np.float32)
    s = Surrogate(ctx, 1)
    s.set_params(p32)
    mu, sg = s.predict(Xb)
    mu_r, sg_r = R.predict(p32.astype(np.float64), Xb.astype(np.float64))
    assert np.all(np.abs(mu - mu_r) <= 0.03 * (1 + np.abs(mu_r)))
    assert np.all(np.abs(sg / sg_r - 1) <= 0.06)
    y = (mu_r[:4096] + rng.normal(scale=0.3, size=4096)).astype(np.float32)
    loss_train, _ = s.grad(Xb[:4096], y)
    ls = np.log(sg[:4096].astype(np.float64))
    loss_tc = float(np.mean(ls + 0.5 * (y - mu[:4096]) ** 2 * np.exp(-2 * ls)))
    print(f"NLL: training forward {loss_train:.5f}, tensor-core inference {loss_tc:.5f}")
    assert loss_tc == pytest.approx(loss_train, rel=2e-3, abs=2e-3)
    s.close()


def test_gradient_matches_fp64_reference(ctx, params, feats):
    """The gradient check of the training kernels against the CPU oracle."""
    import mlp_ref as R
    from mcs import Surrogate

    _, X = feats
    X = X[:1024]
    p32 = params.astype(np.float32)
    mu_r, _ = R.predict(p32.astype(np.float64), X.astype(np.float64))
    y = (mu_r + np.random.default_rng(5).normal(scale=0.5, size=len(X))).astype(np.float32)
    s = Surrogate(ctx, 1)
    s.set_params(p32)
    loss, g = s.grad(X, y)
    loss_r, g_r = R.loss_and_grad(p32.astype(np.float64), X.astype(np.float64), y.astype(np.float64))
    W_, b_, _ = R.layout()
    # the mean loss is near 0: BF16 activations shift it by a few 1e-3
    assert loss == pytest.approx(loss_r, rel=0.02, abs=0.01)
    for l, ((o, k, n), (ob, nb)) in enumerate(zip(W_, b_)):
        for lo, hi in ((o, o + k * n), (ob, ob + nb)):
            a, r = g[lo:hi].astype(np.float64), g_r[lo:hi]
            rel = np.linalg.norm(a - r) / max(np.linalg.norm(r), 1e-30)
            cos = a @ r / max(np.linalg.norm(a) * np.linalg.norm(r), 1e-30)
            print(f"layer {l} [{lo}:{hi}]: rel L2 err {rel:.4f}, cosine {cos:.6f}")
            assert rel < 0.05 and cos > 0.998
    # normalisation entries are not trained
    assert np.all(g[:2 * R.N_IN] == 0)
    s.close()


def test_training_fits_a_smooth_target(ctx, feats):
    from mcs import Surrogate, _abi as A
    from mcs._lib import default_train_opts

    _, X = feats
    Z = (X - X.mean(0)) / (X.std(0) + 1e-6)
    y = (0.6 * Z[:, 0] - 0.4 * Z[:, 11] + 0.3 * np.sin(Z[:, 4]) + 0.2 * Z[:, 12] * Z[:, 13]
         ).astype(np.float32)
    s = Surrogate(ctx, 7)
    o = default_train_opts()
    o.epochs, o.batch, o.lr = 60, 256, 2e-3
    tl, vl = s.train(X[:1536], y[:1536], X[1536:], y[1536:], o)
    mu, sg = s.predict(X[1536:])
    r2 = 1 - np.mean((mu - y[1536:]) ** 2) / np.var(y[1536:])
    print(f"train loss {tl[0]:.3f} -> {tl[-1]:.3f}, val loss {vl[-1]:.3f}, val R^2 {r2:.3f}")
    assert tl[-1] < tl[0] - 0.5
    assert r2 > 0.9
    assert np.all(np.isfinite(sg)) and np.all(sg > 0)
    s.close()


@pytest.fixture(scope="module")
def trained_small(ctx):
    """A surrogate trained on labels the GPU solver makes for 2048 seeded setups
    (20 revolutions per trial to keep the test short) and 512 held-out points."""
    from mcs import Surrogate, surrogate as SG
    from mcs import workloads as W
    from mcs._lib import default_train_opts

    wl = W.hetero(n=2560, first_seed=90000)
    wl.opts.revs = 20
    X = ctx.features(wl.setups, wl.modals, wl.points, wl.opts)
    y, res = SG.labels(ctx, wl)
    s = Surrogate(ctx, 3)
    o = default_train_opts()
    o.epochs, o.batch = 40, 256
    s.train(X[:2048], y[:2048], None, None, o)
    held = wl.subset(np.arange(2048, 2560))
    return s, held, res[2048:]


def wide_guide():
    """The bracket method with its default options, but no point goes straight to the
    plain bisection, so that every path is exercised whatever the small model's sigma."""
    from mcs import _abi as A
    from mcs._lib import default_guide_opts

    g = default_guide_opts()
    g.mode = A.GUIDE_BRACKET
    g.hw_direct = 100.0
    g.hw_max = math.log(2.0)
    return g


def test_guided_solve_against_plain(ctx, trained_small):
    from mcs import _abi as A

    s, wl, plain = trained_small
    res, info = ctx.solve_guided(s, wl.setups, wl.modals, wl.points, wl.opts, wide_guide())
    path = info["path"]
    assert set(np.unique(path)) <= {0, 1, 2, 3}
    counts = {A.PATH_NAMES[k]: int((path == k).sum()) for k in range(4)}
    # paths that end in the plain algorithm give the plain result exactly, and so does an
    # open point (decided by the plain first trial)
    op = path == A.PATH_OPEN
    full = (path == A.PATH_FALLBACK) | (path == A.PATH_DIRECT) | op
    for f in ("alim", "lo", "hi", "open"):
        assert np.array_equal(res[f][full], plain[f][full]), f
    assert np.all(res["open"][op] == 1)
    assert np.all(plain["open"][path == A.PATH_GUIDED] == 0)
    g = path == A.PATH_GUIDED
    rel = np.abs(res["alim"][g] / plain["alim"][g] - 1)
    within = float(np.mean(rel <= 0.03)) if g.any() else 1.0
    trials_g, trials_p = res["trials"].sum(), plain["trials"].sum()
    print(f"paths {counts}; guided within 3 %: {within:.3f}; trials {trials_g} vs plain "
          f"{trials_p}")
    assert counts["direct"] == 0
    assert g.sum() > 0.2 * len(path)
    assert within >= 0.8
    # every guided bracket is what its trials say: stable at lo (a_min is taken as stable,
    # as in the plain method), chatter at hi -- replayed through mcs_chatter_at
    gi = np.where(g)[0]
    tr = np.zeros(2 * len(gi), dtype=A.TRIAL_DTYPE)
    tr["point"] = np.repeat(gi, 2)
    tr["ap"] = np.stack([res["lo"][gi], res["hi"][gi]], 1).ravel()
    ch = ctx.chatter_at(wl.setups, wl.modals, wl.points, tr, wl.opts)["chatter"].reshape(-1, 2)
    at_min = res["lo"][gi] <= wl.opts.a_min
    assert np.all((ch[:, 0] == 0) | at_min)
    assert np.all(ch[:, 1] == 1)
    assert np.all(res["lo"][gi] < res["hi"][gi])
    assert np.all((res["lo"][gi] >= wl.opts.a_min) & (res["hi"][gi] <= wl.opts.a_max))
    # a_max + 2 bracket checks + 3 refinements + ceil(log2(hw / hw_min)) <= 9 < 1 + 10
    assert np.all(res["trials"][g] <= 9) and np.all(res["trials"][g] < plain["trials"][g])
    # the open path is the plain first trial
    assert np.all(res["trials"][op] == 1) and np.all(plain["trials"][op] == 1)
    # a fallback runs the plain algorithm after at most 2 bracket checks (a_max is shared)
    fb = path == A.PATH_FALLBACK
    assert np.all(res["trials"][fb] <= plain["trials"][fb] + 2)
    assert np.all(res["trials"][fb] > plain["trials"][fb])
    # mu and sigma come back with the results
    assert np.all(np.isfinite(info["mu"])) and np.all(info["sigma"] > 0)


def plain_bracket_after(lo_final, hi_final, a_min, a_max, levels):
    """The plain geometric bisection's bracket after `levels` levels on the way to its
    final bracket (every decision of the path is the side the final bracket lies on)."""
    lo = np.full(len(lo_final), a_min)
    hi = np.full(len(lo_final), a_max)
    for _ in range(levels):
        m = np.sqrt(lo * hi)
        c = hi_final <= m
        hi = np.where(c, m, hi)
        lo = np.where(c, lo, m)
    return lo, hi


def test_speculative_guide_is_the_plain_bisection(ctx, trained_small):
    """The default guided method runs the plain bisection's own trials, steered by the
    prediction: after `levels` levels its bracket is exactly the plain bisection's, so the
    limit lies within half that bracket's width of the plain limit (1.12 % for 8 of the
    10 levels over [0.05, 15]); with levels = iters the results are the plain ones byte for
    byte."""
    from mcs import _abi as A
    from mcs._lib import default_guide_opts

    s, wl, plain = trained_small
    g = default_guide_opts()
    assert g.mode == A.GUIDE_SPECULATE and g.levels == 8
    res, info = ctx.solve_guided(s, wl.setups, wl.modals, wl.points, wl.opts, g)
    op = plain["open"] == 1
    assert np.array_equal(res["open"], plain["open"])
    for f in ("alim", "lo", "hi", "trials"):
        assert np.array_equal(res[f][op], plain[f][op]), f
    assert np.all(info["path"][op] == A.PATH_OPEN)
    assert np.all(info["path"][~op] == A.PATH_GUIDED)
    lo8, hi8 = plain_bracket_after(plain["lo"][~op], plain["hi"][~op], wl.opts.a_min,
                                   wl.opts.a_max, 8)
    assert np.array_equal(res["lo"][~op], lo8) and np.array_equal(res["hi"][~op], hi8)
    assert np.array_equal(res["alim"][~op], np.sqrt(lo8 * hi8))
    half = math.exp(math.log(wl.opts.a_max / wl.opts.a_min) / 2 ** 9) - 1
    assert np.all(np.abs(res["alim"][~op] / plain["alim"][~op] - 1) <= half * (1 + 1e-9))
    assert np.all(res["trials"][~op] == 1 + 8)
    assert np.all((info["rounds"] >= 1) & (info["rounds"] <= res["trials"]))
    print(f"speculative: rounds {info['rounds'].sum()} for {res['trials'].sum()} trials")
    # all the levels: the plain solve, byte for byte
    g.levels = wl.opts.iters
    full, finfo = ctx.solve_guided(s, wl.setups, wl.modals, wl.points, wl.opts, g)
    assert full.tobytes() == plain.tobytes()
    # a levels value above iters means iters
    g.levels = 99
    again, _ = ctx.solve_guided(s, wl.setups, wl.modals, wl.points, wl.opts, g)
    assert again.tobytes() == plain.tobytes()
    # skip_top = 1: every point skips the first trial at a_max; the points that chatter
    # there keep their bracket and spend one trial and one round less, the open ones are
    # no longer reported open
    g.levels = 8
    g.skip_top = 1.0
    sk, skinfo = ctx.solve_guided(s, wl.setups, wl.modals, wl.points, wl.opts, g)
    assert np.all(sk["open"] == 0)
    for f in ("alim", "lo", "hi"):
        assert np.array_equal(sk[f][~op], res[f][~op]), f
    assert np.all(sk["trials"][~op] == res["trials"][~op] - 1)
    assert np.array_equal(skinfo["rounds"][~op], info["rounds"][~op] - 1)
    g.skip_top = 0.0
    # serial trials: one trial per round, the same results
    o = wl.opts.__class__.from_buffer_copy(wl.opts)
    o.serial_trials = 1
    g.levels = 8
    ser, sinfo = ctx.solve_guided(s, wl.setups, wl.modals, wl.points, o, g)
    assert ser.tobytes() == res.tobytes()
    assert np.array_equal(sinfo["rounds"], ser["trials"])


def test_direct_guide_reproduces_plain(ctx, trained_small):
    """With the bracket method, a tiny hw_direct sends every point to the plain bisection:
    the plain results."""
    from mcs import _abi as A
    from mcs._lib import default_guide_opts

    s, wl, plain = trained_small
    g = default_guide_opts()
    g.mode = A.GUIDE_BRACKET
    g.hw_direct = 1e-6
    res, info = ctx.solve_guided(s, wl.setups, wl.modals, wl.points, wl.opts, g)
    assert np.all(info["path"] == A.PATH_DIRECT)
    assert res.tobytes() == plain.tobytes()


def test_guided_plan_matches_guided_solve(ctx, trained_small):
    s, wl, _ = trained_small
    a, ia = ctx.solve_guided(s, wl.setups, wl.modals, wl.points, wl.opts)
    plan = ctx.plan(wl.setups, wl.modals, wl.points, wl.opts, surrogate=s)
    for _ in range(2):
        plan.execute()
        b = plan.results()
        ib = plan.guide_info()
        assert a.tobytes() == b.tobytes()
        assert ia.tobytes() == ib.tobytes()
    plan.close()


def test_params_roundtrip(ctx, trained_small):
    from mcs import Surrogate

    s, wl, _ = trained_small
    X = ctx.features(wl.setups, wl.modals, wl.points, wl.opts)
    p = s.get_params()
    t = Surrogate(ctx, 99)
    t.set_params(p)
    assert np.array_equal(s.predict(X)[0], t.predict(X)[0])
    t.close()


def test_surrogate_outlives_its_plans(ctx, trained_small):
    from mcs import MCSError, Surrogate, _abi as A

    _, wl, _ = trained_small
    t = Surrogate(ctx, 5)
    plan = ctx.plan(wl.setups, wl.modals, wl.points[:8], wl.opts, surrogate=t)
    with pytest.raises(MCSError) as e:
        t.close()
    assert e.value.status == A.MCS_ERR_STATE
    plan.execute()
    assert len(plan.results()) == 8
    plan.close()
    t.close()


def test_keep_best_and_warm_start(ctx, feats):
    from mcs import Surrogate
    from mcs._lib import default_train_opts

    _, X = feats
    Z = (X - X.mean(0)) / (X.std(0) + 1e-6)
    y = (0.5 * Z[:, 0] - 0.5 * Z[:, 11] + 0.4 * np.sin(2 * Z[:, 4])).astype(np.float32)
    s = Surrogate(ctx, 9)
    o = default_train_opts()
    o.epochs, o.batch, o.lr, o.keep_best = 12, 256, 3e-3, 1
    tl, vl = s.train(X[:1536], y[:1536], X[1536:], y[1536:], o)
    # the parameters left are those of the epoch of lowest validation loss
    loss, _ = s.grad(X[1536:], y[1536:])
    assert loss == pytest.approx(float(vl.min()), rel=1e-3, abs=1e-4)
    # a warm start continues from them instead of a fresh initialisation
    o.warm, o.epochs, o.keep_best = 1, 3, 0
    tl2, _ = s.train(X[:1536], y[:1536], None, None, o)
    assert tl2[0] < tl[0]
    s.close()


def test_ablation_trained_model_saves_rounds(ctx):
    """What the trained network gains over the method without it.  On 2048 serving
    queries the speculative guided solve with the committed model needs fewer rounds (warp
    passes over the trial loop, the point's cost in time) than the same solve steered by an
    untrained network, with the same limits: both are the plain bisection's after 8
    levels, within 1.12 % of the plain limits."""
    from mcs import Surrogate
    from mcs import surrogate as SG
    from mcs import workloads as W

    assert SG.DEFAULT_MODEL.exists(), "the trained model is part of the package"
    sv = W.serve().subset(np.arange(2048))
    plain = ctx.solve(sv.setups, sv.modals, sv.points, sv.opts)
    trained = SG.load(ctx)
    untrained = Surrogate(ctx, 1)
    rt, it = ctx.solve_guided(trained, sv.setups, sv.modals, sv.points, sv.opts)
    ru, iu = ctx.solve_guided(untrained, sv.setups, sv.modals, sv.points, sv.opts)
    assert rt.tobytes() == ru.tobytes()
    rel = np.abs(rt["alim"] / plain["alim"] - 1)
    nt, nu = int(it["rounds"].sum()), int(iu["rounds"].sum())
    print(f"rounds: trained {nt}, untrained {nu} ({nt / nu:.3f}); max |alim / plain - 1| "
          f"{rel.max():.4f}")
    assert nt < 0.95 * nu
    assert rel.max() <= 0.0113
    trained.close()
    untrained.close()


def test_ablation_trained_model_saves_trials(ctx):
    """The bracket method: on 2048 serving queries the committed model's guided solve
    needs fewer time-domain trials than the plain bisection, and than the same guided
    method with an untrained network, while its limits stay within 2 % of the plain ones
    on at least 99 % of the queries."""
    from mcs import Surrogate
    from mcs import _abi as A
    from mcs import surrogate as SG
    from mcs import workloads as W
    from mcs._lib import default_guide_opts

    assert SG.DEFAULT_MODEL.exists(), "the trained model is part of the package"
    sv = W.serve().subset(np.arange(2048))
    plain = ctx.solve(sv.setups, sv.modals, sv.points, sv.opts)
    trained = SG.load(ctx)
    untrained = Surrogate(ctx, 1)

    def within(r):
        op = (r["open"] == 1) & (plain["open"] == 1)
        return float(np.mean(op | (np.abs(r["alim"] / plain["alim"] - 1) <= 0.02)))

    g = default_guide_opts()
    g.mode = A.GUIDE_BRACKET
    rt, it = ctx.solve_guided(trained, sv.setups, sv.modals, sv.points, sv.opts, g)
    ru, iu = ctx.solve_guided(untrained, sv.setups, sv.modals, sv.points, sv.opts, g)
    tp, tt, tu = plain["trials"].sum(), rt["trials"].sum(), ru["trials"].sum()
    print(f"trials: plain {tp}, trained {tt} ({tt / tp:.3f}), untrained {tu} ({tu / tp:.3f}); "
          f"guided fraction trained {np.mean(it['path'] == 0):.3f} untrained "
          f"{np.mean(iu['path'] == 0):.3f}; within 2 %: trained {within(rt):.4f} untrained "
          f"{within(ru):.4f}")
    assert tt < tp
    assert tt < tu
    assert within(rt) >= 0.99
    trained.close()
    untrained.close()
