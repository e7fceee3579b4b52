"""Surrogate pieces that need no GPU: the FP64 reference MLP (the checker of the BF16
kernels) against finite differences, and the library's feature map against an
independent numpy restatement."""
from __future__ import annotations

import math

import numpy as np
import pytest


def random_params(rng, scale=0.3):
    import mlp_ref as R

    W_, b_, total = R.layout()
    p = np.zeros(total)
    p[:R.N_IN] = rng.normal(size=R.N_IN)
    p[R.N_IN:2 * R.N_IN] = rng.uniform(0.5, 2.0, R.N_IN)
    for l, (o, k, n) in enumerate(W_):
        w = rng.normal(scale=scale / math.sqrt(k), size=(k, n))
        if l == 0:
            w[R.N_IN:, :] = 0
        if l == 3:
            w[:, 2:] = 0
        p[o:o + k * n] = w.ravel()
    for l, (o, n) in enumerate(b_):
        b = rng.normal(scale=0.1, size=n)
        if l == 3:
            b[2:] = 0
        p[o:o + n] = b
    return p


def test_reference_gradient_matches_finite_differences():
    import mlp_ref as R

    rng = np.random.default_rng(3)
    p = random_params(rng)
    X = rng.normal(size=(16, R.N_IN))
    y = rng.normal(size=16)
    loss, g = R.loss_and_grad(p, X, y)
    W_, b_, _ = R.layout()
    idx = []
    for (o, k, n), (ob, nb) in zip(W_, b_):
        idx += list(rng.integers(o, o + min(k, 20) * n, 6)) + list(rng.integers(ob, ob + 2, 2))
    for i in idx:
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (R.loss_and_grad(pp, X, y)[0] - R.loss_and_grad(pm, X, y)[0]) / (2 * h)
        assert fd == pytest.approx(g[i], rel=1e-5, abs=1e-9), i


def numpy_features(wl):
    """The feature map of include/mcs.h restated: dominant modes by min k*zeta."""
    st = wl.setups[wl.points["setup"]]
    md = wl.modals[wl.points["modal"]]
    o = wl.opts
    out = np.zeros((wl.n, 20))
    for r in range(wl.n):
        s, m, S = st[r], md[r], max(100.0, wl.points["S"][r])
        t = s["tool"]
        nx = m["nx"]
        ny = m["ny"] if m["ny"] > 0 else m["nx"]
        xs = m["x"][:nx]
        ys = (m["y"] if m["ny"] > 0 else m["x"])[:ny]

        def dom(ms):
            kz = ms["k"] * ms["zeta"]
            return ms[int(np.argmin(kz))]

        dx, dy = dom(xs), dom(ys)
        ft = S * t["N"] / 60
        out[r] = [math.log(t["R"]), t["N"], math.tan(math.radians(t["helix_deg"])),
                  t["runout"] if o.honor_runout else 0.0, math.log(s["mat"]["Ktc"]),
                  s["mat"]["Krc"] / s["mat"]["Ktc"], s["mat"]["mc"] if o.nonlinear else 0.0,
                  math.log1p(s["mat"]["Ci"] if o.nonlinear else 0.0), s["arc_st"], s["arc_ex"],
                  math.log(s["fz"]), math.log(S), math.log(dx["k"] * max(dx["zeta"], 1e-6)),
                  math.log(dx["fn"]), math.log(dy["k"] * max(dy["zeta"], 1e-6)),
                  math.log(dy["fn"]), math.sin(2 * math.pi * dx["fn"] / ft),
                  math.cos(2 * math.pi * dx["fn"] / ft), math.sin(2 * math.pi * dy["fn"] / ft),
                  math.cos(2 * math.pi * dy["fn"] / ft)]
    return out


def test_feature_map_matches_restatement(mcs_lib):
    import ctypes as C

    from mcs import _abi as A
    from mcs import _lib
    from mcs import workloads as W

    for wl in (W.hetero(n=64), W.sweep(n_speeds=32), W.small()):
        out = np.zeros((wl.n, 20), dtype=np.float32)
        st = mcs_lib.mcs_features(C.c_void_p(wl.setups.ctypes.data), len(wl.setups),
                                  C.c_void_p(wl.modals.ctypes.data), len(wl.modals),
                                  C.c_void_p(wl.points.ctypes.data), wl.n, C.byref(wl.opts),
                                  C.c_void_p(out.ctypes.data))
        assert st == 0, _lib.last_error()
        ref = numpy_features(wl)
        assert np.allclose(out, ref, rtol=2e-6, atol=2e-6)
