"""The seeded synthetic workloads: determinism, per-seed reproducibility, value ranges of
the five benchmark configurations."""
from __future__ import annotations

import math

import numpy as np


def test_small_is_the_documented_case():
    from mcs import workloads as W

    w = W.small()
    assert w.n == 64 and len(w.setups) == 1
    s = w.setups[0]
    assert s["tool"]["N"] == 4 and s["tool"]["R"] == 5 and s["tool"]["helix_deg"] == 30
    assert (s["mat"]["Ktc"], s["mat"]["Krc"], s["mat"]["Kte"], s["mat"]["Kre"]) == (700, 210, 20, 30)
    assert s["arc_st"] == math.pi / 2 and s["arc_ex"] == math.pi and s["fz"] == 0.05
    assert w.modals[0]["nx"] == 1 and tuple(w.modals[0]["x"][0]) == (1e4, 1000.0, 0.02)
    assert np.allclose(w.points["S"], np.linspace(5000, 20000, 64))
    o = w.opts
    assert (o.a_min, o.a_max, o.iters, o.revs, o.steps_per_tooth, o.slices) == (0.1, 10, 10, 60, 200, 40)


def test_sweep_ranges_and_determinism():
    from mcs import workloads as W

    a, b = W.sweep(), W.sweep()
    assert a.n == 4096
    assert a.setups.tobytes() == b.setups.tobytes() and a.modals.tobytes() == b.modals.tobytes()
    m = a.modals[0]
    assert (m["nx"], m["ny"]) == (3, 3)
    for ax in ("x", "y"):
        assert np.all((m[ax]["fn"][:3] >= 600) & (m[ax]["fn"][:3] <= 3000))
        assert np.all((m[ax]["k"][:3] >= 5e3) & (m[ax]["k"][:3] <= 5e4))
        assert np.all((m[ax]["zeta"][:3] >= 0.01) & (m[ax]["zeta"][:3] <= 0.05))
    assert a.setups[0]["tool"]["runout"] == 0.010
    assert a.points["S"].min() == 3000 and a.points["S"].max() == 30000
    assert len(a.meta["fp64_subset"]) == 256 and len(set(a.meta["fp64_subset"])) == 256
    assert W.sweep(seed=2).modals.tobytes() != a.modals.tobytes()


def test_hetero_ranges_and_per_seed_reproducibility():
    from mcs import workloads as W

    w = W.hetero()
    assert w.n == 16384
    st, md = w.setups, w.modals
    t = st["tool"]
    assert np.all((2 * t["R"] >= 3) & (2 * t["R"] <= 20))
    assert set(np.unique(t["N"])) == {2, 3, 4, 5, 6}
    assert np.all((t["helix_deg"] >= 0) & (t["helix_deg"] <= 45))
    assert np.all((t["runout"] >= 0) & (t["runout"] <= 0.020))
    ratio = st["mat"]["Krc"] / st["mat"]["Ktc"]
    assert np.all((ratio >= 0.2) & (ratio <= 0.5))
    assert np.all((st["mat"]["mc"] >= 0.2) & (st["mat"]["mc"] <= 0.3))
    assert np.all((md["nx"] >= 1) & (md["nx"] <= 3) & (md["ny"] >= 1) & (md["ny"] <= 3))
    assert np.all((st["fz"] >= 0.02) & (st["fz"] <= 0.15))
    assert np.all((w.points["S"] >= 3000) & (w.points["S"] <= 30000))
    # immersion arcs lie in [0, pi]; up milling starts at 0, down milling ends at pi
    assert np.all((st["arc_st"] >= 0) & (st["arc_ex"] <= math.pi + 1e-12))
    assert np.all((st["arc_st"] == 0) | (st["arc_ex"] == math.pi))
    # a setup is a pure function of its seed: regenerate a slice on its own
    part = W.hetero(n=16, first_seed=1000)
    assert part.setups.tobytes() == st[1000:1016].tobytes()
    assert part.modals.tobytes() == md[1000:1016].tobytes()


def test_train_and_serve_split():
    from mcs import workloads as W

    tr = W.train(n_setups=512, speeds_per_setup=4)
    assert tr.n == 2048
    val = tr.meta["val_setup"]
    assert 0.05 < val.mean() < 0.15
    sv = W.serve(n=4096, train_setups=512)
    assert 0.25 < sv.meta["outside"].mean() < 0.35
    assert len(sv.meta["fp64_subset"]) == 512


def test_uniform_is_a_pure_hash():
    from mcs import workloads as W

    u = W.uniform(np.arange(100000), 3, 7)
    assert np.all((u >= 0) & (u < 1))
    assert abs(u.mean() - 0.5) < 0.01
    assert np.array_equal(W.uniform(np.arange(10), 3, 7), u[:10])
