"""Surrogate-guided stability limits: labels from the GPU solver, training, storage.

    python -m mcs.surrogate train --out machinig-sim_b200/models/surrogate_hetero.npz

generates labels for the "train" workload (16384 seeded heterogeneous setups x 16
speeds) with the plain GPU bisection, trains the MLP on the 90 % training split (by setup
seed) with the library's BF16 training kernels and stores the parameters with the
training record.  `load()` puts stored parameters into a Surrogate; `Context.solve_guided`
and guided plans use it.
"""
from __future__ import annotations

import argparse
import json
import math
import sys
import time
from pathlib import Path

import numpy as np

from . import _abi as A
from . import workloads as W
from ._lib import Context, Surrogate, default_train_opts

PKG = Path(__file__).resolve().parent.parent
DEFAULT_MODEL = PKG / "models" / "surrogate_hetero.npz"


def labels(ctx: Context, wl: W.Workload, precision: str = "fp32", chunk: int = 65536):
    """log critical depth of every point by the plain GPU bisection (and the results)."""
    opts = A.make_opts(precision=precision)
    for f in ("a_min", "a_max", "iters", "revs", "nonlinear", "honor_runout", "steps_per_tooth",
              "slices", "chatter_idx"):
        setattr(opts, f, getattr(wl.opts, f))
    res = np.concatenate([ctx.solve(wl.setups, wl.modals, wl.points[i:i + chunk], opts)
                          for i in range(0, wl.n, chunk)])
    return np.log(res["alim"]).astype(np.float32), res


def train(ctx: Context, wl: W.Workload | None = None, seed: int = 1, epochs: int = 20,
          batch: int = 4096, keep_best: bool = False, log=print):
    """Labels + training on the seed-split of `wl` (default: the train workload).

    keep_best=False keeps the last epoch: serving queries mostly come from training setups
    at new speeds, where the longer fit predicts better than the epoch of lowest loss on
    unseen setups."""
    wl = wl if wl is not None else W.train()
    t0 = time.time()
    X = ctx.features(wl.setups, wl.modals, wl.points, wl.opts)
    y, res = labels(ctx, wl)
    t_label = time.time() - t0
    val_setup = wl.meta.get("val_setup")
    val = val_setup[wl.points["setup"]] if val_setup is not None else np.zeros(wl.n, bool)
    s = Surrogate(ctx, seed)
    o = default_train_opts()
    o.epochs, o.batch, o.seed, o.keep_best = epochs, batch, seed, int(keep_best)
    t1 = time.time()
    tl, vl = s.train(X[~val], y[~val], X[val], y[val], o)
    t_train = time.time() - t1
    mu, sg = s.predict(X[val])
    err = np.abs(mu - y[val])
    record = {
        "workload": wl.name, "points": int(wl.n), "train_points": int((~val).sum()),
        "val_points": int(val.sum()), "epochs": epochs, "batch": batch, "seed": seed,
        "keep_best": bool(keep_best),
        "label_seconds": round(t_label, 2), "train_seconds": round(t_train, 2),
        "label_points_per_s": round(wl.n / t_label, 1),
        "train_loss": [float(v) for v in tl], "val_loss": [float(v) for v in vl],
        "val_abs_log_err_median": float(np.median(err)),
        "val_within_15pct": float(np.mean(err < math.log(1.15))),
        "val_open_fraction": float(np.mean(res["open"][val])),
        "val_sigma_median": float(np.median(sg)),
    }
    log(json.dumps(record))
    return s, record


def save(s: Surrogate, path: Path, record: dict | None = None) -> None:
    path = Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    np.savez_compressed(path, params=s.get_params(),
                        record=np.array(json.dumps(record or {})))


def load(ctx: Context, path: Path | str = DEFAULT_MODEL) -> Surrogate:
    with np.load(path, allow_pickle=False) as z:
        p = z["params"]
    s = Surrogate(ctx)
    s.set_params(p)
    return s


def record_of(path: Path | str = DEFAULT_MODEL) -> dict:
    with np.load(path, allow_pickle=False) as z:
        return json.loads(str(z["record"]))


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train")
    t.add_argument("--out", default=str(DEFAULT_MODEL))
    t.add_argument("--setups", type=int, default=16384)
    t.add_argument("--speeds", type=int, default=16)
    t.add_argument("--epochs", type=int, default=20)
    t.add_argument("--batch", type=int, default=4096)
    t.add_argument("--seed", type=int, default=1)
    t.add_argument("--device", type=int, default=0)
    t.add_argument("--keep-best", action="store_true")
    a = ap.parse_args(argv)
    ctx = Context(a.device)
    wl = W.train(n_setups=a.setups, speeds_per_setup=a.speeds)
    s, rec = train(ctx, wl, seed=a.seed, epochs=a.epochs, batch=a.batch,
                   keep_best=a.keep_best)
    save(s, Path(a.out), rec)
    return 0


if __name__ == "__main__":
    sys.exit(main())
