"""Cutting coefficients from cutting tests, and validation against a measured force record,
on batched GPU cutting engines: the reference's identify.js and validate.js.

The reference runs every simulation it needs one after the other: six unit-force runs per
test (identify.js:26-40), one revolution per runout candidate (validate.js:137-150, 289 of
them), six unit waveforms per coefficient fit (:119-122).  Here each such set is one batch
of rigid-tool engines in one launch (mcs.engine); the least squares, the synchronous
averaging, the alignment and the comparisons are host arithmetic as in the reference.

    U = unit_forces(ctx, tool, tests)                    # [tests, 6, 3] N per coefficient
    r = identify(ctx, tool, tests, current)              # {coefs, rows, r2, rms, edgeFixed}
    rec = parse_record(csv); sa = sync_average(rec["t"], rec["F"], S)
    f = fit_record(ctx, tool, mat, test, sa["avg"])      # coefficients and runout

Frames and units as the reference: feed along +X, Y 90 degrees to its left, Z up, forces
on the workpiece; tool {D, N, helixDeg, type, fluteLen, runout [um], runoutPhase}.
"""
from __future__ import annotations

import math
import re
from typing import Any, Mapping, Sequence

import numpy as np

from . import engine as E

COEF_KEYS = ("Ktc", "Krc", "Kac", "Kte", "Kre", "Kae")  # identify.js:13
NB = 360                                                 # validate.js:13
COMP = ("Fx", "Fy", "Fz")


def immersion(mode: str, ae: float, D: float) -> tuple[float, float]:
    """Engagement arc of a test (identify.js:18-22)."""
    if mode == "slot" or not (ae < D):
        return 0.0, math.pi
    pe = math.acos(1 - 2 * ae / D)
    return (math.pi - pe, math.pi) if mode == "down" else (0.0, pe)


def _engine_tool(tool: Mapping[str, Any], ap: float, runout=None, phase=None) -> dict:
    return {"N": tool["N"], "R": tool["D"] / 2, "helixDeg": tool.get("helixDeg", 30),
            "type": tool.get("type") or "flat",
            "fluteLen": max(tool.get("fluteLen") or 0, ap + 1),
            "runout": tool.get("runout", 0) if runout is None else runout,
            "runoutPhase": tool.get("runoutPhase", 0) if phase is None else phase}


def _steps_per_rev(cfg) -> int:
    """stepsPerRev of configure() for a rigid-tool config (cutting.js:50, 67)."""
    N = cfg.tool.N
    S = max(100.0, cfg.S)
    Ttooth = 60 / (S * N)
    fTop = max(cfg.modal.x[j].fn for j in range(cfg.modal.nx))
    return N * int(max(48.0, math.ceil(Ttooth * max(fTop, cfg.fn_max) * 24)))


def unit_forces(ctx, tool: Mapping[str, Any], tests: Sequence[Mapping[str, Any]],
                mc: float = 0.0) -> np.ndarray:
    """Mean force on the workpiece [N] of each test with one coefficient at 1 and the
    others 0 (identify.js:26-40): out[test, coefficient, component].  A rigid tool at
    6000 rpm runs two revolutions, its statistics are taken and dropped, and one more
    revolution is averaged; all 6 x len(tests) engines run in one launch."""
    cfgs, gs = [], []
    for t in tests:
        st, ex = immersion(t["mode"], t["ae"], tool["D"])
        # the test's six engines share one engagement (the record is copied per engine)
        g = E.engagement(E.arc_map(st, ex), (1, 0), t["fz"], -t["ap"], t["ap"])
        for key in COEF_KEYS:
            mat = dict.fromkeys(COEF_KEYS, 0.0)
            mat.update({key: 1.0, "mc": mc, "Ci": 0.0})
            tl = _engine_tool(tool, t["ap"], phase=0.0)  # unitForces passes no phase
            tl["nonlinear"] = mc > 0
            cfgs.append(E.config(tl, E.RIGID, mat, 6000))
            gs.append(g)
    if not cfgs:
        return np.zeros((0, 6, 3))
    eng = E.Engines(ctx, len(cfgs))
    try:
        eng.configure(cfgs)
        eng.set_engagement(gs)
        spr = np.array([_steps_per_rev(c) for c in cfgs], dtype=np.int64)
        eng.run(2 * spr)
        eng.take_stats()
        eng.run(spr)
        s = eng.take_stats()
    finally:
        eng.close()
    out = np.stack([-s["sumFx"] / s["n"], -s["sumFy"] / s["n"], -s["sumFz"] / s["n"]], axis=1)
    return out.reshape(len(tests), 6, 3)


def _gauss_jordan(A: np.ndarray, b: np.ndarray, tiny: float = 1e-300, floor: bool = False):
    """solve() of identify.js:43-52: Gauss-Jordan with partial pivoting (None when singular;
    floor=True raises tiny pivots to 1e-12 as fitCoefs does, validate.js:130)."""
    n = len(b)
    M = np.concatenate([np.array(A, dtype=np.float64), np.array(b, dtype=np.float64)[:, None]],
                       axis=1)
    for c in range(n):
        p = c
        for r in range(c + 1, n):
            if abs(M[r][c]) > abs(M[p][c]):
                p = r
        M[[c, p]] = M[[p, c]]
        if abs(M[c][c]) < tiny:
            if not floor:
                return None
            M[c][c] = 1e-12
        for r in range(n):
            if r != c:
                f = M[r][c] / M[c][c]
                M[r, c:] -= f * M[c, c:]
    return M[:, n] / np.diag(M)


def identify_from_units(U: np.ndarray, tests: Sequence[Mapping[str, Any]],
                        current: Mapping[str, float]) -> dict | None:
    """The least squares of identify.js:56-90 on given unit forces U[test, 6, 3]."""
    if not len(tests):
        return None
    feeds = {f"{t['fz']:.4f}" for t in tests}
    edge_fixed = len(feeds) < 2
    free = [0, 1, 2] if edge_fixed else [0, 1, 2, 3, 4, 5]
    A, y = [], []
    for i, t in enumerate(tests):
        for k, c in enumerate(COMP):
            rhs = t[c]
            if edge_fixed:
                for j in (3, 4, 5):
                    rhs -= current[COEF_KEYS[j]] * U[i][j][k]
            A.append([U[i][j][k] for j in free])
            y.append(rhs)
    A, y = np.array(A), np.array(y)
    # each column scaled to unit norm first: shearing and edge columns differ by ~1/fz
    nrm = np.array([math.hypot(*A[:, c]) or 1.0 for c in range(len(free))])
    As = A / nrm
    AtA = As.T @ As
    Aty = As.T @ y
    xs = _gauss_jordan(AtA, Aty)
    if xs is None:
        return None
    coefs = {k: current[k] for k in COEF_KEYS}
    for c, j in enumerate(free):
        coefs[COEF_KEYS[j]] = xs[c] / nrm[c]
    rows = [{"test": t, "pred": [sum(coefs[key] * U[i][j][k] for j, key in enumerate(COEF_KEYS))
                                 for k in range(3)]} for i, t in enumerate(tests)]
    res = [r["test"][c] - r["pred"][k] for r in rows for k, c in enumerate(COMP)]
    allv = [r["test"][c] for r in rows for c in COMP]
    mean = sum(allv) / len(allv)
    ssr = sum(v * v for v in res)
    sst = sum((v - mean) ** 2 for v in allv)
    return {"coefs": coefs, "rows": rows, "r2": 1 - ssr / sst if sst > 0 else 1.0,
            "rms": math.sqrt(ssr / len(res)), "edgeFixed": edge_fixed}


def identify(ctx, tool, tests, current, mc: float = 0.0) -> dict | None:
    """identify(tool, tests, current, mc) of identify.js:56-90 with the unit forces of
    unit_forces: tests [{fz, ap, ae, mode, Fx, Fy, Fz}]; with a single feed the edge terms
    are held at the current values."""
    if not len(tests):
        return None
    return identify_from_units(unit_forces(ctx, tool, tests, mc), tests, current)


def parse_tests(text: str, mode: str = "slot") -> dict:
    """parseTests (identify.js:93-103): "fz ap ae Fx Fy Fz" per line; # comments."""
    tests, bad = [], []
    for i, line in enumerate(text.split("\n")):
        s = re.sub(r"#.*", "", line.rstrip("\r")).strip()
        if not s:
            continue
        v = [_num(x) for x in re.split(r"[\s,;]+", s)]
        if len(v) < 6 or not all(math.isfinite(x) for x in v[:6]) or not (v[0] > 0) or \
                not (v[1] > 0) or not (v[2] > 0):
            if not re.match(r"^[a-zA-Zぁ-んァ-ヶ一-龠]", s):
                bad.append(i + 1)
            continue
        tests.append({"fz": v[0], "ap": v[1], "ae": v[2], "Fx": v[3], "Fy": v[4], "Fz": v[5],
                      "mode": mode})
    return {"tests": tests, "bad": bad}


def _num(x: str) -> float:
    """JS Number(x) for the tokens of a table row: NaN where it is not a number."""
    try:
        return float(x) if x.strip() else 0.0
    except ValueError:
        return math.nan


# ---------------------------------------------------------------- validate.js
def parse_record(text: str) -> dict:
    """parseRecord (validate.js:20-43): "t,Fx,Fy[,Fz]" rows with the test on # key=value."""
    test: dict[str, Any] = {}
    t, F, bad = [], [[], [], []], []
    has_z = False
    for i, line in enumerate(text.split("\n")):
        line = line.rstrip("\r")
        c = re.match(r"^\s*#(.*)$", line)
        if c:
            for m in re.finditer(r"([A-Za-z]+)\s*=\s*([^\s,;]+)", c.group(1)):
                k, v = m.group(1).lower(), m.group(2)
                if k == "mode":
                    test["mode"] = v.lower()
                elif math.isfinite(_num(v)):
                    test[{"s": "S", "d": "D", "n": "N"}.get(k, k)] = _num(v)
            continue
        s = line.strip()
        if not s:
            continue
        v = [_num(x) for x in re.split(r"[\s,;]+", s)]
        if len(v) < 3 or not all(math.isfinite(x) for x in v[:3]):
            if not re.match(r'^[A-Za-z"]', s):
                bad.append(i + 1)
            continue
        t.append(v[0])
        F[0].append(v[1])
        F[1].append(v[2])
        if len(v) > 3 and math.isfinite(v[3]):
            F[2].append(v[3])
            has_z = True
        else:
            F[2].append(0.0)
    test["mode"] = test.get("mode") if test.get("mode") in ("slot", "down", "up") else "slot"
    return {"test": test, "t": t, "F": F, "hasZ": has_z, "bad": bad}


def _bins(t: np.ndarray, S: float) -> np.ndarray:
    a = (t - t[0]) * (S / 60)
    return np.minimum(NB - 1, np.floor((a - np.floor(a)) * NB)).astype(np.int64)


def sync_average(t, F, S: float) -> dict:
    """syncAverage (validate.js:47-71): the record folded onto the spindle angle and
    averaged per bin; empty bins take their neighbours' mean; the asynchronous RMS."""
    t = np.asarray(t, dtype=np.float64)
    F = np.asarray(F, dtype=np.float64)
    b = _bins(t, S)
    cnt = np.bincount(b, minlength=NB).astype(np.float64)
    avg = np.array([np.bincount(b, weights=F[c], minlength=NB) for c in range(3)])
    with np.errstate(invalid="ignore", divide="ignore"):
        avg = np.where(cnt > 0, avg / cnt, np.nan)
    for a in avg:
        for k in range(NB):
            if math.isnan(a[k]):
                lo, hi = k, k
                while math.isnan(a[lo % NB]) and lo > k - NB:
                    lo -= 1
                while math.isnan(a[hi % NB]) and hi < k + NB:
                    hi += 1
                a[k] = (a[lo % NB] + a[hi % NB]) / 2
    async_rms = [float(np.sqrt(np.sum((F[c] - avg[c][b]) ** 2) / max(1, len(t))))
                 for c in range(3)]
    revs = (t[-1] - t[0]) * S / 60 if len(t) > 1 else 0.0
    return {"avg": avg, "revs": revs, "asyncRms": async_rms, "cnt": cnt}


def sim_revolutions(ctx, cases: Sequence[tuple]) -> np.ndarray:
    """simRevolution (validate.js:76-100) of every (tool, mat, test) at once: one
    revolution of the rigid tool's force on the workpiece in NB angle bins, out[case, 3,
    NB].  Two revolutions settle, then the history (sampled every step) holds the third."""
    cfgs, gs = [], []
    for tool, mat, test in cases:
        st, ex = immersion(test["mode"], test["ae"], tool["D"])
        tl = _engine_tool(tool, test["ap"])
        tl["nonlinear"] = (mat.get("mc") or 0) > 0
        m = {"Ci": 0.0, **mat}
        cfgs.append(E.config(tl, E.RIGID, m, test.get("S") or 6000, decim=1))
        gs.append(E.engagement(E.arc_map(st, ex), (1, 0), test["fz"], -test["ap"], test["ap"]))
    eng = E.Engines(ctx, len(cfgs))
    try:
        eng.configure(cfgs)
        eng.set_engagement(gs)
        spr = np.array([_steps_per_rev(c) for c in cfgs], dtype=np.int64)
        if np.any(spr > 4096):
            raise ValueError("one revolution has more steps than the history holds")
        eng.run(2 * spr)
        eng.reset_history()
        eng.run(spr)
        hist, _, _ = eng.history()
    finally:
        eng.close()
    out = np.zeros((len(cases), 3, NB))
    b = np.arange(NB)
    for i, n in enumerate(spr):
        x = (b + 0.5) / NB * n - 0.5
        i0 = np.floor(x).astype(np.int64)
        f = x - i0
        for c in range(3):
            h = hist[i, c].astype(np.float64)
            a, cc = h[(i0 + n) % n], h[(i0 + 1) % n]
            out[i, c] = -(a + (cc - a) * f)
    return out


def sim_revolution(ctx, tool, mat, test) -> np.ndarray:
    return sim_revolutions(ctx, [(tool, mat, test)])[0]


def align(meas, sim) -> int:
    """The circular shift (bins) of sim that best matches meas on Fx and Fy (:103-111)."""
    best, best_v = 0, -math.inf
    m = np.asarray(meas)[:2]
    p = np.asarray(sim)[:2]
    for s in range(NB):
        v = float(np.sum(m * np.roll(p, s, axis=1)))
        if v > best_v:
            best_v, best = v, s
    return best


def shifted(sim, s: int) -> np.ndarray:
    return np.roll(np.asarray(sim), s, axis=1)


def compare(meas, sim, comps=(0, 1, 2)) -> list[dict]:
    """Per component: means, peak-to-peak, RMS error in % of the measured peak-to-peak and
    the correlation (validate.js:115-126)."""
    out = []
    for c in comps:
        m, p = np.asarray(meas[c]), np.asarray(sim[c])
        mm, pm = float(np.mean(m)), float(np.mean(p))
        dm, dp = m - mm, p - pm
        se = float(np.sum((m - p) ** 2))
        sxy, sxx, syy = float(np.sum(dm * dp)), float(np.sum(dm * dm)), float(np.sum(dp * dp))
        ppm = float(m.max() - m.min())
        out.append({"comp": COMP[c], "meanM": mm, "meanS": pm, "ppM": ppm,
                    "ppS": float(p.max() - p.min()),
                    "rmsPct": math.sqrt(se / NB) / max(1e-9, ppm) * 100,
                    "r": sxy / math.sqrt(sxx * syy) if sxx > 0 and syy > 0 else 0.0})
    return out


def _unit_waveforms(ctx, tools, test, mc, Ci) -> np.ndarray:
    """The six unit waveforms (one coefficient at 1) of each tool: out[tool, 6, 3, NB]."""
    cases = []
    for tool in tools:
        for key in COEF_KEYS:
            mat = dict.fromkeys(COEF_KEYS, 0.0)
            mat.update({key: 1.0, "mc": mc, "Ci": Ci})
            cases.append((tool, mat, test))
    return sim_revolutions(ctx, cases).reshape(len(tools), 6, 3, NB)


def _fit_coefs(U: np.ndarray, meas, comps) -> dict:
    """fitCoefs (validate.js:119-146) on given unit waveforms U[6, 3, NB]: least squares of
    the six coefficients at every fourth shift, then around the best."""
    meas = np.asarray(meas)
    y = np.concatenate([meas[c] for c in comps])

    def fit(s):
        rows = np.concatenate([np.roll(U[:, c, :], s, axis=1).T for c in comps])
        nrm = np.array([math.hypot(*rows[:, j]) or 1.0 for j in range(6)])
        A = (rows / nrm).T @ (rows / nrm)
        v = (rows / nrm).T @ y
        x = _gauss_jordan(A, v, tiny=1e-12, floor=True) / nrm
        e = float(np.sum((y - rows @ x) ** 2))
        return x, e

    best = None
    for s in range(0, NB, 4):
        x, e = fit(s)
        if best is None or e < best["e"]:
            best = {"s": s, "x": x, "e": e}
    s0 = best["s"]
    for s in range(s0 - 3, s0 + 4):
        x, e = fit((s + NB) % NB)
        if e < best["e"]:
            best = {"s": (s + NB) % NB, "x": x, "e": e}
    return {"coefs": dict(zip(COEF_KEYS, (float(v) for v in best["x"]))), "shift": best["s"],
            "sse": best["e"]}


def fit_record(ctx, tool, mat, test, meas, comps=(0, 1, 2), runout_max: float = 30) -> dict:
    """fitRecord (validate.js:148-196): the runout by a grid over size and direction (all
    candidate revolutions in one launch), the coefficients by least squares on the unit
    waveforms at the best three, then a pattern search on size and direction with the
    full fit; returns {coefs, runout, runoutPhase, shift, sim, cmp}."""
    mc = mat.get("mc") or 0.0
    Ci = mat.get("Ci") or 0.0
    meas = np.asarray(meas)
    phases = [i / 24 * 2 * math.pi for i in range(24)]
    sizes = [e for e in (0, 1, 2, 3, 4, 6, 8, 10, 13, 16, 20, 25, 30) if e <= runout_max]
    grid = [(e, g) for e in sizes for g in (phases if e else [0.0])]
    sims = sim_revolutions(ctx, [({**tool, "runout": e, "runoutPhase": g}, mat, test)
                                 for e, g in grid])
    cand = []
    for (e, g), sim in zip(grid, sims):
        s = align(meas, sim)
        p = np.roll(sim, s, axis=1)
        num = sum(float(np.sum(meas[c] * p[c])) for c in comps)
        den = sum(float(np.sum(p[c] * p[c])) for c in comps)
        k = num / den if den > 0 else 1.0
        err = sum(float(np.sum((meas[c] - k * p[c]) ** 2)) for c in comps)
        cand.append({"e": e, "g": g, "err": err})
    cand.sort(key=lambda c: c["err"])  # stable, as Array.prototype.sort
    top = cand[:3]
    U = _unit_waveforms(ctx, [{**tool, "runout": c["e"], "runoutPhase": c["g"]} for c in top],
                        test, mc, Ci)
    best = None
    for c, u in zip(top, U):
        f = _fit_coefs(u, meas, comps)
        if best is None or f["sse"] < best["sse"]:
            best = {**f, "runout": c["e"], "runoutPhase": c["g"]}

    def eval_many(points):
        us = _unit_waveforms(ctx, [{**tool, "runout": e, "runoutPhase": g} for e, g in points],
                             test, mc, Ci)
        return [{**_fit_coefs(u, meas, comps), "runout": e, "runoutPhase": g}
                for (e, g), u in zip(points, us)]

    de, dg = 1.0, 7.5 * math.pi / 180
    for _ in range(4):
        moved = True
        while moved:
            moved = False
            steps = [(de, 0.0), (-de, 0.0), (0.0, dg), (0.0, -dg)]
            # the four neighbours of the current best in one batch; after a move the rest
            # are taken around the new best, as the reference's loop takes them
            i = 0
            while i < len(steps):
                pts, idx = [], []
                for j in range(i, len(steps)):
                    a, c = steps[j]
                    e, g = best["runout"] + a, best["runoutPhase"] + c
                    if e < 0 or e > runout_max or (best["runout"] == 0 and c):
                        continue
                    pts.append((e, g))
                    idx.append(j)
                if not pts:
                    break
                fs = eval_many(pts)
                nxt = len(steps)
                for j, f in zip(idx, fs):
                    if f["sse"] < best["sse"] * (1 - 1e-6):
                        best = f
                        moved = True
                        nxt = j + 1
                        break
                i = nxt
        de /= 2
        dg /= 2
    best["runout"] = math.floor(best["runout"] * 10 + 0.5) / 10
    best["runoutPhase"] = ((best["runoutPhase"] % (2 * math.pi)) + 2 * math.pi) % (2 * math.pi)
    coefs = {**mat, **best["coefs"]}
    sim = shifted(sim_revolution(ctx, {**tool, "runout": best["runout"],
                                       "runoutPhase": best["runoutPhase"]}, coefs, test),
                  best["shift"])
    return {"coefs": best["coefs"], "runout": best["runout"], "runoutPhase": best["runoutPhase"],
            "shift": best["shift"], "sim": sim, "cmp": compare(meas, sim, comps)}


def synthetic_record(ctx, tool, mat, test, fs: float = 20000, revs: int = 20,
                     noise: float = 0.03, ring: float = 0.0, ringHz: float = 2317,
                     seed: int = 1) -> str:
    """syntheticRecord (validate.js:200-218): the simulated revolution sampled at fs with
    white noise and an optional asynchronous ringing, as CSV text."""
    sim = sim_revolution(ctx, tool, mat, test)
    pp = float(sim[0].max() - sim[0].min())
    s = seed

    def rnd():
        nonlocal s
        s = (s * 16807) % 2147483647
        return s / 2147483647

    def gauss():
        return math.sqrt(-2 * math.log(rnd() + 1e-12)) * math.cos(2 * math.pi * rnd())

    T = revs * 60 / test["S"]
    n = int(math.floor(T * fs))
    start = rnd()
    lines = ["# synthetic record (made by the simulator; not a measurement)",
             f"# S={test['S']} fz={test['fz']} ap={test['ap']} ae={test['ae']} "
             f"mode={test['mode']} D={tool['D']} N={tool['N']} helix={tool.get('helixDeg', 30)}",
             "t,Fx,Fy,Fz"]
    for i in range(n):
        t = i / fs
        a = (t * test["S"] / 60 + start) % 1
        x = a * NB - 0.5
        b0 = math.floor(x)
        f = x - b0

        def at(c):
            return sim[c][(b0 + NB) % NB] * (1 - f) + sim[c][(b0 + 1) % NB] * f

        r = ring * pp * math.sin(2 * math.pi * ringHz * t)
        vals = [at(c) + noise * pp * gauss() + (r if c < 2 else 0) for c in range(3)]
        lines.append(",".join([f"{t:.6f}"] + [f"{v:.2f}" for v in vals]))
    return "\n".join(lines)


def async_peak(t, F, S: float, N: int, avg, comps=(0, 1)) -> dict | None:
    """asyncPeak (validate.js:224-257): the largest spectral peak of the part of the record
    that does not repeat every revolution, away from the tooth-passing harmonics."""
    t = np.asarray(t, dtype=np.float64)
    n0 = len(t)
    if n0 < 64:
        return None
    fs = (n0 - 1) / (t[n0 - 1] - t[0])
    n = 1
    while n * 2 <= n0:
        n *= 2
    b = _bins(t[:n], S) if n else None
    P = np.zeros(n // 2)
    win = 0.5 - 0.5 * np.cos(2 * math.pi * np.arange(n) / (n - 1))
    for c in comps:
        x = (np.asarray(F[c][:n], dtype=np.float64) - np.asarray(avg[c])[b]) * win
        X = np.fft.fft(x)
        P[1:] += (X.real ** 2 + X.imag ** 2)[1: n // 2]
    df = fs / n
    ftp = S / 60 * N
    best, tot = -1, 0.0
    for k in range(1, n // 2):
        tot += P[k]
        f = k * df
        h = f / ftp
        rh = math.floor(h + 0.5)  # Math.round
        if abs(h - rh) * ftp < 2 * df and rh > 0:
            continue
        if f < 5 * df:
            continue
        if best < 0 or P[k] > P[best]:
            best = k
    if best < 0 or not (tot > 0):
        return None
    pk = P[best - 1] + P[best] + (P[best + 1] if best + 1 < n // 2 else 0.0)
    return {"f": best * df, "amp": math.sqrt(pk / 1.5 / len(comps)) * 4 / n, "share": pk / tot,
            "fs": fs}
