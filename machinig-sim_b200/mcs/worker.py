"""StabWorker: the message protocol of the reference's stability Web Worker
(src/stabworker.js:1-15) over an asynchronous GPU job.

    w = StabWorker(onmessage)
    w.postMessage({"key": k, "points": [{"S": s, "modal": m}, ...], "tool": {...},
                   "mat": {...}, "arc": [a, b], "fz": fz, "nonlinear": True})

onmessage receives {key, S, alim, open} for every point, in point order, then
{key, done: True}.  A newer message replaces an older one: the older job is cancelled at
its next trial boundary on the device and posts nothing more (stabworker.js:7-9).
Replies are posted when the batch completes rather than point by point; the whole sweep
is one persistent launch.
"""
from __future__ import annotations

import threading
import time
from typing import Any, Callable, Mapping

import numpy as np

from . import _abi as A
from ._lib import Context, Job, default_context


class StabWorker:
    def __init__(self, onmessage: Callable[[dict], None], ctx: Context | None = None,
                 poll_interval: float = 0.002):
        self.onmessage = onmessage
        self.ctx = ctx if ctx is not None else default_context()
        self.poll_interval = poll_interval
        self._lock = threading.Lock()
        self._job_id = 0
        self._current: Job | None = None
        self._threads: list[threading.Thread] = []
        self.errors: list[BaseException] = []

    def postMessage(self, m: Mapping[str, Any]) -> None:
        pts = list(m["points"])
        setups = [A.make_setup(m["tool"], m["mat"], m["arc"], m["fz"])]
        modals = [A.make_modal(p["modal"]) for p in pts]
        points = A.points_array(np.zeros(len(pts)), np.arange(len(pts)),
                                [float(p["S"]) for p in pts])
        opts = A.make_opts({"nonlinear": m.get("nonlinear", True)})
        with self._lock:
            self._job_id += 1
            jid = self._job_id
            if self._current is not None:
                self._current.cancel()
            job = self.ctx.solve_async(setups, modals, points, opts)
            self._current = job
        t = threading.Thread(target=self._run, args=(jid, job, m.get("key"), pts), daemon=True)
        self._threads.append(t)
        t.start()

    def _run(self, jid: int, job: Job, key, pts) -> None:
        try:
            while True:
                _, finished = job.poll()
                if finished:
                    break
                time.sleep(self.poll_interval)
            res = job.wait()
            for p, r in zip(pts, res):
                if jid != self._job_id:  # a newer request replaced this one
                    return
                self.onmessage({"key": key, "S": p["S"], "alim": float(r["alim"]),
                                "open": bool(r["open"])})
            if jid == self._job_id:
                self.onmessage({"key": key, "done": True})
        except BaseException as e:  # surfaced to the owner, like a Worker's onerror
            self.errors.append(e)
        finally:
            job.close()

    def join(self, timeout: float | None = None) -> None:
        for t in list(self._threads):
            t.join(timeout)
