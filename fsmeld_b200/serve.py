"""A serving loop: resident target series on one GPU, requests admitted by
HBM footprint and batched continuously.

Requests (`search`, `cutoff`, `exact` of one query against one named target)
arrive from any thread through `Server.submit`, which returns a future.  One
worker thread drains the queue continuously: every pass takes the requests
that are waiting (up to `max_batch`), groups them by target and mode in
arrival order and runs each group as one batched call (`Engine.batch`: the
window statistics and envelopes are computed once per distinct m and (m, w)
inside the group).  A request's answer does not depend on what it is batched
with: every query of a batch runs its own pipeline over its own buffers.

Admission by HBM footprint: each target keeps its series resident (8 bytes a
point) and a grow-only device workspace whose size is the largest request it
has served.  `footprint(n, m, mode)` bounds a request's workspace from the
engine's buffers (window statistics, segment envelopes, the target's forward
windows, the candidate lists of the LB/GLB/DP stages, the result and sort
buffers).  A request is admitted when its footprint alone fits in the room
its target has: the budget less every other target's series and the
workspace its engine holds, and less its own series.  When it does not, the
other targets' engines (idle while this group runs) release their workspace
first; a request that still does not fit fails with FSMELD_E_NOMEM and
nothing else is disturbed.  The admitted requests of a group share the room:
the engine caps its workspace there (`set_workspace_limit`, counted over its
batch workers too) and runs a query refused for workspace while the others
held theirs again alone, once their buffers are released.
"""
from __future__ import annotations

import collections
import concurrent.futures as cf
import threading
import time
from dataclasses import dataclass, field

import numpy as np

E_NOMEM = -3


def macro_length(m: int, n: int) -> int:
    mk = 1
    while mk < 8 * m:
        mk *= 2
    return min(mk, n)


CONCURRENCY = 4  # queries of a batch group running at once (Engine default)


def footprint(n: int, m: int, mode: str, concurrent: int = 1) -> int:
    """Upper estimate of the device workspace (bytes) a request needs on a
    target of n points, with `concurrent` queries of its batch group running
    at once (each holds its own query buffers)."""
    mk = macro_length(m, n)
    kml = mk - m + 1
    tsn = n - m + 1
    S = -(-tsn // kml)
    shared = 16 * S * kml      # window means and sigmas
    shared += 16 * S * mk      # segment envelopes U/L_normal
    shared += 16 * n           # forward windows min/max of the raw target
    q = 40 * tsn               # GLB stage lists (index, boundary, T->Q, survivors, Q->T)
    q += 24 * tsn              # survivors and the (index, distance) result list
    q += 16 * tsn              # sort buffers of the results
    q += 48 * S                # thresholds, segment counters, seeds
    if mode == "cutoff":
        q += 8 * S * kml + 24 * S  # LB values of every window, seed distances
    per_query = int(q * 1.05) + (64 << 20)  # kernel scratch (sort temporaries, work areas)
    return int(shared * 1.05) + max(1, concurrent) * per_query


class ServerError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(msg)
        self.status = status


@dataclass
class _Target:
    engine: object
    n: int
    workspace: int = 0  # footprint of the largest request served (grow-only)


@dataclass
class _Request:
    target: str
    mode: str
    spec: dict
    future: cf.Future
    t_submit: float = field(default_factory=time.perf_counter)


class Server:
    """Serve requests against resident targets on one GPU.

    `engine_factory(target_array)` creates the per-target engine (default: an
    `api.Engine` on `device`); `budget_bytes` defaults to 90% of the device
    memory free when the server starts.
    """

    def __init__(self, device: int = 0, budget_bytes: int | None = None, max_batch: int = 64,
                 engine_factory=None):
        if engine_factory is None:
            from . import api

            def engine_factory(t):
                return api.Engine(t, device=device)
            if budget_bytes is None:
                import torch
                free, _total = torch.cuda.mem_get_info(device)
                budget_bytes = int(free * 0.9)
        if budget_bytes is None:
            raise ValueError("budget_bytes is required with a custom engine factory")
        self.budget = int(budget_bytes)
        self.max_batch = max_batch
        self._factory = engine_factory
        self._targets: dict[str, _Target] = {}
        self._queue: collections.deque[_Request] = collections.deque()
        self._cv = threading.Condition()
        self._stop = False
        self._lock = threading.Lock()  # targets table
        self._thread = threading.Thread(target=self._loop, name="fsmeld-serve", daemon=True)
        self._thread.start()

    # ---------------------------------------------------------------- targets
    @staticmethod
    def _held(t: _Target) -> int:
        """Workspace bytes a target's engine holds: the engine's own count when
        it keeps one (its batch workers included), else the footprint of the
        largest request it has served."""
        held = getattr(t.engine, "workspace_bytes", None)
        return max(t.workspace, int(held())) if held is not None else t.workspace

    def _used(self, exclude: str | None = None) -> int:
        return sum(8 * t.n + self._held(t) for name, t in self._targets.items() if name != exclude)

    def _release_others(self, name: str) -> None:
        """Free the workspace of every other target's engine (idle while this
        worker serves `name`); the caller holds the targets lock."""
        for other, t in self._targets.items():
            rel = getattr(t.engine, "release_workspace", None)
            if other != name and rel is not None:
                rel()
                t.workspace = 0

    def add_target(self, name: str, target) -> None:
        t = np.ascontiguousarray(target, dtype=np.float64)
        with self._lock:
            if name in self._targets:
                raise ValueError(f"target {name!r} exists")
            if self._used() + 8 * len(t) > self.budget:
                raise ServerError(E_NOMEM, "target does not fit in the HBM budget")
            self._targets[name] = _Target(self._factory(t), len(t))

    def remove_target(self, name: str) -> None:
        with self._lock:
            tgt = self._targets.pop(name)
        tgt.engine.close()

    # --------------------------------------------------------------- requests
    def submit(self, target: str, mode: str, query, m: int, metric: str, w: int, arg: float = 0.0,
               cutoff: float | None = None, k: int | None = None, exclude=(-1, -1)) -> cf.Future:
        """Queue one request; the future's result is (idx, counters) for search,
        (idx, dist, counters) for cutoff and exact."""
        if mode not in ("search", "cutoff", "exact"):
            raise ValueError(mode)
        if (mode == "cutoff") != (k is not None):
            raise ValueError("cutoff requests take k; search and exact take a cutoff")
        spec = dict(query=np.ascontiguousarray(query, dtype=np.float64), m=int(m), metric=metric, w=int(w),
                    arg=float(arg), exclude=tuple(exclude))
        if mode == "cutoff":
            spec["k"] = int(k)
        else:
            spec["cutoff"] = float(cutoff)
        fut: cf.Future = cf.Future()
        with self._cv:
            if self._stop:
                raise RuntimeError("server closed")
            self._queue.append(_Request(target, mode, spec, fut))
            self._cv.notify()
        return fut

    def close(self) -> None:
        with self._cv:
            self._stop = True
            self._cv.notify()
        self._thread.join()
        with self._lock:
            for t in self._targets.values():
                t.engine.close()
            self._targets.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ----------------------------------------------------------------- worker
    def _loop(self) -> None:
        while True:
            with self._cv:
                while not self._queue and not self._stop:
                    self._cv.wait()
                if self._stop and not self._queue:
                    return
                take = [self._queue.popleft() for _ in range(min(self.max_batch, len(self._queue)))]
            groups: dict[tuple[str, str], list[_Request]] = collections.OrderedDict()
            for r in take:
                groups.setdefault((r.target, r.mode), []).append(r)
            for (name, mode), reqs in groups.items():
                self._run_group(name, mode, reqs)

    def _run_group(self, name: str, mode: str, reqs: list[_Request]) -> None:
        with self._lock:
            tgt = self._targets.get(name)
            if tgt is None:
                for r in reqs:
                    r.future.set_exception(KeyError(f"unknown target {name!r}"))
                return
            room = self.budget - self._used(exclude=name) - 8 * tgt.n
            # each request must fit alone; several of them share the room as
            # far as it goes (the engine runs a query refused for workspace
            # again alone once the others' buffers are released)
            fps = [footprint(tgt.n, r.spec["m"], mode, 1) if r.spec["m"] <= tgt.n else 0 for r in reqs]
            if fps and max(fps) > room:
                self._release_others(name)
                room = self.budget - self._used(exclude=name) - 8 * tgt.n
        admitted = []
        for r, fp in zip(reqs, fps):
            if fp > room:
                r.future.set_exception(ServerError(E_NOMEM, "request does not fit in the HBM budget"))
            else:
                admitted.append((r, fp))
        if not admitted:
            return
        eng = tgt.engine
        try:
            if hasattr(eng, "set_workspace_limit"):
                eng.set_workspace_limit(room)
            res = eng.batch(mode, [r.spec for r, _ in admitted])
        except Exception as e:  # a failure of the whole call
            for r, _ in admitted:
                r.future.set_exception(e)
            return
        with self._lock:
            tgt.workspace = max([tgt.workspace] + [fp for _, fp in admitted])
        for (r, _), o in zip(admitted, res):
            try:
                if o["status"] != 0:
                    raise ServerError(o["status"], f"request failed with status {o['status']}")
                if o["count"] > len(o["idx"]):  # more matches than the batch buffer: run it alone
                    s = r.spec
                    if mode == "search":
                        r.future.set_result(eng.search(s["query"], s["m"], s["cutoff"], s["metric"], s["w"],
                                                       s["arg"], exclude=s["exclude"]))
                    else:
                        r.future.set_result(eng.exact(s["query"], s["m"], s["cutoff"], s["metric"], s["w"],
                                                      s["arg"], exclude=s["exclude"]))
                    continue
                if mode == "search":
                    r.future.set_result((o["idx"], o["counters"]))
                else:
                    r.future.set_result((o["idx"], o["dist"], o["counters"]))
            except Exception as e:
                r.future.set_exception(e)
