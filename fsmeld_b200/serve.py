"""A serving loop: resident target series on one GPU, requests admitted by
HBM footprint and batched continuously on several slots.

Requests (`search`, `cutoff`, `exact` of one query against one named target)
arrive from any thread through `Server.submit`, which returns a future.
`slots` worker threads serve the queue at once, each with its own engine
(its own CUDA streams and workspace) over every target: the first slot's
engine holds the target series, the others borrow it.  A free worker takes
the oldest waiting request and every other waiting request of the same
target and mode (up to `max_batch`) and runs them as one batched call
(`Engine.batch`: window statistics and envelopes once per distinct m and
(m, w) inside the call).  So a request that arrives while others are on the
GPU starts as soon as a slot is free, and a long request occupies one slot
while the others keep serving.  A request's answer does not depend on what
it is batched with: every query of a batch runs its own pipeline over its
own buffers.

Admission by HBM footprint.  The budget holds every target's series (8 bytes
a point) and the workspace of every slot engine.  `footprint(n, m, mode)`
bounds one request's workspace from the engine's buffers (window
statistics, segment envelopes, the target's forward windows, the candidate
lists of the LB/GLB/DP stages, the result and sort buffers).  A batch starts
when its slot's engine can be granted room for its largest request: the
budget less the series and, for every other engine, the larger of the
workspace it holds and the room granted to it while it runs.  When the room
is short, the idle engines release their workspace first; when it is still
short and other slots are running, the batch waits for one of them to
finish; a request that cannot fit even with every other engine idle fails
with FSMELD_E_NOMEM and nothing else is disturbed.  The engine caps its
workspace at the granted room (`set_workspace_limit`, counted over its batch
workers) and runs a query refused for workspace while the others of its
batch held theirs again alone, once their buffers are released.
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
    engines: list  # one per slot; engines[0] holds the series
    n: int


@dataclass
class _Request:
    target: str
    mode: str
    spec: dict
    future: cf.Future
    t_submit: float = field(default_factory=time.perf_counter)


class Server:
    """Serve requests against resident targets on one GPU.

    `engine_factory(target_array)` creates the engine of the first slot of a
    target (default: an `api.Engine` on `device`); `borrow_factory(engine)`
    creates the engine of another slot over the same resident series
    (default for `api.Engine`: an engine on the first one's device pointer;
    with a custom engine factory and no borrow factory, the engine factory
    again).  `budget_bytes` defaults to 90% of the device memory free when
    the server starts.
    """

    def __init__(self, device: int = 0, budget_bytes: int | None = None, max_batch: int = 16,
                 engine_factory=None, slots: int = 4, borrow_factory=None, capacity: int = 1 << 20):
        if engine_factory is None:
            from . import api

            def engine_factory(t):
                return api.Engine(t, device=device)

            if borrow_factory is None:
                def borrow_factory(e):
                    return api.Engine(device=device, device_ptr=e.target_device_ptr(), n=e.n)
            if budget_bytes is None:
                import torch
                free, _total = torch.cuda.mem_get_info(device)
                budget_bytes = int(free * 0.9)
        if budget_bytes is None:
            raise ValueError("budget_bytes is required with a custom engine factory")
        if slots < 1:
            raise ValueError("slots must be >= 1")
        self.budget = int(budget_bytes)
        self.max_batch = max_batch
        self.slots = slots
        self.capacity = int(capacity)  # matches a batched search/exact returns (more: run alone)
        self._factory = engine_factory
        self._borrow = borrow_factory
        self._targets: dict[str, _Target] = {}
        self._queue: collections.deque[_Request] = collections.deque()
        self._cv = threading.Condition()  # queue, engine states (held, granted, busy)
        self._stop = False
        # per engine (by id): recorded footprint of the largest batch it ran,
        # room granted while it runs, busy flag
        self._recorded: dict[int, int] = {}
        self._granted: dict[int, int] = {}
        self._busy: set[int] = set()
        self._threads = [threading.Thread(target=self._loop, args=(k,), name=f"fsmeld-serve-{k}", daemon=True)
                         for k in range(slots)]
        for th in self._threads:
            th.start()

    # ---------------------------------------------------------------- memory
    def _held(self, e) -> int:
        """Workspace bytes an engine holds: the engine's own count when it
        keeps one (its batch workers included), else the footprint of the
        largest batch it has run."""
        rec = self._recorded.get(id(e), 0)
        held = getattr(e, "workspace_bytes", None)
        return max(rec, int(held())) if held is not None else rec

    def _engines(self):
        for t in self._targets.values():
            yield from t.engines

    def _series(self) -> int:
        return sum(8 * t.n for t in self._targets.values())

    def _room_for(self, e) -> int:
        """Room an engine may be granted now (the caller holds the lock)."""
        other = sum(max(self._held(o), self._granted.get(id(o), 0)) for o in self._engines() if o is not e)
        return self.budget - self._series() - other

    def _release_idle(self, keep) -> None:
        for o in self._engines():
            if o is keep or id(o) in self._busy:
                continue
            rel = getattr(o, "release_workspace", None)
            if rel is not None:
                rel()
                self._recorded[id(o)] = 0

    # ---------------------------------------------------------------- targets
    def add_target(self, name: str, target) -> None:
        t = np.ascontiguousarray(target, dtype=np.float64)
        with self._cv:
            if name in self._targets:
                raise ValueError(f"target {name!r} exists")
            used = self._series() + sum(max(self._held(o), self._granted.get(id(o), 0)) for o in self._engines())
            if used + 8 * len(t) > self.budget:
                raise ServerError(E_NOMEM, "target does not fit in the HBM budget")
            first = self._factory(t)
            engines = [first]
            for _ in range(self.slots - 1):
                engines.append(self._borrow(first) if self._borrow is not None else self._factory(t))
            self._targets[name] = _Target(engines, len(t))

    def remove_target(self, name: str) -> None:
        with self._cv:
            while any(id(e) in self._busy for e in self._targets[name].engines):
                self._cv.wait()
            tgt = self._targets.pop(name)
        for e in reversed(tgt.engines):  # borrowers before the owner of the series
            e.close()

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
            self._cv.notify_all()
        return fut

    def close(self) -> None:
        with self._cv:
            self._stop = True
            self._cv.notify_all()
        for th in self._threads:
            th.join()
        with self._cv:
            for t in self._targets.values():
                for e in reversed(t.engines):
                    e.close()
            self._targets.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ----------------------------------------------------------------- worker
    def _take(self, k: int):
        """The next batch for worker k and its engine, with the room granted;
        None when the server stops.  The caller holds the lock."""
        while True:
            while not self._queue and not self._stop:
                self._cv.wait()
            if not self._queue:
                return None
            head = self._queue[0]
            tgt = self._targets.get(head.target)
            if tgt is None:
                self._queue.popleft().future.set_exception(KeyError(f"unknown target {head.target!r}"))
                continue
            eng = next((e for e in tgt.engines if id(e) not in self._busy), None)
            if eng is None:  # every slot engine of this target runs: wait for one
                self._cv.wait()
                continue
            batch = [r for r in self._queue if r.target == head.target and r.mode == head.mode][: self.max_batch]
            fps = [footprint(tgt.n, r.spec["m"], r.mode, 1) if r.spec["m"] <= tgt.n else 0 for r in batch]
            room = self._room_for(eng)
            if max(fps) > room:
                self._release_idle(eng)
                room = self._room_for(eng)
            if max(fps) > room:
                if self._busy:  # memory frees up when a running batch ends
                    self._cv.wait()
                    continue
                # nothing else runs: what does not fit now never will
                keep = []
                for r, fp in zip(batch, fps):
                    if fp > room:
                        self._queue.remove(r)
                        r.future.set_exception(ServerError(E_NOMEM, "request does not fit in the HBM budget"))
                    else:
                        keep.append((r, fp))
                if not keep:
                    continue
                batch, fps = [r for r, _ in keep], [fp for _, fp in keep]
            for r in batch:
                self._queue.remove(r)
            # grant enough for the engine's concurrent queries, within the room
            want = sum(sorted(fps)[-CONCURRENCY:])
            grant = min(room, max(self._held(eng), want))
            self._granted[id(eng)] = grant
            self._busy.add(id(eng))
            return batch, fps, eng, grant

    def _loop(self, k: int) -> None:
        while True:
            with self._cv:
                got = self._take(k)
            if got is None:
                return
            batch, fps, eng, grant = got
            try:
                self._run(batch, fps, eng, grant)
            finally:
                with self._cv:
                    self._busy.discard(id(eng))
                    self._granted.pop(id(eng), None)
                    self._recorded[id(eng)] = max([self._recorded.get(id(eng), 0)] + fps)
                    self._cv.notify_all()

    @staticmethod
    def _alone(eng, mode: str, s: dict):
        """One request alone on its slot's engine (its batch is done); the
        workspace the batch's concurrent queries left is released first when
        the request does not fit beside it."""
        def call():
            if mode == "search":
                return eng.search(s["query"], s["m"], s["cutoff"], s["metric"], s["w"], s["arg"],
                                  exclude=s["exclude"])
            return eng.exact(s["query"], s["m"], s["cutoff"], s["metric"], s["w"], s["arg"], exclude=s["exclude"])
        try:
            return call()
        except Exception as e:
            rel = getattr(eng, "release_workspace", None)
            if getattr(e, "status", None) != E_NOMEM or rel is None:
                raise
            rel()
            return call()

    def _run(self, reqs: list[_Request], fps: list[int], eng, grant: int) -> None:
        mode = reqs[0].mode
        try:
            if hasattr(eng, "set_workspace_limit"):
                eng.set_workspace_limit(grant)
            res = eng.batch(mode, [r.spec for r in reqs], capacity=self.capacity)
        except Exception as e:  # a failure of the whole call
            for r in reqs:
                r.future.set_exception(e)
            return
        for r, o in zip(reqs, res):
            try:
                if o["status"] != 0:
                    raise ServerError(o["status"], f"request failed with status {o['status']}")
                if o["count"] > len(o["idx"]):  # more matches than the batch buffer: run it alone
                    r.future.set_result(self._alone(eng, mode, r.spec))
                    continue
                if mode == "search":
                    r.future.set_result((o["idx"], o["counters"]))
                else:
                    r.future.set_result((o["idx"], o["dist"], o["counters"]))
            except Exception as e:
                r.future.set_exception(e)
