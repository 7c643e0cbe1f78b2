"""The serving loop's host logic (fsmeld_b200.serve) with a stand-in engine:
requests are grouped by target and mode in arrival order, every answer
reaches its own future, admission by HBM footprint rejects what does not fit
and serves the rest, a result larger than the batch buffer is fetched alone,
a long request holds one slot while the others keep serving, and a batch
whose room is taken by a running one waits for it instead of failing."""
import threading
import time

import numpy as np
import pytest

from fsmeld_b200.serve import E_NOMEM, Server, ServerError, footprint


class FakeEngine:
    """Answers from the query values: idx = [sum-derived index], one batch log."""

    def __init__(self, t, log, gate=None):
        self.n = len(t)
        self.log = log
        self.gate = gate
        self.limit = None

    def set_workspace_limit(self, b):
        self.limit = b

    def batch(self, mode, specs, capacity=1 << 14):
        if self.gate is not None:
            self.gate.wait()
        self.log.append((mode, len(specs)))
        out = []
        for s in specs:
            key = int(round(float(np.sum(s["query"])) * 1000)) % 997
            big = s.get("cutoff", 0.0) == 99.0
            idx = np.array([key], dtype=np.int64)
            out.append({"status": 0, "idx": idx, "dist": np.array([key * 0.5]), "count": 5 if big else 1,
                        "counters": {"valid": key}})
        return out

    def search(self, q, m, cutoff, metric, w, arg, exclude=(-1, -1)):
        return np.arange(5, dtype=np.int64), {"valid": -1}

    def exact(self, q, m, cutoff, metric, w, arg, exclude=(-1, -1)):
        return np.arange(5, dtype=np.int64), np.arange(5.0), {"valid": -1}

    def close(self):
        pass


def _q(i, m=32):
    return np.sin(np.arange(m) * 0.1 * (i + 1))


def test_routing_and_grouping():
    log = []
    gate = threading.Event()
    srv = Server(budget_bytes=1 << 40, max_batch=64, slots=1, engine_factory=lambda t: FakeEngine(t, log, gate))
    try:
        srv.add_target("a", np.zeros(4096))
        srv.add_target("b", np.zeros(8192))
        # the first request occupies the worker; the rest queue up and come as one pass
        first = srv.submit("a", "search", _q(100), 32, "dtw", 3, cutoff=1.0)
        time.sleep(0.2)
        futs = []
        for i in range(12):
            tgt = "a" if i % 2 else "b"
            if i % 3 == 0:
                futs.append((i, srv.submit(tgt, "cutoff", _q(i), 32, "dtw", 3, k=4)))
            else:
                futs.append((i, srv.submit(tgt, "search", _q(i), 32, "msm", 3, 0.5, cutoff=2.0)))
        gate.set()
        first.result(timeout=10)
        for i, f in futs:
            res = f.result(timeout=10)
            key = int(round(float(np.sum(_q(i))) * 1000)) % 997
            assert int(res[0][0]) == key
            assert res[-1]["valid"] == key
        # after the first call: one batch per (target, mode) group
        groups = {("b", "cutoff"), ("a", "search"), ("a", "cutoff"), ("b", "search")}
        assert len(log) == 1 + len(groups)
        assert sum(nq for _, nq in log[1:]) == 12
    finally:
        gate.set()
        srv.close()


def test_admission_by_footprint():
    log = []
    n = 1 << 16
    small = footprint(n, 32, "search")
    big = footprint(n, 4096, "search")
    assert big > small + 4 * n
    # room for target a, its largest small request and half of another series
    srv = Server(budget_bytes=8 * n + small + 4 * n, slots=1, engine_factory=lambda t: FakeEngine(t, log))
    try:
        srv.add_target("a", np.zeros(n))
        ok = srv.submit("a", "search", _q(1), 32, "dtw", 3, cutoff=1.0)
        assert ok.result(timeout=10)[0].shape == (1,)  # alone in its pass: one query's buffers
        bad = srv.submit("a", "search", _q(2, 4096), 4096, "dtw", 3, cutoff=1.0)
        with pytest.raises(ServerError) as ei:
            bad.result(timeout=10)
        assert ei.value.status == E_NOMEM
        with pytest.raises(ServerError):
            srv.add_target("b", np.zeros(n))  # its series does not fit beside a's workspace
    finally:
        srv.close()


def test_large_result_fetched_alone_and_bad_requests():
    log = []
    srv = Server(budget_bytes=1 << 40, engine_factory=lambda t: FakeEngine(t, log))
    try:
        srv.add_target("a", np.zeros(4096))
        idx, cnt = srv.submit("a", "search", _q(3), 32, "dtw", 3, cutoff=99.0).result(timeout=10)
        assert list(idx) == [0, 1, 2, 3, 4] and cnt["valid"] == -1
        with pytest.raises(KeyError):
            srv.submit("nope", "search", _q(3), 32, "dtw", 3, cutoff=1.0).result(timeout=10)
        with pytest.raises(ValueError):
            srv.submit("a", "cutoff", _q(3), 32, "dtw", 3, cutoff=1.0)
    finally:
        srv.close()


class SlowEngine(FakeEngine):
    """Blocks the batches whose first query has cutoff 7.0 until `gate` is set."""

    def __init__(self, t, log, gate, started):
        super().__init__(t, log)
        self.slow_gate = gate
        self.started = started

    def batch(self, mode, specs, capacity=1 << 14):
        self.started.append(tuple(s.get("cutoff") for s in specs))
        if specs[0].get("cutoff") == 7.0:
            self.slow_gate.wait(timeout=20)
        return super().batch(mode, specs, capacity)


def test_long_request_holds_one_slot():
    log, started = [], []
    gate = threading.Event()
    srv = Server(budget_bytes=1 << 40, slots=2, engine_factory=lambda t: SlowEngine(t, log, gate, started))
    try:
        srv.add_target("a", np.zeros(4096))
        slow = srv.submit("a", "search", _q(1), 32, "dtw", 3, cutoff=7.0)
        time.sleep(0.2)
        fast = srv.submit("a", "search", _q(2), 32, "dtw", 3, cutoff=1.0)
        fast.result(timeout=10)  # served by the second slot while the first is held
        assert not slow.done()
        gate.set()
        slow.result(timeout=10)
    finally:
        gate.set()
        srv.close()


def test_batch_waits_for_room_held_by_a_running_one():
    log, started = [], []
    gate = threading.Event()
    n = 1 << 16
    fp = footprint(n, 32, "search")
    # room for the series and one request's workspace: the second request
    # waits until the first one's slot is done, then runs (no FSMELD_E_NOMEM)
    srv = Server(budget_bytes=8 * n + fp + fp // 2, slots=2,
                 engine_factory=lambda t: SlowEngine(t, log, gate, started))
    try:
        srv.add_target("a", np.zeros(n))
        first = srv.submit("a", "search", _q(1), 32, "dtw", 3, cutoff=7.0)
        time.sleep(0.2)
        second = srv.submit("a", "search", _q(2), 32, "dtw", 3, cutoff=1.0)
        time.sleep(0.3)
        assert not second.done() and len(started) == 1
        gate.set()
        first.result(timeout=10)
        assert second.result(timeout=10)[0].shape == (1,)
    finally:
        gate.set()
        srv.close()


class HoldingEngine(FakeEngine):
    """Keeps `held` bytes after a batch (its workers' buffers); a request run
    alone fails with FSMELD_E_NOMEM until that workspace is released."""

    def __init__(self, t, log):
        super().__init__(t, log)
        self.held = 0
        self.released = 0

    def workspace_bytes(self):
        return self.held

    def release_workspace(self):
        self.held = 0
        self.released += 1

    def batch(self, mode, specs, capacity=1 << 14):
        out = super().batch(mode, specs, capacity)
        self.held = 1 << 30
        return out

    def search(self, q, m, cutoff, metric, w, arg, exclude=(-1, -1)):
        if self.held:
            err = RuntimeError("Device workspace budget exceeded")
            err.status = E_NOMEM
            raise err
        return super().search(q, m, cutoff, metric, w, arg, exclude)


def test_large_result_alone_after_release():
    log = []
    engines = []

    def factory(t):
        e = HoldingEngine(t, log)
        engines.append(e)
        return e

    srv = Server(budget_bytes=1 << 40, slots=1, engine_factory=factory)
    try:
        srv.add_target("a", np.zeros(4096))
        # cutoff 99.0: the stand-in reports more matches than the batch buffer
        idx, cnt = srv.submit("a", "search", _q(3), 32, "dtw", 3, cutoff=99.0).result(timeout=10)
        assert list(idx) == [0, 1, 2, 3, 4]
        assert engines[0].released == 1
    finally:
        srv.close()
