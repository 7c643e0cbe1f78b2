"""Targets larger than device memory: stream a headerless little-endian
float64 target file (the reference's target format, src/fsmeld.cpp:740-746)
through the GPU in macro-segment-aligned chunks.

A chunk is a slice of the target that starts at a segment boundary and ends
with the m-1 halo of its last full segment (the last chunk runs to the end of
the file and also holds the EOF-aligned tail segment), exactly the slices of
the multi-GPU partition (`shard.partition`): every per-segment computation
sees the points it sees in a search of the whole target, so the merged
results equal one search of the whole file, bit for bit (match lists
concatenated, counters summed; top-k lists merged by (distance, index)).

The file is memory-mapped; a reader thread copies each chunk into pinned
host memory while the GPU works on the previous one, and two engines (each
with its own CUDA stream) take alternate chunks, so a chunk's upload
overlaps the previous chunk's kernels.  Queries are grouped by length m (the
segment geometry depends on m) and each group streams the file once for all
its queries.
"""
from __future__ import annotations

import concurrent.futures as cf
import threading

import numpy as np

from .shard import FEWER_K, ShardedSearch, local_exclusion, macro_length, partition


def chunk_plan(n: int, m: int, max_points: int):
    """Segment-aligned slices of a length-n target, each at most max_points
    long (a single full segment plus the tail is the smallest chunk)."""
    chunks = 1
    while True:
        plan = [s for s in partition(n, m, chunks) if s is not None]
        if max(s.stop - s.start for s in plan) <= max_points or len(plan) < chunks:
            return plan
        chunks = max(chunks + 1, int(chunks * 1.25))


def _local_exclusions(specs, sh):
    out = []
    for d in specs:
        d2 = dict(d)
        d2["exclude"] = local_exclusion(tuple(d.get("exclude", (-1, -1))), sh)
        out.append(d2)
    return out


class StreamingTarget:
    """Search / exact / cutoff over a target file that need not fit in device
    memory.

    `max_points`: the longest chunk (points) held on the device at a time;
    `chunk_runner(array, mode, specs)`: runs a batch on one chunk and returns
    `Engine.batch`-style results (default: two `api.Engine`s on `device`,
    alternating chunks).
    """

    def __init__(self, path: str, max_points: int, device: int = 0, chunk_runner=None):
        self.path = path
        self.data = np.memmap(path, dtype="<f8", mode="r")
        self.n = len(self.data)
        self.max_points = int(max_points)
        self.device = device
        self._runner = chunk_runner
        self._engines = None
        self._pool = None

    # default runner: two engines, each owned by one worker thread
    def _engine_runner(self):
        if self._engines is None:
            import torch

            from . import api
            self._api = api
            self._torch = torch
            self._engines = [None, None]
            self._pinned = [None, None]
            self._pool = cf.ThreadPoolExecutor(max_workers=2)
            self._locks = [threading.Lock(), threading.Lock()]
        return self._run_on_engine

    def _run_on_engine(self, slot, arr, mode, specs):
        with self._locks[slot]:
            buf = self._pinned[slot]
            if buf is None or buf.numel() < len(arr):
                buf = self._torch.empty(self.max_points, dtype=self._torch.float64).pin_memory()
                self._pinned[slot] = buf
            host = buf.numpy()[:len(arr)]
            np.copyto(host, arr)
            if self._engines[slot] is None:
                self._engines[slot] = self._api.Engine(host, device=self.device)
            else:
                self._engines[slot].load(host)
            return self._engines[slot].batch(mode, specs)

    def close(self):
        if self._engines:
            for e in self._engines:
                if e is not None:
                    e.close()
        if self._pool is not None:
            self._pool.shutdown()
        self._engines = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def batch(self, mode: str, queries: list[dict]):
        """queries as for `Engine.batch`; returns one result dict per query
        (idx, dist, count, counters, status) over the whole file."""
        out: list[dict | None] = [None] * len(queries)
        by_m: dict[int, list[int]] = {}
        for i, d in enumerate(queries):
            by_m.setdefault(int(d["m"]), []).append(i)
        for m, ids in by_m.items():
            specs = [queries[i] for i in ids]
            for i, r in zip(ids, self._stream(mode, m, specs)):
                out[i] = r
        return out

    def _stream(self, mode, m, specs):
        plan = chunk_plan(self.n, m, self.max_points)
        per_query = [[] for _ in specs]

        def run_chunk(k, sh):
            arr = self.data[sh.start:sh.stop]
            local = _local_exclusions(specs, sh)
            if self._runner is not None:
                res = self._runner(np.asarray(arr), mode, local)
            else:
                res = self._engine_runner()(k % 2, arr, mode, local)
            return sh, local, res

        if self._runner is None:
            self._engine_runner()
            futs = [self._pool.submit(run_chunk, k, sh) for k, sh in enumerate(plan)]
            results = [f.result() for f in futs]
        else:
            results = [run_chunk(k, sh) for k, sh in enumerate(plan)]
        for sh, local, res in results:
            for q, r in enumerate(res):
                if mode == "cutoff" and r["status"] == FEWER_K:
                    r = self._chunk_all(sh, local[q])  # the chunk has fewer than k valid windows
                elif r["status"] != 0:
                    raise RuntimeError(f"chunk [{sh.start}, {sh.stop}): status {r['status']}")
                elif r["count"] > len(r["idx"]):
                    r = self._chunk_alone(sh, mode, local[q])
                per_query[q].append((np.asarray(r["idx"], dtype=np.int64) + sh.start,
                                     np.asarray(r["dist"], dtype=np.float64), r["counters"]))
        outs = []
        for q, parts in enumerate(per_query):
            if mode == "search":
                idx, cnt = ShardedSearch.merge_search([(p[0], p[2]) for p in parts], m, self.n, specs[q]["cutoff"])
                dist = np.zeros(0)
            elif mode == "exact":
                idx, dist, cnt = ShardedSearch.merge_exact(parts, m, self.n, specs[q]["cutoff"])
            else:
                idx, dist, cnt = ShardedSearch.merge_cutoff(parts, m, self.n, specs[q]["k"])
            outs.append({"status": 0, "idx": idx, "dist": dist, "count": len(idx), "counters": cnt})
        return outs

    # single-query fallbacks on one chunk (default engines or the runner)
    def _one(self, sh, mode, spec):
        arr = np.asarray(self.data[sh.start:sh.stop])
        if self._runner is not None:
            return self._runner(arr, mode, [spec])[0]
        from . import api
        with api.Engine(arr, device=self.device) as e:
            s = spec
            if mode == "search":
                idx, cnt = e.search(s["query"], s["m"], s["cutoff"], s["metric"], s["w"], s.get("arg", 0.0),
                                    exclude=s["exclude"])
                return {"status": 0, "idx": idx, "dist": np.zeros(0), "count": len(idx), "counters": cnt}
            idx, dist, cnt = e.exact(s["query"], s["m"], s["cutoff"], s["metric"], s["w"], s.get("arg", 0.0),
                                     exclude=s["exclude"])
            return {"status": 0, "idx": idx, "dist": dist, "count": len(idx), "counters": cnt}

    def _chunk_alone(self, sh, mode, spec):
        return self._one(sh, mode, spec)

    def _chunk_all(self, sh, spec):
        s = dict(spec)
        s.pop("k", None)
        s["cutoff"] = float(np.finfo(np.float64).max)
        return self._one(sh, "exact", s)

    def search(self, query, m, cutoff, metric, w, arg=0.0, exclude=(-1, -1)):
        r = self.batch("search", [dict(query=query, m=m, cutoff=cutoff, metric=metric, w=w, arg=arg,
                                       exclude=exclude)])[0]
        return r["idx"], r["counters"]

    def exact(self, query, m, cutoff, metric, w, arg=0.0, exclude=(-1, -1)):
        r = self.batch("exact", [dict(query=query, m=m, cutoff=cutoff, metric=metric, w=w, arg=arg,
                                      exclude=exclude)])[0]
        return r["idx"], r["dist"], r["counters"]

    def cutoff(self, query, m, k, metric, w, arg=0.0, exclude=(-1, -1)):
        r = self.batch("cutoff", [dict(query=query, m=m, k=k, metric=metric, w=w, arg=arg, exclude=exclude)])[0]
        return r["idx"], r["dist"], r["counters"]


__all__ = ["StreamingTarget", "chunk_plan", "macro_length"]
