"""One target series searched by several GPUs: partition by macro segment.

Every per-segment computation of the search (window statistics restarted at
each segment, segment envelopes and LB_IP thresholds, LB_IP, GLB, the exact
DPs) reads only the segment's m_k points (src/fsmeld.cpp:729-746).  A slice of
the target that starts at a segment boundary s0 * k_m_l and ends with the m-1
halo of its last full segment therefore has, as its own geometry, exactly the
global segments s0 .. s1-1, point for point; the slice that runs to the end of
the target also reproduces the EOF-aligned tail segment (src/fsmeld.cpp:
155-168, 658-661) as long as it holds at least one full segment.  Each rank
searches its slice on its own GPU and the results are merged:

* search / exact: match lists concatenated in rank order (the ranks' window
  ranges are disjoint and increasing, so the merged list stays sorted), the
  counters summed -- equal, bit for bit, to one search over the whole target;
* cutoff: each rank's top-k (dist, index) pairs gathered and the k smallest
  taken in the reference's lexicographic order (src/fsmeld.cpp:409-418); every
  global top-k pair is in its own rank's top-k, so the merge is exact.

Global window index = local index + slice start.  Ranks exchange only the
result lists (torch.distributed all_gather_object: NCCL between GPUs, gloo on
the host); there is no data-path collective.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

FEWER_K = -5  # FSMELD_E_FEWER_K: a slice with fewer valid windows than k
SUMMED = ("valid", "invalid", "after_lb", "after_glb", "exact_evals", "matches", "dp_cells", "segments")


def macro_length(m: int, n: int) -> int:
    """m_k = 2^ceil(log2(8m)) clipped to n (src/fsmeld.cpp:28-37)."""
    mk = 1
    while mk < 8 * m:
        mk *= 2
    return min(mk, n)


@dataclass(frozen=True)
class Shard:
    rank: int
    start: int  # first target point of the slice (= first global window index)
    stop: int   # one past the last target point of the slice
    seg_begin: int
    seg_end: int       # full segments [seg_begin, seg_end)
    has_tail: bool


def partition(n: int, m: int, world: int) -> list[Shard | None]:
    """Slices of a length-n target for query length m over `world` ranks (None:
    the rank has no segment; happens when there are fewer full segments than
    ranks)."""
    if m < 1 or n < m:
        raise ValueError("target shorter than the query")
    mk = macro_length(m, n)
    kml = mk - m + 1
    tsn = n - m + 1
    forsize, tail = tsn // kml, tsn % kml
    used = max(1, min(world, forsize))
    shards: list[Shard | None] = [None] * world
    for r in range(used):
        s0 = forsize * r // used
        s1 = forsize * (r + 1) // used
        last = r == used - 1
        stop = n if last else s1 * kml + m - 1
        shards[r] = Shard(r, s0 * kml, stop, s0, s1, last and tail > 0)
    return shards


def local_exclusion(ex: tuple[int, int], shard: Shard) -> tuple[int, int]:
    """The exclusion interval of global window indices in slice coordinates."""
    eb, ee = ex
    if eb < 0 or ee <= eb:
        return (-1, -1)
    lb, le = max(eb - shard.start, 0), ee - shard.start
    nwin = shard.stop - shard.start
    if le <= 0 or lb >= nwin:
        return (-1, -1)
    return (lb, le)


def _sum_counters(parts: list[dict], m_k: int) -> dict:
    out = {k: 0 for k in SUMMED}
    for p in parts:
        for k in SUMMED:
            out[k] += int(p.get(k, 0))
    out["m_k"] = m_k
    out["tail"] = int(parts[-1].get("tail", 0)) if parts else 0
    return out


class ShardedSearch:
    """Search one target with `world` ranks, each on its own slice.

    `shard_engine(start, stop)` returns the object that searches target[start:stop]
    on this rank (an `api.Engine` on this rank's GPU in `ShardedEngine`); it needs
    `search`, `exact` and `cutoff` with `api.Engine`'s signatures.  Every rank
    calls every method with the same arguments, in the same order.
    """

    def __init__(self, n: int, rank: int, world: int, shard_engine, group=None):
        self.n, self.rank, self.world, self.group = n, rank, world, group
        self._shard_engine = shard_engine

    def _gather(self, obj):
        import torch.distributed as dist
        if self.world == 1:
            return [obj]
        out = [None] * self.world
        dist.all_gather_object(out, obj, group=self.group)
        return out

    def _mine(self, m):
        return partition(self.n, m, self.world)[self.rank]

    # rank-local parts (None when the rank holds no segment) ------------------
    def local_search(self, query, m, cutoff, metric, w, arg=0.0, exclude=(-1, -1)):
        sh = self._mine(m)
        if sh is None:
            return None
        eng = self._shard_engine(sh.start, sh.stop)
        idx, cnt = eng.search(query, m, cutoff, metric, w, arg, exclude=local_exclusion(exclude, sh))
        return (np.asarray(idx, dtype=np.int64) + sh.start, cnt)

    def local_exact(self, query, m, cutoff, metric, w, arg=0.0, exclude=(-1, -1)):
        sh = self._mine(m)
        if sh is None:
            return None
        eng = self._shard_engine(sh.start, sh.stop)
        idx, dist, cnt = eng.exact(query, m, cutoff, metric, w, arg, exclude=local_exclusion(exclude, sh))
        return (np.asarray(idx, dtype=np.int64) + sh.start, np.asarray(dist, dtype=np.float64), cnt)

    def local_cutoff(self, query, m, k, metric, w, arg=0.0, exclude=(-1, -1)):
        """This rank's top-k (all its valid windows when it has fewer than k)."""
        sh = self._mine(m)
        if sh is None:
            return None
        eng = self._shard_engine(sh.start, sh.stop)
        ex = local_exclusion(exclude, sh)
        try:
            idx, dist, cnt = eng.cutoff(query, m, k, metric, w, arg, exclude=ex)
        except Exception as e:
            if getattr(e, "status", None) != FEWER_K:
                raise
            idx, dist, cnt = eng.exact(query, m, float(np.finfo(np.float64).max), metric, w, arg, exclude=ex)
        return (np.asarray(idx, dtype=np.int64) + sh.start, np.asarray(dist, dtype=np.float64), cnt)

    # merges of every rank's part, in rank order --------------------------------
    @staticmethod
    def merge_search(parts, m, n, cutoff):
        parts = [p for p in parts if p is not None]
        idx = np.concatenate([p[0] for p in parts]) if parts else np.zeros(0, np.int64)
        cnt = _sum_counters([p[1] for p in parts], macro_length(m, n))
        cnt["threshold"] = float(cutoff)
        return idx, cnt

    @staticmethod
    def merge_exact(parts, m, n, cutoff):
        parts = [p for p in parts if p is not None]
        idx = np.concatenate([p[0] for p in parts]) if parts else np.zeros(0, np.int64)
        dist = np.concatenate([p[1] for p in parts]) if parts else np.zeros(0)
        cnt = _sum_counters([p[2] for p in parts], macro_length(m, n))
        cnt["threshold"] = float(cutoff)
        return idx, dist, cnt

    @staticmethod
    def merge_cutoff(parts, m, n, k):
        parts = [p for p in parts if p is not None]
        idx = np.concatenate([p[0] for p in parts])
        dist = np.concatenate([p[1] for p in parts])
        if len(idx) < k:
            raise ValueError("Fewer valid, non-excluded candidates than requested k.")
        order = np.lexsort((idx, dist))[:k]
        cnt = _sum_counters([p[2] for p in parts], macro_length(m, n))
        cnt["matches"] = k
        cnt["threshold"] = float(dist[order[-1]])
        return idx[order], dist[order], cnt

    # collective calls: every rank calls them with the same arguments ----------
    def search(self, query, m, cutoff, metric, w, arg=0.0, exclude=(-1, -1)):
        parts = self._gather(self.local_search(query, m, cutoff, metric, w, arg, exclude))
        return self.merge_search(parts, m, self.n, cutoff)

    def exact(self, query, m, cutoff, metric, w, arg=0.0, exclude=(-1, -1)):
        parts = self._gather(self.local_exact(query, m, cutoff, metric, w, arg, exclude))
        return self.merge_exact(parts, m, self.n, cutoff)

    def cutoff(self, query, m, k, metric, w, arg=0.0, exclude=(-1, -1)):
        """Global top-k: every rank's top-k merged by (distance, index)."""
        parts = self._gather(self.local_cutoff(query, m, k, metric, w, arg, exclude))
        return self.merge_cutoff(parts, m, self.n, k)


class ShardedEngine(ShardedSearch):
    """`ShardedSearch` over this rank's GPU: the whole target is resident once
    (a torch tensor) and each slice is searched by an `api.Engine` that borrows
    its device memory; engines are cached per slice (one per query length)."""

    def __init__(self, target, rank: int, world: int, device: int = 0, group=None):
        import torch

        from . import api
        self._api = api
        self._device = device
        self._target = torch.from_numpy(np.ascontiguousarray(target, dtype=np.float64)).to(f"cuda:{device}")
        self._engines: dict[tuple[int, int], object] = {}
        super().__init__(len(target), rank, world, self._engine_for, group)

    def _engine_for(self, start: int, stop: int):
        key = (start, stop)
        if key not in self._engines:
            ptr = self._target.data_ptr() + 8 * start
            self._engines[key] = self._api.Engine(device_ptr=ptr, n=stop - start, device=self._device)
        return self._engines[key]

    def close(self):
        for e in self._engines.values():
            e.close()
        self._engines.clear()
