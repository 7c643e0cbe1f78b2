"""One target across several ranks (fsmeld_b200.shard), on the host.

The partition puts each rank on a slice that starts at a macro-segment
boundary (with the m-1 halo), so every per-segment computation sees exactly
the points it sees in a search of the whole target.  Checked here with two
gloo ranks whose per-slice searches run on the oracle: the merged match sets,
counters, exact distances and top-k rankings equal one oracle run over the
whole target, bit for bit.  The GPU path uses the same host logic with an
`api.Engine` per slice.
"""
import os
import socket

import numpy as np
import pytest

from fsmeld_b200.shard import ShardedSearch, local_exclusion, macro_length, partition

CASES = [("dtw", 0.0), ("erp", 0.4), ("edr", 0.25), ("lcss", 0.25), ("msm", 0.5)]


@pytest.mark.parametrize("n,m,world", [(1 << 15, 64, 2), (1 << 15, 64, 3), (1 << 15, 100, 4), (700, 64, 2),
                                       (5000, 40, 7), (2 * 512 + 63, 64, 2), (1 << 14, 128, 1)])
def test_partition_reproduces_segments(n, m, world):
    mk = macro_length(m, n)
    kml = mk - m + 1
    tsn = n - m + 1
    forsize, tail = tsn // kml, tsn % kml
    shards = [s for s in partition(n, m, world) if s is not None]
    assert shards and len(shards) <= world
    covered = []
    for k, sh in enumerate(shards):
        ln = sh.stop - sh.start
        assert sh.start == sh.seg_begin * kml
        # the slice's own geometry is the global segments seg_begin..seg_end (+ the tail)
        assert macro_length(m, ln) == mk
        ltsn = ln - m + 1
        assert ltsn // kml == sh.seg_end - sh.seg_begin
        assert ltsn % kml == (tail if sh.has_tail else 0)
        if sh.has_tail:
            assert sh.stop == n and k == len(shards) - 1 and sh.seg_end > sh.seg_begin
        covered.append((sh.start, sh.start + ltsn))
    # windows covered exactly once, in increasing order
    assert covered[0][0] == 0 and covered[-1][1] == tsn
    for a, b in zip(covered, covered[1:]):
        assert a[1] == b[0]
    assert sum(s.seg_end - s.seg_begin for s in shards) == forsize


def test_local_exclusion():
    from fsmeld_b200.shard import Shard
    sh = Shard(1, 1000, 3000, 1, 3, False)
    assert local_exclusion((-1, -1), sh) == (-1, -1)
    assert local_exclusion((0, 500), sh) == (-1, -1)
    assert local_exclusion((900, 1100), sh) == (0, 100)
    assert local_exclusion((1500, 1600), sh) == (500, 600)
    assert local_exclusion((5000, 6000), sh) == (-1, -1)


class _OracleSlice:
    """The oracle over one slice, with api.Engine's method signatures."""

    def __init__(self, oracle, t):
        self.o, self.t = oracle, t

    def search(self, q, m, cut, metric, w, arg, exclude=(-1, -1)):
        return self.o.search(self.t, q, m, cut, metric, w, arg, excl=exclude)

    def exact(self, q, m, cut, metric, w, arg, exclude=(-1, -1)):
        return self.o.exact(self.t, q, m, cut, metric, w, arg, excl=exclude)

    def cutoff(self, q, m, k, metric, w, arg, exclude=(-1, -1)):
        try:
            return self.o.cutoff(self.t, q, m, k, metric, w, arg, excl=exclude)
        except ValueError as e:
            if "Fewer" in str(e):
                err = RuntimeError(str(e))
                err.status = -5
                raise err from None
            raise


def _bits(a):
    return np.asarray(a, dtype=np.float64).view(np.int64)


def _rank_main(rank, world, port, n, m, w, seed):
    import torch.distributed as dist

    from fsmeld_b200.synth import query_from, walk_with_structure
    from oracle.oracle import Oracle

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        o = Oracle("oracle")
        t = walk_with_structure(n, m, seed=seed, motifs=10, nan_fraction=2e-3, flat_runs=3, nan_spans=4)
        q, _ = query_from(t, m, np.random.default_rng(seed + 1))
        ss = ShardedSearch(n, rank, world, lambda a, b: _OracleSlice(o, t[a:b]))
        excl = (n // 3, n // 3 + 5 * m)
        for metric, arg in CASES:
            fidx, fdist, fc = o.cutoff(t, q, m, 12, metric, w, arg)
            sidx, sdist, sc = ss.cutoff(q, m, 12, metric, w, arg)
            cut = float(fdist[-1])
            gidx, gc = ss.search(q, m, cut, metric, w, arg)
            eidx, edist, ec = ss.exact(q, m, cut, metric, w, arg)
            xidx, xc = ss.search(q, m, cut, metric, w, arg, exclude=excl)
            if rank == 0:
                assert list(sidx) == list(fidx), metric
                assert np.array_equal(_bits(sdist), _bits(fdist)), metric
                assert sc["valid"] == fc["valid"], metric
                oidx, oc = o.search(t, q, m, cut, metric, w, arg)
                assert list(gidx) == list(oidx), metric
                for key in ("valid", "invalid", "after_lb", "after_glb", "exact_evals", "matches", "segments",
                            "tail", "m_k"):
                    assert gc[key] == oc[key], (metric, key, gc[key], oc[key])
                oeidx, oedist, _ = o.exact(t, q, m, cut, metric, w, arg)
                assert list(eidx) == list(oeidx) and np.array_equal(_bits(edist), _bits(oedist)), metric
                ox, oxc = o.search(t, q, m, cut, metric, w, arg, excl=excl)
                assert list(xidx) == list(ox) and xc["invalid"] == oxc["invalid"], metric
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world,n,m,w", [(2, 1 << 15, 64, 5), (3, 6000, 48, 4)])
def test_sharded_search_equals_whole_target(oracle, world, n, m, w):
    import torch.multiprocessing as mp
    mp.spawn(_rank_main, args=(world, _free_port(), n, m, w, 4242 + world), nprocs=world, join=True)
