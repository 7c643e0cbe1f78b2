"""One target split over ranks at macro-segment boundaries, on the CUDA path.

Every rank's slice is searched by an `api.Engine` that borrows the device
memory of one resident copy of the target (slice starts are 8-byte aligned
only); the merged results must equal the oracle over the whole target and
one engine over the whole target, bit for bit, with summed counters.  The ranks run one after another in this
process (the merge is the same host code the collective calls use)."""
import numpy as np
import pytest

from fsmeld_b200.shard import ShardedSearch, partition
from fsmeld_b200.synth import query_from, walk_with_structure

pytestmark = pytest.mark.gpu

CASES = [("dtw", 0.0), ("erp", 0.4), ("edr", 0.25), ("lcss", 0.25), ("msm", 0.5)]


def _bits(a):
    return np.asarray(a, dtype=np.float64).view(np.int64)


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_engine_equals_whole_target(oracle, world):
    import torch

    from fsmeld_b200 import api

    m, w, n = 64, 5, 1 << 16
    t = walk_with_structure(n, m, seed=91, motifs=20, nan_fraction=2e-3, flat_runs=6, nan_spans=5)
    q, _ = query_from(t, m, np.random.default_rng(92))
    t_dev = torch.from_numpy(t).to("cuda:0")
    engines = {}

    def slice_engine(a, b):
        if (a, b) not in engines:
            engines[(a, b)] = api.Engine(device_ptr=t_dev.data_ptr() + 8 * a, n=b - a, device=0)
        return engines[(a, b)]

    ranks = [ShardedSearch(n, r, world, slice_engine) for r in range(world)]
    assert sum(s is not None for s in partition(n, m, world)) == world
    excl = (n // 2, n // 2 + 3 * m)
    try:
        with api.Engine(t) as full:
            for metric, arg in CASES:
                fidx, fdist, fc = full.cutoff(q, m, 20, metric, w, arg)
                sidx, sdist, sc = ShardedSearch.merge_cutoff(
                    [r.local_cutoff(q, m, 20, metric, w, arg) for r in ranks], m, n, 20)
                assert list(sidx) == list(fidx) and np.array_equal(_bits(sdist), _bits(fdist)), metric
                assert sc["valid"] == fc["valid"]
                kidx, kdist, _ = oracle.cutoff(t, q, m, 20, metric, w, arg)
                assert list(sidx) == list(kidx) and np.array_equal(_bits(sdist), _bits(kdist)), metric
                cut = float(fdist[-1])
                oidx, oc = full.search(q, m, cut, metric, w, arg)
                gidx, gc = ShardedSearch.merge_search([r.local_search(q, m, cut, metric, w, arg) for r in ranks],
                                                      m, n, cut)
                assert list(gidx) == list(oidx), metric
                for key in ("valid", "invalid", "after_lb", "after_glb", "matches", "segments", "tail", "m_k"):
                    assert gc[key] == oc[key], (metric, key)
                yidx, yc = oracle.search(t, q, m, cut, metric, w, arg)
                assert list(gidx) == list(yidx), metric
                for key in ("valid", "invalid", "after_lb", "after_glb", "matches"):
                    assert gc[key] == yc[key], (metric, key)
                eidx, edist, _ = full.exact(q, m, cut, metric, w, arg)
                xidx, xdist, _ = ShardedSearch.merge_exact([r.local_exact(q, m, cut, metric, w, arg) for r in ranks],
                                                           m, n, cut)
                assert list(xidx) == list(eidx) and np.array_equal(_bits(xdist), _bits(edist)), metric
                zidx, zdist, _ = oracle.exact(t, q, m, cut, metric, w, arg)
                assert list(xidx) == list(zidx) and np.array_equal(_bits(xdist), _bits(zdist)), metric
                pidx, pc = full.search(q, m, cut, metric, w, arg, exclude=excl)
                hidx, hc = ShardedSearch.merge_search(
                    [r.local_search(q, m, cut, metric, w, arg, exclude=excl) for r in ranks], m, n, cut)
                assert list(hidx) == list(pidx) and hc["invalid"] == pc["invalid"], metric
    finally:
        for e in engines.values():
            e.close()
