"""Raw (non-normalised) mode on the CUDA path against the oracle's raw mode,
bit for bit (needs a B200): top-k rankings and distances, search match sets
and counters, exact matches and distances, for every metric; plus a flat
query (allowed in raw mode only)."""
import numpy as np
import pytest

from fsmeld_b200.synth import query_from, walk_with_structure

pytestmark = pytest.mark.gpu

METRIC_ARGS = [("dtw", 0.0), ("erp", 0.0), ("erp", 0.4), ("edr", 1.0), ("lcss", 1.0), ("msm", 0.5)]


def _bits(a):
    return np.asarray(a, dtype=np.float64).view(np.int64)


@pytest.fixture()
def raw_oracle(oracle):
    oracle.set_normalization("raw")
    yield oracle
    oracle.set_normalization("zscore")


def test_raw_mode_vs_oracle(raw_oracle):
    from fsmeld_b200 import api

    o = raw_oracle
    m, w = 64, 5
    t = walk_with_structure(1 << 16, m, seed=515, motifs=20, nan_fraction=2e-3, flat_runs=6, nan_spans=4)
    q, _ = query_from(t, m, np.random.default_rng(516), noise=0.5)
    with api.Engine(t) as e:
        e.set_normalization("raw")
        assert e.normalization == "raw"
        for metric, arg in METRIC_ARGS:
            gidx, gdist, gc = e.cutoff(q, m, 9, metric, w, arg)
            oidx, odist, oc = o.cutoff(t, q, m, 9, metric, w, arg)
            assert list(gidx) == list(oidx) and np.array_equal(_bits(gdist), _bits(odist)), metric
            cut = float(odist[-1])
            sidx, sc = e.search(q, m, cut, metric, w, arg)
            xidx, xc = o.search(t, q, m, cut, metric, w, arg)
            assert list(sidx) == list(xidx), metric
            for key in ("valid", "invalid", "after_lb", "after_glb", "matches"):
                assert sc[key] == xc[key], (metric, key)
            eidx, edist, ec = e.exact(q, m, cut, metric, w, arg)
            yidx, ydist, yc = o.exact(t, q, m, cut, metric, w, arg)
            assert list(eidx) == list(yidx) and np.array_equal(_bits(edist), _bits(ydist)), metric
            assert ec["valid"] == yc["valid"]
        # back to z-score on the same context
        e.set_normalization("zscore")
        o.set_normalization("zscore")
        gidx, gdist, _ = e.cutoff(q, m, 9, "dtw", w, 0.0)
        oidx, odist, _ = o.cutoff(t, q, m, 9, "dtw", w, 0.0)
        assert list(gidx) == list(oidx) and np.array_equal(_bits(gdist), _bits(odist))


def test_raw_flat_query(raw_oracle):
    from fsmeld_b200 import api

    o = raw_oracle
    m, w = 16, 2
    t = np.concatenate([np.full(200, 3.0), np.cumsum(np.random.default_rng(2).normal(size=3000))])
    q = np.full(m, 3.0)
    with api.Engine(t) as e:
        with pytest.raises(api.FsmeldError):
            e.exact(q, m, 0.0, "dtw", w, 0.0)  # z-score: a flat query is rejected
        e.set_normalization("raw")
        gidx, gdist, _ = e.exact(q, m, 0.5, "dtw", w, 0.0)
        oidx, odist, _ = o.exact(t, q, m, 0.5, "dtw", w, 0.0)
        assert list(gidx) == list(oidx) and np.array_equal(_bits(gdist), _bits(odist))
        assert list(range(0, 200 - m + 1)) == list(gidx[: 200 - m + 1])
