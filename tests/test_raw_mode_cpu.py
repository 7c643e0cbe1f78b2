"""Raw (non-normalised) mode of the oracle restatement, on the host.

The reference declares NormalizationMode::Raw (include/funcs.h:20-28) but
never consults it, so there is no reference output to pin; these checks
pin the restatement's raw mode by properties instead: the exact scan's
distances are the elastic distances of the raw query against the raw
windows, every window of finite points is a candidate (flat ones included)
and no window holding a NaN is, and the LB_IP -> GLB cascade is admissible
(search finds exactly the exact scan's matches)."""
import numpy as np
import pytest

from fsmeld_b200.synth import walk_with_structure

CASES = [("dtw", 0.0), ("erp", 0.4), ("edr", 1.0), ("lcss", 1.0), ("msm", 0.5)]


@pytest.fixture()
def raw_oracle(oracle):
    oracle.set_normalization("raw")
    yield oracle
    oracle.set_normalization("zscore")


@pytest.mark.parametrize("metric,arg", CASES)
def test_raw_exact_equals_direct_and_search(raw_oracle, metric, arg):
    o = raw_oracle
    m, w = 32, 3
    t = walk_with_structure(4000, m, seed=5, motifs=3, nan_fraction=3e-3, flat_runs=2, nan_spans=2)
    q = t[1000:1000 + m] + np.random.default_rng(1).normal(0.0, 0.3, m)
    idx, dist, _ = o.cutoff(t, q, m, 7, metric, w, arg)
    cut = float(dist[-1])
    x, xd, xc = o.exact(t, q, m, cut, metric, w, arg)
    direct = np.array([o.distance(metric, q, t[g:g + m], w, arg) for g in x])
    assert np.array_equal(direct.view(np.int64), np.asarray(xd).view(np.int64))
    s, sc = o.search(t, q, m, cut, metric, w, arg)
    assert list(s) == list(x)
    finite = np.array([np.isfinite(t[g:g + m]).all() for g in range(len(t) - m + 1)])
    assert xc["valid"] == int(finite.sum()) == sc["valid"]


def test_raw_flat_query_and_windows(raw_oracle):
    # a flat query cannot be z-normalised, but is a raw query; flat windows are candidates
    o = raw_oracle
    m, w = 16, 2
    t = np.concatenate([np.full(200, 3.0), np.cumsum(np.random.default_rng(2).normal(size=800))])
    q = np.full(m, 3.0)
    x, xd, xc = o.exact(t, q, m, 0.0, "dtw", w, 0.0)
    assert list(x) == list(range(0, 200 - m + 1))
    assert np.all(xd == 0.0)
    assert xc["valid"] == len(t) - m + 1
