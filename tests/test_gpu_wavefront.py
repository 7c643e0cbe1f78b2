"""The wide-band exact DP (one warp per candidate, anti-diagonal wavefront,
k_dpw) against the oracle, bit for bit (needs a B200).

Wide bands take this kernel automatically (the lane-per-candidate DP's band
and ring no longer fit shared memory); FSMELD_DP_FORM=wave forces it for
every band it supports, so the ordinary fixture also runs through it.
"""
import numpy as np
import pytest

from fsmeld_b200.synth import query_from, walk_with_structure

pytestmark = pytest.mark.gpu

METRIC_ARGS = [("dtw", 0.0), ("erp", 0.0), ("erp", 0.4), ("edr", 0.25), ("lcss", 0.25), ("msm", 0.5)]


def bits_equal(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return a.shape == b.shape and np.array_equal(a.view(np.int64), b.view(np.int64))


_ORACLE_CACHE = {}


def _cached(key, fn):
    # the oracle's answers do not depend on the DP form under test
    if key not in _ORACLE_CACHE:
        _ORACLE_CACHE[key] = fn()
    return _ORACLE_CACHE[key]


@pytest.fixture(scope="module")
def api():
    from fsmeld_b200 import api as a
    a.lib()
    return a


@pytest.mark.parametrize("form", ["auto", "wave"])
@pytest.mark.parametrize("m,w,extra", [(1850, 138, 400), (1025, 51, 1500), (300, 255, 900)])
def test_wide_band_all_distances(api, oracle, monkeypatch, form, m, w, extra):
    # every valid window's distance (the exact scan at an unbounded cutoff)
    monkeypatch.setenv("FSMELD_DP_FORM", form)
    t = walk_with_structure(2 * m + extra, m, seed=3000 + m, motifs=2, nan_fraction=0.0, flat_runs=0)
    q, _ = query_from(t, m, np.random.default_rng(3001 + m))
    with api.Engine(t) as e:
        for metric, arg in METRIC_ARGS:
            gidx, gdist, gc = e.exact(q, m, 1e300, metric, w, arg)
            oidx, odist, oc = _cached(("all", m, w, metric, arg),
                                      lambda: oracle.exact(t, q, m, 1e300, metric, w, arg))
            assert len(oidx) == oc["valid"] == gc["valid"]
            assert list(gidx) == list(oidx), metric
            assert bits_equal(gdist, odist), metric


@pytest.mark.parametrize("form", ["auto", "wave"])
@pytest.mark.parametrize("m,w", [(1025, 51), (700, 120)])
def test_wide_band_cutoff_search(api, oracle, monkeypatch, form, m, w):
    # top-k and search through LB_IP, GLB and the exact DP with its cascading
    # abandon bound (the wavefront for wide bands, or forced)
    monkeypatch.setenv("FSMELD_DP_FORM", form)
    t = walk_with_structure(1 << 16, m, seed=4000 + m, motifs=8, nan_fraction=1e-3, flat_runs=2, nan_spans=2)
    q, _ = query_from(t, m, np.random.default_rng(4001 + m))
    with api.Engine(t) as e:
        for metric, arg in METRIC_ARGS:
            gidx, gdist, _ = e.cutoff(q, m, 6, metric, w, arg)
            oidx, odist, _ = _cached(("cut", m, w, metric, arg), lambda: oracle.cutoff(t, q, m, 6, metric, w, arg))
            assert list(gidx) == list(oidx) and bits_equal(gdist, odist), metric
            cut = float(odist[-1])
            sidx, sc = e.search(q, m, cut, metric, w, arg)
            xidx, xc = _cached(("search", m, w, metric, arg), lambda: oracle.search(t, q, m, cut, metric, w, arg))
            assert list(sidx) == list(xidx), metric
            assert (sc["valid"], sc["after_lb"], sc["after_glb"]) == (xc["valid"], xc["after_lb"], xc["after_glb"])
            # the exact scan (every window through the DP) finds the same set;
            # the distances of the top-k among them equal the oracle's
            eidx, edist, _ = e.exact(q, m, cut, metric, w, arg)
            assert list(eidx) == list(xidx), metric
            pos = {int(g): k for k, g in enumerate(eidx)}
            assert bits_equal([edist[pos[int(g)]] for g in oidx], odist), metric


def test_forced_wavefront_narrow_band(api, oracle, monkeypatch):
    # FSMELD_DP_FORM=wave: the wavefront for a narrow band (one 64-offset
    # chunk), through exact, top-k and search
    monkeypatch.setenv("FSMELD_DP_FORM", "wave")
    m, w = 64, 5
    t = walk_with_structure(1 << 16, m, seed=77, motifs=30, nan_fraction=2e-3, flat_runs=8, nan_spans=6)
    q, _ = query_from(t, m, np.random.default_rng(78))
    with api.Engine(t) as e:
        for metric, arg in METRIC_ARGS:
            gidx, gdist, _ = e.exact(q, m, 1e300, metric, w, arg)
            oidx, odist, _ = oracle.exact(t, q, m, 1e300, metric, w, arg)
            assert list(gidx) == list(oidx) and bits_equal(gdist, odist), metric
            kidx, kdist, _ = e.cutoff(q, m, 9, metric, w, arg)
            pidx, pdist, _ = oracle.cutoff(t, q, m, 9, metric, w, arg)
            assert list(kidx) == list(pidx) and bits_equal(kdist, pdist), metric
            sidx, _ = e.search(q, m, float(pdist[-1]), metric, w, arg)
            xidx, _ = oracle.search(t, q, m, float(pdist[-1]), metric, w, arg)
            assert list(sidx) == list(xidx), metric
