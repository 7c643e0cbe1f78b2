"""The two benchmark configurations at their stated sizes against the
reference's own answers (needs a B200).

tests/golden/config_pins.json was made by tests/golden/make_config_pins.py
from the reference CLI (its own sources) and the reference's functions:

* c1: DTW, m=128, w=6, 2^20-point random walk; the reference's `cutoff
  k=10` ranking and threshold, `search` and `exact` at that threshold;
* c2: the five metrics at m=256, w=13 on the 2^24-point structured walk of
  the benchmark; per metric the k=50 cutoff (proved by the reference's
  `search`: at least 50 matches at the cutoff, fewer just below it), the
  match set at the cutoff and the top-50 ranking by (distance, index) with
  full-precision distances.

The targets are rebuilt from their seeds and checked by SHA-256.  Rankings,
thresholds, match sets and distances must be bit-identical; so must the
valid/invalid counters.  The LB_IP and GLB survivor counters are compared
where the target has no NaN (c1): on targets with NaN the reference sorts
envelope cores that contain NaN with an unspecified order, which changes its
per-segment LB_IP thresholds there (never a match set).
"""
import hashlib
import json
import os

import numpy as np
import pytest

from fsmeld_b200 import synth

pytestmark = pytest.mark.gpu

PINS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "config_pins.json")


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<f8").tobytes()).hexdigest()


def _hex(xs):
    return [float(x).hex() for x in xs]


@pytest.fixture(scope="module")
def pins():
    with open(PINS) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def api():
    from fsmeld_b200 import api as a
    a.lib()
    return a


def test_config1_vs_reference(api, pins):
    p = pins["c1"]
    t, q0, meta = synth.config1()
    assert _sha(t) == p["target_sha256"]
    q = np.array([float.fromhex(x) for x in p["query"]])
    assert np.array_equal(q, np.array([float("%.17g" % x) for x in q0]))
    m, w, metric, arg = p["m"], p["w"], p["metric"], p["arg"]
    with api.Engine(t) as e:
        idx, dist, cnt = e.cutoff(q, m, p["k"], metric, w, arg)
        assert list(idx) == p["cutoff"]["ranks"]
        assert _hex(dist) == p["cutoff"]["dists"]
        assert float(cnt["threshold"]).hex() == p["threshold"]
        assert cnt["valid"] == p["cutoff"]["kk1"]
        thr = float.fromhex(p["threshold"])
        sidx, sc = e.search(q, m, thr, metric, w, arg)
        assert list(sidx) == p["search"]["matches"]
        assert (sc["valid"], sc["invalid"], sc["after_lb"], sc["after_glb"]) == (
            p["search"]["kk1"], p["search"]["invalid"], p["search"]["kk2"], p["search"]["kk3"])
        eidx, edist, ec = e.exact(q, m, thr, metric, w, arg)
        assert list(eidx) == p["exact"]["matches"]
        order = sorted(range(len(eidx)), key=lambda i: (edist[i], eidx[i]))
        assert [int(eidx[i]) for i in order] == p["exact"]["by_distance"]
        assert _hex([edist[i] for i in order]) == p["exact"]["dists"]
        assert (ec["valid"], ec["invalid"]) == (p["exact"]["kk1"], p["exact"]["invalid"])


def test_config2_vs_reference(api, pins):
    p = pins["c2"]
    t, queries, meta = synth.config2()
    assert _sha(t) == p["target_sha256"]
    m, w = p["m"], p["w"]
    with api.Engine(t) as e:
        for metric, mp in p["metrics"].items():
            q = np.array([float.fromhex(x) for x in mp["query"]])
            assert np.array_equal(q, np.array([float("%.17g" % x) for x in queries[metric][0]]))
            arg = mp["arg"]
            idx, dist, cnt = e.cutoff(q, m, p["k"], metric, w, arg)
            assert list(idx) == mp["ranks"], metric
            assert _hex(dist) == mp["dists"], metric
            assert float(cnt["threshold"]).hex() == mp["cutoff"], metric
            cut = float.fromhex(mp["cutoff"])
            sidx, sc = e.search(q, m, cut, metric, w, arg)
            assert list(sidx) == mp["search"]["matches"], metric
            assert (sc["valid"], sc["invalid"]) == (mp["search"]["kk1"], mp["search"]["invalid"]), metric
            below = np.nextafter(cut, 0.0)
            bidx, bc = e.search(q, m, below, metric, w, arg)
            assert len(bidx) == mp["matches_below"] < p["k"], metric


@pytest.mark.parametrize("k", [10, 100])
def test_config4_shape_rankings_vs_oracle(api, oracle, k):
    # the top-k configuration's shape (DTW, m=512, w=26, walk with noise
    # bursts) on a 2^18-point target: GPU rankings (distance, index, ties
    # included) equal the oracle's, through both LB_IP forms of a batch
    from fsmeld_b200.synth import query_from, walk_with_bursts

    m, w = 512, 26
    t = walk_with_bursts(1 << 18, m, seed=44)
    rng = np.random.default_rng(4404)
    qs = [query_from(t, m, rng)[0] for _ in range(2)]
    want = [oracle.cutoff(t, q, m, k, "dtw", w, 0.0) for q in qs]
    with api.Engine(t) as e:
        for form in ("fft", "gemm"):
            e.set_lb_form(form)
            got = e.batch("cutoff", [dict(query=q, m=m, metric="dtw", w=w, arg=0.0, k=k) for q in qs])
            for g_, (oidx, odist, _) in zip(got, want):
                assert g_["status"] == 0
                assert list(g_["idx"]) == list(oidx), form
                assert _hex(g_["dist"]) == _hex(odist), form
