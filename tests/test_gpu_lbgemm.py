"""The tensor-core LB_IP (one tcgen05 BF16x3 product for a group of queries
of equal (m, w) and metric, FP32 accumulation, bounds lowered by a
rounding-error margin) against FP64 and the oracle (needs a B200).

* the bound of every window is a true lower bound of the FP64 LB_IP at the
  same thresholds, and within twice the stated margins of it (the error of
  the product against FP64 is reported per case);
* batched searches through it return the oracle's match sets and valid
  counters for every metric (the exact DP decides every match).
"""
import numpy as np
import pytest

from fsmeld_b200.synth import query_from, walk_with_structure

pytestmark = pytest.mark.gpu

METRIC_ARGS = [("dtw", 0.0), ("erp", 0.4), ("edr", 0.25), ("lcss", 0.25), ("msm", 0.5)]


@pytest.fixture(scope="module")
def target():
    m, w = 96, 6
    t = walk_with_structure(1 << 16, m, seed=808, motifs=20, nan_fraction=1e-3, flat_runs=4, nan_spans=3)
    return t, m, w


def _segments(n, m):
    mk = 1
    while mk < 8 * m:
        mk *= 2
    mk = min(mk, n)
    kml = mk - m + 1
    tsn = n - m + 1
    forsize, tail = tsn // kml, tsn % kml
    return mk, kml, forsize, tail


@pytest.mark.parametrize("metric,arg", METRIC_ARGS)
def test_gemm_bound_below_fp64_within_margin(oracle, target, metric, arg):
    from fsmeld_b200 import api

    t, m, w = target
    q, _ = query_from(t, m, np.random.default_rng(809))
    n = len(t)
    mk, kml, forsize, tail = _segments(n, m)
    S = forsize + (1 if tail else 0)
    with api.Engine(t) as e:
        lb = e.inspect(q, m, metric, w, arg, 6).reshape(S, kml)
        tl, tu, ml, mu = e.inspect(q, m, metric, w, arg, 7)
        Un = e.inspect(q, m, metric, w, arg, 2).reshape(S, mk)
        Ln = e.inspect(q, m, metric, w, arg, 3).reshape(S, mk)
    qn = oracle.normalize_query(q)
    hl = oracle.q_to_h(0, metric, qn, tl, arg)
    hu = oracle.q_to_h(1, metric, qn, tu, arg)
    worst = 0.0
    checked = 0
    for s in range(S):
        gl = (Ln[s] >= tl).astype(np.float64)
        gu = (Un[s] <= tu).astype(np.float64)
        # exact-enough FP64 sliding inner products (sums of at most m terms)
        zl = np.array([np.dot(hl, gl[j:j + m]) for j in range(kml)])
        zu = np.array([np.dot(hu, gu[j:j + m]) for j in range(kml)])
        ok = ~np.isnan(lb[s])
        zz = zl + zu
        if metric in ("dtw", "erp"):
            lb2 = lb[s][ok] ** 2
        elif metric == "lcss":
            lb2 = lb[s][ok] * m
        else:
            lb2 = lb[s][ok]
        exact = zz[ok]
        # a lower bound (up to the FP64 rounding of this check) ...
        assert np.all(lb2 <= exact * (1 + 1e-12) + 1e-12), (metric, s)
        # ... within twice the margins of the FP64 value
        slack = 2.0 * (ml + mu) + 1e-9 * (1.0 + exact)
        assert np.all(exact - lb2 <= slack), (metric, s, float(np.max(exact - lb2)), ml, mu)
        if exact.size:
            worst = max(worst, float(np.max(exact - lb2)))
        checked += int(ok.sum())
    assert checked > 0
    print(f"{metric}: max FP64 - GEMM bound (squared domain) {worst:.3e}, margins {ml:.3e} + {mu:.3e}")


def test_gemm_batched_search_equals_oracle(oracle, target):
    from fsmeld_b200 import api

    t, m, w = target
    rng = np.random.default_rng(810)
    batch = []
    for metric, arg in METRIC_ARGS:
        for _ in range(3):
            q, _ = query_from(t, m, rng)
            _, d, _ = oracle.cutoff(t, q, m, 6, metric, w, arg)
            batch.append(dict(query=q, m=m, metric=metric, w=w, arg=arg, cutoff=float(d[-1])))
    batch[1]["exclude"] = (20_000, 20_400)
    with api.Engine(t) as e:
        e.set_lb_form("gemm")
        got = e.batch("search", batch)
        e.set_lb_form("fft")
        fft = e.batch("search", batch)
    for d, g_, f_ in zip(batch, got, fft):
        ex = d.get("exclude", (-1, -1))
        oidx, oc = oracle.search(t, d["query"], m, d["cutoff"], d["metric"], w, d["arg"], excl=ex)
        assert g_["status"] == 0
        assert list(g_["idx"]) == list(oidx) == list(f_["idx"]), d["metric"]
        assert g_["counters"]["valid"] == oc["valid"] == f_["counters"]["valid"]
        assert g_["counters"]["matches"] == oc["matches"]


def test_gemm_batched_topk_equals_oracle(oracle, target):
    from fsmeld_b200 import api

    t, m, w = target
    rng = np.random.default_rng(811)
    batch = []
    for metric, arg in [("dtw", 0.0), ("msm", 0.5), ("lcss", 0.25)]:
        for _ in range(3):
            q, _ = query_from(t, m, rng)
            batch.append(dict(query=q, m=m, metric=metric, w=w, arg=arg, k=7))
    with api.Engine(t) as e:
        e.set_lb_form("gemm")
        got = e.batch("cutoff", batch)
    for d, g_ in zip(batch, got):
        oidx, odist, _ = oracle.cutoff(t, d["query"], m, 7, d["metric"], w, d["arg"])
        assert g_["status"] == 0
        assert list(g_["idx"]) == list(oidx), d["metric"]
        assert np.array_equal(np.asarray(g_["dist"]).view(np.int64), np.asarray(odist).view(np.int64))
