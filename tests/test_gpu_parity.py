"""CUDA path vs the oracle and the reference's golden outputs (needs a B200).

Bars: match index sets, rankings, window statistics, envelopes, thresholds,
exact distances: bit-identical.  LB_IP values (FFT sliding inner products):
within 1e-9 absolute + 1e-12 relative of the oracle; the prune test's 1e-9
guard makes pruning decisions agree.
"""
import numpy as np
import pytest

from fsmeld_b200.synth import query_from, random_walk, walk_with_structure

pytestmark = pytest.mark.gpu

METRIC_ARGS = [("dtw", 0.0), ("erp", 0.0), ("erp", 0.4), ("edr", 0.25), ("lcss", 0.25), ("msm", 0.5)]


def bits_equal(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    if a.shape != b.shape:
        return False
    na, nb = np.isnan(a), np.isnan(b)
    return np.array_equal(na, nb) and np.array_equal(a[~na].view(np.int64), b[~nb].view(np.int64))


@pytest.fixture(scope="module")
def api():
    from fsmeld_b200 import api as a
    a.lib()
    return a


def _geom(m, n):
    sel = 1
    while sel < 8 * m:
        sel *= 2
    mk = min(sel, n)
    kml = mk - m + 1
    tsn = n - m + 1
    return mk, kml, tsn // kml, tsn % kml


def _segments(t, m):
    n = len(t)
    mk, kml, forsize, tail = _geom(m, n)
    segs = [t[s * kml: s * kml + mk] for s in range(forsize)]
    if tail:
        segs.append(t[n - mk:])
    return segs, mk, kml


@pytest.fixture(scope="module")
def structured():
    m, w = 64, 5
    t = walk_with_structure(1 << 16, m, seed=77, motifs=30, nan_fraction=2e-3, flat_runs=8, nan_spans=6)
    rng = np.random.default_rng(78)
    q, _ = query_from(t, m, rng)
    return t, q, m, w


def test_window_stats_bits(api, oracle, structured):
    t, q, m, w = structured
    segs, mk, kml = _segments(t, m)
    with api.Engine(t) as e:
        mu = e.inspect(q, m, "dtw", w, 0.0, 0).reshape(-1, kml)
        sg = e.inspect(q, m, "dtw", w, 0.0, 1).reshape(-1, kml)
    assert mu.shape[0] == len(segs)
    for s, ts in enumerate(segs):
        omu, osg = oracle.mvmean(ts, m)
        assert bits_equal(mu[s], omu), s
        assert bits_equal(sg[s], osg), s


def test_envelopes_bits(api, oracle, structured):
    t, q, m, w = structured
    segs, mk, kml = _segments(t, m)
    with api.Engine(t) as e:
        un = e.inspect(q, m, "dtw", w, 0.0, 2).reshape(-1, mk)
        ln = e.inspect(q, m, "dtw", w, 0.0, 3).reshape(-1, mk)
    for s, ts in enumerate(segs):
        omu, osg = oracle.mvmean(ts, m)
        mn, mx = oracle.min_max_window(omu, mk, m)
        smn, smx = oracle.min_max_window(osg, mk, m)
        L, U = oracle.lemire(ts, w)
        oun, oln = oracle.normalized(U, L, mx, mn, smx, smn)
        assert bits_equal(un[s], oun), s
        assert bits_equal(ln[s], oln), s


@pytest.mark.parametrize("metric,arg", METRIC_ARGS)
def test_thresholds_bits(api, oracle, structured, metric, arg):
    t, q, m, w = structured
    segs, mk, kml = _segments(t, m)
    qn = oracle.normalize_query(q)
    with api.Engine(t) as e:
        thr = e.inspect(q, m, metric, w, arg, 4).reshape(-1, 2)
        un = e.inspect(q, m, metric, w, arg, 2).reshape(-1, mk)
        ln = e.inspect(q, m, metric, w, arg, 3).reshape(-1, mk)
    bad = []
    for s in range(len(segs)):
        tl = oracle.find_t(0, metric, ln[s], qn, m, arg)
        tu = oracle.find_t(1, metric, un[s], qn, m, arg)
        if not (bits_equal([thr[s, 0], thr[s, 1]], [tl, tu])):
            bad.append((s, thr[s].tolist(), [tl, tu]))
    assert not bad, bad[:5]


@pytest.mark.parametrize("metric,arg", METRIC_ARGS)
def test_lbip_values(api, oracle, structured, metric, arg):
    t, q, m, w = structured
    segs, mk, kml = _segments(t, m)
    qn = oracle.normalize_query(q)
    with api.Engine(t) as e:
        z = e.inspect(q, m, metric, w, arg, 5).reshape(-1, kml)
        thr = e.inspect(q, m, metric, w, arg, 4).reshape(-1, 2)
        un = e.inspect(q, m, metric, w, arg, 2).reshape(-1, mk)
        ln = e.inspect(q, m, metric, w, arg, 3).reshape(-1, mk)
    for s, ts in enumerate(segs[::7]):
        s = s * 7
        omu, osg = oracle.mvmean(segs[s], m)
        valid = np.isfinite(osg) & (osg > 1e-12)
        hl = oracle.q_to_h(0, metric, qn, thr[s, 0], arg)
        hu = oracle.q_to_h(1, metric, qn, thr[s, 1], arg)
        gl = oracle.s_to_g(0, ln[s], thr[s, 0])
        gu = oracle.s_to_g(1, un[s], thr[s, 1])
        zl = oracle.sip(mk, m, hl, gl)
        zu = oracle.sip(mk, m, hu, gu)
        ref = np.zeros(kml)
        for j in range(kml):
            a, b = zl[m - 1 + j], zu[m - 1 + j]
            if metric in ("dtw", "erp"):
                ref[j] = np.sqrt(max(0.0, a + b))
            elif metric == "lcss":
                ref[j] = max(0.0, (a + b) / m)
            else:
                ref[j] = a + b
        got = z[s]
        sel = valid.copy()
        if s == len(segs) - 1:
            _, _, _, tail = _geom(m, len(t))
            if tail:
                sel[: kml - tail] = False
        assert np.all(np.isnan(got[~valid & sel]))
        g, r = got[sel], ref[sel]
        if metric in ("dtw", "erp"):
            # compare before the square root: sqrt turns 1e-14 FFT noise around a
            # zero sum into 1e-7 (the prune test carries a guard for exactly this)
            g, r = g * g, r * r
        diff = np.abs(g - r)
        assert np.all(diff <= 1e-9 + 1e-12 * np.abs(r)), (s, float(diff.max()))


@pytest.mark.parametrize("metric,arg", METRIC_ARGS)
def test_cutoff_search_exact_vs_oracle(api, oracle, structured, metric, arg):
    t, q, m, w = structured
    k = 15
    with api.Engine(t) as e:
        gidx, gdist, gc = e.cutoff(q, m, k, metric, w, arg)
        oidx, odist, oc = oracle.cutoff(t, q, m, k, metric, w, arg)
        assert list(gidx) == list(oidx)
        assert bits_equal(gdist, odist)
        thr = float(odist[-1])
        sidx, sc = e.search(q, m, thr, metric, w, arg)
        oidx2, osc = oracle.search(t, q, m, thr, metric, w, arg)
        assert list(sidx) == list(oidx2)
        assert sc["valid"] == osc["valid"] and sc["invalid"] == osc["invalid"]
        assert sc["after_glb"] == osc["after_glb"]
        assert sc["after_lb"] == osc["after_lb"]
        eidx, edist, ec = e.exact(q, m, thr, metric, w, arg)
        xidx, xdist, xc = oracle.exact(t, q, m, thr, metric, w, arg)
        assert list(eidx) == list(xidx)
        assert bits_equal(edist, xdist)
        assert ec["valid"] == xc["valid"]
        assert set(sidx) == set(eidx)


def test_golden_cli_cases(api, golden_cli):
    z, meta = golden_cli
    engines = {}
    try:
        for case in meta:
            name = case["name"]
            if name not in engines:
                engines[name] = api.Engine(z[name + "_target"])
            e = engines[name]
            q = z[name + "_query"]
            m, w, k, metric, arg = case["m"], case["w"], case["k"], case["metric"], case["arg"]
            t = z[name + "_target"]
            idx, dist, cnt = e.cutoff(q, m, k, metric, w, arg)
            assert list(idx) == case["cutoff"]["ranks"], (name, metric)
            assert float(cnt["threshold"]) == float(case["cutoff"]["threshold"])
            assert cnt["valid"] == case["cutoff"]["kk1"]
            thr = float(case["cutoff"]["threshold"])
            sidx, sc = e.search(q, m, thr, metric, w, arg)
            assert list(sidx) == case["search"]["matches"], (name, metric)
            assert sc["valid"] == case["search"]["kk1"] and sc["invalid"] == case["search"]["invalid"]
            if not np.isnan(t).any():
                assert (sc["after_lb"], sc["after_glb"]) == (case["search"]["kk2"], case["search"]["kk3"])
            eidx, edist, ec = e.exact(q, m, thr, metric, w, arg)
            assert list(eidx) == case["exact"]["matches"]
            assert ["%f" % d for d in edist] == case["exact"]["dists"]
            xidx, xc = e.search(q, m, thr, metric, w, arg, exclude=tuple(case["exclusion"]))
            assert list(xidx) == case["search_excl"]["matches"]
            assert xc["invalid"] == case["search_excl"]["invalid"]
    finally:
        for e in engines.values():
            e.close()


def test_short_target_and_no_tail(api, oracle):
    # target shorter than one macro segment (m_k = n) and a target whose
    # windows fill whole segments (no tail)
    rng = np.random.default_rng(5)
    for n, m, w in [(300, 40, 4), (1024 + 63, 64, 3), (130, 64, 10)]:
        t = random_walk(n, int(rng.integers(1 << 30)))
        q, _ = query_from(t, m, rng)
        with api.Engine(t) as e:
            for metric, arg in METRIC_ARGS:
                gidx, gdist, _ = e.cutoff(q, m, 3, metric, w, arg)
                oidx, odist, _ = oracle.cutoff(t, q, m, 3, metric, w, arg)
                assert list(gidx) == list(oidx) and bits_equal(gdist, odist), (n, metric)
                sidx, _ = e.search(q, m, float(odist[-1]) * 1.5, metric, w, arg)
                oidx2, _ = oracle.search(t, q, m, float(odist[-1]) * 1.5, metric, w, arg)
                assert list(sidx) == list(oidx2)


def test_errors(api):
    t = random_walk(1000, 3)
    with api.Engine(t) as e:
        q = t[10:42].copy()
        with pytest.raises(api.FsmeldError) as ei:
            e.cutoff(q, 32, 10 ** 6, "dtw", 3, 0.0)
        assert ei.value.status == api.E_ARG
        with pytest.raises(api.FsmeldError):
            e.search(np.ones(32), 32, 1.0, "dtw", 3, 0.0)  # flat query cannot be normalised
        with pytest.raises(api.FsmeldError):
            e.search(q, 32, 1.0, "dtw", 32, 0.0)  # w >= m
        with pytest.raises(api.FsmeldError):
            e.search(q, 32, 1.0, "msm", 3, -1.0)
        with pytest.raises(api.FsmeldError):
            e.search(q, 32, 1.0, "dtw", 3, 0.0, exclude=(5, 5))
    # all windows excluded -> fewer than k candidates
    with api.Engine(t) as e:
        with pytest.raises(api.FsmeldError) as ei:
            e.cutoff(q, 32, 5, "dtw", 3, 0.0, exclude=(0, 2000))
        assert ei.value.status == api.E_FEWER_K


def _znorm_max(q):
    q = np.asarray(q, dtype=np.float64)
    return float(np.max(np.abs((q - q.mean()) / q.std())))


def _all_distances(api, oracle, t, q, m, w, metric, arg):
    with api.Engine(t) as e:
        gidx, gdist, gc = e.exact(q, m, 1e300, metric, w, arg)
    oidx, odist, oc = oracle.exact(t, q, m, 1e300, metric, w, arg)
    assert len(oidx) == oc["valid"]  # every valid window is reported
    assert list(gidx) == list(oidx), metric
    assert bits_equal(gdist, odist), metric
    assert gc["valid"] == oc["valid"]


@pytest.mark.parametrize("metric,arg", METRIC_ARGS)
def test_all_window_distances_bits(api, oracle, structured, metric, arg):
    # the full distance profile (every valid window), through the DP's fast mode
    t, q, m, w = structured
    _all_distances(api, oracle, t, q, m, w, metric, arg)


@pytest.mark.parametrize("metric", ["erp", "msm"])
@pytest.mark.parametrize("margin", [1.5, -1e9])
def test_dp_exact_boundary_mode(api, oracle, structured, metric, margin):
    # An ERP gap value g or MSM cost c near sqrt(1e17 / (2m+2)) makes the DP's
    # fast-mode limit on candidate points small (margin 1.5: lanes whose
    # candidate has a point above ~1.5 restart in the exact mode while the
    # others stay fast) or negative (the whole query runs in the exact mode).
    # Cell values reach ~1e16 and column 0 of ERP/MSM takes the reference's
    # column formula; every distance must still equal the oracle's bits.
    t, q, m, w = structured
    big = np.sqrt(1e17 / (2.0 * m + 2.0)) - _znorm_max(q[:m]) - 2.0 - margin
    _all_distances(api, oracle, t, q, m, w, metric, float(big))


def test_dp_forced_exact_mode(api, oracle, structured, monkeypatch):
    # FSMELD_DP_EXACT=1 runs every candidate in the exact boundary mode; the
    # results are the same as the fast mode's
    t, q, m, w = structured
    monkeypatch.setenv("FSMELD_DP_EXACT", "1")
    for metric, arg in METRIC_ARGS:
        _all_distances(api, oracle, t, q, m, w, metric, arg)
        with api.Engine(t) as e:
            gidx, gdist, _ = e.cutoff(q, m, 9, metric, w, arg)
        oidx, odist, _ = oracle.cutoff(t, q, m, 9, metric, w, arg)
        assert list(gidx) == list(oidx) and bits_equal(gdist, odist), metric


@pytest.mark.parametrize("m,w", [(1025, 10), (777, 0)])
def test_long_odd_queries_vs_oracle(api, oracle, m, w):
    # long queries (m_k = 16384 / 8192): thresholds, envelopes and LB_IP run
    # from per-block scratch in global memory; odd m gives odd-sized layouts
    t = walk_with_structure(1 << 17, m, seed=1000 + m, motifs=8, nan_fraction=1e-3, flat_runs=2, nan_spans=2)
    q, _ = query_from(t, m, np.random.default_rng(m))
    with api.Engine(t) as e:
        for metric, arg in [("dtw", 0.0), ("erp", 0.4), ("lcss", 0.25)]:
            gidx, gdist, _ = e.cutoff(q, m, 5, metric, w, arg)
            oidx, odist, _ = oracle.cutoff(t, q, m, 5, metric, w, arg)
            assert list(gidx) == list(oidx) and bits_equal(gdist, odist), metric
            cut = float(odist[-1])
            sidx, sc = e.search(q, m, cut, metric, w, arg)
            xidx, xc = oracle.search(t, q, m, cut, metric, w, arg)
            assert list(sidx) == list(xidx), metric
            assert sc["valid"] == xc["valid"]


def test_cutoff_k_larger_than_segments(api, oracle):
    # k far above the number of macro segments: several seeds per segment
    m, w = 64, 4
    t = walk_with_structure(4000, m, seed=4242, motifs=3, nan_fraction=0.0, flat_runs=1)
    q, _ = query_from(t, m, np.random.default_rng(4243))
    with api.Engine(t) as e:
        for metric, arg in [("dtw", 0.0), ("edr", 0.25), ("msm", 0.5)]:
            for k in (40, 200):
                gidx, gdist, _ = e.cutoff(q, m, k, metric, w, arg)
                oidx, odist, _ = oracle.cutoff(t, q, m, k, metric, w, arg)
                assert list(gidx) == list(oidx) and bits_equal(gdist, odist), (metric, k)


@pytest.mark.parametrize("scale", [1.0, 1e-5, 1e140])
def test_division_paths_vs_oracle(api, oracle, scale):
    # candidate z-normalisation divides by the window's sigma through its
    # reciprocal (reciprocal, two FMA corrections) unless the sigma or the
    # quotient lies outside [2^-450, 2^450]: an integer-valued walk has points
    # equal to their window mean (zero dividends), and at scale 1e140 every
    # sigma is past 2^450 so every division takes the direct path
    rng = np.random.default_rng(17)
    m, w = 64, 4
    t = np.cumsum(rng.integers(-2, 3, 1 << 14)).astype(np.float64) * scale
    q, _ = query_from(t, m, np.random.default_rng(5))
    with api.Engine(t) as e:
        for metric, arg in [("dtw", 0.0), ("erp", 0.3), ("lcss", 0.25), ("msm", 0.5)]:
            gidx, gdist, _ = e.exact(q, m, 1e300, metric, w, arg)
            oidx, odist, _ = oracle.exact(t, q, m, 1e300, metric, w, arg)
            assert list(gidx) == list(oidx) and bits_equal(gdist, odist), metric
            kidx, kdist, _ = oracle.cutoff(t, q, m, 20, metric, w, arg)
            cut = float(kdist[-1])
            sidx, sc = e.search(q, m, cut, metric, w, arg)
            xidx, xc = oracle.search(t, q, m, cut, metric, w, arg)
            assert list(sidx) == list(xidx), metric
            assert (sc["after_lb"], sc["after_glb"]) == (xc["after_lb"], xc["after_glb"]), metric
