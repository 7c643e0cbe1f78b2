"""fsmeld_exact_noalloc: the exact scan for callers that cannot call cudaMalloc.

Some callers cannot allocate device memory (a serving loop whose memory belongs
to another allocator, or code that must not allocate while a request is in
flight).  This entry point takes device-resident inputs and outputs and keeps
its scratch in a static device array.  Checked here against the oracle's exact
scan and against the allocating entry point (fsmeld_exact) on the same
inputs, bit for bit, on two calls in a row; then an output buffer smaller
than the match count (the first entries and the full total), and the size
limits.  The file name sorts last so a run that stops at the first failure
has run every other test first; it also passes alone.
"""
import numpy as np
import pytest

from fsmeld_b200.synth import query_from, walk_with_structure

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.asarray(a, dtype=np.float64).view(np.int64)


def _target():
    m, n = 96, 200_000
    return m, n, walk_with_structure(n, m, seed=606, motifs=20, nan_fraction=1e-3, flat_runs=5, nan_spans=4)


def test_exact_noalloc_matches_oracle_and_exact_twice(oracle):
    import torch

    from fsmeld_b200 import api

    m, n, t = _target()
    w = 6
    rng = np.random.default_rng(607)
    d_target = torch.from_numpy(t).to("cuda:0")
    cap = 4096
    d_idx = torch.empty(cap, dtype=torch.int64, device="cuda:0")
    d_dist = torch.empty(cap, dtype=torch.float64, device="cuda:0")
    with api.Engine(t) as eng:
        for metric, arg in [("dtw", 0.0), ("msm", 0.5)]:
            q, _ = query_from(t, m, rng)
            _, odist, _ = oracle.cutoff(t, q, m, 25, metric, w, arg)
            cutoff = float(odist[-1])
            o_idx, o_dist, _ = oracle.exact(t, q, m, cutoff, metric, w, arg)
            ref_idx, ref_dist, _ = eng.exact(q, m, cutoff, metric, w, arg)
            assert np.array_equal(ref_idx, o_idx) and np.array_equal(_bits(ref_dist), _bits(o_dist)), metric
            for call in range(2):  # two calls in a row share the scratch array
                d_idx.fill_(-7)
                d_dist.fill_(float("nan"))
                count = api.exact_noalloc(d_target.data_ptr(), n, q, m, cutoff, metric, w, arg,
                                          d_idx.data_ptr(), d_dist.data_ptr(), cap)
                assert count == len(o_idx), (metric, call)
                got_idx = d_idx[:count].cpu().numpy()
                got_dist = d_dist[:count].cpu().numpy()
                assert np.array_equal(got_idx, o_idx), (metric, call)
                assert np.array_equal(_bits(got_dist), _bits(o_dist)), (metric, call)
                assert np.array_equal(got_idx, ref_idx) and np.array_equal(_bits(got_dist), _bits(ref_dist))


def test_exact_noalloc_truncates_at_capacity(oracle):
    import torch

    from fsmeld_b200 import api

    m, n, t = _target()
    w = 6
    q, _ = query_from(t, m, np.random.default_rng(611))
    _, odist, _ = oracle.cutoff(t, q, m, 40, "dtw", w, 0.0)
    cutoff = float(odist[-1])
    o_idx, o_dist, _ = oracle.exact(t, q, m, cutoff, "dtw", w, 0.0)
    assert len(o_idx) >= 40
    cap = 7
    d_target = torch.from_numpy(t).to("cuda:0")
    d_idx = torch.full((cap + 1,), -7, dtype=torch.int64, device="cuda:0")
    d_dist = torch.full((cap + 1,), float("nan"), dtype=torch.float64, device="cuda:0")
    count = api.exact_noalloc(d_target.data_ptr(), n, q, m, cutoff, "dtw", w, 0.0, d_idx.data_ptr(),
                              d_dist.data_ptr(), cap)
    assert count == len(o_idx)  # the full total, although only `cap` entries were written
    got_idx, got_dist = d_idx.cpu().numpy(), d_dist.cpu().numpy()
    assert np.array_equal(got_idx[:cap], o_idx[:cap])
    assert np.array_equal(_bits(got_dist[:cap]), _bits(o_dist[:cap]))
    assert got_idx[cap] == -7 and np.isnan(got_dist[cap])  # nothing past the capacity


def test_exact_noalloc_rejects_oversize():
    import torch

    from fsmeld_b200 import api

    m = 64
    n = api_max = 262_144 + m  # one window more than the limit
    d_target = torch.zeros(n, dtype=torch.float64, device="cuda:0")
    d_idx = torch.empty(16, dtype=torch.int64, device="cuda:0")
    d_dist = torch.empty(16, dtype=torch.float64, device="cuda:0")
    q = np.sin(np.arange(m) * 0.3)
    with pytest.raises(api.FsmeldError) as ei:
        api.exact_noalloc(d_target.data_ptr(), api_max, q, m, 1.0, "dtw", 3, 0.0, d_idx.data_ptr(),
                          d_dist.data_ptr(), 16)
    assert ei.value.status == api.E_ARG
    assert "FSMELD_NOALLOC_MAX_WINDOWS" in str(ei.value)
    # a band too wide for the shared-memory DP of this path (w <= 94 on a 227 KB device)
    m2, w2 = 400, 95
    q2 = np.sin(np.arange(m2) * 0.05)
    with pytest.raises(api.FsmeldError) as ei:
        api.exact_noalloc(d_target.data_ptr(), 4096, q2, m2, 1.0, "dtw", w2, 0.0, d_idx.data_ptr(),
                          d_dist.data_ptr(), 16)
    assert ei.value.status == api.E_ARG
    assert "too wide" in str(ei.value)
    # the largest accepted band still runs
    got = api.exact_noalloc(d_target.data_ptr(), 4096, q2, m2, 0.0, "dtw", 94, 0.0, d_idx.data_ptr(),
                            d_dist.data_ptr(), 16)
    assert got == 0  # an all-zero target has no valid window
