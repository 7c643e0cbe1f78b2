"""fsmeld_exact_noalloc: the exact scan for callers that cannot call cudaMalloc.

Some callers cannot allocate device memory (a serving loop whose memory belongs
to another allocator, or code that must not allocate while a request is in
flight).  This entry point takes device-resident inputs and outputs and keeps
its scratch in a static device array.  Checked here against the allocating
entry point (fsmeld_exact) on the same inputs, bit for bit, on two calls in a
row, plus the size limit.  The file name sorts last so a run that stops at the
first failure has run every other test first; it also passes alone.
"""
import numpy as np
import pytest

from fsmeld_b200.synth import query_from, walk_with_structure

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.asarray(a, dtype=np.float64).view(np.int64)


def test_exact_noalloc_matches_exact_twice():
    import torch

    from fsmeld_b200 import api

    m, w = 96, 6
    n = 200_000
    t = walk_with_structure(n, m, seed=606, motifs=20, nan_fraction=1e-3, flat_runs=5, nan_spans=4)
    rng = np.random.default_rng(607)
    d_target = torch.from_numpy(t).to("cuda:0")
    cap = 4096
    d_idx = torch.empty(cap, dtype=torch.int64, device="cuda:0")
    d_dist = torch.empty(cap, dtype=torch.float64, device="cuda:0")
    with api.Engine(t) as eng:
        for metric, arg in [("dtw", 0.0), ("msm", 0.5)]:
            q, _ = query_from(t, m, rng)
            kidx, kdist, _ = eng.cutoff(q, m, 25, metric, w, arg)
            cutoff = float(kdist[-1])
            ref_idx, ref_dist, _ = eng.exact(q, m, cutoff, metric, w, arg)
            for call in range(2):  # two calls in a row share the scratch array
                d_idx.fill_(-7)
                d_dist.fill_(float("nan"))
                count = api.exact_noalloc(d_target.data_ptr(), n, q, m, cutoff, metric, w, arg,
                                          d_idx.data_ptr(), d_dist.data_ptr(), cap)
                assert count == len(ref_idx), (metric, call)
                got_idx = d_idx[:count].cpu().numpy()
                got_dist = d_dist[:count].cpu().numpy()
                assert np.array_equal(got_idx, ref_idx), (metric, call)
                assert np.array_equal(_bits(got_dist), _bits(ref_dist)), (metric, call)


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
