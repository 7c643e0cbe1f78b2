"""Streaming a target file through the device in segment-aligned chunks
(fsmeld_b200.stream), on the host: chunk plans cover every window once with
chunks no longer than the budget, and the merged search / exact / cutoff
results over a file streamed in many chunks equal one oracle run over the
whole target, bit for bit, with summed counters."""
import os
import tempfile

import numpy as np
import pytest

from fsmeld_b200.stream import StreamingTarget, chunk_plan
from fsmeld_b200.synth import query_from, walk_with_structure


@pytest.mark.parametrize("n,m,cap", [(50_000, 64, 4000), (50_000, 64, 30_000), (9000, 100, 2000),
                                     (1 << 15, 40, 1 << 15)])
def test_chunk_plan(n, m, cap):
    plan = chunk_plan(n, m, cap)
    tsn = n - m + 1
    prev = 0
    for sh in plan:
        assert sh.start == prev
        prev = sh.start + (sh.stop - sh.start) - m + 1
        assert sh.stop - sh.start <= max(cap, plan[-1].stop - plan[-1].start)
    assert prev == tsn
    if len(plan) > 1:
        assert all(sh.stop - sh.start <= cap for sh in plan)


def _oracle_runner(o):
    def run(arr, mode, specs):
        out = []
        for s in specs:
            args = (arr, s["query"], s["m"])
            if mode == "search":
                idx, cnt = o.search(arr, s["query"], s["m"], s["cutoff"], s["metric"], s["w"], s["arg"],
                                    excl=s["exclude"])
                out.append({"status": 0, "idx": idx, "dist": np.zeros(0), "count": len(idx), "counters": cnt})
            elif mode == "exact":
                idx, dist, cnt = o.exact(arr, s["query"], s["m"], s["cutoff"], s["metric"], s["w"], s["arg"],
                                         excl=s["exclude"])
                out.append({"status": 0, "idx": idx, "dist": dist, "count": len(idx), "counters": cnt})
            else:
                try:
                    idx, dist, cnt = o.cutoff(arr, s["query"], s["m"], s["k"], s["metric"], s["w"], s["arg"],
                                              excl=s["exclude"])
                    out.append({"status": 0, "idx": idx, "dist": dist, "count": len(idx), "counters": cnt})
                except ValueError:
                    out.append({"status": -5, "idx": np.zeros(0, np.int64), "dist": np.zeros(0), "count": 0,
                                "counters": {}})
            del args
        return out
    return run


def _bits(a):
    return np.asarray(a, dtype=np.float64).view(np.int64)


def test_streamed_file_equals_whole_target(oracle):
    m, w = 64, 5
    t = walk_with_structure(40_000, m, seed=808, motifs=8, nan_fraction=2e-3, flat_runs=3, nan_spans=3)
    rng = np.random.default_rng(809)
    d = tempfile.mkdtemp()
    path = os.path.join(d, "t.bin")
    t.astype("<f8").tofile(path)
    st = StreamingTarget(path, max_points=3500, chunk_runner=_oracle_runner(oracle))
    assert len(chunk_plan(len(t), m, 3500)) > 5
    excl = (12_000, 12_000 + 4 * m)
    for metric, arg in [("dtw", 0.0), ("erp", 0.4), ("lcss", 0.25), ("msm", 0.5)]:
        q, _ = query_from(t, m, rng)
        fidx, fdist, _ = oracle.cutoff(t, q, m, 30, metric, w, arg)
        sidx, sdist, _ = st.cutoff(q, m, 30, metric, w, arg)
        assert list(sidx) == list(fidx) and np.array_equal(_bits(sdist), _bits(fdist)), metric
        cut = float(fdist[-1])
        oidx, oc = oracle.search(t, q, m, cut, metric, w, arg)
        gidx, gc = st.search(q, m, cut, metric, w, arg)
        assert list(gidx) == list(oidx), metric
        for key in ("valid", "invalid", "after_lb", "after_glb", "matches", "segments", "tail"):
            assert gc[key] == oc[key], (metric, key)
        eidx, edist, _ = oracle.exact(t, q, m, cut, metric, w, arg)
        xidx, xdist, _ = st.exact(q, m, cut, metric, w, arg)
        assert list(xidx) == list(eidx) and np.array_equal(_bits(xdist), _bits(edist)), metric
        pidx, _ = oracle.search(t, q, m, cut, metric, w, arg, excl=excl)
        hidx, _ = st.search(q, m, cut, metric, w, arg, exclude=excl)
        assert list(hidx) == list(pidx), metric
