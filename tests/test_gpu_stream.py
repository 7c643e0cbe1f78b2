"""A target file streamed through the GPU in segment-aligned chunks (two
engines alternating, uploads from pinned memory) gives the results of the
oracle over the whole target and of one resident engine, bit for bit, for a
batch of queries of two lengths."""
import os
import tempfile

import numpy as np
import pytest

from fsmeld_b200.synth import query_from, walk_with_structure

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.asarray(a, dtype=np.float64).view(np.int64)


def test_streamed_equals_resident(oracle):
    from fsmeld_b200 import api
    from fsmeld_b200.stream import StreamingTarget, chunk_plan

    t = walk_with_structure(1 << 18, 96, seed=707, motifs=30, nan_fraction=1e-3, flat_runs=6, nan_spans=5)
    rng = np.random.default_rng(708)
    path = os.path.join(tempfile.mkdtemp(), "t.bin")
    t.astype("<f8").tofile(path)
    qs = []
    for i, (metric, arg) in enumerate([("dtw", 0.0), ("erp", 0.4), ("edr", 0.25), ("lcss", 0.25), ("msm", 0.5)]):
        m = 64 if i % 2 else 96
        q, _ = query_from(t, m, rng)
        qs.append(dict(query=q, m=m, metric=metric, w=5, arg=arg))
    for d in qs:
        _, dk, _ = oracle.cutoff(t, d["query"], d["m"], 12, d["metric"], d["w"], d["arg"])
        d["cutoff"] = float(dk[-1])
    orc = {"search": [oracle.search(t, d["query"], d["m"], d["cutoff"], d["metric"], d["w"], d["arg"]) for d in qs],
           "exact": [oracle.exact(t, d["query"], d["m"], d["cutoff"], d["metric"], d["w"], d["arg"]) for d in qs],
           "cutoff": [oracle.cutoff(t, d["query"], d["m"], 12, d["metric"], d["w"], d["arg"]) for d in qs]}
    with api.Engine(t) as full:
        want = {mode: full.batch(mode, [dict(d, k=12) if mode == "cutoff" else d for d in qs])
                for mode in ("search", "exact", "cutoff")}
    with StreamingTarget(path, max_points=40_000) as st:
        assert len(chunk_plan(len(t), 96, 40_000)) >= 6
        for mode in ("search", "exact", "cutoff"):
            got = st.batch(mode, [dict(d, k=12) if mode == "cutoff" else d for d in qs])
            for g, w_, o in zip(got, want[mode], orc[mode]):
                assert list(g["idx"]) == list(w_["idx"]) == list(o[0]), mode
                if mode != "search":
                    assert np.array_equal(_bits(g["dist"]), _bits(o[1])), mode
                else:
                    for key in ("valid", "invalid", "after_lb", "after_glb", "matches"):
                        assert g["counters"][key] == o[1][key], (mode, key)
                if mode != "search":
                    assert np.array_equal(_bits(g["dist"]), _bits(w_["dist"])), mode
                if mode == "search":
                    for key in ("valid", "invalid", "after_lb", "after_glb", "matches"):
                        assert g["counters"][key] == w_["counters"][key], (mode, key)
