"""The serving loop on the CUDA path: a mix of search, cutoff and exact
requests of several lengths, metrics and radii against two resident targets,
submitted from three threads at once, must give exactly the answers of the
same requests run alone on the GPU, and those of the oracle (match lists and
distances bit for bit, counters)."""
import threading

import numpy as np
import pytest

from fsmeld_b200.synth import query_from, walk_with_structure

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.asarray(a, dtype=np.float64).view(np.int64)


def test_mix_equals_alone(oracle):
    from fsmeld_b200 import api
    from fsmeld_b200.serve import Server

    rng = np.random.default_rng(31)
    targets = {"a": walk_with_structure(1 << 16, 64, seed=32, motifs=15, nan_fraction=1e-3, flat_runs=4,
                                        nan_spans=3),
               "b": walk_with_structure(50_000, 96, seed=33, motifs=10, nan_fraction=0.0, flat_runs=2)}
    reqs = []
    for i in range(24):
        tname = "a" if i % 2 == 0 else "b"
        m = [48, 64, 96][i % 3]
        w = [2, 4, 7][(i // 3) % 3]
        metric, arg = [("dtw", 0.0), ("erp", 0.4), ("edr", 0.25), ("lcss", 0.25), ("msm", 0.5)][i % 5]
        q, _ = query_from(targets[tname], m, rng)
        mode = ["search", "cutoff", "exact"][i % 3]
        reqs.append((tname, mode, q, m, metric, w, arg))
    # cutoffs for search/exact: each query's k=8 distance from the oracle;
    # every request's answer from the oracle and from a plain engine alone
    alone, want = {}, {}
    with api.Engine(targets["a"]) as ea, api.Engine(targets["b"]) as eb:
        eng = {"a": ea, "b": eb}
        for j, (tn, mode, q, m, metric, w, arg) in enumerate(reqs):
            e, t = eng[tn], targets[tn]
            _, d8, _ = oracle.cutoff(t, q, m, 8, metric, w, arg)
            cut = float(d8[-1])
            if mode == "search":
                alone[j] = (cut, e.search(q, m, cut, metric, w, arg))
                want[j] = oracle.search(t, q, m, cut, metric, w, arg)
            elif mode == "exact":
                alone[j] = (cut, e.exact(q, m, cut, metric, w, arg))
                want[j] = oracle.exact(t, q, m, cut, metric, w, arg)
            else:
                alone[j] = (None, e.cutoff(q, m, 5, metric, w, arg))
                want[j] = oracle.cutoff(t, q, m, 5, metric, w, arg)
    with Server(device=0) as srv:
        for name, t in targets.items():
            srv.add_target(name, t)
        futs = {}
        lock = threading.Lock()

        def client(ids):
            for j in ids:
                tn, mode, q, m, metric, w, arg = reqs[j]
                cut = alone[j][0]
                f = (srv.submit(tn, mode, q, m, metric, w, arg, k=5) if mode == "cutoff"
                     else srv.submit(tn, mode, q, m, metric, w, arg, cutoff=cut))
                with lock:
                    futs[j] = f

        th = [threading.Thread(target=client, args=(list(range(c, len(reqs), 3)),)) for c in range(3)]
        for x in th:
            x.start()
        for x in th:
            x.join()
        for j, f in sorted(futs.items()):
            got = f.result(timeout=120)
            ref, orc = alone[j][1], want[j]
            assert list(got[0]) == list(ref[0]) == list(orc[0]), j
            if len(ref) == 3:
                assert np.array_equal(_bits(got[1]), _bits(ref[1])), j
                assert np.array_equal(_bits(got[1]), _bits(orc[1])), j
            for key in ("valid", "invalid", "after_lb", "after_glb", "matches"):
                assert got[-1][key] == ref[-1][key], (j, key)
            keys = ("valid", "invalid", "after_lb", "after_glb", "matches") if reqs[j][1] == "search" else ("valid",)
            for key in keys:
                assert got[-1][key] == orc[-1][key], (j, key)
