"""Pin the two benchmark configurations at their stated sizes against the
reference itself.

  c1: DTW, m=128, w=6, 2^20-point random walk (synth.config1); the
      reference's `cutoff k=10`, then `search` and `exact` at that threshold.
  c2: the five metrics at m=256, w=13 on the 2^24-point structured walk
      (synth.config2, the bench workload); for each metric the reference's
      `search` at the workload cutoff and at the next double below it.  At
      least k=50 matches at the cutoff and fewer than 50 just below it prove
      the cutoff is the reference's k=50 exact distance.

Match distances are full-precision values from the reference's own
functions (libfsmeld_ref.so: its mvmean over the window's macro segment and
its elastic distance), so rankings can be compared bit for bit; the CLI
prints distances with six decimals only (src/fsmeld.cpp:1219-1221).

Output: config_pins.json (match lists, counters, distances as float.hex).
The targets are regenerated from their seeds; their SHA-256 is recorded so a
test can check it rebuilt the same input.

Run from the repository root with the reference build present (oracle/_ref):
    python tests/golden/make_config_pins.py            # c1 and c2 (minutes)
"""
from __future__ import annotations

import concurrent.futures as cf
import hashlib
import json
import math
import os
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

from fsmeld_b200 import synth  # noqa: E402
from make_golden import parse_cli  # noqa: E402
from oracle import oracle as orc  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "config_pins.json")
# the workload's k=50 cutoffs of the five c2 queries (bench.py CUTOFFS)
C2_CUTOFFS = {"dtw": 2.80906383446946, "erp": 5.138604886191949, "edr": 48.0, "lcss": 0.265625,
              "msm": 74.7957914893858}
C2_K = 50


def sha256(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<f8").tobytes()).hexdigest()


def geometry(n, m):
    mk = 1
    while mk < 8 * m:
        mk *= 2
    mk = min(mk, n)
    kml = mk - m + 1
    tsn = n - m + 1
    forsize = tsn // kml
    tail = tsn % kml
    return mk, kml, forsize, kml - tail


def window_distance(ref, t, qn, m, g, metric, w, arg):
    """The reference's distance of window g, from its own mvmean over the
    macro segment that holds g (src/fsmeld.cpp:811-851) and its elastic
    distance (src/ElasticMeasures.cpp)."""
    n = len(t)
    mk, kml, forsize, tail_lo = geometry(n, m)
    q = g // kml
    if q < forsize:
        off, j = q * kml, g - q * kml
    else:
        off, j = n - mk, tail_lo + (g - forsize * kml)
    seg = t[off:off + mk]
    mu, si = ref.mvmean(seg, m)
    cand = (seg[j:j + m] - mu[j]) / si[j]
    return ref.distance(metric, qn, cand, w, arg)


def ranking(ref, t, q, m, idx, metric, w, arg):
    qn = orc.Oracle("oracle").normalize_query(q)
    d = [window_distance(ref, t, qn, m, int(g), metric, w, arg) for g in idx]
    order = sorted(range(len(idx)), key=lambda i: (d[i], int(idx[i])))
    return [int(idx[i]) for i in order], [float(d[i]).hex() for i in order]


def run(args, tmp):
    env = dict(os.environ, FSMELD_RESULTS_CSV=os.path.join(tmp, f"r{os.getpid()}_{time.time_ns()}.csv"))
    t0 = time.time()
    rc, out, err = orc.run_reference_cli(args, cwd=tmp, env=env)
    if rc != 0:
        raise RuntimeError(f"reference CLI failed: {args}: {err}")
    return out, time.time() - t0


def config1(ref, tmp):
    t, q, meta = synth.config1()
    m, w, metric, arg = meta["m"], meta["w"], meta["metric"], meta["arg"]
    tp, qp = os.path.join(tmp, "c1.bin"), os.path.join(tmp, "c1.txt")
    t.astype("<f8").tofile(tp)
    np.savetxt(qp, q, fmt="%.17g")
    q = np.loadtxt(qp)
    out, s_cut = run(["cutoff", tp, qp, m, 10, metric, w, arg], tmp)
    cut = parse_cli("cutoff", out)
    thr = cut["threshold"]
    out, s_search = run(["search", tp, qp, m, thr, metric, w, arg], tmp)
    srch = parse_cli("search", out)
    out, s_exact = run(["exact", tp, qp, m, thr, metric, w, arg], tmp)
    ex = parse_cli("exact", out)
    assert sorted(srch["matches"]) == sorted(ex["matches"]), "search and exact disagree"
    assert set(cut["ranks"]) <= set(srch["matches"]), "cutoff ranks missing from the search matches"
    ridx, rdist = ranking(ref, t, q, m, cut["ranks"], metric, w, arg)
    assert ridx == cut["ranks"], "reference ranking disagrees with its own distances"
    assert float.fromhex(rdist[-1]) == float(thr), "k-th distance is not the printed threshold"
    xi, xd = ranking(ref, t, q, m, ex["matches"], metric, w, arg)
    return {
        "n": len(t), "m": m, "w": w, "metric": metric, "arg": arg, "k": 10,
        "target_sha256": sha256(t), "query": [float(x).hex() for x in q],
        "threshold": float(thr).hex(),
        "cutoff": {"ranks": ridx, "dists": rdist, "kk1": cut["kk1"], "lb_pruned": cut["lb_pruned"],
                   "glb_pruned": cut["glb_pruned"], "exact": cut["exact"]},
        "search": srch,
        "exact": {"matches": sorted(ex["matches"]), "by_distance": xi, "dists": xd, "kk1": ex["kk1"],
                  "invalid": ex["invalid"]},
        "reference_seconds": {"cutoff": s_cut, "search": s_search, "exact": s_exact},
    }


def config2(ref, tmp):
    t, queries, meta = synth.config2()
    m, w, args = meta["m"], meta["w"], meta["args"]
    tp = os.path.join(tmp, "c2.bin")
    t.astype("<f8").tofile(tp)
    jobs = {}
    qs = {}
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        for metric, (q, _s) in queries.items():
            qp = os.path.join(tmp, f"c2_{metric}.txt")
            np.savetxt(qp, q, fmt="%.17g")
            qs[metric] = np.loadtxt(qp)
            cut = C2_CUTOFFS[metric]
            below = math.nextafter(cut, 0.0)
            for tag, c in (("at", cut), ("below", below)):
                jobs[(metric, tag)] = ex.submit(run, ["search", tp, qp, m, repr(c), metric, w, args[metric]], tmp)
        res = {k: (parse_cli("search", f.result()[0]), f.result()[1]) for k, f in jobs.items()}
    out = {"n": len(t), "m": m, "w": w, "k": C2_K, "target_sha256": sha256(t), "metrics": {}}
    for metric in queries:
        at, s_at = res[(metric, "at")]
        below, s_below = res[(metric, "below")]
        assert len(at["matches"]) >= C2_K > len(below["matches"]), (metric, len(at["matches"]),
                                                                      len(below["matches"]))
        ridx, rdist = ranking(ref, t, qs[metric], m, at["matches"], metric, w, args[metric])
        assert float.fromhex(rdist[C2_K - 1]) == C2_CUTOFFS[metric], metric
        out["metrics"][metric] = {
            "arg": args[metric], "query": [float(x).hex() for x in qs[metric]],
            "cutoff": float(C2_CUTOFFS[metric]).hex(),
            "search": at, "search_below": {k: below[k] for k in ("kk1", "kk2", "kk3", "invalid")},
            "matches_below": len(below["matches"]),
            "ranks": ridx[:C2_K], "dists": rdist[:C2_K],
            "reference_seconds": {"search": s_at, "search_below": s_below},
        }
    return out


def main():
    if not orc.have_reference():
        raise SystemExit("oracle/_ref is not built: python -c 'from oracle import oracle; oracle.build()'")
    ref = orc.Oracle("ref")
    pins = {}
    with tempfile.TemporaryDirectory() as tmp:
        t0 = time.time()
        pins["c1"] = config1(ref, tmp)
        print(f"c1 pinned in {time.time() - t0:.1f} s", flush=True)
        t0 = time.time()
        pins["c2"] = config2(ref, tmp)
        print(f"c2 pinned in {time.time() - t0:.1f} s", flush=True)
    with open(OUT, "w") as f:
        json.dump(pins, f, indent=1)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
