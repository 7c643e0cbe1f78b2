"""Measure the automatic kernel choices on the GPU and write the tuning table.

Two choices depend on the shape and are settled by measurement:

* the exact DP kernel: the lane-per-candidate DP (band and candidate ring
  per lane in shared memory) or the anti-diagonal wavefront (one warp per
  candidate, band in registers), per metric, macro-segment length m_k and
  radius w; `dp` rules for the DP over the GLB survivors of a search or
  top-k query (timed as a search at the rank-50 distance on a structured
  walk), `dpx` rules for the exact scan of every window (timed at the
  rank-20 distance on a random walk).
* the LB_IP form of batched searches (`lb` rules) and top-k queries (`lbk`):
  per-query thresholds and FP64 FFTs, or one tensor-core product for the
  group, per metric, m_k and group size.  Timed as one batched `search` of
  the group at each query's rank-10 distance, and one batched `cutoff` k=10,
  on a 2^22-point random walk.

A rule departs from the built-in choice (lane DP, FFT LB_IP) only where the
other form measured at least MARGIN (5%) faster, so timing noise between two
nearly equal forms does not flip a shape back and forth.  Shapes where the
lane DP's band does not fit shared memory need no measurement (the wavefront
is the only shared-memory form there).  The table (fsmeld_b200/tune_table.txt)
is loaded by api.Engine into every context.

    python -m fsmeld_b200.tune [--quick] [--out PATH]
    python -m fsmeld_b200.tune --from-log LOG [--out PATH]   # table from a measurement log
"""
from __future__ import annotations

import argparse
import os
import re
import time

import numpy as np

from fsmeld_b200 import api
from fsmeld_b200.synth import query_from, random_walk, walk_with_structure

METRIC_ARGS = {"dtw": 0.0, "erp": 0.0, "edr": 0.25, "lcss": 0.25, "msm": 0.5}
DP_SHAPES = {64: (2, 3, 6, 13, 31), 128: (3, 6, 13, 26, 51), 256: (6, 13, 26, 51, 94),
             512: (13, 26, 51, 94), 1024: (26, 51, 94), 2048: (51, 94)}
LB_SHAPES = {128: (8, 32), 256: (8, 32), 512: (8, 32)}
MARGIN = 0.05
DEFAULT = {"dp": "lane", "dpx": "lane", "lb": "fft", "lbk": "fft"}


def choose(kind, times):
    """The built-in form unless the other one measured MARGIN faster."""
    base = DEFAULT[kind]
    other = min((f for f in times if f != base), key=times.get)
    return other if times[other] < (1.0 - MARGIN) * times[base] else base


def macro_length(m):
    mk = 1
    while mk < 8 * m:
        mk *= 2
    return mk


def lane_fits(w, smem_optin=232448):
    ring = 1
    while ring < 2 * w + 2:
        ring *= 2
    return 2 * 8 * 32 * (2 * w + 2 + ring) <= smem_optin - 4096


def timed(eng, fn, reps=2):
    fn()  # warm-up (workspace)
    best = float("inf")
    for _ in range(reps):
        fn()
        best = min(best, eng.last_call_ms)
    return best


def tune_dp(metrics, shapes, log):
    """dp: the DP over a candidate list (search and top-k), timed as a search
    at the query's rank-50 distance on a structured walk of 2^20 points (the
    search's other stages are the same for both forms); dpx: the exact scan
    (every window), timed at the rank-20 distance on 2^16-2^17 points."""
    rules = []
    for m, ws in shapes.items():
        n = (1 << 17) if m <= 256 else (1 << 16)
        t = random_walk(n, 9000 + m)
        q, _ = query_from(t, m, np.random.default_rng(9001 + m))
        ts = walk_with_structure(1 << 20, m, seed=9002 + m, motifs=40, nan_fraction=1e-3, flat_runs=8)
        qs, _ = query_from(ts, m, np.random.default_rng(9003 + m))
        for metric in metrics:
            arg = METRIC_ARGS[metric]
            for w in ws:
                if w >= m or not lane_fits(w):
                    continue
                mk = macro_length(m)
                for kind in ("dp", "dpx"):
                    times = {}
                    for form in ("lane", "wave"):
                        table = f"{kind} {metric} {mk} 1000 {form}\n"
                        if kind == "dp":
                            with api.Engine(ts, tuning=table) as e:
                                _, d, _ = e.cutoff(qs, m, 50, metric, w, arg)
                                cut = float(d[-1])
                                times[form] = timed(e, lambda: e.search(qs, m, cut, metric, w, arg))
                        else:
                            with api.Engine(t, tuning=table) as e:
                                _, d, _ = e.cutoff(q, m, 20, metric, w, arg)
                                cut = float(d[-1])
                                times[form] = timed(e, lambda: e.exact(q, m, cut, metric, w, arg))
                    choice = choose(kind, times)
                    log(f"{kind} {metric} m={m} w={w}: lane {times['lane']:.2f} ms, wave {times['wave']:.2f} ms "
                        f"-> {choice}")
                    rules.append((kind, metric, mk, w, choice, times))
    return rules


def tune_lb(metrics, shapes, log, n=1 << 22):
    """Search groups (at each query's rank-10 distance) and top-k groups (k=10)."""
    rules = []
    t = random_walk(n, 9100)
    for m, qcounts in shapes.items():
        rng = np.random.default_rng(9101 + m)
        w = max(1, m // 20)
        for metric in metrics:
            arg = METRIC_ARGS[metric]
            with api.Engine(t, tuning="") as e:
                qs = []
                for _ in range(max(qcounts)):
                    q, _ = query_from(t, m, rng)
                    _, d, _ = e.cutoff(q, m, 10, metric, w, arg)
                    qs.append(dict(query=q, m=m, metric=metric, w=w, arg=arg, cutoff=float(d[-1]), k=10))
                for kind, mode in (("lb", "search"), ("lbk", "cutoff")):
                    for nq in qcounts:
                        times = {}
                        for form in ("fft", "gemm"):
                            e.set_lb_form(form)
                            times[form] = timed(e, lambda: e.batch(mode, qs[:nq]))
                        choice = choose(kind, times)
                        log(f"{kind} {metric} m={m} q={nq}: fft {times['fft']:.2f} ms, gemm {times['gemm']:.2f} ms "
                            f"-> {choice}")
                        rules.append((kind, metric, macro_length(m), nq, choice, times))
    return rules


def write_table(path, dp_rules, lb_rules):
    lines = ["# Tuning table: measured by `python -m fsmeld_b200.tune` on one B200.",
             "# kind metric m_k limit choice  (dp: w <= limit; lb: group size >= limit); first match wins",
             f"# a rule departs from the built-in form only where the other measured {MARGIN:.0%} faster"]
    for kind, metric, mk, w, choice, times in dp_rules:
        lines.append(f"{kind} {metric} {mk} {w} {choice}   # lane {times['lane']:.2f} ms, wave {times['wave']:.2f} ms")
    # lb: for each (metric, m_k) the smallest group size from which the product wins at every measured size
    by_shape = {}
    for kind, metric, mk, nq, choice, times in lb_rules:
        by_shape.setdefault((kind, metric, mk), []).append((nq, choice, times))
    for (kind, metric, mk), rows in by_shape.items():
        rows.sort()
        qmin = None
        for i, (nq, _, _) in enumerate(rows):
            if all(ch == "gemm" for _, ch, _ in rows[i:]):
                qmin = nq
                break
        detail = ", ".join(f"q={nq}: fft {tm['fft']:.1f} / gemm {tm['gemm']:.1f} ms" for nq, _, tm in rows)
        if qmin is not None:
            lines.append(f"{kind} {metric} {mk} {qmin} gemm   # {detail}")
        else:
            lines.append(f"# {kind} {metric} {mk}: fft at every measured size ({detail})")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


LOG_LINE = re.compile(r"^(dpx?|lbk?) (\w+) m=(\d+) (w|q)=(\d+): (\w+) ([\d.]+) ms, (\w+) ([\d.]+) ms")


def rules_from_log(path):
    """dp and lb rules from the lines a measurement run logged (the choices
    are made again under the current margin)."""
    dp, lb = [], []
    with open(path) as f:
        for ln in f:
            mt = LOG_LINE.match(ln)
            if not mt:
                continue
            kind, metric, m, _, lim, f1, t1, f2, t2 = mt.groups()
            times = {f1: float(t1), f2: float(t2)}
            rule = (kind, metric, macro_length(int(m)), int(lim), choose(kind, times), times)
            (dp if kind.startswith("dp") else lb).append(rule)
    return dp, lb


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=api.TUNE_TABLE)
    ap.add_argument("--quick", action="store_true", help="DTW and MSM only")
    ap.add_argument("--from-log", help="write the table from the lines of an earlier run's log")
    args = ap.parse_args()
    if args.from_log:
        dp, lb = rules_from_log(args.from_log)
        write_table(args.out, dp, lb)
        print(f"wrote {args.out} from {args.from_log}: {len(dp)} dp rules, {len(lb)} lb measurements")
        return
    metrics = ["dtw", "msm"] if args.quick else list(METRIC_ARGS)
    t0 = time.time()
    log = lambda s: print(s, flush=True)  # noqa: E731
    dp = tune_dp(metrics, DP_SHAPES, log)
    lb = tune_lb(metrics, LB_SHAPES, log)
    write_table(args.out, dp, lb)
    log(f"wrote {args.out} in {time.time() - t0:.0f} s")


if __name__ == "__main__":
    main()
