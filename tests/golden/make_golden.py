"""Generate the golden fixtures in this folder from the reference itself.

The reference ships no tests, fixtures or known-answer vectors, so they are
made here: the reference's own sources are compiled unmodified against the
project's FFTW-API shim (oracle/Makefile -> oracle/_ref) and run on small
seeded inputs.  Outputs:

  kat_functions.npz  per-function vectors (window statistics, masks,
                     envelopes, thresholds, penalties, SIP, GLB, distances)
                     from oracle/_ref/libfsmeld_ref.so
  cli_cases.npz      small targets + queries and the reference CLI's match
                     sets, counters and rankings (oracle/_ref/fsmeld_ref)

Run from the repository root with the reference tree present:
    python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import os
import re
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from fsmeld_b200.synth import query_from, random_walk, walk_with_structure  # noqa: E402
from oracle import oracle as orc  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
METRIC_ARGS = [("dtw", 0.0), ("erp", 0.0), ("erp", 0.4), ("edr", 0.25), ("lcss", 0.25),
               ("msm", 0.5)]


def kat_functions(ref: orc.Oracle) -> dict:
    out = {}
    rng = np.random.default_rng(11)
    cases = [(64, 5, 0), (32, 3, 1), (128, 6, 2)]
    for ci, (m, w, seed) in enumerate(cases):
        n = 1 << 14
        t = walk_with_structure(n, m, seed=100 + seed, motifs=8, nan_fraction=3e-3, flat_runs=4,
                                nan_spans=3)
        mk = orc.Oracle.macro_length(_restatement(), m, n)
        kml = mk - m + 1
        segs = np.arange((n - m + 1) // kml)
        pick = rng.choice(segs, size=min(4, len(segs)), replace=False)
        q, _ = query_from(t, m, rng)
        qn = _restatement().normalize_query(q)
        LQ, UQ = ref.lemire(qn, w)
        p = f"c{ci}_"
        out[p + "target"] = t
        out[p + "query"] = q
        out[p + "params"] = np.array([m, w, mk])
        out[p + "segments"] = pick
        for s in pick:
            ts = t[s * kml: s * kml + mk]
            k = f"{p}s{s}_"
            mu, si = ref.mvmean(ts, m)
            out[k + "mu"], out[k + "si"] = mu, si
            out[k + "mask"] = ref.invalid_mask(ts, si, m)
            mn, mx = ref.min_max_window(mu, mk, m)
            smn, smx = ref.min_max_window(si, mk, m)
            out[k + "mumin"], out[k + "mumax"], out[k + "simin"], out[k + "simax"] = mn, mx, smn, smx
            L, U = ref.lemire(ts, w)
            out[k + "L"], out[k + "U"] = L, U
            Un, Ln = ref.normalized(U, L, mx, mn, smx, smn)
            out[k + "Un"], out[k + "Ln"] = Un, Ln
            core_nan = bool(np.isnan(Un[m - 1: mk - m + 1]).any() or np.isnan(Ln[m - 1: mk - m + 1]).any())
            out[k + "core_nan"] = np.array(core_nan)
            for metric, arg in METRIC_ARGS:
                mm = f"{k}{metric}{arg}_"
                tu = ref.find_t(1, metric, Un, qn, m, arg)
                tl = ref.find_t(0, metric, Ln, qn, m, arg)
                out[mm + "t"] = np.array([tu, tl])
                hl = ref.q_to_h(0, metric, qn, tl, arg)
                hu = ref.q_to_h(1, metric, qn, tu, arg)
                gl = ref.s_to_g(0, Ln, tl)
                gu = ref.s_to_g(1, Un, tu)
                out[mm + "hl"], out[mm + "hu"] = hl, hu
                zl = ref.sip(mk, m, hl, gl)
                zu = ref.sip(mk, m, hu, gu)
                out[mm + "zl"], out[mm + "zu"] = zl, zu
            js = [j for j in range(kml) if np.isfinite(si[j]) and si[j] > 1e-12][::97][:6]
            out[k + "cand"] = np.array(js, dtype=np.int64)
            for j in js:
                T = (ts[j:j + m] - mu[j]) / si[j]
                for metric, arg in METRIC_ARGS:
                    d = ref.distance(metric, qn, T, w, arg)
                    glbs = [ref.glb(metric, qn, T, arg, LQ, UQ, w, b) for b in (0.5 * d, d, 2 * d)]
                    out[f"{k}j{j}_{metric}{arg}_d"] = np.array([d] + glbs)
    return out


_RESTATEMENT = None


def _restatement():
    global _RESTATEMENT
    if _RESTATEMENT is None:
        _RESTATEMENT = orc.Oracle("oracle")
    return _RESTATEMENT


def parse_cli(cmd: str, text: str) -> dict:
    res = {}
    if cmd == "search":
        for key, pat in [("kk1", r"^kk1=(\d+)"), ("kk2", r"^kk2=(\d+)"),
                         ("kk3", r"^Candidates after GLB: (\d+)"),
                         ("invalid", r"^Invalid candidates: (\d+)")]:
            mm = re.search(pat, text, re.M)
            res[key] = int(mm.group(1))
        res["matches"] = [int(x) for x in re.findall(r"^A\[\d+\]=(\d+)$", text, re.M)]
    elif cmd == "exact":
        res["matches"] = [int(x) for x in re.findall(r"^A\[\d+\] = (\d+)$", text, re.M)]
        res["dists"] = [x for x in re.findall(r"^GET \w+: (\S+) \(index", text, re.M)]
        res["kk1"] = int(re.search(r"^Total Valid Candidates: (\d+)", text, re.M).group(1))
        res["invalid"] = int(re.search(r"^Invalid candidates: (\d+)", text, re.M).group(1))
    else:
        res["threshold"] = re.search(r"Final Top-K Threshold:\s+(\S+)", text).group(1)
        res["ranks"] = [int(x) for x in re.findall(r"^Rank \d+: Index A\[\d+\]=(\d+)$", text, re.M)]
        for key, pat in [("kk1", r"Candidates checked by LB:\s+(\d+)"),
                         ("lb_pruned", r"Pruned by LBIP:\s+(\d+)"),
                         ("glb_pruned", r"Pruned by GLB:\s+(\d+)"),
                         ("exact", r"Exact distances computed:\s+(\d+)")]:
            res[key] = int(re.search(pat, text).group(1))
    return res


def cli_cases() -> dict:
    arrays, meta = {}, []
    specs = [
        # name, n, m, w, seed, structured, k
        ("walk_m64", 1 << 15, 64, 5, 21, False, 10),
        ("struct_m32", 1 << 14, 32, 3, 22, True, 20),
        ("short_m40", 300, 40, 4, 23, False, 5),      # target shorter than one macro segment
        ("tail_m48", 5000, 48, 4, 24, True, 8),
    ]
    with tempfile.TemporaryDirectory() as tmp:
        env = dict(os.environ, FSMELD_RESULTS_CSV=os.path.join(tmp, "r.csv"))
        for name, n, m, w, seed, structured, k in specs:
            t = (walk_with_structure(n, m, seed, motifs=6, nan_fraction=2e-3, flat_runs=3, nan_spans=2)
                 if structured else random_walk(n, seed))
            rng = np.random.default_rng(seed + 5)
            q, _ = query_from(t, m, rng)
            tp, qp = os.path.join(tmp, f"{name}.bin"), os.path.join(tmp, f"{name}.txt")
            t.astype("<f8").tofile(tp)
            np.savetxt(qp, q, fmt="%.17g")
            arrays[f"{name}_target"] = t
            arrays[f"{name}_query"] = np.loadtxt(qp)
            for metric, arg in METRIC_ARGS:
                excl = ["-1", "-1"]
                rc, out, err = orc.run_reference_cli(["cutoff", tp, qp, m, k, metric, w, arg], cwd=tmp, env=env)
                assert rc == 0, err
                cut = parse_cli("cutoff", out)
                thr = cut["threshold"]
                rc, out, err = orc.run_reference_cli(["search", tp, qp, m, thr, metric, w, arg], cwd=tmp, env=env)
                assert rc == 0, err
                srch = parse_cli("search", out)
                rc, out, err = orc.run_reference_cli(["exact", tp, qp, m, thr, metric, w, arg], cwd=tmp, env=env)
                assert rc == 0, err
                ex = parse_cli("exact", out)
                # with an exclusion interval around the best match
                b0 = cut["ranks"][0]
                excl = [max(0, b0 - m // 2), b0 + m // 2]
                rc, out, err = orc.run_reference_cli(
                    ["search", tp, qp, m, thr, metric, w, arg, excl[0], excl[1]], cwd=tmp, env=env)
                assert rc == 0, err
                sx = parse_cli("search", out)
                meta.append({"name": name, "n": n, "m": m, "w": w, "k": k, "metric": metric,
                             "arg": arg, "cutoff": cut, "search": srch, "exact": ex,
                             "exclusion": excl, "search_excl": sx})
    arrays["meta_json"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    return arrays


def main() -> None:
    orc.build(reference=True)
    ref = orc.Oracle("ref")
    np.savez_compressed(os.path.join(OUT, "kat_functions.npz"), **kat_functions(ref))
    np.savez_compressed(os.path.join(OUT, "cli_cases.npz"), **cli_cases())
    print("golden fixtures written to", OUT)


if __name__ == "__main__":
    main()
