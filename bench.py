"""Benchmark: FSMELD exact subsequence range search on B200.

Workload (the single-GPU configuration the headline metric is quoted on):
five queries per step, one per metric (DTW, ERP g=0, EDR eps=0.25, LCSS
eps=0.25, MSM c=0.5), m=256, w=13, on a 2^24-point float64 random walk with
200 sine/chirp motifs, NaN spans (0.1% of points) and flat runs; each
query's cutoff is its k=50 exact distance (computed once, untimed).  A step
is one batched `search` of the five queries through the LB_IP -> GLB -> ELD
cascade.  The metric is candidates/s: valid windows scanned per second,
summed over the step's queries.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (torchrun, one rank per GPU) every rank searches its own target
partition (weak scaling, no data-path collective); timings are the max over
ranks.  `--impl reference` times the reference's own CPU code (built from
its sources against the project FFT shim, oracle/_ref) on bounded samples.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_POINTS = 1 << 24
M, W, K_TOP = 256, 13, 50
METRICS = [("dtw", 0.0), ("erp", 0.0), ("edr", 0.25), ("lcss", 0.25), ("msm", 0.5)]
WORKLOAD = ("five queries (dtw; erp g=0; edr eps=0.25; lcss eps=0.25; msm c=0.5), m=256, w=13, "
            "2^24-point float64 random walk + 200 motifs + NaN spans + flat runs; cutoff = k=50 exact distance")
# k=50 exact distance of each query over the full rank-0 target: the
# reference's own values, pinned by tests/golden/make_config_pins.py (the
# reference's `search` finds at least 50 matches at each cutoff and fewer
# than 50 just below it; tests/test_gpu_config_pins.py checks the GPU's top-50
# rankings against the reference's).  The GPU arm re-derives them with its own
# `cutoff` and records whether they agree; the CPU reference arm uses them.
PINS_PATH = os.path.join(ROOT, "tests", "golden", "config_pins.json")


def load_cutoffs():
    with open(PINS_PATH) as f:
        pins = json.load(f)["c2"]["metrics"]
    return {mt: float.fromhex(pins[mt]["cutoff"]) for mt, _ in METRICS}


CUTOFFS = load_cutoffs()
PEAKS_PATH = os.path.join(ROOT, "MEASURED_PEAKS.json")
PROFILE_SUMMARY = os.path.join(ROOT, "profiles", "roofline_traffic.json")
LATENCY_REPS = 10  # plain single-query requests per query for the latency figures
DEFAULT_CONCURRENCY = 4  # the library's default (fsmeld_set_concurrency)


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def make_workload(rank, n_points=N_POINTS):
    from fsmeld_b200.synth import query_from, walk_with_structure
    t = walk_with_structure(n_points, M, seed=2 + 7919 * rank)
    rng = np.random.default_rng(1002 + rank)
    queries = {}
    for metric, _ in METRICS:
        q, _s = query_from(t, M, rng)
        queries[metric] = q
    return t, queries


class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = str(gpu_index)
        try:
            import torch
            self.gpu = "GPU-" + str(torch.cuda.get_device_properties(gpu_index).uuid)
        except Exception:
            vis = os.environ.get("CUDA_VISIBLE_DEVICES")
            if vis:
                self.gpu = vis.split(",")[gpu_index].strip()
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm = []
        mx = None
        reasons = set()
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
                for nm, v in zip(names, r[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def load_peaks():
    try:
        with open(PEAKS_PATH) as f:
            p = json.load(f)
        return {"hbm_gbs": float(p["hbm_gbs"]), "bf16_tflops": float(p["bf16_tflops"]), "source": "measured"}
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback"}


# FP64 operations the reference's recurrence evaluates per band cell
# (src/ElasticMeasures.cpp): DTW dist (sub, mul) + min of three (2) + add;
# ERP three candidates of (sub, mul, add) + min of three; EDR sub, abs,
# compare, three adds, min of three; LCSS sub, abs, compare, add, max of
# three; MSM |x - y| + add, two split/merge costs (4 compares, 2 subs, 2 abs,
# min, add) + adds, min of three.
FLOPS_PER_CELL = {"dtw": 5, "erp": 11, "edr": 8, "lcss": 6, "msm": 27}
# B200 FP64 issue rate: 148 SMs x 64 FP64 lanes x 1.965 GHz (the datasheet's
# 37 TFLOP/s counts a fused multiply-add as two operations)
FP64_PEAK_TOPS = 148 * 64 * 1.965e9 / 1e12


def roofline(stages, cells, peaks):
    """The dominant kernel, the exact DP, is FP64-bound: algorithmic work =
    band cells it computed (device counter; early abandon skips the rest) x
    FP64 operations per cell of the reference's recurrence, over its average
    launch time.  The lane DP (k_dp) and the wavefront (k_dpw, where the
    tuning table selects it) share the counter, so their launches are taken
    together."""
    ms_lane, n_lane = stages.get("k_dp", (0.0, 0))
    ms_wave, n_wave = stages.get("k_dpw", (0.0, 0))
    ms, launches = ms_lane + ms_wave, n_lane + n_wave
    if launches == 0 or ms <= 0.0:
        return None
    kernel = "k_dp" if n_wave == 0 else ("k_dpw" if n_lane == 0 else "k_dp+k_dpw")
    flops = sum(cells[mt] * FLOPS_PER_CELL[mt] for mt in cells)
    avg_s = ms / launches / 1e3
    achieved = flops / launches / avg_s / 1e12
    traffic = None
    try:
        with open(PROFILE_SUMMARY) as f:
            traffic = json.load(f).get(kernel, {}).get("bytes_per_launch")
    except Exception:
        pass
    return {"bound": "fp64", "kernel": kernel, "achieved": round(achieved, 3), "peak": round(FP64_PEAK_TOPS, 2),
            "unit": "TFLOP/s", "frac": round(achieved / FP64_PEAK_TOPS, 4), "traffic": traffic,
            "algorithmic_flops_per_launch": flops / launches, "avg_launch_ms": round(avg_s * 1e3, 4),
            "dp_cells_per_launch": sum(cells.values()) / launches, "flops_per_cell": FLOPS_PER_CELL,
            "peak_source": "nominal FP64 issue rate of B200 (148 SMs x 64 lanes x 1.965 GHz); "
                           "MEASURED_PEAKS.json holds no FP64 figure"}


def roofline_hbm(stages, geom, peaks):
    """The window-statistics scan (k_mvmean), HBM-bound: reads every macro
    segment's m_k target points once (the m-1 halo included) and writes mean and
    sigma of its k_m_l windows."""
    ms, launches = stages["k_mvmean"]
    launches = max(1, launches)
    S, m_k, kml = geom["S"], geom["m_k"], geom["kml"]
    bytes_per_launch = 8.0 * S * m_k + 16.0 * S * kml
    avg_s = ms / launches / 1e3
    achieved = bytes_per_launch / avg_s / 1e9
    traffic = None
    try:
        with open(PROFILE_SUMMARY) as f:
            traffic = json.load(f).get("k_mvmean", {}).get("bytes_per_launch")
    except Exception:
        pass
    return {"bound": "hbm", "kernel": "k_mvmean", "achieved": round(achieved, 1), "peak": peaks["hbm_gbs"],
            "unit": "GB/s", "frac": round(achieved / peaks["hbm_gbs"], 4), "traffic": traffic,
            "algorithmic_bytes_per_launch": bytes_per_launch, "avg_launch_ms": round(avg_s * 1e3, 4),
            "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)" if peaks["source"] == "measured"
            else "fallback 6.65 TB/s"}


def stage_rooflines(stages, geom, n, peaks):
    """HBM fraction of every memory-bound stage, from its algorithmic bytes
    per launch and its average CUDA-event launch time:
      k_mvmean   8 B per segment point read (halo included) + 16 B per window
      k_envelope 8 B per segment point + 16 B per window read, 16 B per point written
      k_fwd_env  8 B per target point read, 16 B written
      k_seed / k_lb_filter (k_select): 8 B per window (top-k only)"""
    S, m_k, kml = geom["S"], geom["m_k"], geom["kml"]
    per_launch = {"k_mvmean": 8.0 * S * m_k + 16.0 * S * kml,
                  "k_envelope": 8.0 * S * m_k + 16.0 * S * kml + 16.0 * S * m_k,
                  "k_fwd_env": 24.0 * n}
    out = {}
    for k, b in per_launch.items():
        if k not in stages or stages[k][1] == 0:
            continue
        ms, launches = stages[k]
        avg_s = ms / launches / 1e3
        gbs = b / avg_s / 1e9
        out[k] = {"bound": "hbm", "algorithmic_bytes_per_launch": b, "avg_launch_ms": round(avg_s * 1e3, 4),
                  "achieved_gbs": round(gbs, 1), "frac": round(gbs / peaks["hbm_gbs"], 4)}
    return out


def geometry(n, m):
    sel = 1
    while sel < 8 * m:
        sel *= 2
    m_k = min(sel, n)
    kml = m_k - m + 1
    tsn = n - m + 1
    forsize, tail = tsn // kml, tsn % kml
    return {"m_k": m_k, "kml": kml, "forsize": forsize, "tail": tail, "S": forsize + (1 if tail else 0)}


# ------------------------------------------------------------------ reference arm

def ref_binary():
    return os.path.join(ROOT, "oracle", "_ref", "fsmeld_ref")


def run_ref(args, env):
    p = subprocess.run([ref_binary()] + [str(a) for a in args], capture_output=True, text=True, env=env)
    if p.returncode != 0:
        raise RuntimeError(p.stderr.strip())
    return p.stdout


def parse_valid(out):
    for line in out.splitlines():
        if line.startswith("Total Valid Candidates: "):
            return int(line.split(": ")[1])
    raise RuntimeError("no candidate count in reference output")


def reference_setup(tmp, target, queries, cutoffs, slice_points):
    """Write sample slices and query files for the reference binary."""
    env = dict(os.environ, FSMELD_QUIET_MATCHES="1", FSMELD_RESULTS_CSV=os.path.join(tmp, "ref.csv"))
    files = {}
    for metric, _ in METRICS:
        qp = os.path.join(tmp, f"q_{metric}.txt")
        np.savetxt(qp, queries[metric], fmt="%.17g")
        files[metric] = qp
    slices = []
    nslices = max(1, len(target) // slice_points)
    for i in range(nslices):
        sp = os.path.join(tmp, f"slice_{i}.bin")
        target[i * slice_points:(i + 1) * slice_points].astype("<f8").tofile(sp)
        slices.append(sp)
    return env, files, slices


def reference_step(env, files, slices, cutoffs, procs, offset):
    """`procs` concurrent reference processes, each one search over one sample slice."""
    jobs = []
    for i in range(procs):
        metric, arg = METRICS[(offset + i) % len(METRICS)]
        sp = slices[(offset + i) % len(slices)]
        jobs.append((sp, metric, arg))
    t0 = time.perf_counter()
    ps = [subprocess.Popen([ref_binary(), "search", sp, files[mt], str(M), repr(cutoffs[mt]), mt, str(W), ag],
                           stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True, env=env)
          for sp, mt, ag in [(a, b, str(c)) for a, b, c in jobs]]
    total = 0
    for p in ps:
        out, err = p.communicate()
        if p.returncode != 0:
            raise RuntimeError(err.strip())
        total += parse_valid(out)
    return total, time.perf_counter() - t0


def impl_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    if not os.path.exists(ref_binary()):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/fsmeld_ref was not built"}))
        return 0
    target, queries = make_workload(0)
    slice_points = 1 << 17
    cores = os.cpu_count() or 1
    cutoffs = dict(CUTOFFS)
    with tempfile.TemporaryDirectory() as tmp:
        env, files, slices = reference_setup(tmp, target, queries, cutoffs, slice_points)
        procs = max(1, min(cores, 5 * len(slices)))
        for i in range(args.warmup):
            reference_step(env, files, slices, cutoffs, procs, i * procs)
        cand, secs = 0, 0.0
        for i in range(args.steps):
            c, s = reference_step(env, files, slices, cutoffs, procs, (args.warmup + i) * procs)
            cand += c
            secs += s
    value = cand / secs
    sample = (f"per step {procs} concurrent reference `search` processes (one per host thread), each over a "
              f"2^17-point slice of the workload's target with one of the five queries and its k=50 cutoff")
    line = {"impl": "reference", "metric": "candidates/s", "value": value, "unit": "candidates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": secs / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "n": N_POINTS, "m": M, "w": W, "k": K_TOP, "queries_per_step": procs},
            "cpu_baseline": {"value": value, "unit": "candidates/s", "cores": procs, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": "candidates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def cpu_baseline_single(target, queries, cutoffs):
    """The reference's CPU path, one core, five searches over a 2^21-point sample."""
    if not os.path.exists(ref_binary()):
        return None
    with tempfile.TemporaryDirectory() as tmp:
        env = dict(os.environ, FSMELD_QUIET_MATCHES="1", FSMELD_RESULTS_CSV=os.path.join(tmp, "ref.csv"))
        sp = os.path.join(tmp, "sample.bin")
        target[: 1 << 18].astype("<f8").tofile(sp)
        cand, secs = 0, 0.0
        for metric, arg in METRICS:
            qp = os.path.join(tmp, f"q_{metric}.txt")
            np.savetxt(qp, queries[metric], fmt="%.17g")
            t0 = time.perf_counter()
            out = run_ref(["search", sp, qp, M, repr(cutoffs[metric]), metric, W, arg], env)
            secs += time.perf_counter() - t0
            cand += parse_valid(out)
    return {"value": cand / secs, "unit": "candidates/s", "cores": 1, "kind": "reference",
            "sample": "the reference's `search` (its own sources + project FFT shim), single thread, the five "
                      "queries with the workload's cutoffs over the first 2^18 points of the target"}


# ------------------------------------------------------------------ our arm

def impl_ours(args):
    import torch
    import torch.distributed as dist

    from fsmeld_b200 import api

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    target, queries = make_workload(rank, args.n_points or N_POINTS)
    geom = geometry(len(target), M)
    eng = api.Engine(target, device=local)
    conc = args.concurrency or DEFAULT_CONCURRENCY
    eng.set_concurrency(conc)
    metrics = [(mt, ag) for mt, ag in METRICS if args.case in (None, mt)]
    if args.case or args.fixed_cutoffs or (args.n_points or N_POINTS) != N_POINTS:
        cutoffs = dict(CUTOFFS)  # profiling cases: the workload's constants, no setup launches
        cutoffs_match = None
    else:
        cutoffs = {}
        for metric, arg in METRICS:
            _idx, dist_k, _c = eng.cutoff(queries[metric], M, K_TOP, metric, W, arg)
            cutoffs[metric] = float(dist_k[-1])
        cutoffs_match = (rank != 0) or all(cutoffs[k] == CUTOFFS[k] for k in CUTOFFS)
    batch = [dict(query=queries[mt], m=M, metric=mt, w=W, arg=ag, cutoff=cutoffs[mt]) for mt, ag in metrics]

    def step():
        res = eng.batch("search", batch)
        for r in res:
            if r["status"] != 0:
                raise RuntimeError(f"query failed: {r['status']}")
        return res

    for _ in range(args.warmup):
        step()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = eng.launches
    dev_ms = 0.0
    cand = 0
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            res = step()
            dev_ms += eng.last_call_ms
            cand += sum(r["counters"]["valid"] for r in res)
    torch.cuda.synchronize()
    launches = eng.launches - launches0
    # per-kernel figures (stage times, DP cells, roofline) from a separate pass
    # with the queries one after another and CUDA events around every launch,
    # so that each kernel is timed alone; the timed steps above run the batch
    # as the library does by default (queries of a group on concurrent streams)
    prof_steps = 2
    eng.set_concurrency(1)
    eng.set_profiling(True)
    cells = {mt: 0 for mt, _ in metrics}
    for _ in range(prof_steps):
        for (mt, _), r in zip(metrics, step()):
            cells[mt] += r["counters"]["dp_cells"]
    stages = eng.stage_times()
    eng.set_profiling(False)
    eng.set_concurrency(conc)
    t_local = torch.tensor([dev_ms], dtype=torch.float64, device="cuda")
    c_local = torch.tensor([float(cand)], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t_local, op=dist.ReduceOp.MAX)
        dist.all_reduce(c_local, op=dist.ReduceOp.SUM)
        dist.barrier()
    t_max_ms = float(t_local.item())
    cand_all = float(c_local.item())
    value = cand_all / (t_max_ms / 1e3)

    # end to end through the public API: every step uploads the target from pinned host
    # memory into the engine (fsmeld_load) and runs the batch, whose results come back to
    # host memory
    pinned = torch.from_numpy(target).pin_memory()
    pinned_np = pinned.numpy()
    e2e_secs = 0.0
    e2e_cand = 0
    d2h = 0
    for i in range(0 if args.no_e2e else args.warmup + args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        eng.load(pinned_np)
        res = eng.batch("search", batch)
        t1 = time.perf_counter()
        if i >= args.warmup:
            e2e_secs += t1 - t0
            e2e_cand += sum(r["counters"]["valid"] for r in res)
            d2h = sum(int(r["count"]) * 8 + 96 for r in res)
    e2e_value = e2e_cand / e2e_secs * world if e2e_secs > 0 else None

    # request latency: every query issued alone through the plain (unbatched)
    # search call, device time per request; and the batched call's speed-up
    # over issuing the same queries one by one
    lat = []
    for _ in range(0 if args.no_e2e else LATENCY_REPS):
        for b in batch:
            eng.search(b["query"], b["m"], b["cutoff"], b["metric"], b["w"], b["arg"])
            lat.append(eng.last_call_ms)
    latency = None
    if lat:
        lat_a = np.asarray(lat)
        plain_ms = float(lat_a.sum()) / LATENCY_REPS
        batched_ms = t_max_ms / args.steps
        latency = {"requests": len(lat), "p50_ms": round(float(np.percentile(lat_a, 50)), 3),
                   "p99_ms": round(float(np.percentile(lat_a, 99)), 3),
                   "plain_ms_per_step": round(plain_ms, 3), "batched_ms_per_step": round(batched_ms, 3),
                   "batched_speedup": round(plain_ms / batched_ms, 3)}
    h2d = len(target) * 8 + sum(M * 8 for _ in METRICS)

    if rank == 0:
        peaks = load_peaks()
        line = {
            "metric": "candidates/s", "value": value, "unit": "candidates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_max_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded random walks with motifs, NaN spans and flat runs; stands in for the "
                    "reference's recorded datasets)",
            "config": {"workload": WORKLOAD if not args.case else f"{args.case} query of: {WORKLOAD}",
                       "n": args.n_points or N_POINTS, "m": M, "w": W, "k": K_TOP,
                       "queries_per_step": len(metrics), "parallelism": f"{world} GPU(s), one target partition each",
                       "l2": "inputs larger than L2 (134 MB target per GPU)",
                       "cutoffs": cutoffs, "cutoffs_source": "reference k=50 distances (tests/golden/config_pins.json)",
                       "cutoffs_match_reference_pins": cutoffs_match},
            "queries_per_s": len(metrics) * world / (t_max_ms / 1e3 / args.steps),
            "roofline": roofline(stages, cells, peaks),
            "roofline_hbm": roofline_hbm(stages, geom, peaks),
            "stage_rooflines": stage_rooflines(stages, geom, len(target), peaks),
            "dominant_kernel": max(stages.items(), key=lambda kv: kv[1][0])[0],
            "stage_timing": f"{prof_steps} steps, queries one after another, CUDA events around each launch",
            "stage_ms_per_step": {k: round(v[0] / prof_steps, 4) for k, v in stages.items()},
            "e2e": {"value": e2e_value, "unit": "candidates/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "latency": latency,
            "gpu_launches": launches,
            "clocks": clk.summary(),
        }
        if world == 1 and not args.no_cpu_baseline and not args.case and (args.n_points or N_POINTS) == N_POINTS:
            line["cpu_baseline"] = cpu_baseline_single(target, queries, cutoffs)
        print(json.dumps(line))
    eng.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


C4_M, C4_W, C4_KS = 512, 26, (10, 100)


def workload_c4(args):
    """Many DTW top-k queries (m=512, w=26, k=10 and 100) over one 2^27-point
    walk with bursts: queries/s of the batched device-resident `cutoff`, with
    LB_IP per query by FFT and for the whole group as one tensor-core product
    (the rankings of the two must be identical).  A consistency check on a
    2^22-point prefix: the exact scan (every window through the DP) at the
    returned threshold must give the same k smallest (distance, index) pairs
    (the rankings against the oracle, ties included, are checked by the GPU
    tests)."""
    import torch

    from fsmeld_b200 import api
    from fsmeld_b200.synth import query_from, walk_with_bursts

    n = args.n_points or (1 << 27)
    t = walk_with_bursts(n, C4_M, seed=4)
    rng = np.random.default_rng(404)
    qs = [query_from(t, C4_M, rng)[0] for _ in range(args.queries)]
    eng = api.Engine(t)
    out = {}
    forms = {}
    for k in C4_KS:
        batch = [dict(query=q, m=C4_M, metric="dtw", w=C4_W, arg=0.0, k=k) for q in qs]
        per_form = {}
        ranks = {}
        for form in ("fft", "gemm"):
            eng.set_lb_form(form)
            eng.batch("cutoff", batch[:2])  # warm-up (workspace, statistics)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            res = eng.batch("cutoff", batch)
            wall = time.perf_counter() - t0
            dev_ms = eng.last_call_ms
            bad = [r["status"] for r in res if r["status"] != 0]
            if bad:
                raise RuntimeError(f"cutoff failed ({form}): {bad}")
            ranks[form] = [(list(r["idx"]), np.asarray(r["dist"]).view(np.int64).tolist()) for r in res]
            per_form[form] = {"device_ms": round(dev_ms, 2), "queries_per_s": len(qs) / (dev_ms / 1e3),
                              "wall_queries_per_s": len(qs) / wall,
                              "lb_survivors_mean": float(np.mean([r["counters"]["after_lb"] for r in res]))}
        if ranks["fft"] != ranks["gemm"]:
            raise RuntimeError("c4: rankings of the two LB_IP forms differ")
        best = max(per_form, key=lambda f: per_form[f]["queries_per_s"])
        out[k] = dict(per_form[best], queries=len(qs), lb_form=best,
                      mean_threshold=float(np.mean([r["counters"]["threshold"] for r in res])))
        forms[k] = per_form
    eng.set_lb_form("auto")
    # independent check on a prefix: cutoff ranking == k smallest of the exact scan at its threshold
    pre = t[:1 << 22]
    checked = 0
    with api.Engine(pre) as e2:
        for q in qs[:4]:
            for k in C4_KS:
                idx, dist, _ = e2.cutoff(q, C4_M, k, "dtw", C4_W, 0.0)
                xi, xd, _ = e2.exact(q, C4_M, float(dist[-1]), "dtw", C4_W, 0.0)
                order = np.lexsort((xi, xd))[:k]
                if not (np.array_equal(xi[order], idx) and np.array_equal(xd[order].view(np.int64),
                                                                             np.asarray(dist).view(np.int64))):
                    raise RuntimeError("cutoff ranking differs from the exact scan at its threshold")
                checked += 1
    eng.close()
    peaks = load_peaks()
    line = {"metric": "queries/s", "value": out[10]["queries_per_s"], "unit": "queries/s", "n_gpus": 1,
            "higher_is_better": True, "dtype": "f64", "data": "synthetic (seeded random walk with bursts)",
            "config": {"workload": f"c4: {len(qs)} DTW top-k queries, m={C4_M}, w={C4_W}, k=10 and k=100, "
                                   f"n={n} walk + bursts on 1% of points (N(0,5))", "n": n},
            "per_k": out, "lb_forms": forms, "rankings_identical_across_lb_forms": True,
            "rankings_checked_against_exact_scan": checked,
            "hbm_peak_gbs": peaks["hbm_gbs"]}
    print(json.dumps(line))
    return 0


C3_METRICS = [("dtw", 0.0), ("erp", 0.0), ("edr", 0.25), ("lcss", 0.25), ("msm", 0.5)]
C3_M_RANGE = (64, 1024)
C3_K = 10


def c3_queries(t, count, seed=303):
    """count queries: m uniform on [64, 1024], metrics round-robin, w = floor(0.05 m)."""
    from fsmeld_b200.synth import query_from
    rng = np.random.default_rng(seed)
    qs = []
    for i in range(count):
        m = int(rng.integers(C3_M_RANGE[0], C3_M_RANGE[1] + 1))
        metric, arg = C3_METRICS[i % len(C3_METRICS)]
        q, _ = query_from(t, m, rng)
        qs.append(dict(query=q, m=m, metric=metric, w=(m * 5) // 100, arg=arg))
    return qs


def workload_c3(args):
    """Batched mixed queries: 512 queries of uneven length (m uniform on
    [64, 1024], metrics round-robin, w = floor(0.05 m)) over one 2^26-point
    random walk, each at its own rank-10 exact distance.  queries/s of one
    batched call (fsmeld_batch) against the plain form (one fsmeld_search per
    query on the same resident target) and the plain drop-in command (one
    `fsmeld search` process per query: file read, upload, search, print; a
    sample of the queries).  The match sets of the batched and plain forms
    must be identical."""
    import torch

    from fsmeld_b200 import api
    from fsmeld_b200.synth import random_walk

    n = args.n_points or (1 << 26)
    count = args.queries if args.queries != 32 else 512
    t = random_walk(n, 3)
    qs = c3_queries(t, count)
    eng = api.Engine(t)
    if args.concurrency:
        eng.set_concurrency(args.concurrency)
    t0 = time.perf_counter()
    cres = eng.batch("cutoff", [dict(d, k=C3_K) for d in qs], capacity=C3_K)
    for d, r in zip(qs, cres):
        if r["status"] != 0:
            raise RuntimeError(f"cutoff failed: {r['status']}")
        d["cutoff"] = float(r["dist"][C3_K - 1])
    setup_s = time.perf_counter() - t0
    eng.batch("search", qs[:8])  # warm-up (workspace)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    bres = eng.batch("search", qs)
    wall_b = time.perf_counter() - t0
    dev_b = eng.last_call_ms
    t0 = time.perf_counter()
    pres = [eng.search(d["query"], d["m"], d["cutoff"], d["metric"], d["w"], d["arg"]) for d in qs]
    wall_p = time.perf_counter() - t0
    same = all(r["status"] == 0 and list(r["idx"]) == list(p[0]) for r, p in zip(bres, pres))
    if not same:
        raise RuntimeError("batched and plain match sets differ")
    cand = sum(r["counters"]["valid"] for r in bres)
    eng.close()
    # the plain drop-in: one process per query, as the reference command runs
    from fsmeld_b200.api import CLI_PATH
    sample = qs[:args.dropin_sample]
    dropin_s = None
    if sample and os.path.exists(CLI_PATH):
        with tempfile.TemporaryDirectory() as tmp:
            tp = os.path.join(tmp, "target.bin")
            t.astype("<f8").tofile(tp)
            env = dict(os.environ, FSMELD_RESULTS_CSV=os.path.join(tmp, "r.csv"), FSMELD_QUIET_MATCHES="1")
            t0 = time.perf_counter()
            for i, d in enumerate(sample):
                qp = os.path.join(tmp, f"q{i}.txt")
                np.savetxt(qp, d["query"], fmt="%.17g")
                subprocess.run([CLI_PATH, "search", tp, qp, str(d["m"]), repr(d["cutoff"]), d["metric"],
                                str(d["w"]), repr(d["arg"])], env=env, stdout=subprocess.DEVNULL, check=True)
            dropin_s = (time.perf_counter() - t0) / len(sample)
    qps_b = count / wall_b
    qps_p = count / wall_p
    line = {"metric": "queries/s", "value": qps_b, "unit": "queries/s", "n_gpus": 1, "higher_is_better": True,
            "dtype": "f64", "data": "synthetic (seeded random walk)",
            "config": {"workload": f"c3: {count} queries, m uniform on [64, 1024], metrics round-robin "
                                   f"(dtw, erp g=0, edr eps=0.25, lcss eps=0.25, msm c=0.5), w=floor(0.05 m), "
                                   f"cutoff = rank-{C3_K} exact distance, n={n} random walk",
                       "n": n, "queries": count, "distinct_m": len({d["m"] for d in qs}),
                       "concurrency": args.concurrency or DEFAULT_CONCURRENCY},
            "batched": {"queries_per_s": qps_b, "wall_s": wall_b, "device_ms": dev_b,
                        "candidates_per_s": cand / wall_b},
            "plain": {"queries_per_s": qps_p, "wall_s": wall_p},
            "batched_speedup": qps_b / qps_p,
            "plain_dropin": ({"queries_per_s": 1.0 / dropin_s, "sample": len(sample),
                              "speedup_batched_vs_dropin": qps_b * dropin_s} if dropin_s else None),
            "match_sets_identical": same, "cutoff_setup_s": setup_s}
    print(json.dumps(line))
    return 0


def workload_c5(args):
    """Serving: requests with Poisson arrivals against two resident targets
    through `fsmeld_b200.serve.Server` (continuous batching, admission by HBM
    footprint).  m log-uniform in [64, 2048], metric uniform, w uniform in
    [0, floor(0.1 m)], cutoff = the request's rank-ceil(1e-4 (n-m+1)) exact
    distance (computed before the timed run).  Reports request latency
    (submit to answer) and throughput; a sample of answers is checked against
    the same request run alone."""
    import math
    import threading

    import torch

    from fsmeld_b200 import api
    from fsmeld_b200.serve import Server
    from fsmeld_b200.synth import query_from, random_walk

    big, small = args.c5_log2
    sizes = {f"t{big}": 1 << big, f"t{small}": 1 << small}  # the stated 2^28 and 2^25 by default
    targets = {name: random_walk(n, seed=50 + i) for i, (name, n) in enumerate(sizes.items())}
    rng = np.random.default_rng(505)
    metrics = [("dtw", 0.0), ("erp", 0.0), ("edr", 0.25), ("lcss", 0.25), ("msm", 0.5)]
    reqs = []
    for _ in range(args.queries):
        name = list(sizes)[int(rng.integers(0, 2))]
        m = int(round(math.exp(rng.uniform(math.log(64), math.log(2048)))))
        metric, arg = metrics[int(rng.integers(0, 5))]
        w = int(rng.integers(0, int(0.1 * m) + 1))
        q, _ = query_from(targets[name], m, rng)
        reqs.append([name, q, m, metric, w, arg, None])
    # cutoffs: rank ceil(1e-4 (n-m+1)) distance of each request (untimed)
    t_pre = time.perf_counter()
    for name, t in targets.items():
        with api.Engine(t) as e:
            for r in reqs:
                if r[0] == name:
                    k = math.ceil(1e-4 * (len(t) - r[2] + 1))
                    _i, d, _c = e.cutoff(r[1], r[2], k, r[3], r[4], r[5])
                    r[6] = float(d[-1])
                    print(f"c5 cutoff {name} m={r[2]} w={r[4]} {r[3]} k={k}: {e.last_call_ms:.1f} ms",
                          file=sys.stderr, flush=True)
    t_pre = time.perf_counter() - t_pre
    lat = [None] * len(reqs)
    answers = [None] * len(reqs)
    with Server(device=0) as srv:
        for name, t in targets.items():
            srv.add_target(name, t)
        for r in reqs[:4]:  # warm-up: workspaces of the largest lengths come later and grow then
            srv.submit(r[0], "search", r[1], r[2], r[3], r[4], r[5], cutoff=r[6]).result()
        torch.cuda.synchronize()
        gaps = rng.exponential(1.0 / args.rate, size=len(reqs))
        done = threading.Event()
        left = [len(reqs)]
        lk = threading.Lock()

        errors = []

        def finish(i, t0):
            def cb(f):
                lat[i] = time.perf_counter() - t0
                answers[i] = f.result()[0] if f.exception() is None else None
                if f.exception() is not None and len(errors) < 5:
                    r = reqs[i]
                    errors.append(f"{r[0]} m={r[2]} w={r[4]} {r[3]}: {f.exception()}")
                with lk:
                    left[0] -= 1
                    if left[0] == 0:
                        done.set()
            return cb

        t_start = time.perf_counter()
        t_next = t_start
        for i, r in enumerate(reqs):
            t_next += gaps[i]
            delay = t_next - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            t0 = time.perf_counter()
            srv.submit(r[0], "search", r[1], r[2], r[3], r[4], r[5], cutoff=r[6]).add_done_callback(finish(i, t0))
        if not done.wait(timeout=600):
            raise RuntimeError("c5: requests still pending after 600 s")
        span = time.perf_counter() - t_start
        budget_gb = srv.budget / 1e9
    failed = sum(1 for a in answers if a is None)
    # answers in the mix against the same requests alone
    checked = 0
    for name, t in targets.items():
        with api.Engine(t) as e:
            for i, r in enumerate(reqs[: min(len(reqs), 40)]):
                if r[0] != name or answers[i] is None:
                    continue
                idx, _c = e.search(r[1], r[2], r[6], r[3], r[4], r[5])
                if not np.array_equal(idx, answers[i]):
                    raise RuntimeError(f"request {i}: answer in the mix differs from the request alone")
                checked += 1
    lat_ms = np.asarray([x for x in lat if x is not None]) * 1e3
    line = {"metric": "requests/s", "value": len(reqs) / span, "unit": "requests/s", "n_gpus": 1,
            "higher_is_better": True, "dtype": "f64", "data": "synthetic (seeded random walks)",
            "config": {"workload": f"c5 serving: {len(reqs)} search requests (a sample of the 20k-request "
                                   f"stream), Poisson arrivals at {args.rate}/s, targets 2^{big} and 2^{small} "
                                   "points resident, m log-uniform [64, 2048], metric uniform, w uniform "
                                   "[0, 0.1 m], cutoff = rank ceil(1e-4 (n-m+1)) distance",
                       "rate_per_s": args.rate, "requests": len(reqs)},
            "latency_ms": {"p50": round(float(np.percentile(lat_ms, 50)), 2),
                           "p99": round(float(np.percentile(lat_ms, 99)), 2),
                           "max": round(float(lat_ms.max()), 2)},
            "failed": failed, "failures": errors, "hbm_budget_gb": round(budget_gb, 1),
            "answers_checked_against_alone": checked,
            "cutoff_precompute_s": round(t_pre, 1)}
    print(json.dumps(line))
    return 0


def workload_stream(args):
    """Target ingestion: the headline workload's target written to a file and
    streamed through the GPU in segment-aligned chunks of at most 2^22 points
    (file read + pinned upload overlapped with the previous chunk's search),
    against the same batch on the resident target.  Candidates/s, end to end
    from the file; every answer is checked against the resident run."""
    import tempfile

    from fsmeld_b200 import api
    from fsmeld_b200.stream import StreamingTarget, chunk_plan

    target, queries = make_workload(0, args.n_points or N_POINTS)
    batch = [dict(query=queries[mt], m=M, metric=mt, w=W, arg=ag, cutoff=CUTOFFS[mt]) for mt, ag in METRICS]
    path = os.path.join(tempfile.mkdtemp(), "target.bin")
    target.astype("<f8").tofile(path)
    chunk = 1 << 22
    with api.Engine(target) as e:
        e.batch("search", batch)
        t0 = time.perf_counter()
        want = e.batch("search", batch)
        resident_s = time.perf_counter() - t0
    cand = sum(r["counters"]["valid"] for r in want)
    with StreamingTarget(path, max_points=chunk) as st:
        st.batch("search", batch)  # warm-up: engines, pinned buffers, page cache
        t0 = time.perf_counter()
        got = st.batch("search", batch)
        stream_s = time.perf_counter() - t0
    for g, w_ in zip(got, want):
        if not np.array_equal(g["idx"], w_["idx"]) or g["counters"]["after_glb"] != w_["counters"]["after_glb"]:
            raise RuntimeError("streamed search differs from the resident search")
    line = {"metric": "candidates/s", "value": cand / stream_s, "unit": "candidates/s", "n_gpus": 1,
            "higher_is_better": True, "dtype": "f64", "data": "synthetic (the headline workload's target)",
            "config": {"workload": f"five searches streamed from a {len(target)}-point target file in chunks of "
                                   f"at most {chunk} points ({len(chunk_plan(len(target), M, chunk))} chunks)",
                       "n": len(target)},
            "resident_candidates_per_s": cand / resident_s, "streamed_over_resident": resident_s / stream_s,
            "answers_checked_against_resident": len(got)}
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (profiling runs)")
    ap.add_argument("--case", choices=[m for m, _ in METRICS], help="one metric's query only (profiling runs)")
    ap.add_argument("--n-points", type=int, default=None,
                    help="target length (default: the workload's own: 2^24 search5/stream, 2^26 c3, 2^27 c4)")
    ap.add_argument("--workload", choices=["search5", "c3", "c4", "c5", "stream"], default="search5",
                    help="c3: 512 mixed queries, batched vs plain (queries/s); "
                         "c4: batched DTW top-k queries over a 2^27-point target (queries/s); "
                         "c5: serving loop with Poisson arrivals (latency)")
    ap.add_argument("--rate", type=float, default=50.0, help="c5: request arrivals per second")
    ap.add_argument("--c5-log2", type=int, nargs=2, default=(28, 25),
                    help="c5: log2 sizes of the two resident targets (stated: 28 25)")
    ap.add_argument("--queries", type=int, default=32, help="c4: number of queries (c3: 512 unless given)")
    ap.add_argument("--dropin-sample", type=int, default=8,
                    help="c3: queries timed through the plain drop-in command, one process each")
    ap.add_argument("--concurrency", type=int, default=None,
                    help="queries of the batch running at once on worker streams (default: the library's)")
    ap.add_argument("--fixed-cutoffs", action="store_true",
                    help="use the workload's cutoff constants without recomputing them (profiling runs)")
    args = ap.parse_args()
    if args.impl == "reference":
        return impl_reference(args)
    if args.workload == "c3":
        return workload_c3(args)
    if args.workload == "c4":
        return workload_c4(args)
    if args.workload == "c5":
        return workload_c5(args)
    if args.workload == "stream":
        return workload_stream(args)
    return impl_ours(args)


if __name__ == "__main__":
    sys.exit(main())
