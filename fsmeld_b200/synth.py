"""Seeded synthetic targets and queries with the shapes of the FSMELD benchmark
configurations.

The reference's published runs use recorded datasets (ECG, TEMP, THCHS, PLA,
PLETH) that are not available here; seeded float64 random walks with injected
structure stand in for them.  Targets are native-endian IEEE-754 doubles with
no header and queries are text numbers, the reference's input conventions
(README "Input").
"""
from __future__ import annotations

import numpy as np


def random_walk(n: int, seed) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.standard_normal(n))


def query_from(target: np.ndarray, m: int, rng, noise: float = 0.1, start=None):
    """A target window plus N(0, noise) noise, avoiding non-finite or flat windows."""
    n = len(target)
    for _ in range(1000):
        s = int(rng.integers(0, n - m)) if start is None else int(start)
        w = target[s:s + m]
        if np.all(np.isfinite(w)) and np.std(w) > 1e-6:
            return w + rng.normal(0.0, noise, m), s
        start = None
    raise RuntimeError("no usable query window")


def walk_with_structure(n: int, m: int, seed, motifs: int = 200, nan_fraction: float = 1e-3,
                        flat_runs: int = 50, nan_spans: int = None) -> np.ndarray:
    """Random walk with sine/chirp motifs, NaN spans and flat (zero-variance) runs.

    Motifs: amplitude U(0.5, 3), period U(20, 400), length U(m, 4m); half are
    chirps.  NaN spans total `nan_fraction` of the points.  Flat runs have
    length U(m, 3m) and make the windows inside them invalid (sigma <= 1e-12).
    """
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.standard_normal(n))
    for k in range(motifs):
        L = int(rng.integers(m, 4 * m + 1))
        if L >= n:
            continue
        s = int(rng.integers(0, n - L))
        amp = rng.uniform(0.5, 3.0)
        period = rng.uniform(20.0, 400.0)
        x = np.arange(L, dtype=np.float64)
        if k % 2:
            f1 = period * rng.uniform(0.3, 0.9)
            phase = 2 * np.pi * (x / period + (1.0 / f1 - 1.0 / period) * x * x / (2 * L))
        else:
            phase = 2 * np.pi * x / period
        t[s:s + L] += amp * np.sin(phase)
    for _ in range(flat_runs):
        L = int(rng.integers(m, 3 * m + 1))
        if L >= n:
            continue
        s = int(rng.integers(0, n - L))
        t[s:s + L] = t[s]
    total_nan = int(round(nan_fraction * n))
    if total_nan > 0:
        spans = nan_spans if nan_spans is not None else max(1, total_nan // 100)
        per = max(1, total_nan // spans)
        for _ in range(spans):
            s = int(rng.integers(0, n - per))
            t[s:s + per] = np.nan
    return t


CONFIG_METRIC_ARGS = {"dtw": 0.0, "erp": 0.0, "edr": 0.25, "lcss": 0.25, "msm": 0.5}


def config1(n: int = 1 << 20, m: int = 128, seed: int = 1):
    """Plain DTW search: random walk, query = target window + N(0, 0.1), w = 6."""
    t = random_walk(n, seed)
    rng = np.random.default_rng(seed + 1000)
    q, s = query_from(t, m, rng)
    return t, q, {"m": m, "w": 6, "metric": "dtw", "arg": 0.0, "query_start": s}


def config2(n: int = 1 << 24, m: int = 256, seed: int = 2):
    """All five metrics at m=256, w=13 on a structured walk (motifs, NaN spans,
    flat runs, natural tail).  Returns the target and one query per metric."""
    t = walk_with_structure(n, m, seed)
    rng = np.random.default_rng(seed + 1000)
    queries = {}
    for metric in ("dtw", "erp", "edr", "lcss", "msm"):
        q, s = query_from(t, m, rng)
        queries[metric] = (q, s)
    return t, queries, {"m": m, "w": 13, "args": dict(CONFIG_METRIC_ARGS)}


def walk_with_bursts(n: int, m: int, seed, burst_fraction: float = 0.01, burst_sigma: float = 5.0) -> np.ndarray:
    """Random walk with bursts: spans of length U(m, 8m) covering `burst_fraction`
    of the points carry extra N(0, burst_sigma) noise (the top-k workload with
    k=10/100 over a 2^27-point target)."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.standard_normal(n))
    covered = 0
    while covered < burst_fraction * n:
        ln = int(rng.integers(m, 8 * m + 1))
        s = int(rng.integers(0, max(1, n - ln)))
        t[s:s + ln] += rng.normal(0.0, burst_sigma, size=min(ln, n - s))
        covered += ln
    return t
