"""The drop-in `fsmeld` command against the reference CLI's own stdout and
experiment CSV, line by line (needs a B200).

tests/golden/cli_stdout.json.gz holds what the reference printed for the
golden CLI cases (4 targets x 6 metric/argument pairs x cutoff, search,
exact, search and exact with an exclusion interval; made by
tests/golden/make_cli_stdout.py).  The drop-in runs the same argument lists
in a folder holding the same files.  Every line must be identical except:

* timings: `LP_IP Lower Bound Time taken: ...` (twice), `T_LB: ...`,
  `T_total: ...`, and the CSV columns lb_time, total_time, lbip_time and
  timestamp;
* the `cutoff` command's pruning counters (`Pruned by LBIP`, `Pruned by
  GLB`, `Exact distances computed`): the device selects the top k with its
  own bound (the k-th smallest distance among per-segment seeds) instead of
  the reference's running heap threshold, so it prunes a different number of
  candidates on the way to the same ranking and threshold;
* on targets that contain NaN, the LB_IP and GLB survivor counts and the
  rates derived from them (`kk2=`, `Candidates after LP/IP`, `Candidates
  after GLB`, both `Pruning Power` lines, the CSV's pruned_candidates,
  pruning_rate, survivors, lbip_pruning_rate): the reference sorts envelope
  cores that contain NaN with std::sort, whose order is unspecified there,
  so its per-segment LB_IP thresholds in those segments are not
  reproducible (match sets never depend on them).
"""
import gzip
import json
import os
import subprocess

import numpy as np
import pytest

from fsmeld_b200 import api as fapi

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TIMING_PREFIXES = ("LP_IP Lower Bound Time taken:", "T_LB:", "T_total:")
CUTOFF_DEVICE_COUNTERS = ("  - Pruned by LBIP:", "  - Pruned by GLB:", "  - Exact distances computed:")
CSV_TIMING_COLUMNS = ("lb_time", "total_time", "lbip_time", "timestamp")
NAN_TARGET_COUNTERS = ("kk2=", "Candidates after LP/IP:", "Candidates after GLB:", "Pruning Power (guolv)=",
                       "Pruning Power (guolv2)=")
NAN_TARGET_CSV_COLUMNS = ("pruned_candidates", "pruning_rate", "survivors", "lbip_pruning_rate")


def _lines(text, cmd, nan_target):
    out = []
    for ln in text.splitlines():
        if ln.startswith(TIMING_PREFIXES):
            continue
        if cmd == "cutoff" and ln.startswith(CUTOFF_DEVICE_COUNTERS):
            continue
        if nan_target and ln.startswith(NAN_TARGET_COUNTERS):
            continue
        out.append(ln)
    return out


def _csv_rows(rows, header, nan_target):
    cols = header.split(",")
    drop = {cols.index(c) for c in CSV_TIMING_COLUMNS + (NAN_TARGET_CSV_COLUMNS if nan_target else ())}
    return [[v for i, v in enumerate(r.split(",")) if i not in drop] for r in rows]


def _strip_csv_line(ln, header, nan_target):
    if ln.startswith("EXPERIMENT_CSV="):
        return "EXPERIMENT_CSV=" + ",".join(_csv_rows([ln[len("EXPERIMENT_CSV="):]], header, nan_target)[0])
    return ln


@pytest.fixture(scope="module")
def runs(tmp_path_factory):
    fapi.lib()
    assert os.path.exists(fapi.CLI_PATH), "the fsmeld command is not built"
    with gzip.open(os.path.join(GOLDEN, "cli_stdout.json.gz"), "rt") as f:
        ref = json.load(f)
    z = np.load(os.path.join(GOLDEN, "cli_cases.npz"))
    folder = tmp_path_factory.mktemp("cli")
    nan_targets = set()
    for name in {r["args"][1][:-4] for r in ref}:
        z[f"{name}_target"].astype("<f8").tofile(folder / f"{name}.bin")
        np.savetxt(folder / f"{name}.txt", z[f"{name}_query"], fmt="%.17g")
        if np.isnan(z[f"{name}_target"]).any():
            nan_targets.add(name)
    return ref, folder, nan_targets


def test_cli_stdout_and_csv_match_reference(runs):
    ref, folder, nan_targets = runs
    header = None
    for r in ref:
        for ln in r["stdout"].splitlines():
            if ln.startswith("EXPERIMENT_CSV_HEADER="):
                header = ln[len("EXPERIMENT_CSV_HEADER="):]
    assert header
    diffs = []
    for r in ref:
        csv = folder / "results.csv"
        if csv.exists():
            csv.unlink()
        env = dict(os.environ, FSMELD_RESULTS_CSV="results.csv", FSMELD_DEVICE="0")
        env.pop("FSMELD_QUIET_MATCHES", None)
        p = subprocess.run([fapi.CLI_PATH] + r["args"], cwd=folder, env=env, capture_output=True, text=True,
                           timeout=300)
        cmd = r["args"][0]
        nt = r["args"][1][:-4] in nan_targets
        assert p.returncode == r["rc"], (r["args"], p.stderr)
        got = [_strip_csv_line(ln, header, nt) for ln in _lines(p.stdout, cmd, nt)]
        want = [_strip_csv_line(ln, header, nt) for ln in _lines(r["stdout"], cmd, nt)]
        if got != want:
            first = next(i for i in range(min(len(got), len(want)) + 1)
                         if i >= min(len(got), len(want)) or got[i] != want[i])
            diffs.append((r["args"], first, want[first:first + 3], got[first:first + 3]))
        rows = csv.read_text().splitlines() if csv.exists() else []
        if _csv_rows(rows, header, nt) != _csv_rows(r["csv"], header, nt):
            diffs.append((r["args"], "csv", r["csv"], rows))
    assert not diffs, diffs[:5]
