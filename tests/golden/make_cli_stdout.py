"""Record the reference CLI's stdout and experiment-CSV rows on the golden
CLI cases (cli_cases.npz), for a line-by-line diff of the drop-in `fsmeld`
command on the GPU.

For each of the 4 targets x 6 metric/argument pairs: `cutoff k`, `search`
and `exact` at the reference's k-th distance, and `search` / `exact` with an
exclusion interval around the best match.  Paths are relative to the working
folder (`<name>.bin`, `<name>.txt`) so the dataset column of the CSV, which
the reference derives from the path, is the same for any folder.

Output: cli_stdout.json.gz.  Run from the repository root with the reference
build present (oracle/_ref):
    python tests/golden/make_cli_stdout.py
"""
from __future__ import annotations

import gzip
import json
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as orc  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "cli_stdout.json.gz")


def commands(case):
    """The argument lists run for one golden case (shared with the GPU test)."""
    name, m, w, k = case["name"], case["m"], case["w"], case["k"]
    metric, arg = case["metric"], case["arg"]
    thr = case["cutoff"]["threshold"]
    b, e = case["exclusion"]
    base = [f"{name}.bin", f"{name}.txt", str(m)]
    tail = [metric, str(w), repr(float(arg))]
    return [
        ["cutoff"] + base + [str(k)] + tail,
        ["search"] + base + [thr] + tail,
        ["exact"] + base + [thr] + tail,
        ["search"] + base + [thr] + tail + [str(b), str(e)],
        ["exact"] + base + [thr] + tail + [str(b), str(e)],
    ]


def write_inputs(z, case, folder):
    name = case["name"]
    tp, qp = os.path.join(folder, f"{name}.bin"), os.path.join(folder, f"{name}.txt")
    if not os.path.exists(tp):
        z[f"{name}_target"].astype("<f8").tofile(tp)
        np.savetxt(qp, z[f"{name}_query"], fmt="%.17g")


def main():
    if not orc.have_reference():
        raise SystemExit("oracle/_ref is not built")
    z = np.load(os.path.join(HERE, "cli_cases.npz"))
    meta = json.loads(bytes(z["meta_json"]).decode())
    out = []
    with tempfile.TemporaryDirectory() as tmp:
        for case in meta:
            write_inputs(z, case, tmp)
            for args in commands(case):
                csv = os.path.join(tmp, "results.csv")
                if os.path.exists(csv):
                    os.remove(csv)
                env = dict(os.environ, FSMELD_RESULTS_CSV="results.csv")  # relative: same text in any folder
                env.pop("FSMELD_QUIET_MATCHES", None)
                rc, so, se = orc.run_reference_cli(args, cwd=tmp, env=env)
                rows = open(csv).read().splitlines() if os.path.exists(csv) else []
                out.append({"args": args, "rc": rc, "stdout": so, "stderr": se, "csv": rows})
    with gzip.open(OUT, "wt") as f:
        json.dump(out, f)
    print(f"wrote {len(out)} runs to {OUT}")


if __name__ == "__main__":
    main()
