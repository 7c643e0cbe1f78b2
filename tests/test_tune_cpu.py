"""The tuning table's host side: the committed table follows the grammar the
library parses (fsmeld_set_tuning: `kind metric m_k limit choice`, `#`
comments), the margin rule keeps the built-in form unless the other one
measured 5% faster, and a table rebuilt from a measurement log keeps the
rules of the committed one."""
import os
import re

from fsmeld_b200 import api, tune

KINDS = {"dp": ("lane", "wave"), "dpx": ("lane", "wave"), "lb": ("fft", "gemm"), "lbk": ("fft", "gemm")}
METRICS = {"dtw", "erp", "edr", "lcss", "msm"}


def _rules(text):
    out = []
    for ln in text.splitlines():
        body = ln.split("#", 1)[0].strip()
        if not body:
            continue
        kind, metric, mk, lim, choice = body.split()
        out.append((kind, metric, int(mk), int(lim), choice))
    return out


def test_committed_table_grammar():
    assert os.path.exists(api.TUNE_TABLE)
    with open(api.TUNE_TABLE) as f:
        rules = _rules(f.read())
    assert rules
    for kind, metric, mk, lim, choice in rules:
        assert kind in KINDS and metric in METRICS and choice in KINDS[kind]
        assert mk >= 64 and mk & (mk - 1) == 0  # macro-segment lengths are powers of two
        assert lim >= 0


def test_margin_rule():
    assert tune.choose("dp", {"lane": 1.0, "wave": 0.96}) == "lane"
    assert tune.choose("dp", {"lane": 1.0, "wave": 0.94}) == "wave"
    assert tune.choose("lb", {"fft": 10.0, "gemm": 9.6}) == "fft"
    assert tune.choose("lbk", {"fft": 10.0, "gemm": 9.0}) == "gemm"
    assert tune.choose("dpx", {"lane": 1.0, "wave": 2.0}) == "lane"


def test_table_from_log(tmp_path):
    log = tmp_path / "tune.log"
    log.write_text("\n".join([
        "dp dtw m=128 w=6: lane 1.40 ms, wave 1.03 ms -> wave",
        "dpx dtw m=128 w=6: lane 0.82 ms, wave 0.65 ms -> wave",
        "dp msm m=128 w=6: lane 1.96 ms, wave 3.43 ms -> lane",
        "lb dtw m=128 q=8: fft 7.64 ms, gemm 5.90 ms -> gemm",
        "lb dtw m=128 q=32: fft 28.01 ms, gemm 12.97 ms -> gemm",
        "lbk msm m=128 q=8: fft 65.17 ms, gemm 66.19 ms -> fft",
        "lbk msm m=128 q=32: fft 242.07 ms, gemm 237.37 ms -> gemm",
        "some other line",
    ]) + "\n")
    dp, lb = tune.rules_from_log(str(log))
    out = tmp_path / "table.txt"
    tune.write_table(str(out), dp, lb)
    rules = _rules(out.read_text())
    assert ("dp", "dtw", 1024, 6, "wave") in rules
    assert ("dpx", "dtw", 1024, 6, "wave") in rules
    assert ("dp", "msm", 1024, 6, "lane") in rules
    assert ("lb", "dtw", 1024, 8, "gemm") in rules  # the product wins from 8 queries on
    # top-k MSM: the product is within the margin at 32 queries and slower at 8
    assert not [r for r in rules if r[0] == "lbk" and r[1] == "msm"]
    assert re.search(r"# lbk msm 1024: fft at every measured size", out.read_text())
