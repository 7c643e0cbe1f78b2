"""The drop-in boundary without a GPU: the C ABI library loads and exports every
symbol include/fsmeld_cuda.h declares, and the `fsmeld` CLI validates its
arguments with the reference's messages (src/main.cpp:46-88) before any device
work."""
import ctypes
import os
import subprocess
import tempfile

import numpy as np
import pytest

from fsmeld_b200 import api
from oracle import oracle as orc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def built():
    from fsmeld_b200 import build
    build.build()
    return True


def test_library_exports_header_symbols(built):
    lib = ctypes.CDLL(api.LIB_PATH)
    names = api.exported_symbols()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert lib.fsmeld_strerror  # callable without a device


def _run(binary, args, cwd):
    p = subprocess.run([binary] + [str(a) for a in args], capture_output=True, text=True, cwd=cwd,
                       env=dict(os.environ, FSMELD_RESULTS_CSV=os.path.join(cwd, "r.csv")))
    return p.returncode, p.stdout, p.stderr


@pytest.fixture(scope="module")
def files():
    d = tempfile.mkdtemp()
    t = np.cumsum(np.random.default_rng(1).standard_normal(600))
    t.astype("<f8").tofile(os.path.join(d, "t.bin"))
    t[:50].astype("<f8").tofile(os.path.join(d, "short.bin"))
    with open(os.path.join(d, "odd.bin"), "wb") as f:
        f.write(b"\0" * 801)
    np.savetxt(os.path.join(d, "q.txt"), t[100:132], fmt="%.17g")
    with open(os.path.join(d, "flat.txt"), "w") as f:
        f.write("1 " * 40)
    with open(os.path.join(d, "bad.txt"), "w") as f:
        f.write("1 2 x 4")
    return d


CASES = [
    ([], 0),
    (["search"], 1),
    (["find", "t.bin", "q.txt", 32, 1.0, "dtw", 3, 0], 1),
    (["search", "t.bin", "q.txt", 1, 1.0, "dtw", 0, 0], 1),
    (["search", "t.bin", "q.txt", "3x", 1.0, "dtw", 0, 0], 1),
    (["search", "t.bin", "q.txt", 32, 1.0, "swale", 3, 0], 1),
    (["search", "t.bin", "q.txt", 32, 1.0, "dtw", 32, 0], 1),
    (["search", "t.bin", "q.txt", 32, 1.0, "dtw", -1, 0], 1),
    (["search", "t.bin", "q.txt", 32, 1.0, "edr", 3, -0.5], 1),
    (["search", "t.bin", "q.txt", 32, 1.0, "msm", 3, "nan"], 1),
    (["search", "short.bin", "q.txt", 32, 1.0, "dtw", 3, 0], 1),
    (["search", "odd.bin", "q.txt", 32, 1.0, "dtw", 3, 0], 1),
    (["search", "t.bin", "flat.txt", 32, 1.0, "dtw", 3, 0], 1),
    (["search", "t.bin", "bad.txt", 4, 1.0, "dtw", 1, 0], 1),
    (["search", "t.bin", "q.txt", 32, -1.0, "dtw", 3, 0], 1),
    (["search", "t.bin", "q.txt", 32, "inf", "dtw", 3, 0], 1),
    (["cutoff", "t.bin", "q.txt", 32, 0, "dtw", 3, 0], 1),
    (["cutoff", "t.bin", "q.txt", 32, 100000, "dtw", 3, 0], 1),
    (["search", "t.bin", "q.txt", 32, 1.0, "dtw", 3, 0, 5, 5], 1),
    (["search", "t.bin", "q.txt", 32, 1.0, "dtw", 3, 0, -1, 5], 1),
]


@pytest.mark.parametrize("args,rc", CASES)
def test_cli_validation(built, files, args, rc):
    code, out, err = _run(api.CLI_PATH, args, files)
    assert code == rc, (args, out, err)
    if rc:
        assert err.startswith("Error: "), err
    if orc.have_reference():
        rcode, rout, rerr = _run(orc.BIN_REF, args, files)
        assert rcode == code
        assert rerr == err
        assert rout == out  # usage text on the argument-count errors


def test_help_matches_reference(built, files):
    for flag in ([], ["--help"], ["-h"]):
        code, out, _ = _run(api.CLI_PATH, flag, files)
        assert code == 0 and out.startswith("FSMELD: exact z-normalized subsequence search")
        if orc.have_reference():
            assert out == _run(orc.BIN_REF, flag, files)[1]
