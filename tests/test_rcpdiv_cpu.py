"""The reciprocal-and-FMA division of the kernels (fsmeld_b200/csrc/rcpdiv.h)
against IEEE division on the CPU: random operands, all-ones and power-of-two
significands, quotients next to rounding boundaries and z-normalisation-like
operands must all give the bits of a / b."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc not available")
def test_rcp_division_matches_ieee(tmp_path):
    exe = tmp_path / "rcpdiv_check"
    subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-o", str(exe), os.path.join(HERE, "rcpdiv_check.c"), "-lm"],
                   check=True)
    for seed in (1, 2):
        out = subprocess.run([str(exe), "2000000", str(seed)], capture_output=True, text=True)
        assert out.returncode == 0, out.stdout
        assert out.stdout.strip().endswith("tested 24000000"), out.stdout
        assert "mismatches 0 " in out.stdout
