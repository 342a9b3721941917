"""The division by 12 of the reference-arithmetic kernels is the IEEE
quotient for every finite float outside 0 < |t| < 2^-124 (where the kernels
use the IEEE division instead), and the kernels' integer test of that range
agrees with the floating-point one: an exhaustive check of all 2^32 bit
patterns, compiled here from tests/c/div12_check.c."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_div12_fast_path_is_ieee_outside_the_tiny_range(tmp_path):
    exe = str(tmp_path / "div12_check")
    subprocess.run(["gcc", "-O3", "-march=native", "-fopenmp", "-ffp-contract=off", "-fno-fast-math",
                    os.path.join(HERE, "c", "div12_check.c"), "-o", exe, "-lm"], check=True)
    out = subprocess.run([exe], check=True, capture_output=True, text=True, timeout=600).stdout
    words = out.split()
    outside, inside, key = int(words[1]), int(words[3]), int(words[5])
    assert outside == 0, out
    assert key == 0, out  # the kernels' integer test of the range is exact
    assert inside > 0  # the tiny range does need the IEEE division
