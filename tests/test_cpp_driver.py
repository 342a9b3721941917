"""The C++ mirror of the reference's classes (include/coffee_b200.hpp): a
driver in the shape of the reference's main-alfven3d.cpp compiles and links
against libcoffee_b200.so (CPU), and on a GPU its result matches the oracle."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from coffee_b200 import problems
from coffee_b200.fld import read_fld
from helpers import fp32_parity
from oracle import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "alfven_driver.cpp")
LIBDIR = os.path.join(ROOT, "coffee_b200")


def build_driver(outdir):
    exe = os.path.join(outdir, "alfven_driver")
    cmd = ["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), SRC, "-o", exe,
           "-L", LIBDIR, "-lcoffee_b200", f"-Wl,-rpath,{LIBDIR}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_driver_compiles_and_links(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("no g++")
    exe = build_driver(str(tmp_path))
    assert os.path.exists(exe)


@pytest.mark.gpu
def test_driver_matches_oracle(tmp_path):
    exe = build_driver(str(tmp_path))
    p = problems.alfven_params(32)
    p.max_steps = 8
    p.write_toml(str(tmp_path / "config.toml"))
    r = subprocess.run([exe], cwd=str(tmp_path), capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    fin = read_fld(str(tmp_path / "in.fld"))
    fout = read_fld(str(tmp_path / "out.fld"))
    f32 = [a.copy() for a in fin.arrays]
    ref32, _ = oracle.run_port(p, f32, 8, taper_lanes=16)
    ref64, _ = oracle.run_port(p, [a.astype(np.float64) for a in f32], 8, taper_lanes=16)
    ok, rep = fp32_parity([a for a in fout.arrays], ref32, ref64)
    assert ok, rep
