"""The inverse-radius transport run outwards (the escape leg of star-map frames on the mixed path),
checked on the host: tests/far_transport_check.cpp compiles the package's so_kerr.cuh with g++ and
compares far_approach from r ~ 60 M to 1000 M with the Mino-time DP5(4) at tolerance 1e-13 on
escaping rays past their periapsis.  Bars: u, u' within 1e-10, phi within 1e-8 rad, t within 1e-6 M,
r' from the radial constraint equal to 1e-12, in at most 20 attempts where Mino time takes hundreds.
(The inward leg is pinned through so_approach_state in test_host_abi.py.)"""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_far_transport_outwards_matches_mino_time(tmp_path):
    exe = tmp_path / "far_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-I",
                    os.path.join(ROOT, "spacetime-optics_b200", "csrc"), "-o", str(exe),
                    os.path.join(ROOT, "tests", "far_transport_check.cpp")], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    rows = np.array([[float(v) for v in l.split()] for l in out if l and l != "skip"])
    assert len(rows) >= 10
    applies, nm, nf, dr, dpr, du, dpu, dph, dt = rows.T
    assert (applies == 1).all() and (nf > 0).all() and (nf <= 20).all() and (nm >= 300).all()
    assert dr.max() == 0.0 and dpr.max() <= 1e-12
    assert du.max() <= 1e-10 and dpu.max() <= 1e-10
    assert dph.max() <= 1e-8 and dt.max() <= 1e-6
