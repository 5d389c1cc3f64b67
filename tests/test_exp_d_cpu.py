"""The FP64 exponential of the Tersoff pair terms (exp_d.cuh) on the host.

The batched Tersoff kernels evaluate fr = cr e^{-lr t} and fa = ca e^{-la t} with it; the
same source compiles for the host, where this test builds it with g++ (FMA contraction off,
so every fma in the source is the only fused operation) and checks the relative error
against the exponential in long double."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")
def test_exp_d_error_bound(tmp_path):
    exe = str(tmp_path / "exp_d_check")
    subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-o", exe,
                    os.path.join(HERE, "exp_d_check.cpp")], check=True)
    out = subprocess.run([exe, "2000000"], capture_output=True, text=True, check=True).stdout.split()
    n, max_rel, mean_rel, bad, max10 = int(out[0]), float(out[1]), float(out[2]), int(out[3]), float(out[4])
    max9c = float(out[5])
    assert n == 2000000
    assert max_rel <= 3e-16, max_rel      # measured 1.4e-16 (about one unit in the last place)
    assert mean_rel <= 1e-16, mean_rel    # measured 4e-17
    assert bad == 0
    assert max10 <= 4e-13, max10          # degree 10: truncation 2.3e-13
    assert max9c <= 1.2e-11, max9c        # exp_d_clamped, degree 9: truncation 7.3e-12
