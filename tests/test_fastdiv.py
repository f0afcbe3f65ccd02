"""The FFT kernels divide shared-memory indices by block-uniform divisors with
a multiply-high (fast_div / fdiv in csrc/fft_smem.cuh).  fastdiv_check.c
restates both forms of the multiplier (the device's rounded-up
single-precision reciprocal and the host's integer one) and checks every
divisor 2..65000 against every dividend below 2^16 (CPU, gcc)."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc not available")
def test_fastdiv_exact_for_every_divisor_and_dividend(tmp_path):
    exe = str(tmp_path / "fastdiv_check")
    cmd = ["gcc", "-O2", "-frounding-math", "-fopenmp", os.path.join(HERE, "fastdiv_check.c"), "-o", exe, "-lm"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:   # no OpenMP runtime: build the serial form
        cmd.remove("-fopenmp")
        r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([exe, "65000"], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.strip() == "ok 64999"
