"""Register DFTs of the FFT engine (cmblensing_b200/csrc/lf_fft.cuh) checked on the CPU.

The radix-2..32 DFTs that every transform kernel applies in registers are
plain arithmetic, compiled here for the host by nvcc, and compared with a
direct float64 DFT on seeded random inputs, forward and inverse, in float32
and float64.
"""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.skipif(shutil.which("nvcc") is None, reason="nvcc not found")
def test_register_dfts_match_direct_dft(tmp_path):
    exe = tmp_path / "dft_check"
    subprocess.check_call(["nvcc", "-O2", "-std=c++17", "-Wno-deprecated-gpu-targets", "-o", str(exe),
                           os.path.join(HERE, "native", "dft_check.cu")])
    # float32: a few units in the last place of the rms output; float64 the same at its precision
    r = subprocess.run([str(exe), "3e-7", "1e-15"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert len(r.stdout.strip().splitlines()) == 20
