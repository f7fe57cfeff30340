"""The register-resident square FFT (jsd_fftsq.cuh) on the host: prime-factor
S-point DFTs and the two-stage S*S transform, lanes emulated one after another,
and the half-split form (a line on 2 S lanes), against a direct DFT in long
double. Compiles host code with nvcc; no GPU."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def _nvcc():
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    return None


@pytest.mark.skipif(_nvcc() is None, reason="nvcc not available")
def test_square_fft_matches_direct_dft(tmp_path):
    exe = tmp_path / "fftsq_check"
    subprocess.run([_nvcc(), "-std=c++17", "-O2", "-Wno-deprecated-gpu-targets", "-o", str(exe),
                    os.path.join(HERE, "host_kernels", "fftsq_check.cu")], check=True, capture_output=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    rows = [ln.split() for ln in out if ln.strip()]
    sizes = {r[0] for r in rows}
    assert {str(s) for s in (2, 3, 4, 5, 6, 7, 8, 10, 12, 14, 15, 20, 21, 24, 28, 30)} <= sizes
    assert {"h4", "h6", "h8", "h10", "h14"} <= sizes  # half-split forms
    for s, fwd, inv in rows:
        assert float(fwd) < 1e-14 and float(inv) < 1e-14, (s, fwd, inv)
