"""The Ozaki int8 product (jsd_ozaki.cuh) on the host: A packed by
oz_pack_a, B tiles sliced like the converter warps, the tensor-core products
emulated through the canonical-layout offsets with int32 accumulation per
diagonal, combined like the epilogue (FP64 extras for a 129th row / column),
against a long-double product. Compiles with nvcc for sm_100a; no GPU."""
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
def test_ozaki_product_is_fp64_accurate(tmp_path):
    exe = tmp_path / "ozaki_check"
    subprocess.run([_nvcc(), "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a", "-o", str(exe),
                    os.path.join(HERE, "host_kernels", "ozaki_check.cu")], check=True, capture_output=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    assert "overflow" not in out
    rows = [ln.split() for ln in out.split("\n") if ln.strip()]
    assert {(r[0], r[1]) for r in rows} == {("127", "129"), ("127", "127"), ("129", "127"), ("65", "63")}
    for m, k, emax, efro, dmax, dfro in rows:
        # relative Frobenius error within a small factor of a plain FP64 product's
        assert float(efro) < 5e-15 and float(efro) < 10 * float(dfro), (m, k, efro, dfro)
        assert float(emax) < 1e-12, (m, k, emax)
