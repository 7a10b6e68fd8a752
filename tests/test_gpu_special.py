"""Accuracy of the special functions the kernels build on: necg::rsq (the
hardware rsqrt approximation refined by one Householder step) and necg::rcp
(the hardware reciprocal approximation refined by one third-order step), both
in csrc/necg_math.cuh, against IEEE 1/sqrt(x) and 1/x over 2^24 inputs in
[2^-40, 2^41).  The probe is compiled from tests/probe/special_probe.cu with
the library's own header and run on the GPU."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "nbo_correlatedgaussians_b200", "csrc")


def _nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    pytest.skip("nvcc not found")


@pytest.mark.gpu
def test_rsq_rcp_accuracy(tmp_path):
    exe = str(tmp_path / "special_probe")
    subprocess.run([_nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "-I", CSRC,
                    os.path.join(HERE, "probe", "special_probe.cu"), "-o", exe], check=True,
                   capture_output=True, text=True)
    out = subprocess.run([exe], check=True, capture_output=True, text=True, timeout=120).stdout.split()
    rsq_ulp, rcp_ulp = int(out[1]), int(out[3])
    # 1/sqrt(x) and 1/x each round once or twice; the refined approximations stay
    # within a few units of them (measured: rsq 2-3, rcp 1)
    assert rsq_ulp <= 3, rsq_ulp
    assert rcp_ulp <= 1, rcp_ulp
