"""The SFU-based helpers that replace CUDA's cbrtf, powf, sqrtf and IEEE division in the per-pixel
terms of FLIP, FSIM, SSIM and M-SVD (iqm_b200/csrc/iqm_internal.cuh), checked on the GPU against a
double-precision reference over seeded inputs spanning the ranges the kernels use, beside CUDA's own
functions on the same inputs (tests/native/sfu_check.cu).

Bounds (largest relative error), about twice the values measured on a B200 (helper / CUDA's function):
cube root 2e-7 (7.8e-8 / 9.3e-8; exp2(log2(v)/3) refined by one Newton-Raphson step), reciprocal 2e-7
(9.8e-8 / 6.0e-8) and square root 3e-7 (1.5e-7 / 6.0e-8), single SFU operations; power 4e-6 over
twelve decades of bases (2.0e-6 / 7.2e-8: the absolute error of the SFU log2, scaled by the
exponent); the special values pow(0, y) and sqrt(0) exact.  Each bound is far inside the 1e-5 score
tolerance that the metric tests hold."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BOUNDS = {"cbrt": 2e-7, "pow": 4e-6, "sqrt": 3e-7, "rcp": 2e-7}


@pytest.fixture(scope="module")
def sfu_results(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("native") / "sfu_check")
    subprocess.run(["/usr/local/cuda/bin/nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17",
                    "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include"),
                    "-I", os.path.join(ROOT, "iqm_b200", "csrc"), "-o", exe,
                    os.path.join(ROOT, "tests", "native", "sfu_check.cu")], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, check=True, timeout=120).stdout
    res = {}
    for line in out.splitlines():
        name, ours, cuda, exact = line.split()
        res[name] = (float(ours), float(cuda), exact == "1")
    return res


@pytest.mark.parametrize("name", sorted(BOUNDS))
def test_sfu_helper_within_bound(sfu_results, name):
    ours, cuda, exact = sfu_results[name]
    print("%s: helper %.3e, CUDA %.3e" % (name, ours, cuda))
    assert ours <= BOUNDS[name]
    assert exact
