"""The host FFT planner (iqm_b200/csrc/fft.cu), built into a small host program: every plan
multiplies out to its length, uses only radices the engines implement, stays within the stage
limit, and Bluestein lengths are 2,3,5-smooth and long enough; the benchmark's plane lengths keep
the radix sequences that their compiled engines (fsim.cu) expect."""
import os
import subprocess
from functools import reduce

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REG = {2, 3, 4, 5, 6, 8, 9, 10, 12, 15}


def is_prime(p):
    return p > 1 and all(p % d for d in range(2, int(p ** 0.5) + 1))


@pytest.fixture(scope="module")
def planner(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("native") / "fft_plan_check")
    csrc = os.path.join(ROOT, "iqm_b200", "csrc")
    subprocess.run(["/usr/local/cuda/bin/nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include"),
                    "-I", csrc, "-o", exe, os.path.join(ROOT, "tests", "native", "fft_plan_check.cu"),
                    os.path.join(csrc, "fft.cu")], check=True)
    return exe


def plans(exe, ns):
    out = subprocess.run([exe] + [str(n) for n in ns], capture_output=True, text=True, check=True).stdout
    res = {}
    for line in out.splitlines():
        f = line.split()
        n = int(f[0])
        if f[1] == "direct":
            res[n] = ("direct", n, [int(x) for x in f[2:]])
        else:
            res[n] = ("bluestein", int(f[2]), [int(x) for x in f[3:]])
    return res


def smooth235(m):
    for p in (2, 3, 5):
        while m % p == 0:
            m //= p
    return m == 1


def test_plans_are_valid_for_all_plane_lengths(planner):
    ns = list(range(2, 1100)) + list(np.random.Generator(np.random.PCG64(5)).integers(1100, 4097, 200))
    res = plans(planner, ns)
    assert set(res) == set(int(n) for n in ns)
    for n, (kind, length, radices) in res.items():
        assert reduce(lambda a, b: a * b, radices, 1) == length, (n, radices)
        assert len(radices) <= 16
        for p in radices:
            assert p in REG or (is_prime(p) and p <= 251), (n, p)
        if kind == "bluestein":
            assert length >= 2 * n - 1 and smooth235(length)
            assert all(p in REG for p in radices)
        else:
            assert length == n
    # odd radices first (bank-conflict-free first stage)
    for n, (kind, length, radices) in res.items():
        odd = [p & 1 for p in radices]
        assert odd == sorted(odd, reverse=True), (n, radices)


def test_benchmark_lengths_match_the_compiled_engines(planner):
    res = plans(planner, [270, 480])
    assert res[270] == ("direct", 270, [9, 3, 10])
    assert res[480] == ("direct", 480, [15, 8, 4])


def test_large_prime_lengths_use_bluestein(planner):
    res = plans(planner, [131, 263, 1999, 4093, 61])
    for n in (131, 263, 1999, 4093, 61):
        assert res[n][0] == "bluestein"
