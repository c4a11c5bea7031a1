"""M-SVD on the GPU through the C ABI.  Pinned against OpenCV (the reference's own library) via
tests/golden/msvd.npz, and against the FP64 oracle.  Tolerance: relative 1e-5 on the score (the
reference itself accumulates in float, whose rounding is ~1e-6 relative at 1080p)."""
import os

import numpy as np
import pytest

import iqm_b200
from iqm_b200 import synth

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
RTOL = 1e-5


def close(a, b):
    return abs(a - b) <= RTOL * max(1.0, abs(b))


def test_msvd_matches_opencv_golden(rt):
    d = np.load(os.path.join(GOLD, "msvd.npz"))
    s = iqm_b200.SVD(rt)
    for i in range(len(d["sizes"])):
        r = s.compute_metric(d["img%d" % i], d["ref%d" % i])
        assert close(r.msvd, float(d["scores"][i])), (i, r.msvd, d["scores"][i])
        dist = d["dist%d" % i]
        mx = dist.max()
        assert np.allclose(r.image_data, dist / mx, rtol=1e-4, atol=1e-4)


@pytest.mark.parametrize("h,w", [(1080, 1920), (64, 64), (65, 65), (73, 250), (8, 8), (9, 17), (300, 47)])
def test_msvd_matches_oracle(rt, o64, o32, h, w):
    a, b = synth.rgb_blockquant_pair(h, w, config=2, pair=h % 5)
    got = iqm_b200.SVD(rt).compute_metric(a, b).msvd
    want = o64.msvd(a, b)
    assert close(got, want), (got, want)
    assert close(got, o32.msvd(a, b))


def test_msvd_identical_is_zero(rt):
    a, b = synth.rgb_blockquant_pair(96, 96, config=2, pair=3)
    assert iqm_b200.SVD(rt).compute_metric(b, b).msvd == 0.0


def test_msvd_batch_uneven(rt, o64):
    sizes = [(64, 64), (33, 130), (250, 17), (128, 300), (1080, 1920)]
    pairs = [synth.rgb_blockquant_pair(h, w, config=2, pair=i) for i, (h, w) in enumerate(sizes)]
    got = iqm_b200.SVD(rt).compute_batch(pairs)
    for (a, b), g in zip(pairs, got):
        assert close(g, o64.msvd(a, b))


def test_msvd_rejects_tiny(rt):
    a = np.zeros((7, 20, 4), np.uint8)
    with pytest.raises(iqm_b200.IQMError):
        iqm_b200.SVD(rt).compute_metric(a, a)
