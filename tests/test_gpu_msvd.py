"""M-SVD on the GPU through the C ABI.  Pinned against OpenCV (the reference's own library) via
tests/golden/msvd.npz, and against the FP64 and FP32 oracle builds.

Tolerance: |delta| <= 1e-5 * max(1, |score|) + 2e-4 / sqrt(n_blocks).  The second term is the
rounding of FP32 singular values: the reference's cv::SVD runs in float on blocks whose largest
singular value reaches ~2040 (ulp ~1.2e-4), so two correct FP32 SVDs differ by ~1e-4 in D; the
score is a mean over n blocks, which averages those differences down by ~sqrt(n)."""
import os

import numpy as np
import pytest

import iqm_b200
from iqm_b200 import synth

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
RTOL = 1e-5


def close(a, b, nblocks=1):
    return abs(a - b) <= RTOL * max(1.0, abs(b)) + 2e-4 / np.sqrt(max(1, nblocks))


def computed_blocks(h, w):
    return max(0, (w - 1) // 8) * max(0, (h - 1) // 8)


def test_msvd_matches_opencv_golden(rt):
    d = np.load(os.path.join(GOLD, "msvd.npz"))
    s = iqm_b200.SVD(rt)
    for i in range(len(d["sizes"])):
        r = s.compute_metric(d["img%d" % i], d["ref%d" % i])
        h, w = d["sizes"][i]
        assert close(r.msvd, float(d["scores"][i]), computed_blocks(h, w)), (i, r.msvd, d["scores"][i])
        dist = d["dist%d" % i]
        mx = dist.max()
        assert np.allclose(r.image_data, dist / mx, rtol=1e-4, atol=1e-4)


@pytest.mark.parametrize("h,w", [(1080, 1920), (64, 64), (65, 65), (73, 250), (8, 8), (9, 17), (300, 47)])
def test_msvd_matches_oracle(rt, o64, o32, h, w):
    a, b = synth.rgb_blockquant_pair(h, w, config=2, pair=h % 5)
    got = iqm_b200.SVD(rt).compute_metric(a, b).msvd
    want = o64.msvd(a, b)
    n = computed_blocks(h, w)
    assert close(got, want, n), (got, want)
    assert close(got, o32.msvd(a, b), n)


def test_msvd_identical_is_zero(rt):
    a, b = synth.rgb_blockquant_pair(96, 96, config=2, pair=3)
    assert iqm_b200.SVD(rt).compute_metric(b, b).msvd == 0.0


def test_msvd_batch_uneven(rt, o64):
    sizes = [(64, 64), (33, 130), (250, 17), (128, 300), (1080, 1920)]
    pairs = [synth.rgb_blockquant_pair(h, w, config=2, pair=i) for i, (h, w) in enumerate(sizes)]
    got = iqm_b200.SVD(rt).compute_batch(pairs)
    for (a, b), g, (h, w) in zip(pairs, got, sizes):
        assert close(g, o64.msvd(a, b), computed_blocks(h, w))


def test_msvd_rejects_tiny(rt):
    a = np.zeros((7, 20, 4), np.uint8)
    with pytest.raises(iqm_b200.IQMError):
        iqm_b200.SVD(rt).compute_metric(a, a)


def test_msvd_constant_blocks_known_answer(rt, o64):
    """A block of one grey value v is the rank-1 matrix v 1 1^T: singular values (8 v, 0, ..., 0).
    Two images of constant blocks a_ij and b_ij therefore have D_ij = 8 |a_ij - b_ij| on every
    computed block (the last block row and column of a size that is a multiple of 8 are not
    computed), and the map is D / max D."""
    nb = 8
    i, j = np.meshgrid(np.arange(nb), np.arange(nb), indexing="ij")
    a = 10 + 3 * i + 5 * j
    b = a + (i * j) % 4 + (i == 2) * 7
    def image(v):
        g = np.repeat(np.repeat(v.astype(np.uint8), 8, 0), 8, 1)
        img = np.repeat(g[..., None], 4, 2)
        img[..., 3] = 255
        return np.ascontiguousarray(img)
    A, B = image(a), image(b)
    res = iqm_b200.SVD(rt).compute_metric(A, B)
    d = 8.0 * np.abs(a - b).astype(np.float64)
    d[nb - 1, :] = 0.0
    d[:, nb - 1] = 0.0
    assert np.allclose(res.image_data.reshape(nb, nb), d / d.max(), atol=2e-5)
    want = o64.msvd(A, B)
    assert abs(res.msvd - want) <= 1e-5 * max(1.0, abs(want))
