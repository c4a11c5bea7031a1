"""SSIM on the GPU through the C ABI, against the CPU oracle (FP64 and reference-faithful FP32).
Tolerance: |delta MSSIM| <= 1e-5 against both; SSIM map max |delta| <= 5e-5 per pixel."""
import ctypes

import numpy as np
import pytest

import iqm_b200
from iqm_b200 import synth

pytestmark = pytest.mark.gpu
TOL = 1e-5


@pytest.mark.parametrize("h,w", [(512, 512), (37, 45), (77, 129), (11, 11), (300, 260), (1080, 1920)])
def test_ssim_matches_oracle(rt, o64, o32, h, w):
    a, b = synth.grey_pair(h, w, config=0, pair=h % 7)
    res = iqm_b200.SSIM(rt).compute_metric(a, b)
    want64, m64 = o64.ssim(a, b, want_map=True)
    want32 = o32.ssim(a, b)
    assert abs(res.mssim - want64) <= TOL
    assert abs(res.mssim - want32) <= TOL
    assert np.abs(res.image_data - m64).max() <= 5e-5


def test_ssim_rgb_input(rt, o64):
    a, b = synth.rgb_gain_pair(200, 333, config=1, pair=2)
    assert abs(iqm_b200.SSIM(rt).compute_metric(a, b).mssim - o64.ssim(a, b)) <= TOL


@pytest.mark.parametrize("ks,sigma", [(3, 0.8), (7, 1.2), (15, 2.5), (10, 1.5)])
def test_ssim_other_windows(rt, o64, ks, sigma):
    a, b = synth.grey_pair(90, 70, config=0, pair=5)
    s = iqm_b200.SSIM(rt)
    s.kernel_size, s.sigma = ks, sigma
    assert abs(s.compute_metric(a, b).mssim - o64.ssim(a, b, kernel_size=ks, sigma=sigma)) <= TOL


def test_ssim_identical_and_constant(rt):
    a, b = synth.grey_pair(64, 64, config=0, pair=1)
    assert iqm_b200.SSIM(rt).compute_metric(b, b).mssim == pytest.approx(1.0, abs=1e-6)
    c1 = np.full((40, 50, 4), 100, np.uint8)
    c2 = np.full((40, 50, 4), 140, np.uint8)
    la, lb = 0.994 * 100 / 255, 0.994 * 140 / 255
    want = (2 * la * lb + 1e-4) / (la * la + lb * lb + 1e-4)
    assert iqm_b200.SSIM(rt).compute_metric(c1, c2).mssim == pytest.approx(want, abs=TOL)


def test_ssim_batch_uneven_matches_single(rt, o64):
    sizes = [(64, 64), (33, 130), (250, 17), (128, 300), (11, 40)]
    pairs = [synth.grey_pair(h, w, config=0, pair=i) for i, (h, w) in enumerate(sizes)]
    s = iqm_b200.SSIM(rt)
    got = s.compute_batch(pairs)
    for (a, b), g in zip(pairs, got):
        assert abs(g - o64.ssim(a, b)) <= TOL
        assert g == s.compute_metric(a, b, want_map=False).mssim  # same kernel, same order


def test_ssim_dev_unaligned_rows(rt, o64):
    torch = pytest.importorskip("torch")
    h, w = 45, 61
    a, b = synth.grey_pair(h, w, config=0, pair=9)
    # device rows 4*w + 4 bytes apart, base offset by 4 bytes: forces the scalar-load path
    pitch = 4 * w + 4
    buf = torch.zeros(2 * (h * pitch + 16), dtype=torch.uint8, device="cuda")
    host = np.zeros(buf.numel(), np.uint8)
    off_a, off_b = 4, h * pitch + 20
    for off, img in ((off_a, a), (off_b, b)):
        for y in range(h):
            host[off + y * pitch: off + y * pitch + 4 * w] = img[y].ravel()
    buf.copy_(torch.from_numpy(host))
    scores = torch.zeros(1, dtype=torch.float64, device="cuda")
    base = buf.data_ptr()
    iqm_b200.SSIM(rt).compute_dev([(base + off_a, base + off_b, w, h, pitch)], scores.data_ptr())
    rt.synchronize()
    assert abs(scores.item() - o64.ssim(a, b)) <= TOL


def test_ssim_deterministic(rt):
    a, b = synth.grey_pair(300, 400, config=0, pair=4)
    s = iqm_b200.SSIM(rt)
    v = [s.compute_metric(a, b, want_map=False).mssim for _ in range(3)]
    assert v[0] == v[1] == v[2]


def test_ssim_errors(rt):
    s = iqm_b200.SSIM(rt)
    a = np.zeros((20, 20, 4), np.uint8)
    with pytest.raises(iqm_b200.IQMError):
        s.compute_metric(a, np.zeros((20, 21, 4), np.uint8))
    s.kernel_size = 17
    with pytest.raises(iqm_b200.IQMError) as e:
        s.compute_metric(a, a)
    assert e.value.code == iqm_b200.IQM_EINVAL
    s.kernel_size = 11
    out = ctypes.c_double()
    assert rt.L.iqm_ssim(rt.h, a.ctypes.data, a.ctypes.data, 20, 20, 40, None, None,
                         ctypes.byref(out)) == iqm_b200.IQM_EINVAL  # row_bytes < 4*w
