"""Tensor-core SSIM (IQM_MIXED: split FP16 products; IQM_MIXED_FAST: single FP16 products) through
the C ABI, against the FP64 oracle.  Tolerance on MSSIM: 1e-5 for the split form, which carries
about 21 significant bits per product (inside the 1e-4 bound of the mixed-precision forms), and
2e-4 for single FP16 products: 11-bit moments and taps leave ~5e-5 on large images and up to
~1.1e-4 on small ones, where fewer pixels average the rounding.  The
per-pixel map is held to 2e-3 (split) and 5e-2 (single products) at worst and to 1e-4 / 2e-3 on
average: a single FP16 product keeps 11 bits, and low-contrast pixels divide by small variances."""
import ctypes

import numpy as np
import pytest

import iqm_b200
from iqm_b200 import synth

pytestmark = pytest.mark.gpu
TOL = 2e-4
SPLIT_TOL = 1e-5
FORMS = [(iqm_b200.IQM_MIXED, "mixed"), (iqm_b200.IQM_MIXED_FAST, "mixed_fast")]
MAP_MAX = {iqm_b200.IQM_MIXED: 2e-3, iqm_b200.IQM_MIXED_FAST: 5e-2}
MAP_MEAN = {iqm_b200.IQM_MIXED: 1e-4, iqm_b200.IQM_MIXED_FAST: 2e-3}


def ssim(rt, precision, **kw):
    s = iqm_b200.SSIM(rt)
    s.precision = precision
    for k, v in kw.items():
        setattr(s, k, v)
    return s


def check(got, want, precision):
    assert abs(got - want) <= TOL
    if precision == iqm_b200.IQM_MIXED:
        assert abs(got - want) <= SPLIT_TOL


def ramp_pair(h, w, seed=1):
    """A vertical 0..255 ramp with noise and a 3% gain: local means sweep the whole range, the
    worst case for moments taken about a per-tile shift."""
    rng = np.random.default_rng(seed)
    ramp = np.linspace(0, 255, h)[:, None] * np.ones((1, w))
    out = []
    for gain in (1.0, 0.97):
        g = np.clip(ramp * gain + rng.normal(0, 3, (h, w)), 0, 255).astype(np.uint8)
        img = np.repeat(g[..., None], 4, 2)
        img[..., 3] = 255
        out.append(np.ascontiguousarray(img))
    return out


@pytest.mark.parametrize("precision,name", FORMS)
@pytest.mark.parametrize("h,w", [(512, 512), (37, 45), (77, 129), (11, 11), (300, 260), (270, 480),
                                 (1080, 1920)])
def test_mixed_ssim_matches_oracle(rt, o64, precision, name, h, w):
    a, b = synth.grey_pair(h, w, config=0, pair=h % 7)
    res = ssim(rt, precision).compute_metric(a, b)
    want, m64 = o64.ssim(a, b, want_map=True)
    check(res.mssim, want, precision)
    err = np.abs(res.image_data.astype(np.float64) - m64)
    assert err.max() <= MAP_MAX[precision]
    assert err.mean() <= MAP_MEAN[precision]


@pytest.mark.parametrize("precision,name", FORMS)
def test_mixed_ssim_ramp(rt, o64, precision, name):
    a, b = ramp_pair(512, 384)
    check(ssim(rt, precision).compute_metric(a, b, want_map=False).mssim, o64.ssim(a, b), precision)


@pytest.mark.parametrize("precision,name", FORMS)
def test_mixed_ssim_rgb_input(rt, o64, precision, name):
    a, b = synth.rgb_gain_pair(200, 333, config=1, pair=2)
    check(ssim(rt, precision).compute_metric(a, b, want_map=False).mssim, o64.ssim(a, b), precision)


@pytest.mark.parametrize("precision,name", FORMS)
@pytest.mark.parametrize("ks,sigma", [(3, 0.8), (5, 1.0), (7, 1.2), (9, 2.0), (13, 2.0), (15, 2.5), (10, 1.5)])
def test_mixed_ssim_other_windows(rt, o64, precision, name, ks, sigma):
    a, b = synth.grey_pair(90, 170, config=0, pair=5)
    got = ssim(rt, precision, kernel_size=ks, sigma=sigma).compute_metric(a, b, want_map=False).mssim
    check(got, o64.ssim(a, b, kernel_size=ks, sigma=sigma), precision)


@pytest.mark.parametrize("precision,name", FORMS)
def test_mixed_ssim_identical_and_constant(rt, precision, name):
    a, b = synth.grey_pair(64, 96, config=0, pair=1)
    assert ssim(rt, precision).compute_metric(b, b).mssim == pytest.approx(1.0, abs=1e-6)
    c1 = np.full((40, 50, 4), 100, np.uint8)
    c2 = np.full((40, 50, 4), 140, np.uint8)
    la, lb = 0.994 * 100 / 255, 0.994 * 140 / 255
    want = (2 * la * lb + 1e-4) / (la * la + lb * lb + 1e-4)
    assert ssim(rt, precision).compute_metric(c1, c2).mssim == pytest.approx(want, abs=1e-5)


@pytest.mark.parametrize("precision,name", FORMS)
def test_mixed_ssim_batch_uneven(rt, o64, precision, name):
    sizes = [(64, 64), (33, 130), (250, 17), (128, 300), (11, 40), (700, 1300)]
    pairs = [synth.grey_pair(h, w, config=0, pair=i) for i, (h, w) in enumerate(sizes)]
    s = ssim(rt, precision)
    got = s.compute_batch(pairs)
    for (a, b), g in zip(pairs, got):
        check(g, o64.ssim(a, b), precision)
        assert g == s.compute_metric(a, b, want_map=False).mssim  # same kernel, same order


@pytest.mark.parametrize("precision,name", FORMS)
def test_mixed_ssim_dev_unaligned_rows(rt, o64, precision, name):
    torch = pytest.importorskip("torch")
    h, w = 45, 61
    a, b = synth.grey_pair(h, w, config=0, pair=9)
    pitch = 4 * w + 4  # rows 4-byte aligned only: the scalar-load path of the staging
    buf = torch.zeros(2 * (h * pitch + 16), dtype=torch.uint8, device="cuda")
    host = np.zeros(buf.numel(), np.uint8)
    off_a, off_b = 4, h * pitch + 20
    for off, img in ((off_a, a), (off_b, b)):
        for y in range(h):
            host[off + y * pitch: off + y * pitch + 4 * w] = img[y].ravel()
    buf.copy_(torch.from_numpy(host))
    scores = torch.zeros(1, dtype=torch.float64, device="cuda")
    base = buf.data_ptr()
    ssim(rt, precision).compute_dev([(base + off_a, base + off_b, w, h, pitch)], scores.data_ptr())
    rt.synchronize()
    check(scores.item(), o64.ssim(a, b), precision)


@pytest.mark.parametrize("precision,name", FORMS)
def test_mixed_ssim_deterministic(rt, precision, name):
    a, b = synth.grey_pair(300, 400, config=0, pair=4)
    s = ssim(rt, precision)
    r1 = s.compute_metric(a, b)
    r2 = s.compute_metric(a, b)
    assert r1.mssim == r2.mssim
    assert np.array_equal(r1.image_data, r2.image_data)


def test_mixed_ssim_unknown_precision_rejected(rt):
    a, b = synth.grey_pair(32, 32, config=0, pair=1)
    s = ssim(rt, 3)
    with pytest.raises(iqm_b200.IQMError) as e:
        s.compute_metric(a, b)
    assert e.value.code == iqm_b200.IQM_EINVAL


def test_noalloc_refuses_mixed(rt):
    torch = pytest.importorskip("torch")
    a, b = synth.grey_pair(64, 64, config=0, pair=1)
    da = torch.from_numpy(a).cuda()
    db = torch.from_numpy(b).cuda()
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    p = ssim(rt, iqm_b200.IQM_MIXED).params()
    L = rt.L
    rc = L.iqm_ssim_noalloc(ctypes.c_void_p(da.data_ptr()), ctypes.c_void_p(db.data_ptr()), 64, 64, 256,
                            ctypes.byref(p), None, ctypes.c_void_p(out.data_ptr()), None)
    assert rc == iqm_b200.IQM_EINVAL
