"""CPU tests of the oracle: golden vectors (OpenCV, the reference's own library), known-answer
properties of each metric, and FP32-vs-FP64 agreement."""
import os

import numpy as np
import pytest

from iqm_b200 import synth

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_gray_matches_opencv(o64):
    d = np.load(os.path.join(GOLD, "gray.npz"))
    rgba = d["rgba"]
    r, g, b = [rgba[:, i].astype(np.uint32) for i in range(3)]
    mine = np.array([o64.L.oracle_gray_u8(int(x), int(y), int(z)) for x, y, z in zip(r, g, b)])
    assert np.array_equal(mine, d["gray"].astype(np.int64))


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_svd8_matches_opencv(prec, o32, o64):
    o = o32 if prec == "f32" else o64
    d = np.load(os.path.join(GOLD, "svd8.npz"))
    for blk, sv in zip(d["blocks"], d["sv"]):
        mine = o.svd8(blk)
        # OpenCV computes in float: agreement to float rounding of values up to ~2040
        assert np.allclose(mine, sv, rtol=2e-6, atol=1e-3), (mine, sv)


def test_msvd_matches_opencv_pipeline(o32, o64):
    d = np.load(os.path.join(GOLD, "msvd.npz"))
    for i in range(len(d["sizes"])):
        a, b = d["img%d" % i], d["ref%d" % i]
        ref_score = float(d["scores"][i])
        s32, dist = o32.msvd(a, b, want_dist=True)
        assert abs(s32 - ref_score) <= 1e-5 * max(1.0, abs(ref_score))
        assert abs(o64.msvd(a, b) - ref_score) <= 1e-5 * max(1.0, abs(ref_score))
        # per-block distances: float rounding of singular values up to ~2040 (ulp 1.2e-4)
        assert np.allclose(dist, d["dist%d" % i], rtol=1e-5, atol=5e-4)


def test_oracle_regression_anchors(o32, o64):
    d = np.load(os.path.join(GOLD, "scores.npz"))
    for j, metric in enumerate(d["metrics"]):
        a, b = d["img%d" % j], d["ref%d" % j]
        if metric == "ssim":
            v64, v32 = [o64.ssim(a, b)], [o32.ssim(a, b)]
        elif metric == "fsim":
            v64, v32 = list(o64.fsim(a, b)), list(o32.fsim(a, b))
        else:
            v64, v32 = [o64.flip(a, b, ppd=67.0)], [o32.flip(a, b, ppd=67.0)]
        assert np.allclose(v64, d["f64_%d" % j], rtol=0, atol=1e-12)
        assert np.allclose(v32, d["f32_%d" % j], rtol=0, atol=1e-7)
        # reference-faithful FP32 restatement within the parity tolerance of FP64
        assert np.allclose(v32, v64, rtol=0, atol=1e-5)


def test_fft_matches_numpy(o64, o32):
    rng = np.random.default_rng(3)
    for h, w in [(8, 8), (27, 40), (30, 48), (67, 131), (263, 17)]:
        z = rng.standard_normal((h, w)) + 1j * rng.standard_normal((h, w))
        ref = np.fft.fft2(z)
        assert np.abs(o64.fft2(z) - ref).max() < 1e-9 * np.abs(ref).max()
        assert np.abs(o32.fft2(z) - ref).max() < 2e-5 * np.abs(ref).max()
        inv = o64.fft2(ref, sign=+1, normalize=True)
        assert np.abs(inv - z).max() < 1e-10


def test_identical_pairs(o64):
    a, b = synth.rgb_gain_pair(96, 120, config=1, pair=7)
    assert o64.ssim(b, b) == pytest.approx(1.0, abs=1e-12)
    f, fc = o64.fsim(b, b)
    assert f == pytest.approx(1.0, abs=1e-12) and fc == pytest.approx(1.0, abs=1e-12)
    assert o64.msvd(b, b) == 0.0
    assert o64.flip(b, b) == 0.0


def test_ssim_constant_images(o64):
    # constant images: variances vanish, SSIM = (2 mu_a mu_b + C1)/(mu_a^2 + mu_b^2 + C1)
    a = np.full((40, 50, 4), 100, np.uint8)
    b = np.full((40, 50, 4), 140, np.uint8)
    la, lb = 0.994 * 100 / 255, 0.994 * 140 / 255
    c1 = 0.01 ** 2
    want = (2 * la * lb + c1) / (la * la + lb * lb + c1)
    assert o64.ssim(a, b) == pytest.approx(want, rel=1e-9)


def test_ssim_small_sizes_pool_count(o64):
    # pooled region is x, y in [5, dim-5] inclusive (src/gpu/ssim/ssim.cpp:386-401)
    a, b = synth.grey_pair(20, 23, config=0, pair=3)
    v, m = o64.ssim(a, b, want_map=True)
    assert v == pytest.approx(m[5:16, 5:19].astype(np.float64).mean(), rel=1e-6)


def test_msvd_skips_last_block_row_and_column_on_multiples_of_8(o64):
    a, b = synth.rgb_blockquant_pair(64, 64, config=2, pair=1)
    _, d = o64.msvd(a, b, want_dist=True)
    assert np.all(d[-1, :] == 0) and np.all(d[:, -1] == 0)
    a, b = synth.rgb_blockquant_pair(65, 65, config=2, pair=1)
    _, d = o64.msvd(a, b, want_dist=True)
    assert np.all(d[-1, :] > 0) and np.all(d[:, -1] > 0)


def test_fsim_downscale_factor(o64):
    # F = max(1, round(min(W, H) / 256)) (src/gpu/fsim/fsim.cpp:165-168)
    assert o64.L.oracle_fsim_downscale_factor(1920, 1080) == 4
    assert o64.L.oracle_fsim_downscale_factor(3840, 2160) == 8
    assert o64.L.oracle_fsim_downscale_factor(300, 2048) == 1
    assert o64.L.oracle_fsim_downscale_factor(100, 100) == 1
    from oracle import fsim_plane_size
    assert fsim_plane_size(1920, 1080, 4) == (480, 270)
    assert fsim_plane_size(1001, 385, 2) == (501, 193)  # roundf: half away from zero


def test_fsim_energy_modes_differ(o64):
    em, an2_ref, aiaj_ref = o64.fsim_constants(64, 48, energy_full=False)
    _, an2_full, aiaj_full = o64.fsim_constants(64, 48, energy_full=True)
    assert np.all(em > 0)
    assert np.all(an2_full >= an2_ref) and not np.allclose(an2_full, an2_ref)


def test_flip_ppd_and_taps(o64):
    ppd = o64.flip_ppd(2560, 0.7, 0.6)
    assert ppd == pytest.approx(0.7 * (2560 / 0.6) * np.pi / 180)
    t = o64.flip_feature_taps(67.0)
    assert t.shape == (3, 19)
    assert t[0].sum() == pytest.approx(1.0)
    for c in (1, 2):
        assert t[c][t[c] > 0].sum() == pytest.approx(1.0)
        assert -t[c][t[c] < 0].sum() == pytest.approx(1.0)


def _opencv_mssim(img, ref, ks=11, sigma=1.5, k1=0.01, k2=0.03):
    """MSSIM built from OpenCV's Gaussian kernel and filtering (the classic OpenCV SSIM recipe) with
    the reference's luma weights (shaders/ssim/ssim_lumapack.glsl: 0.299, 0.581, 0.114 on unorm RGB)
    and pooled region x, y in [r, dim - r] (src/gpu/ssim/ssim.cpp:386-401).  Inside x, y < dim - r
    every window lies in the image (OpenCV's filtering applies unchanged); the last pooled column and
    row are computed directly with the reference's truncated, renormalised window."""
    import cv2

    def luma(x):
        x = x.astype(np.float64) / 255.0
        return 0.299 * x[..., 0] + 0.581 * x[..., 1] + 0.114 * x[..., 2]

    a, b = luma(img), luma(ref)
    g = cv2.getGaussianKernel(ks, sigma, cv2.CV_64F)
    blur = lambda x: cv2.sepFilter2D(x, cv2.CV_64F, g, g, borderType=cv2.BORDER_REFLECT)
    mu_a, mu_b = blur(a), blur(b)
    var_a = blur(a * a) - mu_a * mu_a
    var_b = blur(b * b) - mu_b * mu_b
    cov = blur(a * b) - mu_a * mu_b
    c1, c2 = k1 * k1, k2 * k2
    m = ((2 * mu_a * mu_b + c1) * (2 * cov + c2)) / ((mu_a ** 2 + mu_b ** 2 + c1) * (var_a + var_b + c2))
    r = ks // 2
    h, w = a.shape
    # The pooled region's last column (x = w - r) and row (y = h - r) have windows that reach one
    # pixel past the image; there the reference truncates the window and renormalises its weights.
    g1 = g[:, 0]
    for y in range(r, h - r + 1):
        for x in range(r, w - r + 1):
            if x < w - r and y < h - r:
                continue
            ys, xs = slice(max(0, y - r), min(h, y + r + 1)), slice(max(0, x - r), min(w, x + r + 1))
            wy = g1[ys.start - (y - r): ys.stop - (y - r)]
            wx = g1[xs.start - (x - r): xs.stop - (x - r)]
            wt = np.outer(wy, wx)
            wt = wt / wt.sum()
            pa, pb = a[ys, xs], b[ys, xs]
            ma, mb = (wt * pa).sum(), (wt * pb).sum()
            va, vb = (wt * (pa - ma) ** 2).sum(), (wt * (pb - mb) ** 2).sum()
            cv = (wt * (pa - ma) * (pb - mb)).sum()
            m[y, x] = ((2 * ma * mb + c1) * (2 * cv + c2)) / ((ma * ma + mb * mb + c1) * (va + vb + c2))
    return float(m[r:h - r + 1, r:w - r + 1].mean())


@pytest.mark.parametrize("h,w,ks,sigma", [(64, 80, 11, 1.5), (97, 131, 11, 1.5), (512, 512, 11, 1.5), (70, 90, 7, 1.2)])
def test_ssim_matches_opencv_gaussian_ssim(o64, o32, h, w, ks, sigma):
    """Pins the SSIM restatement to an independent third-party Gaussian filter (OpenCV 4.13)."""
    a, b = synth.rgb_gain_pair(h, w, config=0, pair=w % 5)
    want = _opencv_mssim(a, b, ks=ks, sigma=sigma)
    assert abs(o64.ssim(a, b, kernel_size=ks, sigma=sigma) - want) <= 1e-9
    assert abs(o32.ssim(a, b, kernel_size=ks, sigma=sigma) - want) <= 1e-5


# ---- second, independent restatement (oracle/np_restatement.py): whole-plane numpy from the shaders
@pytest.fixture(scope="module")
def npr():
    import np_restatement
    return np_restatement


@pytest.mark.parametrize("h,w", [(96, 128), (270, 480), (1080, 1920), (57, 61), (131, 263), (263, 131),
                                 (2160, 3840), (300, 2048)])
@pytest.mark.parametrize("energy_full", [False, True])
def test_fsim_two_restatements_agree(o64, npr, h, w, energy_full):
    """FSIM/FSIMc of the C oracle and of the independent numpy restatement: every shader read twice
    (downscale F = 1, 4, 8 and odd plane sizes for the integer n/2 frequency grid, both ways of
    pooling the noise-energy estimates)."""
    a, b = synth.rgb_gain_pair(h, w, config=1, pair=7)
    want = npr.fsim(a, b, energy_full=energy_full)
    got = o64.fsim(a, b, energy_full=energy_full)
    assert np.abs(np.asarray(got) - np.asarray(want)).max() <= 1e-9, (got, want)


def test_fsim_restatements_agree_on_size_constants(o64, npr):
    for w2, h2 in ((480, 270), (61, 57), (131, 263)):
        H = npr.fsim_filters(w2, h2)
        for full in (False, True):
            em, an2, aiaj = npr.fsim_noise_constants(H, full)
            cem, can2, caiaj = o64.fsim_constants(w2, h2, full)
            assert np.allclose(em, cem, rtol=1e-12) and np.allclose(an2, can2, rtol=1e-9)
            assert np.allclose(aiaj, caiaj, rtol=1e-9, atol=1e-9 * np.abs(can2).max())


@pytest.mark.parametrize("h,w", [(96, 128), (131, 263), (270, 480)])
@pytest.mark.parametrize("ppd", [67.0, 52.127, 37.0])
def test_flip_two_restatements_agree(o64, npr, h, w, ppd):
    """Mean FLIP of the C oracle and of the independent numpy restatement."""
    a, b = synth.rgb_blockquant_pair(h, w, config=2, pair=1)
    assert abs(o64.flip(a, b, ppd=ppd) - npr.flip(a, b, ppd)) <= 1e-9


def test_flip_ppd_two_restatements_agree(o64, npr):
    for r, d, wd in ((2560, 0.7, 0.6), (3840, 0.7, 0.7), (1920, 0.5, 0.53)):
        assert npr.flip_ppd(r, d, wd) == o64.flip_ppd(r, d, wd)
