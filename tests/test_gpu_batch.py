"""Batches over several metrics (iqm_batch) and CUDA-graph batch plans (iqm_batch_plan_*), against
the per-metric entry points (bit-exact) and the FP64 oracle (|delta| <= 1e-5)."""
import numpy as np
import pytest

import iqm_b200
from iqm_b200 import synth

pytestmark = pytest.mark.gpu
TOL = 1e-5
ALL = iqm_b200.METRIC_SSIM | iqm_b200.METRIC_FSIM | iqm_b200.METRIC_FLIP | iqm_b200.METRIC_MSVD


def _pairs(sizes, seed_pair=0):
    return [synth.rgb_blockquant_pair(h, w, config=2, pair=seed_pair + i) for i, (w, h) in enumerate(sizes)]


def test_batch_all_metrics_equals_single_metric_calls(rt):
    sizes = [(128, 96), (301, 170), (64, 64), (480, 270), (97, 211)]
    pairs = _pairs(sizes)
    got = iqm_b200.batch(rt, ALL, pairs)
    assert np.array_equal(got["ssim"], iqm_b200.SSIM(rt).compute_batch(pairs))
    assert np.array_equal(got["fsim"], np.asarray(iqm_b200.FSIM(rt).compute_batch(pairs)).reshape(-1, 2))
    assert np.array_equal(got["flip"], iqm_b200.FLIP(rt).compute_batch(pairs))
    assert np.array_equal(got["msvd"], iqm_b200.SVD(rt).compute_batch(pairs))


def test_batch_rejects_bad_mask(rt):
    a = np.zeros((32, 32, 4), np.uint8)
    with pytest.raises(iqm_b200.IQMError):
        iqm_b200.batch(rt, 0, [(a, a)])
    with pytest.raises(iqm_b200.IQMError):
        iqm_b200.batch(rt, 16, [(a, a)])


def _to_device(pairs):
    import torch
    bufs, items = [], []
    for a, b in pairs:
        da = torch.from_numpy(np.ascontiguousarray(a).reshape(-1)).cuda()
        db = torch.from_numpy(np.ascontiguousarray(b).reshape(-1)).cuda()
        bufs += [da, db]
        items.append((da.data_ptr(), db.data_ptr(), a.shape[1], a.shape[0], a.shape[1] * 4))
    return bufs, items


def test_plan_replays_match_batch_and_follow_inputs(rt):
    import torch
    sizes = [(200, 150), (480, 270), (333, 121), (200, 150)]
    pairs = _pairs(sizes, seed_pair=10)
    bufs, items = _to_device(pairs)
    k = iqm_b200.scores_per_pair(ALL)
    d_scores = torch.zeros(k * len(pairs), dtype=torch.float64, device="cuda")
    plan = iqm_b200.BatchPlan(rt, ALL, items, d_scores.data_ptr(), autotune=True)
    try:
        info, launches = plan.info()
        assert "fsim:" in info and launches > 0
        want = iqm_b200.batch(rt, ALL, pairs)
        for _ in range(2):
            d_scores.zero_()
            torch.cuda.synchronize()
            plan.run()
            rt.synchronize()
            got = iqm_b200._split_scores(ALL, len(pairs), d_scores.cpu().numpy())
            for m in want:
                assert np.array_equal(got[m], want[m]), m
        # same buffers, new content: the replay reads the current pixels
        new = _pairs(sizes, seed_pair=20)
        for i, (a, b) in enumerate(new):
            bufs[2 * i].copy_(torch.from_numpy(np.ascontiguousarray(a).reshape(-1)))
            bufs[2 * i + 1].copy_(torch.from_numpy(np.ascontiguousarray(b).reshape(-1)))
        torch.cuda.synchronize()
        plan.run()
        rt.synchronize()
        got = iqm_b200._split_scores(ALL, len(pairs), d_scores.cpu().numpy())
        want = iqm_b200.batch(rt, ALL, new)
        for m in want:
            assert np.array_equal(got[m], want[m]), m
    finally:
        plan.close()


def test_plan_uneven_batch_matches_oracle(rt, o64):
    """Uneven sizes drawn uniformly from [256, 2048] (seeded): SSIM on grey pairs, FSIM on RGB
    pairs, each through its own plan."""
    import torch
    sizes = synth.uneven_sizes(6, seed=3000)
    grey = [synth.grey_pair(h, w, config=3, pair=i) for i, (w, h) in enumerate(sizes)]
    rgb = [synth.rgb_gain_pair(h, w, config=3, pair=i) for i, (w, h) in enumerate(sizes)]
    for mask, pairs in ((iqm_b200.METRIC_SSIM, grey), (iqm_b200.METRIC_FSIM, rgb)):
        bufs, items = _to_device(pairs)
        k = iqm_b200.scores_per_pair(mask)
        d_scores = torch.zeros(k * len(pairs), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        plan = iqm_b200.BatchPlan(rt, mask, items, d_scores.data_ptr(), autotune=False)
        try:
            plan.run()
            rt.synchronize()
            got = d_scores.cpu().numpy()
        finally:
            plan.close()
        for i, (a, b) in enumerate(pairs):
            if mask == iqm_b200.METRIC_SSIM:
                assert abs(got[i] - o64.ssim(a, b)) <= TOL
            else:
                f, fc = o64.fsim(a, b)
                assert abs(got[2 * i] - f) <= TOL and abs(got[2 * i + 1] - fc) <= TOL


def test_plan_error_leaves_context_usable(rt):
    import torch
    tiny = np.zeros((1, 1, 4), np.uint8)
    bufs, items = _to_device([(tiny, tiny)])
    d_scores = torch.zeros(2, dtype=torch.float64, device="cuda")
    with pytest.raises(iqm_b200.IQMError):
        iqm_b200.BatchPlan(rt, iqm_b200.METRIC_FSIM, items, d_scores.data_ptr())
    a, b = synth.grey_pair(64, 64, config=0, pair=1)
    assert 0.0 < iqm_b200.SSIM(rt).compute_metric(a, b).mssim <= 1.0


def test_images_of_2_31_pixels_are_rejected(rt):
    """Pair validation (before any copy or launch) refuses images of 2^31 pixels or more, whose
    pixel counts would overflow 32-bit plane indices."""
    import ctypes
    buf = np.zeros(64, np.uint8)  # never read: validation fails first
    arr = iqm_b200._pairs([(buf.ctypes.data, buf.ctypes.data, 50000, 50000, 200000)])
    out = (ctypes.c_double * 4)()
    sp, fp = iqm_b200.SSIM(rt).params(), iqm_b200.FLIPArguments().c()
    L = rt.L
    for rc in (L.iqm_ssim_batch(rt.h, arr, 1, ctypes.byref(sp), out),
               L.iqm_msvd_batch(rt.h, arr, 1, out),
               L.iqm_flip_batch(rt.h, arr, 1, ctypes.byref(fp), out),
               L.iqm_fsim_batch(rt.h, arr, 1, 0, 0, out)):
        assert rc == iqm_b200.IQM_EINVAL
        assert "too large" in L.iqm_last_error(rt.h).decode()


def test_dev_entry_points_reject_misaligned_images(rt):
    """Device-resident images are read in place with 4-byte loads: a pointer or pitch that is not a
    multiple of 4 is refused with IQM_EINVAL before anything is enqueued."""
    import torch
    w, h = 64, 64
    buf = torch.zeros(w * h * 4 + 64, dtype=torch.uint8, device="cuda")
    d_scores = torch.zeros(4, dtype=torch.float64, device="cuda")
    base = buf.data_ptr()
    metrics = [iqm_b200.SSIM(rt), iqm_b200.SVD(rt), iqm_b200.FLIP(rt), iqm_b200.FSIM(rt)]
    for item in ((base + 1, base, w, h, 4 * w), (base, base + 2, w, h, 4 * w), (base, base, w, h - 1, 4 * w + 2)):
        for m in metrics:
            with pytest.raises(iqm_b200.IQMError) as e:
                m.compute_dev([item], d_scores.data_ptr())
            assert e.value.code == iqm_b200.IQM_EINVAL


def _largest_prime_factor(n):
    p, best = 2, 1
    while p * p <= n:
        while n % p == 0:
            best, n = p, n // p
        p += 1
    return max(best, n) if n > 1 else best


def test_uneven_256_batch_as_benchmarked_matches_oracle(rt, o64):
    """The uneven batch exactly as `bench.py --batch` runs it: the same 256 seeded sizes and crops,
    the SSIM plan without and the FSIM plan with autotuned launch shapes.  Every SSIM score is
    checked against the FP64 oracle; FSIM on a seeded subset that holds every transform class the
    batch reaches (the longest planes, which run CTA-wide, Bluestein lengths, lengths with direct
    odd-prime butterflies, and others)."""
    import torch
    import bench
    from oracle import fsim_plane_size
    sizes, grey, rgb = bench.batch_pairs()
    assert len(sizes) == 256
    plane = []
    for w, h in sizes:
        F = max(1, int(np.floor(min(w, h) / 256.0 + 0.5)))
        plane.append(fsim_plane_size(w, h, F))
    lpf = [max(_largest_prime_factor(w2), _largest_prime_factor(h2)) for w2, h2 in plane]
    order = np.argsort([-(w2 * h2) for w2, h2 in plane], kind="stable")
    picks = list(order[:6])                                                  # longest planes
    picks += [i for i in range(256) if lpf[i] > 61][:6]                      # Bluestein lengths
    picks += [i for i in range(256) if 15 < lpf[i] <= 61][:6]                # direct odd primes
    picks += list(np.random.default_rng(11).choice(256, 6, replace=False))   # anything else
    picks = sorted(set(int(i) for i in picks))
    results = {}
    for name, mask, pairs, tune in (("ssim", iqm_b200.METRIC_SSIM, grey, False),
                                    ("fsim", iqm_b200.METRIC_FSIM, rgb, True)):
        bufs, items = _to_device(pairs)
        d_scores = torch.zeros(iqm_b200.scores_per_pair(mask) * len(pairs), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        plan = iqm_b200.BatchPlan(rt, mask, items, d_scores.data_ptr(), autotune=tune)
        try:
            for _ in range(2):  # replays are identical
                plan.run()
                rt.synchronize()
                got = d_scores.cpu().numpy()
                if name in results:
                    assert np.array_equal(results[name], got)
                results[name] = got
        finally:
            plan.close()
        del bufs
    for i, (a, b) in enumerate(grey):
        assert abs(results["ssim"][i] - o64.ssim(a, b)) <= TOL, (i, sizes[i])
    for i in picks:
        f, fc = o64.fsim(*rgb[i])
        assert abs(results["fsim"][2 * i] - f) <= TOL and abs(results["fsim"][2 * i + 1] - fc) <= TOL, (i, sizes[i])


@pytest.mark.parametrize("precision,tol", [(iqm_b200.IQM_MIXED, 1e-5), (iqm_b200.IQM_MIXED_FAST, 2e-4)])
def test_plan_with_mixed_precision_forms(rt, o64, precision, tol):
    """A batch plan built with the tensor-core forms: SSIM (ssim->precision) and FSIM (the plan's
    precision) replay the same scores as the per-metric calls of those forms and stay within the
    forms' bounds of the FP64 oracle (FSIM: 1e-4 for both forms)."""
    import torch
    sizes = [(480, 270), (1920, 1080), (333, 121), (97, 211)]
    pairs = _pairs(sizes, seed_pair=40)
    bufs, items = _to_device(pairs)
    mask = iqm_b200.METRIC_SSIM | iqm_b200.METRIC_FSIM
    d_scores = torch.zeros(iqm_b200.scores_per_pair(mask) * len(pairs), dtype=torch.float64, device="cuda")
    s = iqm_b200.SSIM(rt)
    s.precision = precision
    f = iqm_b200.FSIM(rt)
    f.precision = precision
    plan = iqm_b200.BatchPlan(rt, mask, items, d_scores.data_ptr(), ssim=s.params(), precision=precision,
                              autotune=False)
    try:
        plan.run()
        rt.synchronize()
        got = iqm_b200._split_scores(mask, len(pairs), d_scores.cpu().numpy())
    finally:
        plan.close()
    assert np.array_equal(got["ssim"], s.compute_batch(pairs))
    assert np.array_equal(np.asarray(got["fsim"]).reshape(-1, 2), np.asarray(f.compute_batch(pairs)).reshape(-1, 2))
    for (a, b), gs, gf in zip(pairs, got["ssim"], np.asarray(got["fsim"]).reshape(-1, 2)):
        assert abs(gs - o64.ssim(a, b)) <= tol
        assert np.abs(np.asarray(gf) - np.asarray(o64.fsim(a, b))).max() <= 1e-4


@pytest.mark.parametrize("precision", [iqm_b200.IQM_FP32, iqm_b200.IQM_MIXED, iqm_b200.IQM_MIXED_FAST])
@pytest.mark.parametrize("h,w", [(16, 4000), (3000, 13), (11, 70)])
def test_ssim_extreme_aspect_ratios(rt, o64, precision, h, w):
    """Thin and wide images: a single tile row or column of the tiled kernels, halos on both sides."""
    a, b = synth.grey_pair(h, w, config=0, pair=7)
    s = iqm_b200.SSIM(rt)
    s.precision = precision
    tol = {iqm_b200.IQM_FP32: 1e-5, iqm_b200.IQM_MIXED: 1e-5, iqm_b200.IQM_MIXED_FAST: 2e-4}[precision]
    assert abs(s.compute_metric(a, b, want_map=False).mssim - o64.ssim(a, b)) <= tol
