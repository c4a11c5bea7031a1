"""The allocation-free SSIM entry point (iqm_ssim_noalloc), for callers that cannot let a library
allocate device memory: its scores and map must match the regular entry points' and the FP64
oracle, call after call (its scratch array is shared and keeps the previous call's contents)."""
import ctypes

import numpy as np
import pytest

import iqm_b200
from iqm_b200 import synth

pytestmark = pytest.mark.gpu
TOL = 1e-5  # the SSIM tolerance used throughout the GPU tests


@pytest.mark.parametrize("h,w,ksize", [(1080, 1920, 11), (301, 517, 11), (301, 517, 7)])
def test_noalloc_matches_regular_entry_points(rt, o64, h, w, ksize):
    torch = pytest.importorskip("torch")
    L = iqm_b200.load_library()
    a, b = synth.grey_pair(h, w, config=0, pair=11)
    da = torch.from_numpy(a.reshape(-1)).cuda()
    db = torch.from_numpy(b.reshape(-1)).cuda()
    s = iqm_b200.SSIM(rt)
    s.kernel_size = ksize
    want = s.compute_metric(a, b)  # host entry point: score and map
    d_want = torch.zeros(1, dtype=torch.float64, device="cuda")
    s.compute_dev([(da.data_ptr(), db.data_ptr(), w, h, 4 * w)], d_want.data_ptr())
    rt.synchronize()
    oracle = o64.ssim(a, b, kernel_size=ksize)
    p = s.params()
    stream = torch.cuda.current_stream()
    for _ in range(2):  # the second call must not see the first call's counter or partials
        d_score = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
        d_map = torch.zeros(h * w, dtype=torch.float32, device="cuda")
        rc = L.iqm_ssim_noalloc(da.data_ptr(), db.data_ptr(), w, h, 4 * w, ctypes.byref(p), d_map.data_ptr(),
                                d_score.data_ptr(), stream.cuda_stream)
        assert rc == iqm_b200.IQM_OK
        stream.synchronize()
        got = d_score.item()
        assert abs(got - want.mssim) <= TOL
        assert abs(got - d_want.item()) <= TOL
        assert abs(got - oracle) <= TOL
        assert np.abs(d_map.cpu().numpy().reshape(h, w) - want.image_data).max() <= 5e-5


def test_noalloc_rejects_sizes_beyond_its_scratch(rt):
    torch = pytest.importorskip("torch")
    L = iqm_b200.load_library()
    buf = torch.zeros(64, dtype=torch.uint8, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    p = iqm_b200.SSIM(rt).params()
    w, h = 128 * 65, 122 * 65  # 4225 tiles > IQM_SSIM_NOALLOC_MAX_TILES
    rc = L.iqm_ssim_noalloc(buf.data_ptr(), buf.data_ptr(), w, h, 4 * w, ctypes.byref(p), None, out.data_ptr(),
                            None)
    assert rc == iqm_b200.IQM_EINVAL
    assert L.iqm_ssim_noalloc(None, buf.data_ptr(), 64, 64, 256, ctypes.byref(p), None, out.data_ptr(),
                              None) == iqm_b200.IQM_EINVAL


def test_noalloc_rejects_misaligned_pointers(rt):
    """Misaligned device pointers or pitches are refused with IQM_EINVAL before any launch (the
    call returns without touching the GPU)."""
    torch = pytest.importorskip("torch")
    L = iqm_b200.load_library()
    buf = torch.zeros(64 * 64 * 4 + 64, dtype=torch.uint8, device="cuda")
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    p = iqm_b200.SSIM(rt).params()
    base, w, h = buf.data_ptr(), 64, 64
    for args in ((base + 1, base, 4 * w, None, out.data_ptr()),
                 (base, base + 2, 4 * w, None, out.data_ptr()),
                 (base, base, 4 * w + 2, None, out.data_ptr()),
                 (base, base, 4 * w, base + 2, out.data_ptr()),
                 (base, base, 4 * w, None, out.data_ptr() + 4)):
        a, r, rb, m, o = args
        assert L.iqm_ssim_noalloc(a, r, w, h, rb, ctypes.byref(p), m, o, None) == iqm_b200.IQM_EINVAL
