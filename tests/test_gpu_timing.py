"""Per-kernel device timing (iqm_set_kernel_timing / iqm_kernel_times): every launch is charged to
its kernel name, launch counts match the launches enqueued, and timing off records nothing."""
import numpy as np
import pytest

import iqm_b200
from iqm_b200 import synth

pytestmark = pytest.mark.gpu


def test_kernel_times_count_launches(rt):
    a, b = synth.grey_pair(256, 320, config=0, pair=3)
    s = iqm_b200.SSIM(rt)
    f = iqm_b200.FSIM(rt)
    rgb_a, rgb_b = synth.rgb_gain_pair(270, 480, config=1, pair=1)
    f.compute_metric(rgb_a, rgb_b)  # plan for this size built before timing starts
    rt.set_kernel_timing(True)
    calls = 3
    fsim_launches = 0
    for _ in range(calls):
        s.compute_metric(a, b)
        f.compute_metric(rgb_a, rgb_b)
        fsim_launches += rt.last_launch_count()
    t = rt.kernel_times()
    rt.set_kernel_timing(False)
    assert t["ssim_kernel"][0] == calls
    assert t["ssim_kernel"][1] > 0.0
    fsim_kernels = {k: v for k, v in t.items() if k.startswith("fsim_")}
    assert sum(n for n, _ in fsim_kernels.values()) == fsim_launches
    assert all(ms > 0.0 for _, ms in fsim_kernels.values())
    # timing off: the next report is empty
    s.compute_metric(a, b)
    assert rt.kernel_times() == {}


def test_kernel_times_match_stream_time(rt):
    """The charged intervals tile the stream: their sum is close to the events around the calls."""
    import torch
    a, b = synth.grey_pair(1080, 1920, config=0, pair=1)
    B = 8
    dev = torch.empty((B, 2, a.size), dtype=torch.uint8, device="cuda")
    for i in range(B):
        dev[i, 0].copy_(torch.from_numpy(a.reshape(-1)))
        dev[i, 1].copy_(torch.from_numpy(b.reshape(-1)))
    pairs = [(dev[i, 0].data_ptr(), dev[i, 1].data_ptr(), 1920, 1080, 1920 * 4) for i in range(B)]
    sc = torch.zeros(B, dtype=torch.float64, device="cuda")
    st = torch.cuda.Stream()
    rt.set_stream(st.cuda_stream)
    try:
        s = iqm_b200.SSIM(rt)
        s.compute_dev(pairs, sc.data_ptr())
        rt.set_kernel_timing(True)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(5):
            s.compute_dev(pairs, sc.data_ptr())
        e1.record(st)
        t = rt.kernel_times()
        rt.set_kernel_timing(False)
        total = e0.elapsed_time(e1)
        n, ms = t["ssim_kernel"]
        assert n == 5
        assert 0.5 * total <= ms <= 1.01 * total
        assert np.isfinite(sc.cpu().numpy()).all()
    finally:
        rt.set_stream(0)
