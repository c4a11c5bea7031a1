"""FLIP on the GPU through the C ABI, against the CPU oracle (FP64 and FP32 builds).
Tolerance |delta mean FLIP| <= 1e-5; per-pixel map |delta| <= 1e-4."""
import numpy as np
import pytest

import iqm_b200
from iqm_b200 import synth

pytestmark = pytest.mark.gpu
TOL = 1e-5
ARGS_67 = iqm_b200.FLIPArguments(3840.0, 0.7, 0.7)  # 67.02 pixels per degree, radii 9/10
ARGS_37 = iqm_b200.FLIPArguments(2560.0, 0.5, 0.6)  # 37.2 pixels per degree, radii 5/6 (generic kernel)


def test_ppd_matches_reference_formula(rt, o64):
    f = iqm_b200.FLIP(rt)
    for args in (iqm_b200.FLIPArguments(), ARGS_67, iqm_b200.FLIPArguments(1920.0, 1.0, 0.5)):
        assert f.ppd(args) == o64.flip_ppd(args.monitor_resolution_x, args.monitor_distance, args.monitor_width)


@pytest.mark.parametrize("h,w", [(64, 96), (41, 59), (300, 517), (1080, 1920), (5, 7)])
@pytest.mark.parametrize("args", [ARGS_67, iqm_b200.FLIPArguments(), ARGS_37])
def test_flip_matches_oracle(rt, o64, o32, h, w, args):
    a, b = synth.rgb_blockquant_pair(h, w, config=2, pair=w % 5)
    f = iqm_b200.FLIP(rt)
    ppd = f.ppd(args)
    r = f.compute_metric(a, b, args, want_map=True)
    v64, m64 = o64.flip(a, b, ppd=ppd, want_map=True)
    assert abs(r.mean_flip - v64) <= TOL
    assert abs(r.mean_flip - o32.flip(a, b, ppd=ppd)) <= TOL
    assert np.abs(r.image_data - m64).max() <= 1e-4


@pytest.mark.parametrize("args", [ARGS_67, iqm_b200.FLIPArguments(), ARGS_37])
def test_flip_identical_is_zero(rt, args):
    a, b = synth.rgb_blockquant_pair(300, 200, config=2, pair=1)
    r = iqm_b200.FLIP(rt).compute_metric(b, b, args, want_map=True)
    assert r.mean_flip == 0.0
    assert not r.image_data.any()


def test_flip_batch_uneven(rt, o64):
    sizes = [(64, 96), (33, 130), (250, 17), (128, 300)]
    pairs = [synth.rgb_blockquant_pair(h, w, config=2, pair=i) for i, (h, w) in enumerate(sizes)]
    f = iqm_b200.FLIP(rt)
    got = f.compute_batch(pairs, ARGS_67)
    ppd = f.ppd(ARGS_67)
    for (a, b), g in zip(pairs, got):
        assert abs(g - o64.flip(a, b, ppd=ppd)) <= TOL


def test_flip_rejects_bad_params(rt):
    a = np.zeros((16, 16, 4), np.uint8)
    with pytest.raises(iqm_b200.IQMError):
        iqm_b200.FLIP(rt).compute_metric(a, a, iqm_b200.FLIPArguments(2560.0, 0.7, 0.0))


@pytest.mark.parametrize("args", [ARGS_67, iqm_b200.FLIPArguments()])
def test_flip_matches_independent_restatement(rt, args):
    """Against the whole-plane numpy restatement (oracle/np_restatement.py), written from the
    shaders independently of the C oracle."""
    import np_restatement
    a, b = synth.rgb_blockquant_pair(270, 480, config=2, pair=2)
    f = iqm_b200.FLIP(rt)
    want = np_restatement.flip(a, b, f.ppd(args))
    assert abs(f.compute_metric(a, b, args).mean_flip - want) <= TOL
