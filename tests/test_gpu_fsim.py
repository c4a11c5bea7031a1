"""FSIM / FSIMc on the GPU through the C ABI, against the CPU oracle (FP64 and the
reference-faithful FP32 build).  Tolerance |delta| <= 1e-5 on both scores."""
import numpy as np
import pytest

import iqm_b200
from iqm_b200 import synth

pytestmark = pytest.mark.gpu
TOL = 1e-5


@pytest.mark.parametrize("w2,h2", [(128, 96), (480, 270), (270, 480), (263, 131), (200, 130), (64, 64)])
@pytest.mark.parametrize("mode", [0, 1])
def test_plan_constants_match_oracle(rt, o64, w2, h2, mode):
    em, an2, aiaj = iqm_b200.FSIM(rt, energy_mode=mode).plan_constants(w2, h2)
    oem, oan2, oaiaj = o64.fsim_constants(w2, h2, energy_full=bool(mode))
    assert np.allclose(em, oem, rtol=1e-5)
    assert np.allclose(an2, oan2, rtol=1e-4, atol=1e-6 * np.abs(oan2).max())
    assert np.allclose(aiaj, oaiaj, rtol=1e-4, atol=1e-6 * np.abs(oan2).max())


@pytest.mark.parametrize("h,w", [(96, 128), (130, 200), (270, 480), (480, 270), (600, 800), (1080, 1920), (1920, 1080),
                                 (131, 263), (57, 61), (2160, 3840),
                                 # full-resolution planes with long runtime-planned transforms, which run
                                 # CTA-wide: rows of 1100; columns of 1100 in groups of four (the last of a
                                 # 301-wide plane holds one); a 1031-point Bluestein row
                                 (300, 1100), (1100, 301), (290, 1031)])
def test_fsim_matches_oracle(rt, o64, o32, h, w):
    a, b = synth.rgb_gain_pair(h, w, config=1, pair=w % 7)
    r = iqm_b200.FSIM(rt).compute_metric(a, b)
    f64, fc64 = o64.fsim(a, b)
    f32, fc32 = o32.fsim(a, b)
    assert abs(r.fsim - f64) <= TOL and abs(r.fsimc - fc64) <= TOL, (r, f64, fc64)
    assert abs(r.fsim - f32) <= TOL and abs(r.fsimc - fc32) <= TOL, (r, f32, fc32)


def test_fsim_full_energy_mode(rt, o64):
    a, b = synth.rgb_gain_pair(200, 260, config=1, pair=3)
    r = iqm_b200.FSIM(rt, energy_mode=1).compute_metric(a, b)
    f, fc = o64.fsim(a, b, energy_full=True)
    assert abs(r.fsim - f) <= TOL and abs(r.fsimc - fc) <= TOL


def test_fsim_identical_is_one(rt):
    a, b = synth.rgb_gain_pair(120, 160, config=1, pair=2)
    r = iqm_b200.FSIM(rt).compute_metric(b, b)
    assert r.fsim == pytest.approx(1.0, abs=1e-6) and r.fsimc == pytest.approx(1.0, abs=1e-6)


def test_fsim_batch_uneven_matches_single(rt, o64):
    sizes = [(96, 128), (270, 480), (96, 128), (130, 200), (600, 800)]
    pairs = [synth.rgb_gain_pair(h, w, config=1, pair=i) for i, (h, w) in enumerate(sizes)]
    f = iqm_b200.FSIM(rt)
    got = f.compute_batch(pairs)
    for (a, b), g in zip(pairs, got):
        single = f.compute_metric(a, b)
        assert g[0] == single.fsim and g[1] == single.fsimc
        w64 = o64.fsim(a, b)
        assert abs(g[0] - w64[0]) <= TOL and abs(g[1] - w64[1]) <= TOL


@pytest.mark.parametrize("count", [3, 9])
def test_fsim_same_size_batch_matches_single(rt, count):
    # 1080p planes take one pair per inverse-pass chunk when several chunks are in flight, and
    # consecutive chunks alternate between two streams.  Every pair's arithmetic is the same in all
    # schedules, so the scores are identical.
    pairs = [synth.rgb_gain_pair(1080, 1920, config=1, pair=i) for i in range(count)]
    f = iqm_b200.FSIM(rt)
    got = f.compute_batch(pairs)
    for (a, b), g in zip(pairs, got):
        single = f.compute_metric(a, b)
        assert g[0] == single.fsim and g[1] == single.fsimc


def test_fsim_deterministic(rt):
    a, b = synth.rgb_gain_pair(270, 480, config=1, pair=5)
    f = iqm_b200.FSIM(rt)
    v = [f.compute_metric(a, b) for _ in range(3)]
    assert v[0] == v[1] == v[2]


def test_fsim_errors(rt):
    f = iqm_b200.FSIM(rt)
    a = np.zeros((40, 40, 4), np.uint8)
    with pytest.raises(iqm_b200.IQMError):
        f.compute_metric(a, np.zeros((40, 41, 4), np.uint8))
    f.energy_mode = 3
    with pytest.raises(iqm_b200.IQMError) as e:
        f.compute_metric(a, a)
    assert e.value.code == iqm_b200.IQM_EINVAL


MIXED_TOL = 1e-4  # the mixed forms' bound against the FP64 oracle
MIXED = [iqm_b200.IQM_MIXED, iqm_b200.IQM_MIXED_FAST]


@pytest.mark.parametrize("precision", MIXED)
@pytest.mark.parametrize("h,w,pair", [(1080, 1920, 0), (1080, 1920, 1), (2160, 3840, 0), (1920, 1080, 2)])
def test_fsim_mixed_within_bound_of_fp64(rt, o64, precision, h, w, pair):
    """Tensor-core inverse transforms (1080p and 4K pairs: 480x270 planes) and FP16 intermediate
    planes: both scores within 1e-4 of the FP64 oracle.  The portrait pair has a 270x480 plane,
    which has no tensor-core engines and runs the FP32 transforms."""
    a, b = synth.rgb_gain_pair(h, w, config=1, pair=pair)
    r = iqm_b200.FSIM(rt, precision=precision).compute_metric(a, b)
    f64, fc64 = o64.fsim(a, b)
    assert abs(r.fsim - f64) <= MIXED_TOL and abs(r.fsimc - fc64) <= MIXED_TOL, (r, f64, fc64)


@pytest.mark.parametrize("precision", MIXED)
def test_fsim_mixed_energy_mode_and_identity(rt, o64, precision):
    a, b = synth.rgb_gain_pair(1080, 1920, config=1, pair=4)
    r = iqm_b200.FSIM(rt, precision=precision, energy_mode=1).compute_metric(a, b)
    f, fc = o64.fsim(a, b, energy_full=True)
    assert abs(r.fsim - f) <= MIXED_TOL and abs(r.fsimc - fc) <= MIXED_TOL
    same = iqm_b200.FSIM(rt, precision=precision).compute_metric(b, b)
    assert same.fsim == pytest.approx(1.0, abs=1e-6) and same.fsimc == pytest.approx(1.0, abs=1e-6)


@pytest.mark.parametrize("precision", MIXED)
def test_fsim_mixed_batch_matches_single_and_oracle(rt, o64, precision):
    """A batch mixing tensor-core (1080p) and FP32-transform plane sizes; several 1080p pairs so the
    inverse passes run in more than one chunk."""
    sizes = [(1080, 1920)] * 5 + [(130, 200), (600, 800), (1080, 1920)]
    pairs = [synth.rgb_gain_pair(h, w, config=1, pair=i) for i, (h, w) in enumerate(sizes)]
    f = iqm_b200.FSIM(rt, precision=precision)
    got = f.compute_batch(pairs)
    for (a, b), g in zip(pairs, got):
        single = f.compute_metric(a, b)
        assert g[0] == single.fsim and g[1] == single.fsimc
        w64 = o64.fsim(a, b)
        assert abs(g[0] - w64[0]) <= MIXED_TOL and abs(g[1] - w64[1]) <= MIXED_TOL


def test_fsim_mixed_deterministic(rt):
    a, b = synth.rgb_gain_pair(1080, 1920, config=1, pair=6)
    f = iqm_b200.FSIM(rt, precision=iqm_b200.IQM_MIXED)
    v = [f.compute_metric(a, b) for _ in range(3)]
    assert v[0] == v[1] == v[2]


def test_fsim_unknown_precision_rejected(rt):
    a, b = synth.rgb_gain_pair(64, 80, config=1, pair=1)
    with pytest.raises(iqm_b200.IQMError) as e:
        iqm_b200.FSIM(rt, precision=7).compute_metric(a, b)
    assert e.value.code == iqm_b200.IQM_EINVAL
    # the context stays usable
    assert 0.0 < iqm_b200.FSIM(rt).compute_metric(a, b).fsim <= 1.0


@pytest.mark.parametrize("h,w", [(1080, 1920), (131, 263), (300, 2048)])
def test_fsim_matches_independent_restatement(rt, h, w):
    """Against the whole-plane numpy restatement (oracle/np_restatement.py), written from the
    shaders independently of the C oracle."""
    import np_restatement
    a, b = synth.rgb_gain_pair(h, w, config=1, pair=9)
    want = np_restatement.fsim(a, b)
    r = iqm_b200.FSIM(rt).compute_metric(a, b)
    assert abs(r.fsim - want[0]) <= TOL and abs(r.fsimc - want[1]) <= TOL
    m = iqm_b200.FSIM(rt, precision=iqm_b200.IQM_MIXED).compute_metric(a, b)
    assert abs(m.fsim - want[0]) <= MIXED_TOL and abs(m.fsimc - want[1]) <= MIXED_TOL
