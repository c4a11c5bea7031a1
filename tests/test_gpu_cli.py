"""The C++ command line on the GPU: the reference's output lines (src/main.cpp:96,161,206) and
maps, against the Python API on the same PNG files."""
import os
import subprocess

import numpy as np
import pytest

import iqm_b200
from iqm_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cli():
    from iqm_b200 import build
    build.build()
    return build.build_cli()


def save(tmp_path, name, rgba):
    from PIL import Image
    p = str(tmp_path / name)
    Image.fromarray(rgba, "RGBA").save(p)
    return p


def run(cli, *args):
    r = subprocess.run([cli] + list(args), capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return r.stdout


def value(out, key):
    for line in out.splitlines():
        if line.startswith(key + ": "):
            return float(line.split(": ", 1)[1])
    raise AssertionError("%s not in %r" % (key, out))


def test_cli_scores_match_api(cli, rt, tmp_path):
    a, b = synth.rgb_blockquant_pair(120, 200, config=2, pair=3)
    pa, pb = save(tmp_path, "a.png", a), save(tmp_path, "b.png", b)
    out = run(cli, "--method", "SSIM", "--input", pa, "--ref", pb, "--output", str(tmp_path / "ssim.png"))
    want = iqm_b200.SSIM(rt).compute_metric(a, b)
    assert value(out, "MSSIM") == pytest.approx(want.mssim, rel=2e-6)
    from PIL import Image
    m = np.asarray(Image.open(str(tmp_path / "ssim.png")))
    assert m.shape == (120, 200)
    assert np.array_equal(m, (want.image_data * np.float32(255)).astype(np.uint8))
    out = run(cli, "--method", "SVD", "--input", pa, "--ref", pb, "--output", str(tmp_path / "svd.png"))
    assert value(out, "M-SVD") == pytest.approx(iqm_b200.SVD(rt).compute_metric(a, b).msvd, rel=2e-6)
    assert np.asarray(Image.open(str(tmp_path / "svd.png"))).shape == (15, 25)
    out = run(cli, "--method", "FSIM", "--input", pa, "--ref", pb)
    f = iqm_b200.FSIM(rt).compute_metric(a, b)
    assert value(out, "FSIM") == pytest.approx(f.fsim, rel=2e-6)
    assert value(out, "FSIMc") == pytest.approx(f.fsimc, rel=2e-6)
    out = run(cli, "--method", "FLIP", "--input", pa, "--ref", pb, "FLIP_RES", "3840", "FLIP_WIDTH", "0.7", "-v")
    fl = iqm_b200.FLIP(rt).compute_metric(a, b, iqm_b200.FLIPArguments(3840.0, 0.7, 0.7))
    assert value(out, "FLIP") == pytest.approx(fl.mean_flip, rel=2e-6)
    assert "Selected method: FLIP" in out and "FLIP monitor resolution: 3840" in out and "TOTAL" in out
