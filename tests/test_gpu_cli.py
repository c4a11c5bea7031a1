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


def test_cli_batch_mode_matches_api(cli, rt, tmp_path):
    """--batch: decode on worker threads into page-locked buffers, one batch call per chunk; every
    pair's line matches the single-pair API; unreadable or mismatched pairs get an error line and the
    rest are still evaluated."""
    sizes = [(96, 130), (64, 64), (121, 77), (200, 150), (96, 130)]
    lines, want = [], []
    for i, (h, w) in enumerate(sizes):
        a, b = synth.rgb_gain_pair(h, w, config=1, pair=i)
        pa, pb = save(tmp_path, "a%d.png" % i, a), save(tmp_path, "b%d.png" % i, b)
        lines.append("%s %s" % (pa, pb))
        want.append(iqm_b200.FSIM(rt).compute_metric(a, b))
    c, d = synth.rgb_gain_pair(40, 50, config=1, pair=9)
    pc, pd = save(tmp_path, "c.png", c), save(tmp_path, "d.png", d[:, :48].copy())
    lines.insert(2, "%s %s" % (pc, pd))                       # size mismatch
    lines.insert(4, "%s %s" % (str(tmp_path / "nope.png"), pc))  # unreadable
    lst = tmp_path / "list.txt"
    lst.write_text("# pairs\n" + "\n".join(lines) + "\n")
    r = subprocess.run([cli, "--method", "FSIM", "--batch", str(lst), "--chunk", "2", "--threads", "3", "-v"],
                       capture_output=True, text=True)
    assert r.returncode == 1, r.stderr
    out = [l for l in r.stdout.splitlines() if not l.startswith("Selected method:")]  # -v header line
    assert len(out) == len(lines)
    assert "error: Compared images must have the same size" in out[2]
    assert "error: Failed to load image" in out[4]
    good = [l for k, l in enumerate(out) if k not in (2, 4)]
    for l, f in zip(good, want):
        parts = l.split()
        assert parts[2] == "FSIM:" and parts[4] == "FSIMc:"
        assert float(parts[3]) == pytest.approx(f.fsim, rel=2e-6)
        assert float(parts[5]) == pytest.approx(f.fsimc, rel=2e-6)
    assert "batch: 7 pairs, 2 failed" in r.stderr


def test_cli_repeat_loop(cli, rt, tmp_path):
    a, b = synth.grey_pair(90, 110, config=0, pair=2)
    pa, pb = save(tmp_path, "a.png", a), save(tmp_path, "b.png", b)
    out = run(cli, "--method", "SSIM", "--input", pa, "--ref", pb, "--repeat", "4", "-v")
    assert "Iterations: 4" in out
    assert value(out, "MSSIM") == pytest.approx(iqm_b200.SSIM(rt).compute_metric(a, b).mssim, rel=2e-6)


def test_cli_flip_output_is_viridis_of_the_flip_map(cli, rt, tmp_path):
    """FLIP --output writes the per-pixel FLIP value as viridis colours (entry floor(v * 255)),
    as the reference's combine pass colours its output image."""
    from PIL import Image
    import cv2
    a, b = synth.rgb_blockquant_pair(90, 130, config=2, pair=4)
    pa, pb = save(tmp_path, "a.png", a), save(tmp_path, "b.png", b)
    out_png = str(tmp_path / "flip.png")
    out = run(cli, "--method", "FLIP", "--input", pa, "--ref", pb, "--output", out_png)
    res = iqm_b200.FLIP(rt).compute_metric(a, b, want_map=True)
    assert value(out, "FLIP") == pytest.approx(res.mean_flip, rel=2e-6)
    img = np.asarray(Image.open(out_png))
    assert img.shape == (90, 130, 4) and np.all(img[..., 3] == 255)
    lut = cv2.applyColorMap(np.arange(256, dtype=np.uint8).reshape(-1, 1), cv2.COLORMAP_VIRIDIS).reshape(256, 3)[:, ::-1]
    idx = np.clip(np.floor(res.image_data.astype(np.float32) * np.float32(255.0)), 0, 255).astype(int)
    assert np.array_equal(img[..., :3], lut[idx])


def test_cli_fsim_precision_and_energy_options(cli, rt, o64, tmp_path):
    a, b = synth.rgb_gain_pair(1080, 1920, config=1, pair=2)
    pa, pb = save(tmp_path, "a.png", a), save(tmp_path, "b.png", b)
    f, fc = o64.fsim(a, b)
    for prec in ("mixed", "mixed_fast"):
        out = run(cli, "--method", "FSIM", "--input", pa, "--ref", pb, "--precision", prec)
        assert abs(value(out, "FSIM") - f) <= 1e-4 and abs(value(out, "FSIMc") - fc) <= 1e-4
    out = run(cli, "--method", "FSIM", "--input", pa, "--ref", pb, "FSIM_ENERGY_SUM", "full")
    ff, ffc = o64.fsim(a, b, energy_full=True)
    assert abs(value(out, "FSIM") - ff) <= 2e-6 and abs(value(out, "FSIMc") - ffc) <= 2e-6


def test_cli_ssim_precision_option(cli, rt, o64, tmp_path):
    """--precision reaches SSIM too: the split tensor-core form within 1e-5 of the FP64 oracle, single
    FP16 products within their 2e-4 bound; the batch mode takes the same option."""
    a, b = synth.grey_pair(600, 700, config=0, pair=3)
    pa, pb = save(tmp_path, "a.png", a), save(tmp_path, "b.png", b)
    want = o64.ssim(a, b)
    for prec, tol in (("mixed", 1e-5), ("mixed_fast", 2e-4)):
        out = run(cli, "--method", "SSIM", "--input", pa, "--ref", pb, "--precision", prec)
        assert abs(value(out, "MSSIM") - want) <= tol
    lst = tmp_path / "list.txt"
    lst.write_text("%s %s\n%s %s\n" % (pa, pb, pb, pa))
    out = run(cli, "--method", "SSIM", "--batch", str(lst), "--precision", "mixed")
    assert out.count("MSSIM") == 2
