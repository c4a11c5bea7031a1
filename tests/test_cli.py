"""CPU tests of the C++ command line: argument handling and error behaviour of src/main.cpp and
src/args.cpp, and the PNG/PNM decoder against PIL (colour types, bit depths, palettes,
transparency, Adam7 interlacing)."""
import os
import struct
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HOST = os.path.join(ROOT, "iqm_b200", "host")


@pytest.fixture(scope="module")
def cli():
    from iqm_b200 import build
    build.build()
    return build.build_cli()


@pytest.fixture(scope="module")
def png_check(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("native") / "png_check")
    subprocess.run(["/usr/bin/g++", "-O1", "-std=c++20", "-I", HOST, "-o", exe,
                    os.path.join(ROOT, "tests", "native", "png_check.cpp"), os.path.join(HOST, "png_io.cpp"),
                    os.path.join(HOST, "image_formats.cpp"), os.path.join(HOST, "jpeg_decode.cpp"), "-lz"],
                   check=True)
    return exe


def decode(png_check, path):
    out = subprocess.run([png_check, path], capture_output=True, check=True).stdout
    w, h = struct.unpack("<II", out[:8])
    return np.frombuffer(out[8:], np.uint8).reshape(h, w, 4)


def pil_rgba(path):
    from PIL import Image
    im = Image.open(path)
    if im.mode in ("I;16", "I;16B", "I"):
        a = (np.asarray(im).astype(np.uint32) >> 8).astype(np.uint8)
        rgba = np.stack([a, a, a, np.full_like(a, 255)], -1)
        return rgba
    return np.asarray(im.convert("RGBA"))


@pytest.mark.parametrize("mode", ["L", "LA", "RGB", "RGBA", "P", "1", "I;16"])
@pytest.mark.parametrize("interlace", [False, True])
def test_png_decoder_matches_pil(png_check, tmp_path, mode, interlace):
    from PIL import Image
    rng = np.random.default_rng(hash(mode) % 1000)
    h, w = 37, 53
    if mode == "I;16":
        im = Image.fromarray(rng.integers(0, 65536, (h, w), dtype=np.uint16))
    elif mode == "1":
        im = Image.fromarray(rng.integers(0, 2, (h, w), dtype=np.uint8) * 255).convert("1")
    elif mode == "P":
        im = Image.fromarray(rng.integers(0, 256, (h, w, 3), dtype=np.uint8)).convert("P", palette=Image.ADAPTIVE, colors=50)
    else:
        ch = {"L": 1, "LA": 2, "RGB": 3, "RGBA": 4}[mode]
        arr = rng.integers(0, 256, (h, w, ch), dtype=np.uint8)
        im = Image.fromarray(arr[..., 0] if ch == 1 else arr, mode=mode)
    path = str(tmp_path / "t.png")
    im.save(path, interlace=interlace)
    assert np.array_equal(decode(png_check, path), pil_rgba(path))


def test_pnm_decoder(png_check, tmp_path):
    from PIL import Image
    rng = np.random.default_rng(5)
    arr = rng.integers(0, 256, (20, 30, 3), dtype=np.uint8)
    path = str(tmp_path / "t.ppm")
    Image.fromarray(arr).save(path)
    got = decode(png_check, path)
    assert np.array_equal(got[..., :3], arr) and np.all(got[..., 3] == 255)


@pytest.mark.parametrize("mode", ["RGB", "RGBA", "P", "L"])
def test_bmp_decoder_matches_pil(png_check, tmp_path, mode):
    from PIL import Image
    rng = np.random.default_rng(8)
    arr = rng.integers(0, 256, (23, 37, 3), dtype=np.uint8)
    im = Image.fromarray(arr)
    im = im.convert("P", palette=Image.ADAPTIVE, colors=64) if mode == "P" else im.convert(mode)
    path = str(tmp_path / "t.bmp")
    im.save(path)
    got = decode(png_check, path)
    want = np.asarray(Image.open(path).convert("RGBA"))
    assert np.array_equal(got[..., :3], want[..., :3])


@pytest.mark.parametrize("mode", ["RGB", "RGBA", "L", "P"])
@pytest.mark.parametrize("rle", [False, True])
@pytest.mark.parametrize("origin", ["bl", "tl"])
def test_tga_decoder_matches_pil(png_check, tmp_path, mode, rle, origin):
    from PIL import Image
    rng = np.random.default_rng(9)
    arr = rng.integers(0, 256, (19, 31, 3), dtype=np.uint8)
    arr[5:9, :, :] = 77  # runs for the run-length form
    im = Image.fromarray(arr)
    im = im.convert("P", palette=Image.ADAPTIVE, colors=32) if mode == "P" else im.convert(mode)
    path = str(tmp_path / "t.tga")
    im.save(path, compression="tga_rle" if rle else None, orientation=1 if origin == "tl" else -1)
    got = decode(png_check, path)
    want = np.asarray(Image.open(path).convert("RGBA"))
    assert np.array_equal(got[..., :3], want[..., :3])


@pytest.mark.parametrize("subsampling", [0, 1, 2])
@pytest.mark.parametrize("size", [(48, 64), (37, 53)])
def test_jpeg_decoder_close_to_pil(png_check, tmp_path, subsampling, size):
    """Baseline JPEG (4:4:4, 4:2:2, 4:2:0; odd sizes): a lossy format decodes to slightly different
    bytes in different decoders, so the bound is a few levels per channel."""
    from PIL import Image
    from iqm_b200 import synth
    h, w = size
    a, _ = synth.rgb_gain_pair(h, w, config=1, pair=1)
    path = str(tmp_path / "t.jpg")
    Image.fromarray(a[..., :3]).save(path, quality=90, subsampling=subsampling)
    got = decode(png_check, path)[..., :3].astype(int)
    want = np.asarray(Image.open(path).convert("RGB")).astype(int)
    d = np.abs(got - want)
    assert d.max() <= 4 and d.mean() <= 0.6, (d.max(), d.mean())


def test_jpeg_grey_and_restart_intervals(png_check, tmp_path):
    from PIL import Image
    from iqm_b200 import synth
    a, _ = synth.grey_pair(45, 70, config=0, pair=2)
    for name, im, kw in (("g.jpg", Image.fromarray(a[..., 0]), {}),
                         ("r.jpg", Image.fromarray(a[..., :3]), {"restart_marker_blocks": 3})):
        path = str(tmp_path / name)
        im.save(path, quality=85, **kw)
        got = decode(png_check, path)[..., :3].astype(int)
        want = np.asarray(Image.open(path).convert("RGB")).astype(int)
        assert np.abs(got - want).max() <= 4


def test_progressive_jpeg_is_refused(png_check, tmp_path):
    from PIL import Image
    path = str(tmp_path / "p.jpg")
    Image.fromarray(np.zeros((16, 16, 3), np.uint8)).save(path, progressive=True)
    r = subprocess.run([png_check, path], capture_output=True, text=True)
    assert r.returncode != 0 and "progressive" in r.stderr


def test_unknown_image_type_is_rejected(png_check, tmp_path):
    path = str(tmp_path / "x.bin")
    open(path, "wb").write(b"\x00\x01not an image at all")
    r = subprocess.run([png_check, path], capture_output=True, text=True)
    assert r.returncode != 0 and "unknown image type" in r.stderr


def test_grey_png_encoder_round_trip(png_check, tmp_path):
    from PIL import Image
    rng = np.random.default_rng(6)
    px = rng.integers(0, 256, (23, 41), dtype=np.uint8)
    png = subprocess.run([png_check, "--encode", "41", "23"], input=px.tobytes(), capture_output=True, check=True).stdout
    path = str(tmp_path / "g.png")
    open(path, "wb").write(png)
    assert np.array_equal(np.asarray(Image.open(path)), px)


@pytest.mark.parametrize("channels", [3, 4])
def test_colour_png_encoder_round_trip(png_check, tmp_path, channels):
    from PIL import Image
    rng = np.random.default_rng(7)
    px = rng.integers(0, 256, (17, 29, channels), dtype=np.uint8)
    png = subprocess.run([png_check, "--encode", "29", "17", str(channels)], input=px.tobytes(), capture_output=True,
                         check=True).stdout
    path = str(tmp_path / "c.png")
    open(path, "wb").write(png)
    img = Image.open(path)
    assert img.mode == ("RGB" if channels == 3 else "RGBA")
    assert np.array_equal(np.asarray(img), px)


def test_viridis_table_matches_opencv():
    """The FLIP --output colour map (iqm_b200/host/viridis_table.h, written by make_viridis.py)."""
    import re
    import cv2
    text = open(os.path.join(ROOT, "iqm_b200", "host", "viridis_table.h")).read()
    rgb = np.array([int(v) for v in re.findall(r"\d+", text.split("= {", 1)[1])[:768]]).reshape(256, 3)
    want = cv2.applyColorMap(np.arange(256, dtype=np.uint8).reshape(-1, 1), cv2.COLORMAP_VIRIDIS).reshape(256, 3)
    assert np.array_equal(rgb, want[:, ::-1])


def test_cli_option_value_errors(cli, tmp_path):
    for opt in (["--precision", "half"], ["FSIM_ENERGY_SUM", "most"]):
        r = subprocess.run([cli, "--method", "FSIM", "--input", "a.png", "--ref", "b.png"] + opt,
                           capture_output=True, text=True)
        assert r.returncode != 0 and "must be" in r.stderr


def test_cli_argument_errors(cli):
    # src/args.cpp:32-34 and :52-60: unknown or missing arguments throw outside main's try block
    r = subprocess.run([cli, "--method", "SSIM_CPU", "--input", "a", "--ref", "b"], capture_output=True, text=True)
    assert r.returncode != 0 and "Unknown method" in r.stderr
    r = subprocess.run([cli, "--input", "a", "--ref", "b"], capture_output=True, text=True)
    assert r.returncode != 0 and "missing method" in r.stderr
    r = subprocess.run([cli, "--method", "FSIM", "--ref", "b"], capture_output=True, text=True)
    assert r.returncode != 0 and "missing input" in r.stderr


def test_cli_load_and_size_errors(cli, tmp_path):
    from PIL import Image
    r = subprocess.run([cli, "--method", "SSIM", "--input", str(tmp_path / "none.png"), "--ref", "x"],
                       capture_output=True, text=True)
    assert r.returncode == 255 and "Failed to load image" in r.stderr
    a, b = str(tmp_path / "a.png"), str(tmp_path / "b.png")
    Image.new("RGB", (10, 12)).save(a)
    Image.new("RGB", (11, 12)).save(b)
    r = subprocess.run([cli, "--method", "FLIP", "--input", a, "--ref", b], capture_output=True, text=True)
    assert r.returncode == 255 and "Compared images must have the same size" in r.stderr


def test_cli_cw_ssim_is_a_no_op(cli, tmp_path):
    # src/main.cpp:275-276: CW_SSIM_CPU is accepted and does nothing
    r = subprocess.run([cli, "--method", "CW_SSIM_CPU", "--input", "a", "--ref", "b", "-v"], capture_output=True,
                       text=True)
    assert r.returncode == 0 and r.stdout.strip() == "Selected method: CW-SSIM"


def test_cli_batch_list_errors(cli, tmp_path):
    # batch mode needs no --input/--ref, but a readable list of "<input> <ref>" lines
    r = subprocess.run([cli, "--method", "SSIM", "--batch", str(tmp_path / "missing.txt")], capture_output=True,
                       text=True)
    assert r.returncode == 255 and "Failed to open batch list" in r.stderr
    bad = tmp_path / "bad.txt"
    bad.write_text("# comment\n\nonly_one_path.png\n")
    r = subprocess.run([cli, "--method", "SSIM", "--batch", str(bad)], capture_output=True, text=True)
    assert r.returncode == 255 and "without a reference image" in r.stderr
    ok = tmp_path / "ok.txt"
    ok.write_text("a.png b.png\n")
    r = subprocess.run([cli, "--method", "SSIM", "--batch", str(ok), "--chunk", "0"], capture_output=True, text=True)
    assert r.returncode == 255 and "--chunk must be >= 1" in r.stderr
    # CW-SSIM stays a no-op in batch mode (no device needed)
    r = subprocess.run([cli, "--method", "CW_SSIM_CPU", "--batch", str(ok)], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout == ""
