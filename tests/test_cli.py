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
    bytes in different decoders, so the bound is a few levels per channel.  With 4:2:2 the column
    before the last chroma pair's second output follows the reference loader's edge rule, not PIL's
    filter, and is left out here (tests/test_loader_vs_reference.py holds it to the loader)."""
    from PIL import Image
    from iqm_b200 import synth
    h, w = size
    a, _ = synth.rgb_gain_pair(h, w, config=1, pair=1)
    path = str(tmp_path / "t.jpg")
    Image.fromarray(a[..., :3]).save(path, quality=90, subsampling=subsampling)
    got = decode(png_check, path)[..., :3].astype(int)
    want = np.asarray(Image.open(path).convert("RGB")).astype(int)
    if subsampling == 1:
        keep = np.ones(w, bool)
        keep[2 * ((w + 1) // 2 - 1)] = False
        got, want = got[:, keep], want[:, keep]
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


@pytest.mark.parametrize("subsampling", [0, 2])
@pytest.mark.parametrize("size", [(48, 64), (37, 53), (130, 97)])
def test_progressive_jpeg_close_to_baseline_decode(png_check, tmp_path, subsampling, size):
    """Progressive JPEG (spectral selection and successive approximation scans): the coefficients
    of all scans are the baseline file's, so the decode matches PIL's within the same few levels,
    and the progressive and baseline encodings of one image decode to the same bytes here."""
    from PIL import Image
    from iqm_b200 import synth
    h, w = size
    a, _ = synth.rgb_gain_pair(h, w, config=1, pair=3)
    prog, base = str(tmp_path / "p.jpg"), str(tmp_path / "b.jpg")
    Image.fromarray(a[..., :3]).save(prog, quality=88, subsampling=subsampling, progressive=True)
    Image.fromarray(a[..., :3]).save(base, quality=88, subsampling=subsampling, optimize=True)
    assert open(prog, "rb").read().find(b"\xff\xc2") > 0
    got = decode(png_check, prog)
    want = np.asarray(Image.open(prog).convert("RGB")).astype(int)
    d = np.abs(got[..., :3].astype(int) - want)
    assert d.max() <= 4 and d.mean() <= 0.6, (d.max(), d.mean())
    assert np.array_equal(got, decode(png_check, base))


def test_progressive_grey_jpeg_with_restarts(png_check, tmp_path):
    from PIL import Image
    from iqm_b200 import synth
    a, _ = synth.grey_pair(61, 90, config=0, pair=4)
    path = str(tmp_path / "pg.jpg")
    Image.fromarray(a[..., 0]).save(path, quality=80, progressive=True, restart_marker_blocks=2)
    got = decode(png_check, path)[..., :3].astype(int)
    want = np.asarray(Image.open(path).convert("RGB")).astype(int)
    assert np.abs(got - want).max() <= 4


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


# ---- GIF, Radiance HDR and PSD, decoded as stbi_load(..., 4) decodes them ----------------------------

def _lzw_literal_stream(indices, min_size):
    """GIF LZW data that codes every pixel as a literal, with a clear code before the table would
    widen the codes (a valid stream any decoder must read)."""
    clear, end, size = 1 << min_size, (1 << min_size) + 1, min_size + 1
    codes, since = [clear], 0
    for v in indices:
        if since == (1 << size) - (clear + 2) - 1:
            codes.append(clear)
            since = 0
        codes.append(int(v))
        since += 1
    codes.append(end)
    acc, nbits, out = 0, 0, bytearray()
    for c in codes:
        acc |= c << nbits
        nbits += size
        while nbits >= 8:
            out.append(acc & 255)
            acc >>= 8
            nbits -= 8
    if nbits:
        out.append(acc & 255)
    blocks = bytearray([min_size])
    for i in range(0, len(out), 255):
        chunk = out[i:i + 255]
        blocks += bytes([len(chunk)]) + chunk
    return bytes(blocks + b"\x00")


def _gif(screen_w, screen_h, palette, bg, frame, x0=0, y0=0, transparent=None):
    import struct as st
    n = len(palette)
    bits = max(1, (n - 1).bit_length())
    pal = bytes(c for rgb in palette for c in rgb) + bytes(3 * ((1 << bits) - n))
    out = b"GIF89a" + st.pack("<HHBBB", screen_w, screen_h, 0x80 | (bits - 1), bg, 0) + pal
    if transparent is not None:
        out += b"\x21\xf9\x04" + bytes([1, 0, 0, transparent, 0])
    fh, fw = frame.shape
    out += b"\x2c" + st.pack("<HHHHB", x0, y0, fw, fh, 0)
    out += _lzw_literal_stream(frame.ravel(), max(2, bits)) + b"\x3b"
    return out


def test_gif_decoder_matches_palette(png_check, tmp_path):
    from PIL import Image
    rng = np.random.default_rng(4)
    idx = rng.integers(0, 16, (23, 37)).astype(np.uint8)
    pal = rng.integers(0, 256, (16, 3)).astype(np.uint8)
    want = np.concatenate([pal[idx], np.full(idx.shape + (1,), 255, np.uint8)], -1)
    for name, kw in (("flat", {"interlace": False}), ("interlaced", {"interlace": True})):
        im = Image.fromarray(idx, "P")
        im.putpalette(pal.ravel().tolist())
        path = str(tmp_path / (name + ".gif"))
        im.save(path, **kw)
        assert np.array_equal(decode(png_check, path), want), name


def test_gif_transparency_and_background(png_check, tmp_path):
    rng = np.random.default_rng(5)
    pal = [tuple(int(v) for v in rng.integers(0, 256, 3)) for _ in range(8)]
    frame = rng.integers(0, 8, (5, 6)).astype(np.uint8)
    frame[0, 0] = frame[2, 3] = 6
    path = str(tmp_path / "t.gif")
    open(path, "wb").write(_gif(11, 9, pal, 2, frame, x0=3, y0=2, transparent=6))
    got = decode(png_check, path)
    want = np.zeros((9, 11, 4), np.uint8)
    r, g, b = pal[2]
    want[...] = (b, g, r, 255)  # pixels outside the frame: the background entry in B, G, R order
    for y in range(5):
        for x in range(6):
            v = frame[y, x]
            want[2 + y, 3 + x] = (0, 0, 0, 0) if v == 6 else pal[v] + (255,)
    assert np.array_equal(got, want)


def _hdr_expected(rgbe):
    m = rgbe[..., :3].astype(np.float32)
    e = rgbe[..., 3].astype(np.int32)
    scale = np.where(e > 0, np.ldexp(np.float32(1), e - 136).astype(np.float32), np.float32(0))
    v = (m * scale[..., None]).astype(np.float32)
    p = np.power(v.astype(np.float64), np.float64(np.float32(1) / np.float32(2.2))).astype(np.float32)
    z = p * np.float32(255) + np.float32(0.5)
    z = np.clip(z, 0, 255)
    out = np.empty(rgbe.shape[:2] + (4,), np.uint8)
    out[..., :3] = z.astype(np.int32).astype(np.uint8)
    out[..., 3] = 255
    return out


def _hdr_rle_scanline(sl):
    out = bytearray([2, 2, sl.shape[0] >> 8, sl.shape[0] & 255])
    for k in range(4):
        comp = sl[:, k].tolist()
        i = 0
        while i < len(comp):
            j = i
            while j < len(comp) and j - i < 127 and comp[j] == comp[i]:
                j += 1
            if j - i >= 3:
                out += bytes([128 + j - i, comp[i]])
                i = j
            else:
                lit = comp[i:i + min(128, len(comp) - i)]
                out += bytes([len(lit)]) + bytes(lit)
                i += len(lit)
    return bytes(out)


@pytest.mark.parametrize("w,rle", [(5, False), (40, True), (40, False)])
def test_hdr_decoder(png_check, tmp_path, w, rle):
    rng = np.random.default_rng(6)
    h = 7
    rgbe = rng.integers(0, 256, (h, w, 4)).astype(np.uint8)
    rgbe[..., 0] |= 0x80  # a valid pixel has one mantissa >= 128, so a flat scanline never looks run-length coded
    rgbe[:, :w // 3, :] = rgbe[:, :1, :]  # runs
    rgbe[1, 2, 3] = 0  # zero exponent
    body = b"".join(_hdr_rle_scanline(rgbe[y]) for y in range(h)) if rle else rgbe.tobytes()
    path = str(tmp_path / "x.hdr")
    open(path, "wb").write(b"#?RADIANCE\n# made by a test\nFORMAT=32-bit_rle_rgbe\n\n-Y %d +X %d\n" % (h, w) + body)
    assert np.array_equal(decode(png_check, path), _hdr_expected(rgbe))


def test_hdr_written_by_opencv(png_check, tmp_path):
    import cv2
    rng = np.random.default_rng(7)
    img = (rng.random((12, 33, 3)) * 4).astype(np.float32)
    path = str(tmp_path / "cv.hdr")
    assert cv2.imwrite(path, img)
    got = decode(png_check, path)
    back = cv2.imread(path, cv2.IMREAD_UNCHANGED)[..., ::-1].astype(np.float32)  # OpenCV's RGBE decode
    p = np.power(back.astype(np.float64), np.float64(np.float32(1) / np.float32(2.2))).astype(np.float32)
    want = np.clip(p * np.float32(255) + np.float32(0.5), 0, 255).astype(np.int32)
    assert got.shape == (12, 33, 4) and (got[..., 3] == 255).all()
    assert np.abs(got[..., :3].astype(int) - want).max() <= 1


def _packbits(row):
    out, i = bytearray(), 0
    while i < len(row):
        j = i
        while j < len(row) and j - i < 128 and row[j] == row[i]:
            j += 1
        if j - i >= 2:
            out += bytes([257 - (j - i), row[i]])
            i = j
        else:
            lit = row[i:i + min(128, len(row) - i)]
            out += bytes([len(lit) - 1]) + bytes(lit)
            i += len(lit)
    return bytes(out)


def _psd(planes, depth, rle):
    import struct as st
    c, h, w = planes.shape
    out = b"8BPS" + st.pack(">H6xHIIHH", 1, c, h, w, depth, 3) + st.pack(">III", 0, 0, 0)  # empty sections
    if not rle:
        data = planes.astype(">u2").tobytes() if depth == 16 else planes.astype(np.uint8).tobytes()
        return out + st.pack(">H", 0) + data
    chunks = [_packbits(planes[k].ravel().tolist()) for k in range(c)]
    counts = st.pack(">%dH" % (c * h), *([0] * (c * h)))
    return out + st.pack(">H", 1) + counts + b"".join(chunks)


def _unpremultiply(px):
    out = px.copy()
    a = px[..., 3]
    m = (a != 0) & (a != 255)
    af = a.astype(np.float32) / np.float32(255)
    ra = np.float32(1) / np.where(m, af, np.float32(1))
    inv = np.float32(255) * (np.float32(1) - ra)
    for c in range(3):
        v = px[..., c].astype(np.float32) * ra + inv
        out[..., c] = np.where(m, (np.trunc(v).astype(np.int64) & 255).astype(np.uint8), px[..., c])
    return out


@pytest.mark.parametrize("channels,depth,rle", [(3, 8, False), (3, 8, True), (4, 8, False), (4, 8, True),
                                                (3, 16, False), (5, 16, False)])
def test_psd_decoder(png_check, tmp_path, channels, depth, rle):
    rng = np.random.default_rng(8)
    h, w = 9, 14
    planes = rng.integers(0, 1 << depth, (channels, h, w)).astype(np.uint32)
    planes[:, :, :5] = planes[:, :, :1]  # runs
    if channels >= 4:
        planes[3, 0, 0], planes[3, 1, 1] = 0, (1 << depth) - 1
    path = str(tmp_path / "x.psd")
    open(path, "wb").write(_psd(planes, depth, rle))
    hi = (planes >> 8) if depth == 16 else planes
    want = np.zeros((h, w, 4), np.uint8)
    want[..., 3] = 255
    for k in range(min(channels, 4)):
        want[..., k] = hi[k]
    if channels >= 4:
        want = _unpremultiply(want)
    assert np.array_equal(decode(png_check, path), want)
    if channels == 3 and depth == 8 and not rle:
        assert np.array_equal(decode(png_check, path), pil_rgba(path))


def test_psd_non_rgb_is_refused(png_check, tmp_path):
    import struct as st
    path = str(tmp_path / "g.psd")
    open(path, "wb").write(b"8BPS" + st.pack(">H6xHIIHH", 1, 1, 2, 2, 8, 1) + b"\x00" * 14 + b"\x00" * 4)
    r = subprocess.run([png_check, path], capture_output=True, text=True)
    assert r.returncode != 0 and "RGB" in r.stderr


def _pic(w, h, packets, rows):
    """Softimage PIC: header, packet chain [(coding, mask)], then per row each packet's bytes."""
    import struct as st
    head = st.pack(">I", 0x5380F634) + b"\x00" * 84 + b"PICT" + st.pack(">HHIHH", w, h, 0, 0, 0)
    chain = b"".join(bytes([1 if i + 1 < len(packets) else 0, 8, t, m]) for i, (t, m) in enumerate(packets))
    return head + chain + b"".join(rows)


def _pic_channels(mask):
    return [c for c in range(4) if mask & (0x80 >> c)]


def _pic_encode_row(px, coding, mask):
    ch = _pic_channels(mask)
    vals = [bytes(int(px[x, c]) for c in ch) for x in range(px.shape[0])]
    if coding == 0:
        return b"".join(vals)
    out, i = bytearray(), 0
    while i < len(vals):
        j = i
        while j < len(vals) and vals[j] == vals[i] and j - i < (255 if coding == 1 else 300):
            j += 1
        n = j - i
        if coding == 1:
            out += bytes([n]) + vals[i]
            i = j
        elif n >= 2:
            out += (bytes([128]) + n.to_bytes(2, "big") if n > 128 else bytes([n + 127])) + vals[i]
            i = j
        else:
            k = i
            while k < len(vals) and k - i < 128 and (k + 1 >= len(vals) or vals[k + 1] != vals[k]):
                k += 1
            k = max(k, i + 1)
            out += bytes([k - i - 1]) + b"".join(vals[i:k])
            i = k
    return bytes(out)


@pytest.mark.parametrize("codings", [(0,), (1,), (2,), (2, 1)])
def test_pic_decoder(png_check, tmp_path, codings):
    rng = np.random.default_rng(9)
    h, w = 6, 150
    img = rng.integers(0, 256, (h, w, 4)).astype(np.uint8)
    img[:, 3:140] = img[:, 3:4]  # a run longer than 128 (a 16-bit count in mixed coding)
    packets = [(codings[0], 0xE0)] + ([(codings[1], 0x10)] if len(codings) > 1 else [])
    rows = [b"".join(_pic_encode_row(img[y], t, m) for t, m in packets) for y in range(h)]
    path = str(tmp_path / "x.pic")
    open(path, "wb").write(_pic(w, h, packets, rows))
    want = img.copy()
    if len(codings) == 1:
        want[..., 3] = 255  # no packet carries alpha
    assert np.array_equal(decode(png_check, path), want)


# ---- BMP and TGA layouts beyond what PIL writes: files built here, expected pixels from the rules
# stb_image applies (bit-field channels widened by repeating their bits, 15/16-bit TGA channels as
# v * 255 / 31, TGA colour maps read after skipping the first-entry field's bytes).

def _bmp(w, h, bpp, pixels_rows, hsz=40, comp=0, masks=None, palette=None, top_down=False):
    """A BMP file: rows given top to bottom as bytes (unpadded); stored bottom-up unless top_down."""
    stride = ((w * bpp + 7) // 8 + 3) & ~3
    rows = [r + b"\0" * (stride - len(r)) for r in pixels_rows]
    data = b"".join(rows if top_down else rows[::-1])
    pal = b""
    if palette is not None:
        pal = b"".join(bytes([b, g, r]) + (b"" if hsz == 12 else b"\0") for r, g, b in palette)
    extra = b""
    if hsz == 12:
        info = struct.pack("<IHHHH", 12, w, h, 1, bpp)
    else:
        info = struct.pack("<IiiHHIIiiII", hsz, w, -h if top_down else h, 1, bpp, comp, len(data), 2835, 2835, 0, 0)
        if hsz >= 108:
            m = list(masks or (0, 0, 0, 0))
            info += struct.pack("<IIII", *m) + b"\0" * (hsz - 56)
        elif masks is not None and comp == 3:
            extra = struct.pack("<III", *masks[:3])
    off = 14 + len(info) + len(extra) + len(pal)
    return b"BM" + struct.pack("<IHHI", off + len(data), 0, 0, off) + info + extra + pal + data


def _widen(v, n):
    r, have = 0, 0
    while have < 8:
        r, have = (r << n) | v, have + n
    return (r >> (have - 8)) & 0xff


def _field(v, mask):
    lo = (mask & -mask).bit_length() - 1
    n = bin(mask).count("1")
    return _widen((v & mask) >> lo, n)


def test_bmp_1_bit_matches_pil(png_check, tmp_path):
    from PIL import Image
    arr = (np.random.default_rng(3).random((13, 21)) > 0.5).astype(np.uint8) * 255
    path = str(tmp_path / "b1.bmp")
    Image.fromarray(arr).convert("1").save(path)
    got = decode(png_check, path)
    assert np.array_equal(got[..., :3], np.asarray(Image.open(path).convert("RGB")))
    assert (got[..., 3] == 255).all()


@pytest.mark.parametrize("hsz", [12, 40, 124])
@pytest.mark.parametrize("bpp", [4, 8])
def test_bmp_palettes_and_headers(png_check, tmp_path, hsz, bpp):
    rng = np.random.default_rng(hsz + bpp)
    w, h, ncol = 11, 7, (16 if bpp == 4 else 200)
    pal = [tuple(int(x) for x in rng.integers(0, 256, 3)) for _ in range(ncol)]
    idx = rng.integers(0, ncol, (h, w))
    rows = []
    for y in range(h):
        if bpp == 8:
            rows.append(bytes(int(i) for i in idx[y]))
        else:
            v = list(idx[y]) + [0]
            rows.append(bytes((int(v[2 * k]) << 4) | int(v[2 * k + 1]) for k in range((w + 1) // 2)))
    path = tmp_path / "p.bmp"
    path.write_bytes(_bmp(w, h, bpp, rows, hsz=hsz, palette=pal))
    got = decode(png_check, str(path))
    want = np.array(pal, np.uint8)[idx]
    assert np.array_equal(got[..., :3], want) and (got[..., 3] == 255).all()


def test_bmp_index_past_palette_reads_black(png_check, tmp_path):
    rows = [bytes([0, 1, 5])]
    path = tmp_path / "i.bmp"
    path.write_bytes(_bmp(3, 1, 8, rows, palette=[(10, 20, 30), (40, 50, 60)]))
    got = decode(png_check, str(path))
    assert got[0, :, :3].tolist() == [[10, 20, 30], [40, 50, 60], [0, 0, 0]]


@pytest.mark.parametrize("masks", [None, (0xF800, 0x07E0, 0x001F), (0x7C00, 0x03E0, 0x001F), (0x0F00, 0x00F0, 0x000F)])
@pytest.mark.parametrize("top_down", [False, True])
def test_bmp_16_bit(png_check, tmp_path, masks, top_down):
    rng = np.random.default_rng(16)
    w, h = 9, 5
    px = rng.integers(0, 1 << 16, (h, w))
    rows = [b"".join(struct.pack("<H", int(v)) for v in px[y]) for y in range(h)]
    path = tmp_path / "s.bmp"
    path.write_bytes(_bmp(w, h, 16, rows, comp=3 if masks else 0, masks=masks, top_down=top_down))
    got = decode(png_check, str(path))
    m = masks or (0x7C00, 0x03E0, 0x001F)
    want = np.array([[[_field(int(v), m[c]) for c in range(3)] for v in row] for row in px], np.uint8)
    assert np.array_equal(got[..., :3], want) and (got[..., 3] == 255).all()


@pytest.mark.parametrize("alpha", ["zero", "mixed"])
def test_bmp_32_bit_alpha_rule(png_check, tmp_path, alpha):
    rng = np.random.default_rng(32)
    w, h = 6, 4
    bgra = rng.integers(0, 256, (h, w, 4), dtype=np.uint8)
    if alpha == "zero":
        bgra[..., 3] = 0
    path = tmp_path / "a.bmp"
    path.write_bytes(_bmp(w, h, 32, [bgra[y].tobytes() for y in range(h)]))
    got = decode(png_check, str(path))
    assert np.array_equal(got[..., :3], bgra[..., 2::-1])
    assert np.array_equal(got[..., 3], np.full((h, w), 255, np.uint8) if alpha == "zero" else bgra[..., 3])


def test_bmp_v5_bitfields_with_alpha(png_check, tmp_path):
    rng = np.random.default_rng(5)
    w, h = 5, 3
    masks = (0x0000FF00, 0x00FF0000, 0xFF000000, 0x000000FF)  # R, G, B, A
    px = rng.integers(0, 1 << 32, (h, w), dtype=np.uint64)
    rows = [b"".join(struct.pack("<I", int(v)) for v in px[y]) for y in range(h)]
    path = tmp_path / "v5.bmp"
    path.write_bytes(_bmp(w, h, 32, rows, hsz=124, comp=3, masks=masks))
    got = decode(png_check, str(path))
    want = np.array([[[_field(int(v), masks[c]) for c in range(4)] for v in row] for row in px], np.uint8)
    assert np.array_equal(got, want)


def test_bmp_run_length_is_refused(png_check, tmp_path):
    path = tmp_path / "r.bmp"
    data = bytearray(_bmp(2, 2, 8, [b"\0\0", b"\0\0"], palette=[(0, 0, 0)]))
    data[30:34] = struct.pack("<I", 1)  # BI_RLE8
    path.write_bytes(bytes(data))
    assert subprocess.run([png_check, str(path)], capture_output=True).returncode != 0


def _tga(w, h, img_type, bpp, body, desc=0, cmap=None, cmap_first=0, cmap_bits=0, skip=b""):
    cmap_len = 0 if cmap is None else len(cmap) // ((cmap_bits + 7) // 8)
    head = struct.pack("<BBBHHBHHHHBB", 0, 1 if cmap is not None else 0, img_type, cmap_first, cmap_len, cmap_bits,
                       0, 0, w, h, bpp, desc)
    return head + skip + (cmap or b"") + body


def _rgb16(v):
    return [((v >> 10) & 31) * 255 // 31, ((v >> 5) & 31) * 255 // 31, (v & 31) * 255 // 31]


@pytest.mark.parametrize("bpp", [15, 16])
def test_tga_16_bit_true_colour(png_check, tmp_path, bpp):
    rng = np.random.default_rng(bpp)
    w, h = 7, 3
    px = rng.integers(0, 1 << 16, (h, w))
    body = b"".join(struct.pack("<H", int(v)) for v in px[::-1].ravel())  # bottom-up
    path = tmp_path / "t16.tga"
    path.write_bytes(_tga(w, h, 2, bpp, body))
    got = decode(png_check, str(path))
    want = np.array([[_rgb16(int(v)) for v in row] for row in px], np.uint8)
    assert np.array_equal(got[..., :3], want) and (got[..., 3] == 255).all()


def test_tga_grey_with_alpha(png_check, tmp_path):
    w, h = 4, 2
    ga = np.arange(w * h * 2, dtype=np.uint8).reshape(h, w, 2) * 7
    path = tmp_path / "ga.tga"
    path.write_bytes(_tga(w, h, 3, 16, ga[::-1].tobytes()))
    got = decode(png_check, str(path))
    assert np.array_equal(got[..., 0], ga[..., 0]) and np.array_equal(got[..., 2], ga[..., 0])
    assert np.array_equal(got[..., 3], ga[..., 1])


@pytest.mark.parametrize("cmap_bits,index_bits", [(16, 8), (24, 16), (32, 8), (8, 8)])
def test_tga_colour_maps(png_check, tmp_path, cmap_bits, index_bits):
    rng = np.random.default_rng(cmap_bits + index_bits)
    w, h, n = 6, 3, 40
    eb = (cmap_bits + 7) // 8
    cmap = rng.integers(0, 256, n * eb, dtype=np.uint8).tobytes()
    idx = rng.integers(0, n + 5, (h, w))  # indices past the map take entry 0
    body = b"".join((struct.pack("<H", int(i)) if index_bits == 16 else bytes([int(i)])) for i in idx[::-1].ravel())
    path = tmp_path / "cm.tga"
    path.write_bytes(_tga(w, h, 1, index_bits, body, cmap=cmap, cmap_bits=cmap_bits, cmap_first=3, skip=b"\x11" * 3))

    def entry(i):
        i = i if i < n else 0
        e = cmap[i * eb:(i + 1) * eb]
        if cmap_bits == 8:
            return [e[0]] * 3 + [255]
        if cmap_bits == 16:
            return _rgb16(e[0] | e[1] << 8) + [255]
        return [e[2], e[1], e[0], e[3] if cmap_bits == 32 else 255]
    want = np.array([[entry(int(i)) for i in row] for row in idx], np.uint8)
    got = decode(png_check, str(path))
    assert np.array_equal(got, want)


def test_tga_right_to_left_bit_is_ignored_and_runs_end_with_the_image(png_check, tmp_path):
    w, h = 3, 2
    px = np.arange(w * h * 3, dtype=np.uint8).reshape(h, w, 3)
    body = px[::-1, :, ::-1].tobytes()  # bottom-up BGR
    path = tmp_path / "rl.tga"
    path.write_bytes(_tga(w, h, 2, 24, body, desc=0x10))
    assert np.array_equal(decode(png_check, str(path))[..., :3], px)
    # a run-length packet of 128 repeats covers the 6 pixels and ends with the image
    path.write_bytes(_tga(w, h, 10, 24, bytes([0xFF, 1, 2, 3])))
    got = decode(png_check, str(path))
    assert (got[..., :3] == np.array([3, 2, 1], np.uint8)).all()


@pytest.mark.parametrize("magic,ch", [(b"P5", 1), (b"P6", 3)])
def test_pnm_16_bit_and_small_maxval(png_check, tmp_path, magic, ch):
    """maxval > 255: two bytes a sample, the loader keeps the second; maxval < 255: samples as they
    are, not rescaled; comments end at CR or LF."""
    rng = np.random.default_rng(ch)
    w, h = 5, 4
    s16 = rng.integers(0, 65536, (h, w, ch)).astype(">u2")
    path = tmp_path / "d.pnm"
    path.write_bytes(magic + b"\n# made here\r%d %d\n65535\n" % (w, h) + s16.tobytes())
    got = decode(png_check, str(path))
    low = (s16.astype(np.uint32) & 0xFF).astype(np.uint8)
    want = np.repeat(low, 3, axis=2) if ch == 1 else low
    assert np.array_equal(got[..., :3], want) and (got[..., 3] == 255).all()
    s8 = rng.integers(0, 16, (h, w, ch), dtype=np.uint8)
    path.write_bytes(magic + b" %d %d 15\n" % (w, h) + s8.tobytes())
    got = decode(png_check, str(path))
    assert np.array_equal(got[..., :3], np.repeat(s8, 3, axis=2) if ch == 1 else s8)


def test_malformed_files_are_refused_not_crashed(png_check, tmp_path):
    """Truncated and byte-mutated files of every input format end with a decoded image or an error
    exit (status 1), never a crash.  (Sanitizer runs of the same mutations, thousands per format,
    found no invalid memory access either.)"""
    from PIL import Image
    rng = np.random.default_rng(12)
    arr = rng.integers(0, 256, (19, 23, 3), dtype=np.uint8)
    seeds = []
    for ext, kw in ((".png", {}), (".png", {"interlace": True}), (".bmp", {}), (".tga", {"compression": "tga_rle"}),
                    (".gif", {}), (".ppm", {}), (".jpg", {"quality": 80}), (".jpg", {"progressive": True})):
        p = tmp_path / ("seed%d%s" % (len(seeds), ext))
        Image.fromarray(arr).save(str(p), **kw)
        seeds.append((ext, p.read_bytes()))
    seeds.append((".psd", _psd(rng.integers(0, 256, (4, 9, 14)).astype(np.uint32), 8, True)))
    seeds.append((".bmp", _bmp(9, 5, 16, [bytes(18)] * 5, comp=3, masks=(0xF800, 0x07E0, 0x001F))))
    seeds.append((".tga", _tga(6, 3, 1, 16, bytes(36), cmap=bytes(120), cmap_bits=24)))
    for ext, data in seeds:
        for it in range(12):
            b = bytearray(data)
            if it % 2 == 0:
                b = b[:int(rng.integers(0, len(b)))]
            else:
                for i in rng.integers(0, len(b), 6):
                    b[i] = int(rng.integers(0, 256))
            p = tmp_path / ("m" + ext)
            p.write_bytes(bytes(b))
            r = subprocess.run([png_check, str(p)], capture_output=True, timeout=30)
            assert r.returncode in (0, 1), (ext, it, r.returncode)
