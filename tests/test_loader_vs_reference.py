"""The command line's image decoders against the reference's own loader: cadik/IQM reads every input
with stbi_load(path, ..., 4) from the stb_image.h it vendors (src/main.cpp:37-57).  `make -C oracle
ref` builds that call from the reference's tree into oracle/_ref/ref_loader (test infrastructure,
never part of the product); these tests skip where the reference tree is absent.

Lossless formats (PNG in every colour type, bit depth and interlace; PNM; BMP and TGA layouts;
GIF; Radiance HDR; PSD; Softimage PIC) must decode to the same RGBA bytes, alpha included.  JPEG is lossy, and the
loader's integer IDCT and fixed-point colour conversion are its own: the bound there is 3 levels
per channel and a mean below 0.15 (chroma upsampling, including the loader's 4:2:2 edge rule,
follows the loader)."""
import os
import struct
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HOST = os.path.join(ROOT, "iqm_b200", "host")
REF_TREE = "/root/reference/lib/stb/stb_image.h"


@pytest.fixture(scope="module")
def ref_loader():
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_loader")
    if not os.path.exists(exe):
        if not os.path.exists(REF_TREE):
            pytest.skip("the reference tree is not available")
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True)
    return exe


@pytest.fixture(scope="module")
def ours(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("native") / "png_check")
    subprocess.run(["/usr/bin/g++", "-O1", "-std=c++20", "-I", HOST, "-o", exe,
                    os.path.join(ROOT, "tests", "native", "png_check.cpp"), os.path.join(HOST, "png_io.cpp"),
                    os.path.join(HOST, "image_formats.cpp"), os.path.join(HOST, "jpeg_decode.cpp"), "-lz"],
                   check=True)
    return exe


def run(exe, path):
    out = subprocess.run([exe, path], capture_output=True, check=True).stdout
    w, h = struct.unpack("<II", out[:8])
    return np.frombuffer(out[8:], np.uint8).reshape(h, w, 4)


def noise(h, w, seed):
    return np.random.default_rng(seed).integers(0, 256, (h, w, 3), dtype=np.uint8)


def lossless_files(tmp_path):
    """A spread of lossless files written by PIL and OpenCV."""
    from PIL import Image
    arr = noise(37, 53, 1)
    files = []
    for mode in ["L", "LA", "RGB", "RGBA", "P", "1"]:
        for inter in (False, True):
            im = Image.fromarray(arr)
            im = im.convert("P", palette=Image.ADAPTIVE, colors=50) if mode == "P" else im.convert(mode)
            p = str(tmp_path / ("png_%s_%d.png" % (mode, inter)))
            im.save(p, interlace=inter)
            files.append(p)
    p = str(tmp_path / "png_16.png")
    Image.fromarray(arr[..., 0].astype(np.uint16) * 257).save(p)
    files.append(p)
    for mode in ["RGB", "RGBA", "P", "L", "1"]:
        im = Image.fromarray(arr)
        im = im.convert("P", palette=Image.ADAPTIVE, colors=64) if mode == "P" else im.convert(mode)
        p = str(tmp_path / ("bmp_%s.bmp" % mode))
        im.save(p)
        files.append(p)
    for mode in ["RGB", "RGBA", "L", "P"]:
        for rle in (False, True):
            im = Image.fromarray(arr)
            im = im.convert("P", palette=Image.ADAPTIVE, colors=32) if mode == "P" else im.convert(mode)
            p = str(tmp_path / ("tga_%s_%d.tga" % (mode, rle)))
            im.save(p, compression="tga_rle" if rle else None)
            files.append(p)
    p = str(tmp_path / "a.gif")
    Image.fromarray(arr).convert("P", palette=Image.ADAPTIVE, colors=64).save(p)
    files.append(p)
    for ext in ("ppm", "pgm"):
        p = str(tmp_path / ("a." + ext))
        (Image.fromarray(arr) if ext == "ppm" else Image.fromarray(arr[..., 1])).save(p)
        files.append(p)
    cv2 = pytest.importorskip("cv2")
    p = str(tmp_path / "a.hdr")
    cv2.imwrite(p, arr.astype(np.float32) / 40.0)
    files.append(p)
    return files


def test_lossless_formats_decode_to_the_loaders_bytes(ref_loader, ours, tmp_path):
    for p in lossless_files(tmp_path):
        assert np.array_equal(run(ours, p), run(ref_loader, p)), os.path.basename(p)


def test_bmp_and_tga_layouts_decode_to_the_loaders_bytes(ref_loader, ours, tmp_path):
    """The hand-built layouts of tests/test_cli.py: 4-bit palettes, the V5 header, 16-bit and
    bit-field pixels, the BI_RGB 32-bit alpha rule, 15/16-bit TGA pixels and colour maps, 16-bit
    indices, grey with alpha.  (OS/2 core-header palettes are left out: the loader reads four entries
    fewer than such a file holds and returns unset values for the last four indices.)"""
    import test_cli as t
    rng = np.random.default_rng(7)
    files = []
    pal = [tuple(int(x) for x in rng.integers(0, 256, 3)) for _ in range(16)]
    idx = rng.integers(0, 16, (7, 11))
    def pack4(r):  # two 4-bit indices a byte, high nibble first
        v = [int(x) for x in r] + [0]
        return bytes((v[2 * k] << 4) | v[2 * k + 1] for k in range((len(r) + 1) // 2))
    rows = [pack4(r) for r in idx]
    for hsz in (40, 124):
        files.append(("b4_%d.bmp" % hsz, t._bmp(11, 7, 4, rows, hsz=hsz, palette=pal)))
    px16 = rng.integers(0, 1 << 16, (5, 9))
    rows16 = [b"".join(struct.pack("<H", int(v)) for v in r) for r in px16]
    files.append(("b16.bmp", t._bmp(9, 5, 16, rows16)))
    files.append(("b565.bmp", t._bmp(9, 5, 16, rows16, comp=3, masks=(0xF800, 0x07E0, 0x001F))))
    bgra = rng.integers(0, 256, (4, 6, 4), dtype=np.uint8)
    files.append(("b32.bmp", t._bmp(6, 4, 32, [r.tobytes() for r in bgra])))
    bgra[..., 3] = 0
    files.append(("b32z.bmp", t._bmp(6, 4, 32, [r.tobytes() for r in bgra])))
    px32 = rng.integers(0, 1 << 32, (3, 5), dtype=np.uint64)
    files.append(("b5.bmp", t._bmp(5, 3, 32, [b"".join(struct.pack("<I", int(v)) for v in r) for r in px32], hsz=124,
                                   comp=3, masks=(0x0000FF00, 0x00FF0000, 0xFF000000, 0x000000FF))))
    t16 = rng.integers(0, 1 << 16, (3, 7))
    files.append(("t16.tga", t._tga(7, 3, 2, 16, b"".join(struct.pack("<H", int(v)) for v in t16.ravel()))))
    files.append(("tga.tga", t._tga(4, 2, 3, 16, rng.integers(0, 256, 16, dtype=np.uint8).tobytes())))
    cmap = rng.integers(0, 256, 40 * 2, dtype=np.uint8).tobytes()
    files.append(("tcm16.tga", t._tga(6, 3, 1, 8, rng.integers(0, 40, 18, dtype=np.uint8).tobytes(), cmap=cmap,
                                      cmap_bits=16)))
    cmap24 = rng.integers(0, 256, 300 * 3, dtype=np.uint8).tobytes()
    ix = b"".join(struct.pack("<H", int(v)) for v in rng.integers(0, 300, 18))
    files.append(("tcm24i16.tga", t._tga(6, 3, 1, 16, ix, cmap=cmap24, cmap_bits=24)))
    for name, data in files:
        p = tmp_path / name
        p.write_bytes(data)
        assert np.array_equal(run(ours, str(p)), run(ref_loader, str(p))), name


@pytest.mark.parametrize("subsampling", [0, 1, 2])
@pytest.mark.parametrize("progressive", [False, True])
@pytest.mark.parametrize("size", [(37, 53), (48, 64), (9, 7)])
def test_jpeg_within_three_levels_of_the_loader(ref_loader, ours, tmp_path, subsampling, progressive, size):
    from PIL import Image
    p = str(tmp_path / "j.jpg")
    Image.fromarray(noise(*size, 2)).save(p, quality=90, subsampling=subsampling, progressive=progressive)
    d = np.abs(run(ours, p).astype(int) - run(ref_loader, p).astype(int))
    assert d.max() <= 3 and d.mean() < 0.15, (d.max(), d.mean())


def test_gif_hdr_psd_pic_layouts_decode_to_the_loaders_bytes(ref_loader, ours, tmp_path):
    """The hand-built files of tests/test_cli.py: a GIF frame inside a larger screen with a
    transparent index and a background entry; flat and run-length HDR scanlines; PSD with 3 to 5
    channels, 8 and 16 bits, raw and PackBits (alpha un-premultiplied); PIC with raw, pure and mixed
    run-length packets."""
    import test_cli as t
    rng = np.random.default_rng(11)
    files = []
    pal = [tuple(int(v) for v in rng.integers(0, 256, 3)) for _ in range(8)]
    frame = rng.integers(0, 8, (5, 6)).astype(np.uint8)
    files.append(("t.gif", t._gif(11, 9, pal, 2, frame, x0=3, y0=2, transparent=6)))
    for w, rle in ((5, False), (40, True)):
        rgbe = rng.integers(0, 256, (7, w, 4)).astype(np.uint8)
        rgbe[..., 0] |= 0x80
        rgbe[:, :w // 3, :] = rgbe[:, :1, :]
        body = b"".join(t._hdr_rle_scanline(rgbe[y]) for y in range(7)) if rle else rgbe.tobytes()
        files.append(("x%d.hdr" % w, b"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n-Y 7 +X %d\n" % w + body))
    for channels, depth, rle in [(3, 8, False), (3, 8, True), (4, 8, False), (4, 8, True), (3, 16, False),
                                 (5, 16, False)]:
        planes = rng.integers(0, 1 << depth, (channels, 9, 14)).astype(np.uint32)
        planes[:, :, :5] = planes[:, :, :1]
        files.append(("p%d%d%d.psd" % (channels, depth, rle), t._psd(planes, depth, rle)))
    img = rng.integers(0, 256, (6, 150, 4)).astype(np.uint8)
    img[:, 3:140] = img[:, 3:4]
    for codings in [(0,), (1,), (2,), (2, 1)]:
        packets = [(codings[0], 0xE0)] + ([(codings[1], 0x10)] if len(codings) > 1 else [])
        rows = [b"".join(t._pic_encode_row(img[y], c, m) for c, m in packets) for y in range(6)]
        files.append(("x%s.pic" % "".join(map(str, codings)), t._pic(150, 6, packets, rows)))
    for name, data in files:
        p = tmp_path / name
        p.write_bytes(data)
        assert np.array_equal(run(ours, str(p)), run(ref_loader, str(p))), name
