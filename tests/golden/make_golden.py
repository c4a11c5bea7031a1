"""Regenerates the golden fixtures in this directory (run from the repository root, CPU only).

The reference (cadik/IQM) ships no tests or golden data and its GPU path cannot run here, so the
fixtures come from two sources:

* OpenCV (cv2), the library the reference's M-SVD stage calls (src/gpu/svd/svd.cpp:50-87):
    gray.npz   -- cv::cvtColor(COLOR_RGB2GRAY) on random RGBA pixels
    svd8.npz   -- cv::SVD(.., NO_UV) singular values of random 8x8 blocks
    msvd.npz   -- whole M-SVD scores of small seeded pairs, computed by a line-by-line Python
                  restatement of src/gpu/svd/svd.cpp:39-164 and shaders/svd/svd.glsl that calls
                  cv2 for the grey conversion and every block SVD (float32 arithmetic and the
                  float running sum over the sorted distances, as the reference does)
* the FP64 and FP32 oracle builds (regression anchors for SSIM, FSIM and FLIP, whose reference
  arithmetic exists only as GLSL):
    scores.npz -- small seeded pairs and their oracle scores

Usage:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import cv2  # noqa: E402

from iqm_b200 import synth  # noqa: E402
from oracle import Oracle  # noqa: E402


def cv2_msvd(img, ref):
    """src/gpu/svd/svd.cpp:39-164 restated with cv2 for every library call."""
    h, w = img.shape[:2]
    gi = cv2.cvtColor(np.ascontiguousarray(img), cv2.COLOR_RGB2GRAY).astype(np.float32)
    gr = cv2.cvtColor(np.ascontiguousarray(ref), cv2.COLOR_RGB2GRAY).astype(np.float32)
    bw, bh = w // 8, h // 8
    D = np.zeros(bw * bh, np.float32)
    y = 0
    while y + 8 < h:
        x = 0
        while x + 8 < w:
            si = cv2.SVDecomp(np.ascontiguousarray(gi[y:y + 8, x:x + 8]), flags=cv2.SVD_NO_UV)[0].ravel()
            sr = cv2.SVDecomp(np.ascontiguousarray(gr[y:y + 8, x:x + 8]), flags=cv2.SVD_NO_UV)[0].ravel()
            acc = np.float32(0)
            for k in range(8):  # shaders/svd/svd.glsl:41-52, float, in order
                d = np.float32(si[k] - sr[k])
                acc = np.float32(acc + d * d)
            D[(y // 8) * bw + x // 8] = np.sqrt(acc)
            x += 8
        y += 8
    s = np.sort(D)
    mid = s[len(s) // 2]
    run = np.add.accumulate(np.abs(s - mid).astype(np.float32), dtype=np.float32)
    msvd = np.float32(run[-1] / np.float32(len(s)))
    return float(msvd), D.reshape(bh, bw)


def main():
    rng = np.random.default_rng(20241)
    # grey conversion
    rgba = rng.integers(0, 256, (1, 8192, 4), dtype=np.uint8)
    rgba[0, :256, 0] = np.arange(256)
    rgba[0, 256:512, 1] = np.arange(256)
    rgba[0, 512:768, 2] = np.arange(256)
    gray = cv2.cvtColor(rgba, cv2.COLOR_RGB2GRAY).ravel()
    np.savez_compressed(os.path.join(HERE, "gray.npz"), rgba=rgba[0], gray=gray)

    # 8x8 singular values
    blocks = []
    for i in range(512):
        b = rng.integers(0, 256, (8, 8)).astype(np.float32)
        if i % 4 == 1:
            b = np.round(b / 64) * 64
        elif i % 4 == 2:
            b[:] = b[0]
        elif i % 4 == 3:
            b = np.clip(np.round(np.outer(rng.random(8), rng.random(8)) * 255 + rng.normal(0, 2, (8, 8))), 0, 255).astype(np.float32)
        blocks.append(b)
    blocks = np.stack(blocks)
    sv = np.stack([cv2.SVDecomp(b, flags=cv2.SVD_NO_UV)[0].ravel() for b in blocks])
    np.savez_compressed(os.path.join(HERE, "svd8.npz"), blocks=blocks, sv=sv)

    # whole M-SVD
    sizes = [(48, 64), (77, 101), (72, 136), (64, 64)]
    imgs, refs, scores, dists = [], [], [], []
    for i, (h, w) in enumerate(sizes):
        a, b = synth.rgb_blockquant_pair(h, w, config=2, pair=90 + i)
        m, d = cv2_msvd(a, b)
        imgs.append(a)
        refs.append(b)
        scores.append(m)
        dists.append(d)
    np.savez_compressed(os.path.join(HERE, "msvd.npz"), sizes=np.array(sizes),
                        scores=np.array(scores), **{"img%d" % i: v for i, v in enumerate(imgs)},
                        **{"ref%d" % i: v for i, v in enumerate(refs)},
                        **{"dist%d" % i: v for i, v in enumerate(dists)})

    # oracle regression anchors for SSIM / FSIM / FLIP
    o64, o32 = Oracle("f64"), Oracle("f32")
    out = {}
    cases = [("ssim", (64, 80), synth.grey_pair, 0), ("ssim", (37, 45), synth.grey_pair, 0),
             ("fsim", (96, 128), synth.rgb_gain_pair, 1), ("fsim", (130, 200), synth.rgb_gain_pair, 1),
             ("flip", (64, 96), synth.rgb_blockquant_pair, 2), ("flip", (41, 59), synth.rgb_blockquant_pair, 2)]
    for j, (metric, (h, w), gen, cfg) in enumerate(cases):
        a, b = gen(h, w, config=cfg, pair=50 + j)
        out["img%d" % j] = a
        out["ref%d" % j] = b
        if metric == "ssim":
            v64, v32 = [o64.ssim(a, b)], [o32.ssim(a, b)]
        elif metric == "fsim":
            v64, v32 = list(o64.fsim(a, b)), list(o32.fsim(a, b))
        else:
            v64, v32 = [o64.flip(a, b, ppd=67.0)], [o32.flip(a, b, ppd=67.0)]
        out["f64_%d" % j] = np.array(v64)
        out["f32_%d" % j] = np.array(v32)
    out["metrics"] = np.array([c[0] for c in cases])
    np.savez_compressed(os.path.join(HERE, "scores.npz"), **out)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
