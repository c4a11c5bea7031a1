"""Seeded synthetic image pairs for the benchmarks and tests.

No dataset ships with IQM and none is named for its benchmarks, so every image is generated:
RGBA8 (A = 255), grey images stored as R = G = B.

* base image: white Gaussian noise, shaped in the Fourier domain by 1/|f| (power ~ 1/f^2, DC
  removed), min-max rescaled to [0, 255] and rounded to uint8;
* RGB images use an independent seed per channel; seeds are 1000*config + 10*pair + channel and
  the distortion RNG uses seed + 500.

Distortions per workload:
  ssim_512   (grey)  ref + N(0, 8^2), 3x3 box blur with replicated edges, clamp, round
  fsim_1080p (RGB)   ref + N(0, 10^2), times a per-channel gain U(0.9, 1.1), clamp, round
  flip_1080p (RGB)   per 8x8 block and channel, uniform quantisation with step U(4, 24)
                     (round(v/step)*step), then + N(0, 4^2), clamp, round   (also used for M-SVD)
"""
import numpy as np


def _pink(h, w, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    noise = rng.standard_normal((h, w))
    fy = np.fft.fftfreq(h)[:, None]
    fx = np.fft.fftfreq(w)[None, :]
    f = np.sqrt(fx * fx + fy * fy)
    amp = np.zeros_like(f)
    nz = f > 0
    amp[nz] = 1.0 / f[nz]
    img = np.real(np.fft.ifft2(np.fft.fft2(noise) * amp))
    lo, hi = img.min(), img.max()
    img = (img - lo) / (hi - lo if hi > lo else 1.0) * 255.0
    return np.clip(np.rint(img), 0, 255)


def _rgba(channels):
    h, w = channels[0].shape
    out = np.empty((h, w, 4), np.uint8)
    for c in range(3):
        out[..., c] = channels[c if len(channels) == 3 else 0].astype(np.uint8)
    out[..., 3] = 255
    return out


def _box3(x):
    p = np.pad(x, 1, mode="edge")
    acc = np.zeros_like(x)
    for dy in range(3):
        for dx in range(3):
            acc += p[dy:dy + x.shape[0], dx:dx + x.shape[1]]
    return acc / 9.0


def grey_pair(h, w, config=0, pair=0):
    """SSIM-style grey pair: returns (distorted, reference) RGBA8 arrays."""
    seed = 1000 * config + 10 * pair
    ref = _pink(h, w, seed)
    rng = np.random.Generator(np.random.PCG64(seed + 500))
    dist = _box3(ref + rng.normal(0.0, 8.0, ref.shape))
    dist = np.clip(np.rint(dist), 0, 255)
    return _rgba([dist]), _rgba([ref])


def rgb_gain_pair(h, w, config=1, pair=0):
    """FSIM-style RGB pair: noise sigma 10 and a per-channel gain U(0.9, 1.1)."""
    base = 1000 * config + 10 * pair
    refc = [_pink(h, w, base + c) for c in range(3)]
    rng = np.random.Generator(np.random.PCG64(base + 500))
    distc = []
    for c in range(3):
        gain = rng.uniform(0.9, 1.1)
        d = (refc[c] + rng.normal(0.0, 10.0, refc[c].shape)) * gain
        distc.append(np.clip(np.rint(d), 0, 255))
    return _rgba(distc), _rgba(refc)


def rgb_blockquant_pair(h, w, config=2, pair=0):
    """FLIP / M-SVD pair: 8x8-block uniform quantisation (step U(4, 24)) plus noise sigma 4."""
    base = 1000 * config + 10 * pair
    refc = [_pink(h, w, base + c) for c in range(3)]
    rng = np.random.Generator(np.random.PCG64(base + 500))
    bh, bw = (h + 7) // 8, (w + 7) // 8
    distc = []
    for c in range(3):
        steps = rng.uniform(4.0, 24.0, (bh, bw))
        step = np.kron(steps, np.ones((8, 8)))[:h, :w]
        q = np.rint(refc[c] / step) * step
        d = q + rng.normal(0.0, 4.0, q.shape)
        distc.append(np.clip(np.rint(d), 0, 255))
    return _rgba(distc), _rgba(refc)


def uneven_sizes(n, seed=3000, lo=256, hi=2048):
    """Widths and heights drawn independently and uniformly from [lo, hi] (batched workload)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return [(int(rng.integers(lo, hi + 1)), int(rng.integers(lo, hi + 1))) for _ in range(n)]
