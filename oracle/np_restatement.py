"""A second, independent FP64 restatement of FSIM/FSIMc and FLIP in numpy.

TEST INFRASTRUCTURE ONLY: tests import it to cross-check the C oracle (oracle/iqm_oracle.c).  The
product library never imports, links or calls anything here.

The reference's FSIM and FLIP exist only as GLSL compute shaders run through Vulkan and VkFFT (none
of which can run here), and the reference ships no tests or golden data for them, so no output of the
reference itself can pin these metrics.  This module is written directly from the shaders and host
code, whole-plane and vectorised, with numpy.fft in place of VkFFT and no code in common with the C
oracle (which follows the shaders pixel by pixel).  Agreement between the two restatements pins the
reading of every shader: a misreading in one of them shows up as a disagreement.

Every function cites the reference file:line it restates (paths within cadik/IQM).
"""
import math

import numpy as np

GLSL_PI = 3.141592653589  # the literal the FSIM and FLIP shaders use for PI


def _round_half_away(v):
    """std::round (half away from zero)."""
    return math.floor(v + 0.5) if v >= 0 else -math.floor(-v + 0.5)


# ============================================================================================= FSIM
def fsim_downscale_factor(w, h):
    """src/gpu/fsim/fsim.cpp:165-168: max(1, round(min(W, H) / 256.0))."""
    return max(1, int(_round_half_away(min(w, h) / 256.0)))


def fsim_plane_size(w, h, F):
    """src/gpu/fsim/fsim.cpp:91-92: round((float)W / (float)F), likewise for H."""
    return (int(_round_half_away(float(np.float32(w) / np.float32(F)))),
            int(_round_half_away(float(np.float32(h) / np.float32(F)))))


def fsim_yiq_planes(img, F, w2, h2):
    """shaders/fsim/fsim_downsample.glsl:21-55: unorm x 255 (the byte value), colorConvert to
    (I, Q, Y), summed over the F x F window starting at (x F - F/2, y F - F/2) with samples outside
    the image skipped, divided by F^2.  Returns I, Q, Y as (h2, w2) float64 arrays."""
    h, w = img.shape[:2]
    rgb = img[..., :3].astype(np.float64)
    r, g, b = rgb[..., 0], rgb[..., 1], rgb[..., 2]
    chans = (r * 0.596 - g * 0.274 - b * 0.322,
             r * 0.211 - g * 0.523 + b * 0.312,
             r * 0.299 + g * 0.587 + b * 0.114)
    off = F // 2
    out = []
    for c in chans:
        # window (x2, y2) covers rows y2 F - off .. y2 F - off + F - 1: place the image at offset
        # `off` inside a zero canvas of h2 F x w2 F and sum F x F blocks
        canvas = np.zeros((h2 * F + F, w2 * F + F))
        hh, ww = min(h, h2 * F - off), min(w, w2 * F - off)
        canvas[off:off + hh, off:off + ww] = c[:hh, :ww]
        blocks = canvas[:h2 * F, :w2 * F].reshape(h2, F, w2, F).sum(axis=(1, 3))
        out.append(blocks / float(F * F))
    return out


def fsim_gradient(Y):
    """shaders/fsim/fsim_gradientmap.glsl:16-57: 3x3 weights (vertical: x-derivative 3/10/3,
    horizontal: y-derivative), zero outside the plane, magnitude of the sums / 16."""
    h2, w2 = Y.shape
    P = np.zeros((h2 + 2, w2 + 2))
    P[1:-1, 1:-1] = Y
    vert = np.array([3.0, 0.0, -3.0, 10.0, 0.0, -10.0, 3.0, 0.0, -3.0])
    hor = np.array([3.0, 10.0, 3.0, 0.0, 0.0, 0.0, -3.0, -10.0, -3.0])
    vs = np.zeros_like(Y)
    hs = np.zeros_like(Y)
    for j in (-1, 0, 1):          # x offset
        for k in (-1, 0, 1):      # y offset
            idx = (j + 1) + (k + 1) * 3
            win = P[1 + k:1 + k + h2, 1 + j:1 + j + w2]
            vs += win * vert[idx]
            hs += win * hor[idx]
    return np.sqrt((vs / 16.0) ** 2 + (hs / 16.0) ** 2)


def _freq_grid(n):
    """The ifftshifted coordinate of fsim_lowpassfilter.glsl:32-35 (integer n/2, also for odd n)."""
    i = np.arange(n)
    return (((i + n // 2) % n) - n // 2) / float(n)


def fsim_filters(w2, h2):
    """16 frequency-domain filters H[z], z = 4 o + s, shape (16, h2, w2):
    log-Gabor (fsim_log_gabor.glsl:16-49, minWaveLength 6, mult 2, sigmaOnf 0.55, DC = 0) times the
    Butterworth lowpass (fsim_lowpassfilter.glsl:21-42, cutoff 0.45, order 15) times the angular
    spread (fsim_angular.glsl:16-48), combined as fsim_filter_combinations.glsl:40-51."""
    sx = _freq_grid(w2)[None, :]
    sy = _freq_grid(h2)[:, None]
    radius = np.sqrt(sx * sx + sy * sy)
    lowpass = 1.0 / (1.0 + (radius / 0.45) ** (2.0 * 15))
    gabor = []
    with np.errstate(divide="ignore"):
        for s in range(4):
            freq = 1.0 / (6.0 * 2.0 ** s)
            v = np.exp(-np.log(radius / freq) ** 2 / (2.0 * np.log(0.55) ** 2)) * lowpass
            v[0, 0] = 0.0
            gabor.append(v)
    theta = np.arctan2(-sy, sx) + 0.0 * sx
    sint, cost = np.sin(theta), np.cos(theta)
    theta_sigma = GLSL_PI / 4 / 1.2
    H = np.empty((16, h2, w2))
    for o in range(4):
        angle = o * GLSL_PI / 4
        ds = sint * math.cos(angle) - cost * math.sin(angle)
        dc = cost * math.cos(angle) + sint * math.sin(angle)
        dtheta = np.abs(np.arctan2(ds, dc))
        ang = np.exp(-dtheta ** 2 / (2.0 * theta_sigma ** 2))
        for s in range(4):
            H[4 * o + s] = gabor[s] * ang
    return H


def fsim_noise_constants(H, energy_full=False):
    """Size-only constants of the noise model.
    EM[o] = sum over the frequency grid of H[4 o]^2 (fsim_filter_combinations.cpp:76-134 with
    fsim_filter_noise.glsl, which squares block 0's values on the first pass);
    An2[o], AiAj[o]: from the inverse transforms of the filters themselves (block 0 after the
    normalised inverse FFT, fsim.cpp:403-431), sum_s Re^2 N and sum_{i<j} Re_i Re_j N
    (fsim_mult_filters.glsl:26-59), pooled over pixels p < ceil(N/2) as the shader writes them
    (the rest of each buffer stays 0), or over all N pixels with energy_full."""
    h2, w2 = H.shape[1:]
    N = h2 * w2
    lim = N if energy_full else (N + 1) // 2
    em, an2, aiaj = np.empty(4), np.empty(4), np.empty(4)
    for o in range(4):
        em[o] = np.sum(H[4 * o] ** 2)
        re = [np.fft.ifft2(H[4 * o + s]).real.reshape(-1)[:lim] for s in range(4)]
        an2[o] = sum(np.sum(r * r * N) for r in re)
        aiaj[o] = sum(np.sum(re[i] * re[j] * N) for i in range(3) for j in range(i + 1, 4))
    return em, an2, aiaj


def fsim_responses(Y, H, ifft2=np.fft.ifft2):
    """Forward transform of luma (fsim.cpp:439-537, sign -1, unnormalised), the 16 filtered spectra
    (fsim_filter_combinations.glsl:53-56), the normalised inverse transforms (fsim.cpp:539-551) and,
    per orientation, the response sums of fsim_sum_filter_responses.glsl:37-80:
    amplitude sum_s |EO|, energy sum_s [E mE + O mO - |E mO - O mE|] with (mE, mO) = (sum E, sum O) /
    (|(sum E, sum O)| + 1e-4); plus |EO(s = 0)|^2 per orientation (fsim_pack_for_median.glsl:39-43).
    `ifft2` is the inverse 2-D transform used (numpy's by default)."""
    S = np.fft.fft2(Y)
    amp, energy, eo0 = [], [], []
    for o in range(4):
        eo = [ifft2(H[4 * o + s] * S) for s in range(4)]
        sE = sum(e.real for e in eo)
        sO = sum(e.imag for e in eo)
        xe = np.sqrt(sE * sE + sO * sO) + 0.0001
        mE, mO = sE / xe, sO / xe
        amp.append(sum(np.abs(e) for e in eo))
        energy.append(sum(e.real * mE + e.imag * mO - np.abs(e.real * mO - e.imag * mE) for e in eo))
        eo0.append(eo[0].real ** 2 + eo[0].imag ** 2)
    return amp, energy, eo0


def fsim_threshold(eo0, em, an2, aiaj):
    """Noise power from the upper median of a full sort (fsim_noise_power.cpp:193-203: v[N/2],
    mean = -median / ln 0.5, divided by EM) and the threshold T of fsim_phase_congruency.glsl:42-53
    (k = 2, divided by 1.7)."""
    v = np.sort(eo0.reshape(-1))
    median = v[v.size // 2]
    noise_power = (-median / math.log(0.5)) / em
    e2 = 2.0 * noise_power * an2 + 4.0 * noise_power * aiaj
    tau = math.sqrt(e2 / 2.0)
    mu = tau * math.sqrt(GLSL_PI / 2)
    sigma = math.sqrt((2 - GLSL_PI / 2) * tau * tau)
    return (mu + 2.0 * sigma) / 1.7


def fsim_phase_congruency(amp, energy, eo0, consts):
    """fsim_phase_congruency.glsl:39-64: sum_o max(E_o - T_o, 0) / sum_o A_o (no epsilon)."""
    em, an2, aiaj = consts
    num = sum(np.maximum(energy[o] - fsim_threshold(eo0[o], em[o], an2[o], aiaj[o]), 0.0) for o in range(4))
    with np.errstate(invalid="ignore", divide="ignore"):
        return num / sum(amp)


def fsim_pool(pc1, pc2, g1, g2, iq1, iq2):
    """fsim_final_multiply.glsl:18-58 (T1 0.85, T2 160, T3 = T4 200, lambda 0.03) and the host's
    division of the pooled sums (fsim_final_multiply.cpp:294-300)."""
    pcm = np.maximum(pc1, pc2)
    pcsim = (2.0 * pc1 * pc2 + 0.85) / (pc1 ** 2 + pc2 ** 2 + 0.85)
    gsim = (2.0 * g1 * g2 + 160.0) / (g1 ** 2 + g2 ** 2 + 160.0)
    isim = (2.0 * iq1[0] * iq2[0] + 200.0) / (iq1[0] ** 2 + iq2[0] ** 2 + 200.0)
    qsim = (2.0 * iq1[1] * iq2[1] + 200.0) / (iq1[1] ** 2 + iq2[1] ** 2 + 200.0)
    sim = gsim * pcsim * pcm
    simc = gsim * pcsim * np.abs(isim * qsim) ** 0.03 * pcm
    s_pcm = np.sum(pcm)
    return float(np.sum(sim) / s_pcm), float(np.sum(simc) / s_pcm)


def fsim(img, ref, energy_full=False, ifft2=np.fft.ifft2):
    """FSIM, FSIMc of an RGBA8 pair (h, w, 4): IQM::GPU::FSIM::computeMetric, fsim.cpp:80-163."""
    h, w = img.shape[:2]
    F = fsim_downscale_factor(w, h)
    w2, h2 = fsim_plane_size(w, h, F)
    H = fsim_filters(w2, h2)
    consts = fsim_noise_constants(H, energy_full)
    planes = [fsim_yiq_planes(x, F, w2, h2) for x in (img, ref)]
    pcs, grads = [], []
    for I, Q, Y in planes:
        amp, energy, eo0 = fsim_responses(Y, H, ifft2)
        pcs.append(fsim_phase_congruency(amp, energy, eo0, consts))
        grads.append(fsim_gradient(Y))
    return fsim_pool(pcs[0], pcs[1], grads[0], grads[1], planes[0][:2], planes[1][:2])


# ============================================================================================= FLIP
# The shaders' matrices are GLSL float constants (float(a) / b in float), kept at float precision.
# GLSL's mat3(...) is column-major and the shaders multiply row vectors (v * M): v * M = M_cols^T v,
# so the rows below (the constructor's columns) are the rows of the usual sRGB -> XYZ matrix.
_RGB_TO_XYZ = np.array([[10135552 / 24577794, 8788810 / 24577794, 4435075 / 24577794],
                        [2613072 / 12288897, 8788810 / 12288897, 887015 / 12288897],
                        [1425312 / 73733382, 8788810 / 73733382, 70074185 / 73733382]],
                       dtype=np.float32).astype(np.float64)
_XYZ_TO_RGB = np.array([[3.241003275, -1.537398934, -0.498615861],
                        [-0.969224334, 1.875930071, 0.041554224],
                        [0.055639423, -0.204011202, 1.057148933]], dtype=np.float32).astype(np.float64)
_WHITE = _RGB_TO_XYZ.sum(axis=1)  # vec3(1.0) * RGB_TO_XYZ


def flip_ppd(resolution_x=2560.0, distance=0.7, width=0.6):
    """src/gpu/flip/flip.cpp:125 with FLIPArguments' float fields (flip.h:21-25)."""
    d, r, wd = np.float32(distance), np.float32(resolution_x), np.float32(width)
    return float(np.float32(d * np.float32(r / wd))) * (math.pi / 180.0)


def _srgb_to_ycxcz(img):
    """shaders/flip/srgb_to_ycxcz.glsl:42-57."""
    c = img[..., :3].astype(np.float64) / 255.0
    lin = np.where(c > 0.04045, ((c + 0.055) / 1.055) ** 2.4, c / 12.92)
    xyz = lin @ _RGB_TO_XYZ.T / _WHITE
    return np.stack([116 * xyz[..., 1] - 16, 500 * (xyz[..., 0] - xyz[..., 1]), 200 * (xyz[..., 1] - xyz[..., 2])], -1)


def flip_feature_taps(ppd):
    """Taps (g, edge, point) of feature_filter.glsl:17-38 over the host's kernel width
    2 ceil(3 * 0.5 * 0.082 ppd) + 1 (flip.cpp:126), each normalised by the sum of its positive or
    negative taps (feature_filter_normalize.glsl:30-46).  Returns an array (K, 3)."""
    K = 2 * int(math.ceil(3 * 0.5 * 0.082 * ppd)) + 1
    sd = 0.5 * 0.082 * float(np.float32(ppd))  # the shader's float push constant
    radius = int(math.ceil(3.0 * sd))
    xc = np.arange(K) - radius
    g = np.exp(-(xc.astype(np.float64) ** 2) / (2.0 * sd ** 2))
    taps = np.stack([g, -xc * g, (xc ** 2 / sd ** 2 - 1) * g], -1)
    pos = np.maximum(taps, 0).sum(axis=0)
    neg = -np.minimum(taps, 0).sum(axis=0)
    return np.where(taps > 0, taps / np.where(pos > 0, pos, 1), taps / np.where(neg > 0, neg, 1))


def _conv_clamped(plane, taps, axis):
    """sum_j taps[j + r] * plane[clamp(i - j)] along `axis` (the shaders' loops, edge clamp)."""
    r = len(taps) // 2
    n = plane.shape[axis]
    out = np.zeros(plane.shape)
    for j in range(-r, r + 1):
        idx = np.clip(np.arange(n) - j, 0, n - 1)
        out += taps[j + r] * np.take(plane, idx, axis=axis)
    return out


def _csf_weights(ppd):
    """Per-channel CSF weights of spatial_prefilter_horizontal.glsl:20-61 (sum of two Gaussians with
    the luma / red-green / blue-yellow parameters), radius ceil(3 sqrt(0.04 / (2 pi^2)) ppd).
    Returns (3, 2r + 1), each row divided by its own sum (Q9: each pass normalises separately)."""
    r = int(math.ceil(3.0 * math.sqrt(0.04 / (2.0 * GLSL_PI * GLSL_PI)) * ppd))
    d = (np.arange(-r, r + 1) / ppd) ** 2
    rows = []
    params = np.array([(1.0, 0.0047, 0.0, 0.00001), (1.0, 0.0053, 0.0, 0.00001), (34.1, 0.04, 13.5, 0.025)],
                      dtype=np.float32).astype(np.float64)  # const vec4s of the shader
    for a1, b1, a2, b2 in params:
        v = a1 * math.sqrt(GLSL_PI / b1) * np.exp(-GLSL_PI ** 2 * d / b1) + \
            a2 * math.sqrt(GLSL_PI / b2) * np.exp(-GLSL_PI ** 2 * d / b2)
        rows.append(v / v.sum())
    return np.array(rows)


def _lab(xyz_over_white):
    """The L*a*b* conversion shared by spatial_prefilter.glsl:84-93 and spatial_detection.glsl:35-45."""
    delta = 6.0 / 29.0
    t = xyz_over_white
    f = np.where(t > 0.008856, np.cbrt(t), t / (3.0 * delta * delta) + 4.0 / 29.0)
    return np.stack([116.0 * f[..., 1] - 16.0, 500.0 * (f[..., 0] - f[..., 1]), 200.0 * (f[..., 1] - f[..., 2])], -1)


def _hunt(lab):
    out = lab.copy()
    out[..., 1] *= 0.01 * lab[..., 0]
    out[..., 2] *= 0.01 * lab[..., 0]
    return out


def _hyab(a, b):
    d = a - b
    return np.abs(d[..., 0]) + np.sqrt(d[..., 1] ** 2 + d[..., 2] ** 2)


def flip_map(img, ref, ppd):
    """Per-pixel FLIP value deltaEc^(1 - deltaEf) (combine_error_maps.glsl:28) of an RGBA8 pair.
    The shaders receive ppd as a float push constant (flip.cpp:326-364 and the prefilter passes);
    the host's kernel width uses the double value."""
    ycc = [_srgb_to_ycxcz(x) for x in (img, ref)]
    # feature pipeline: feature_filter_horizontal.glsl:37-48 then feature_detection.glsl:32-53
    taps = flip_feature_taps(ppd)
    ppd = float(np.float32(ppd))
    grads, lapl = [], []
    for c in ycc:
        L = (c[..., 0] + 16.0) / 116.0
        dx = _conv_clamped(L, taps[:, 1], axis=1)
        ddx = _conv_clamped(L, taps[:, 2], axis=1)
        val = _conv_clamped(L, taps[:, 0], axis=1)
        d = np.hypot(_conv_clamped(dx, taps[:, 0], axis=0), _conv_clamped(val, taps[:, 1], axis=0))
        dd = np.hypot(_conv_clamped(ddx, taps[:, 0], axis=0), _conv_clamped(val, taps[:, 2], axis=0))
        grads.append(d)
        lapl.append(dd)
    diff = np.maximum(np.abs(grads[0] - grads[1]), np.abs(lapl[0] - lapl[1]))
    dEf = (diff / math.sqrt(2.0)) ** 0.5
    # colour pipeline: spatial_prefilter_horizontal.glsl then spatial_prefilter.glsl:58-100
    wts = _csf_weights(ppd)
    labs = []
    for c in ycc:
        f = np.stack([_conv_clamped(_conv_clamped(c[..., i], wts[i], axis=1), wts[i], axis=0) for i in range(3)], -1)
        yy = (f[..., 0] + 16.0) / 116.0
        xyz = np.stack([yy + f[..., 1] / 500.0, yy, yy - f[..., 2] / 200.0], -1) * _WHITE
        lin = np.clip(xyz @ _XYZ_TO_RGB.T, 0.0, 1.0)
        labs.append(_hunt(_lab(lin @ _RGB_TO_XYZ.T / _WHITE)))
    # spatial_detection.glsl:57-85
    green = _hunt(_lab(np.array([0.0, 1.0, 0.0]) @ _RGB_TO_XYZ.T / _WHITE))
    blue = _hunt(_lab(np.array([0.0, 0.0, 1.0]) @ _RGB_TO_XYZ.T / _WHITE))
    cmax = _hyab(green, blue) ** 0.7
    dE = _hyab(labs[0], labs[1]) ** 0.7
    pc, pt = 0.4, 0.95
    dEc = np.where(dE < pc * cmax, (pt / (pc * cmax)) * dE, pt + ((dE - pc * cmax) / (cmax - pc * cmax)) * (1.0 - pt))
    return dEc ** (1.0 - dEf)


def flip(img, ref, ppd):
    """Mean of the per-pixel FLIP value (the reference computes the map but pools nothing)."""
    return float(np.mean(flip_map(img, ref, ppd)))
