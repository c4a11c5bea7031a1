"""ctypes front end of the CPU oracle (oracle/iqm_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
leg, as the reference that GPU results are compared with.  The product library never imports,
links or calls anything here.

Two builds of the same C source are exposed:
  Oracle("f32") -- float arithmetic in the reference's order (reference-faithful restatement)
  Oracle("f64") -- the same steps in double (the accuracy oracle)
"""
import ctypes
import math
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_u8p = ctypes.POINTER(ctypes.c_uint8)
_fp = ctypes.POINTER(ctypes.c_float)
_dp = ctypes.POINTER(ctypes.c_double)


def fsim_plane_size(w, h, F):
    """W' = roundf((float)W / F), H' likewise (src/gpu/fsim/fsim.cpp:91-92), half away from zero."""
    fw = float(np.float32(w) / np.float32(F))
    fh = float(np.float32(h) / np.float32(F))
    return int(math.floor(fw + 0.5)), int(math.floor(fh + 0.5))


def build():
    """Compile both oracle builds with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def _lib_path(prec):
    return os.path.join(_HERE, "liboracle_%s.so" % prec)


def _u8(a):
    a = np.ascontiguousarray(a, dtype=np.uint8)
    return a, a.ctypes.data_as(_u8p)


class Oracle:
    def __init__(self, prec="f64"):
        path = _lib_path(prec)
        if not os.path.exists(path):
            build()
        self.prec = prec
        L = ctypes.CDLL(path)
        L.oracle_ssim.restype = ctypes.c_double
        L.oracle_ssim.argtypes = [_u8p, _u8p, ctypes.c_int, ctypes.c_int, ctypes.c_long, ctypes.c_int,
                                  ctypes.c_double, ctypes.c_double, ctypes.c_double, _fp]
        L.oracle_fsim.restype = ctypes.c_int
        L.oracle_fsim.argtypes = [_u8p, _u8p, ctypes.c_int, ctypes.c_int, ctypes.c_long, ctypes.c_int,
                                  _dp, _dp, _fp, _dp]
        L.oracle_fsim_constants.restype = None
        L.oracle_fsim_constants.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, _dp, _dp]
        L.oracle_fsim_filters.restype = None
        L.oracle_fsim_filters.argtypes = [ctypes.c_int, ctypes.c_int, _dp]
        L.oracle_fsim_downscale_factor.restype = ctypes.c_int
        L.oracle_fsim_downscale_factor.argtypes = [ctypes.c_int, ctypes.c_int]
        L.oracle_flip.restype = ctypes.c_double
        L.oracle_flip.argtypes = [_u8p, _u8p, ctypes.c_int, ctypes.c_int, ctypes.c_long, ctypes.c_double, _fp]
        L.oracle_flip_ppd.restype = ctypes.c_double
        L.oracle_flip_ppd.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double]
        L.oracle_flip_feature_taps.restype = ctypes.c_int
        L.oracle_flip_feature_taps.argtypes = [ctypes.c_double, _dp]
        L.oracle_msvd.restype = ctypes.c_double
        L.oracle_msvd.argtypes = [_u8p, _u8p, ctypes.c_int, ctypes.c_int, ctypes.c_long, _fp, _fp]
        L.oracle_gray_u8.restype = ctypes.c_uint
        L.oracle_gray_u8.argtypes = [ctypes.c_uint, ctypes.c_uint, ctypes.c_uint]
        L.oracle_svd8.restype = None
        L.oracle_svd8.argtypes = [_fp, _fp]
        L.oracle_fft2.restype = None
        L.oracle_fft2.argtypes = [_dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        self.L = L

    # ---- metrics (images: uint8 arrays of shape (h, w, 4), RGBA8) ----
    def ssim(self, img, ref, kernel_size=11, k1=0.01, k2=0.03, sigma=1.5, want_map=False):
        h, w = img.shape[:2]
        a, pa = _u8(img)
        b, pb = _u8(ref)
        m = np.empty((h, w), np.float32) if want_map else None
        v = self.L.oracle_ssim(pa, pb, w, h, w * 4, kernel_size, k1, k2, sigma,
                               m.ctypes.data_as(_fp) if want_map else None)
        return (v, m) if want_map else v

    def fsim(self, img, ref, energy_full=False, want_pc=False):
        h, w = img.shape[:2]
        a, pa = _u8(img)
        b, pb = _u8(ref)
        f = ctypes.c_double()
        fc = ctypes.c_double()
        F = self.L.oracle_fsim_downscale_factor(w, h)
        w2, h2 = fsim_plane_size(w, h, F)
        pc = np.empty((2, h2, w2), np.float32) if want_pc else None
        noise = np.empty(8, np.float64)
        self.L.oracle_fsim(pa, pb, w, h, w * 4, int(energy_full), ctypes.byref(f), ctypes.byref(fc),
                           pc.ctypes.data_as(_fp) if want_pc else None, noise.ctypes.data_as(_dp))
        if want_pc:
            return f.value, fc.value, pc, noise
        return f.value, fc.value

    def fsim_constants(self, w2, h2, energy_full=False):
        em = np.empty(4)
        an2 = np.empty(4)
        aiaj = np.empty(4)
        self.L.oracle_fsim_constants(w2, h2, int(energy_full), em.ctypes.data_as(_dp),
                                     an2.ctypes.data_as(_dp), aiaj.ctypes.data_as(_dp))
        return em, an2, aiaj

    def fsim_filters(self, w2, h2):
        out = np.empty((16, h2, w2), np.float64)
        self.L.oracle_fsim_filters(w2, h2, out.ctypes.data_as(_dp))
        return out

    def flip(self, img, ref, ppd=67.0, want_map=False):
        h, w = img.shape[:2]
        a, pa = _u8(img)
        b, pb = _u8(ref)
        m = np.empty((h, w), np.float32) if want_map else None
        v = self.L.oracle_flip(pa, pb, w, h, w * 4, ppd, m.ctypes.data_as(_fp) if want_map else None)
        return (v, m) if want_map else v

    def flip_ppd(self, res_x=2560.0, distance=0.7, width=0.6):
        return self.L.oracle_flip_ppd(res_x, distance, width)

    def flip_feature_taps(self, ppd):
        k = self.L.oracle_flip_feature_taps(ppd, None)
        t = np.empty((3, k), np.float64)
        self.L.oracle_flip_feature_taps(ppd, t.ctypes.data_as(_dp))
        return t

    def msvd(self, img, ref, want_map=False, want_dist=False):
        h, w = img.shape[:2]
        a, pa = _u8(img)
        b, pb = _u8(ref)
        nb = (w // 8) * (h // 8)
        m = np.empty((h // 8, w // 8), np.float32) if want_map else None
        d = np.empty((h // 8, w // 8), np.float32) if want_dist else None
        v = self.L.oracle_msvd(pa, pb, w, h, w * 4, m.ctypes.data_as(_fp) if want_map else None,
                               d.ctypes.data_as(_fp) if want_dist else None)
        out = [v]
        if want_map:
            out.append(m)
        if want_dist:
            out.append(d)
        return out[0] if len(out) == 1 else tuple(out)

    # ---- stage hooks ----
    def gray(self, rgb):
        rgb = np.asarray(rgb, dtype=np.uint32).reshape(-1, 3)
        return np.array([self.L.oracle_gray_u8(int(r), int(g), int(b)) for r, g, b in rgb], np.uint8)

    def svd8(self, block):
        blk = np.ascontiguousarray(block, dtype=np.float32).reshape(8, 8)
        sv = np.empty(8, np.float32)
        self.L.oracle_svd8(blk.ctypes.data_as(_fp), sv.ctypes.data_as(_fp))
        return sv

    def fft2(self, z, sign=-1, normalize=False):
        h, w = z.shape
        d = np.empty((h, w, 2), np.float64)
        d[..., 0] = z.real
        d[..., 1] = z.imag
        self.L.oracle_fft2(d.ctypes.data_as(_dp), w, h, sign, int(normalize))
        return d[..., 0] + 1j * d[..., 1]
