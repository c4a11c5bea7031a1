"""iqm_b200 -- B200 (sm_100a) implementation of cadik/IQM's metric-evaluation path.

Python front end over the C ABI of libiqm_cuda.so (include/iqm_cuda.h).  It mirrors the
reference's per-metric classes (src/gpu/{ssim,fsim,flip,svd}/*.h): construct a metric object on a
runtime, call compute_metric(image, ref) with RGBA8 images, get a result carrying the score(s)
and, where the reference returns one, the map.

There is no CPU fallback: if the CUDA library is missing or no GPU is present, constructing a
Runtime raises.
"""
import ctypes
import os
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libiqm_cuda.so")

IQM_OK = 0
IQM_EINVAL = -1
IQM_ECUDA = -2
IQM_ENOMEM = -3
IQM_EUNSUPPORTED = -4

IQM_FP32 = 0
IQM_MIXED = 1       # tensor-core transforms, split-precision (hi + lo) FP16 products
IQM_MIXED_FAST = 2  # tensor-core transforms, single FP16 products

# every symbol include/iqm_cuda.h declares
EXPORTS = (
    "iqm_create", "iqm_destroy", "iqm_last_error", "iqm_set_stream", "iqm_synchronize",
    "iqm_device_name", "iqm_ssim_default_params", "iqm_ssim", "iqm_msvd", "iqm_flip_default_params",
    "iqm_flip_ppd", "iqm_flip", "iqm_fsim", "iqm_ssim_dev", "iqm_msvd_dev", "iqm_flip_dev",
    "iqm_fsim_dev", "iqm_ssim_batch", "iqm_msvd_batch", "iqm_flip_batch", "iqm_fsim_batch",
    "iqm_last_launch_count", "iqm_fsim_plan_constants", "iqm_ssim_noalloc", "iqm_set_kernel_timing",
    "iqm_kernel_times", "iqm_batch", "iqm_batch_plan_create", "iqm_batch_plan_run", "iqm_batch_plan_info",
    "iqm_batch_plan_destroy", "iqm_host_alloc", "iqm_host_free",
)

METRIC_SSIM, METRIC_FSIM, METRIC_FLIP, METRIC_MSVD = 1, 2, 4, 8
_SCORES = ((METRIC_SSIM, 1), (METRIC_FSIM, 2), (METRIC_FLIP, 1), (METRIC_MSVD, 1))


class IQMError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (code %d)" % (msg, code))
        self.code = code


class SSIMParams(ctypes.Structure):
    _fields_ = [("kernel_size", ctypes.c_int), ("k1", ctypes.c_float), ("k2", ctypes.c_float),
                ("sigma", ctypes.c_float), ("precision", ctypes.c_int)]


class FLIPParams(ctypes.Structure):
    _fields_ = [("monitor_resolution_x", ctypes.c_float), ("monitor_distance", ctypes.c_float),
                ("monitor_width", ctypes.c_float)]


class Pair(ctypes.Structure):
    _fields_ = [("input", ctypes.c_void_p), ("ref", ctypes.c_void_p), ("w", ctypes.c_int),
                ("h", ctypes.c_int), ("row_bytes", ctypes.c_size_t)]


_lib = None


def load_library(path=LIB_PATH):
    """Loads libiqm_cuda.so and declares its signatures; raises if the library is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError("libiqm_cuda.so not built (run python -m iqm_b200.build): %s" % path)
    L = ctypes.CDLL(path)
    vp, ip, dp, fp = ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_float)
    u8 = ctypes.c_void_p
    L.iqm_create.argtypes = [ip, ctypes.POINTER(vp)]
    L.iqm_destroy.argtypes = [vp]
    L.iqm_last_error.argtypes = [vp]
    L.iqm_last_error.restype = ctypes.c_char_p
    L.iqm_set_stream.argtypes = [vp, vp]
    L.iqm_synchronize.argtypes = [vp]
    L.iqm_device_name.argtypes = [vp, ctypes.c_char_p, ctypes.c_size_t]
    L.iqm_ssim_default_params.argtypes = [ctypes.POINTER(SSIMParams)]
    L.iqm_ssim_default_params.restype = None
    L.iqm_flip_default_params.argtypes = [ctypes.POINTER(FLIPParams)]
    L.iqm_flip_default_params.restype = None
    L.iqm_flip_ppd.argtypes = [ctypes.POINTER(FLIPParams)]
    L.iqm_flip_ppd.restype = ctypes.c_double
    L.iqm_ssim.argtypes = [vp, u8, u8, ip, ip, ctypes.c_size_t, ctypes.POINTER(SSIMParams), fp, dp]
    L.iqm_msvd.argtypes = [vp, u8, u8, ip, ip, ctypes.c_size_t, fp, dp]
    L.iqm_flip.argtypes = [vp, u8, u8, ip, ip, ctypes.c_size_t, ctypes.POINTER(FLIPParams), fp, dp]
    L.iqm_fsim.argtypes = [vp, u8, u8, ip, ip, ctypes.c_size_t, ip, ip, dp, dp]
    PP = ctypes.POINTER(Pair)
    L.iqm_ssim_dev.argtypes = [vp, PP, ip, ctypes.POINTER(SSIMParams), vp]
    L.iqm_msvd_dev.argtypes = [vp, PP, ip, vp]
    L.iqm_flip_dev.argtypes = [vp, PP, ip, ctypes.POINTER(FLIPParams), vp]
    L.iqm_fsim_dev.argtypes = [vp, PP, ip, ip, ip, vp]
    L.iqm_ssim_batch.argtypes = [vp, PP, ip, ctypes.POINTER(SSIMParams), dp]
    L.iqm_msvd_batch.argtypes = [vp, PP, ip, dp]
    L.iqm_flip_batch.argtypes = [vp, PP, ip, ctypes.POINTER(FLIPParams), dp]
    L.iqm_fsim_batch.argtypes = [vp, PP, ip, ip, ip, dp]
    L.iqm_last_launch_count.argtypes = [vp]
    L.iqm_fsim_plan_constants.argtypes = [vp, ip, ip, ip, dp, dp, dp]
    L.iqm_ssim_noalloc.argtypes = [vp, vp, ip, ip, ctypes.c_size_t, ctypes.POINTER(SSIMParams), vp, vp, vp]
    L.iqm_set_kernel_timing.argtypes = [vp, ip]
    L.iqm_kernel_times.argtypes = [vp, ctypes.c_char_p, ctypes.c_size_t]
    L.iqm_batch.argtypes = [vp, ip, PP, ip, ctypes.POINTER(SSIMParams), ctypes.POINTER(FLIPParams), ip, ip, dp]
    L.iqm_batch_plan_create.argtypes = [vp, ip, PP, ip, ctypes.POINTER(SSIMParams), ctypes.POINTER(FLIPParams),
                                        ip, ip, ip, vp, ctypes.POINTER(vp)]
    L.iqm_batch_plan_run.argtypes = [vp]
    L.iqm_batch_plan_info.argtypes = [vp, ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(ip)]
    L.iqm_batch_plan_destroy.argtypes = [vp]
    L.iqm_host_alloc.argtypes = [ctypes.c_size_t, ctypes.POINTER(vp)]
    L.iqm_host_free.argtypes = [vp]
    _lib = L
    return L


def fsim_downscale_factor(w, h):
    """F = max(1, round(min(w, h) / 256)) (src/gpu/fsim/fsim.cpp:165-168), as the library computes it."""
    x = min(w, h) / 256.0
    return max(1, int(np.floor(x + 0.5)))


def fsim_plane_size(w, h):
    """(W', H') of the FSIM working planes: roundf(W / F), roundf(H / F) in float
    (src/gpu/fsim/fsim.cpp:91-92)."""
    F = fsim_downscale_factor(w, h)
    fw = float(np.float32(w) / np.float32(F))
    fh = float(np.float32(h) / np.float32(F))
    return int(np.floor(fw + 0.5)), int(np.floor(fh + 0.5))


def _img(a):
    """RGBA8 host image (h, w, 4) -> contiguous uint8 array."""
    a = np.ascontiguousarray(a, dtype=np.uint8)
    if a.ndim != 3 or a.shape[2] != 4:
        raise ValueError("images must be (height, width, 4) RGBA8 arrays")
    return a


def _check_same(image, ref):
    if image.shape != ref.shape:
        # src/main.cpp:74-76
        raise IQMError(IQM_EINVAL, "Compared images must have the same size")


class Runtime:
    """One CUDA device + stream + arena (stands in for the reference's VulkanRuntime)."""

    def __init__(self, device=0):
        self.L = load_library()
        h = ctypes.c_void_p()
        rc = self.L.iqm_create(device, ctypes.byref(h))
        if rc != IQM_OK:
            raise IQMError(rc, self.L.iqm_last_error(None).decode())
        self.h = h
        buf = ctypes.create_string_buffer(256)
        self.L.iqm_device_name(self.h, buf, 256)
        self.selected_device = buf.value.decode()

    def check(self, rc):
        if rc != IQM_OK:
            raise IQMError(rc, self.L.iqm_last_error(self.h).decode())

    def set_stream(self, stream_handle):
        self.check(self.L.iqm_set_stream(self.h, ctypes.c_void_p(stream_handle)))

    def synchronize(self):
        self.check(self.L.iqm_synchronize(self.h))

    def last_launch_count(self):
        return self.L.iqm_last_launch_count(self.h)

    def set_kernel_timing(self, enable):
        """Per-kernel device timing on this context's stream (clears the totals)."""
        self.check(self.L.iqm_set_kernel_timing(self.h, 1 if enable else 0))

    def kernel_times(self):
        """{kernel name: (launches, total ms)} since timing was enabled; waits for the stream."""
        buf = ctypes.create_string_buffer(1 << 16)
        self.check(self.L.iqm_kernel_times(self.h, buf, len(buf)))
        out = {}
        for line in buf.value.decode().splitlines():
            name, n, ms = line.rsplit(" ", 2)
            out[name] = (int(n), float(ms))
        return out

    def close(self):
        if getattr(self, "h", None):
            self.L.iqm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _fptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float)) if a is not None else None


def _pairs(items):
    """items: (input_ptr, ref_ptr, w, h, row_bytes) tuples -> ctypes array of Pair."""
    arr = (Pair * len(items))()
    for i, (a, b, w, h, rb) in enumerate(items):
        arr[i] = Pair(a, b, w, h, rb)
    return arr


# ---------------------------------------------------------------- results (mirror src/gpu/*/*.h)
@dataclass
class SSIMResult:  # src/gpu/ssim/ssim.h:17-23
    mssim: float
    image_data: Optional[np.ndarray] = None
    width: int = 0
    height: int = 0


@dataclass
class SVDResult:  # src/gpu/svd/svd.h:17-23
    msvd: float
    image_data: Optional[np.ndarray] = None
    width: int = 0
    height: int = 0


@dataclass
class FSIMResult:  # src/gpu/fsim/fsim.h:27-31
    fsim: float
    fsimc: float


@dataclass
class FLIPResult:  # src/gpu/flip/flip.h:16-19 (mean_flip is assigned here)
    mean_flip: float
    image_data: Optional[np.ndarray] = None


@dataclass
class FLIPArguments:  # src/gpu/flip/flip.h:21-25
    monitor_resolution_x: float = 2560.0
    monitor_distance: float = 0.7
    monitor_width: float = 0.6

    def c(self):
        return FLIPParams(self.monitor_resolution_x, self.monitor_distance, self.monitor_width)


# ---------------------------------------------------------------- metric classes
class SSIM:
    """src/gpu/ssim/ssim.h:25-35: public parameters kernel_size, k_1, k_2, sigma."""

    def __init__(self, runtime):
        self.rt = runtime
        self.kernel_size = 11
        self.k_1 = 0.01
        self.k_2 = 0.03
        self.sigma = 1.5
        self.precision = IQM_FP32  # IQM_MIXED / IQM_MIXED_FAST: tensor-core window sums

    def params(self):
        return SSIMParams(self.kernel_size, self.k_1, self.k_2, self.sigma, self.precision)

    def compute_metric(self, image, ref, want_map=True):
        image, ref = _img(image), _img(ref)
        _check_same(image, ref)
        h, w = image.shape[:2]
        m = np.empty((h, w), np.float32) if want_map else None
        out = ctypes.c_double()
        p = self.params()
        self.rt.check(self.rt.L.iqm_ssim(self.rt.h, image.ctypes.data, ref.ctypes.data, w, h, w * 4,
                                         ctypes.byref(p), _fptr(m), ctypes.byref(out)))
        return SSIMResult(out.value, m, w, h)

    def compute_batch(self, pairs):
        """pairs: list of (image, ref) host arrays, sizes may differ -> list of MSSIM."""
        keep = [(_img(a), _img(b)) for a, b in pairs]
        for a, b in keep:
            _check_same(a, b)
        arr = _pairs([(a.ctypes.data, b.ctypes.data, a.shape[1], a.shape[0], a.shape[1] * 4) for a, b in keep])
        out = np.empty(len(keep), np.float64)
        p = self.params()
        self.rt.check(self.rt.L.iqm_ssim_batch(self.rt.h, arr, len(keep), ctypes.byref(p),
                                               out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return out

    def compute_dev(self, dev_pairs, d_scores):
        """dev_pairs: (in_ptr, ref_ptr, w, h, row_bytes) with device pointers; d_scores: device ptr."""
        arr = _pairs(dev_pairs)
        p = self.params()
        self.rt.check(self.rt.L.iqm_ssim_dev(self.rt.h, arr, len(dev_pairs), ctypes.byref(p),
                                             ctypes.c_void_p(d_scores)))


class SVD:
    """src/gpu/svd/svd.h:25-28 (M-SVD)."""

    def __init__(self, runtime):
        self.rt = runtime

    def compute_metric(self, image, ref, want_map=True):
        image, ref = _img(image), _img(ref)
        _check_same(image, ref)
        h, w = image.shape[:2]
        m = np.empty((h // 8, w // 8), np.float32) if want_map else None
        out = ctypes.c_double()
        self.rt.check(self.rt.L.iqm_msvd(self.rt.h, image.ctypes.data, ref.ctypes.data, w, h, w * 4,
                                         _fptr(m), ctypes.byref(out)))
        return SVDResult(out.value, m, w // 8, h // 8)

    def compute_batch(self, pairs):
        keep = [(_img(a), _img(b)) for a, b in pairs]
        arr = _pairs([(a.ctypes.data, b.ctypes.data, a.shape[1], a.shape[0], a.shape[1] * 4) for a, b in keep])
        out = np.empty(len(keep), np.float64)
        self.rt.check(self.rt.L.iqm_msvd_batch(self.rt.h, arr, len(keep),
                                               out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return out

    def compute_dev(self, dev_pairs, d_scores):
        arr = _pairs(dev_pairs)
        self.rt.check(self.rt.L.iqm_msvd_dev(self.rt.h, arr, len(dev_pairs), ctypes.c_void_p(d_scores)))


class FLIP:
    """src/gpu/flip/flip.h:27-30."""

    def __init__(self, runtime):
        self.rt = runtime

    def compute_metric(self, image, ref, args=None, want_map=False):
        args = args or FLIPArguments()
        image, ref = _img(image), _img(ref)
        _check_same(image, ref)
        h, w = image.shape[:2]
        m = np.empty((h, w), np.float32) if want_map else None
        out = ctypes.c_double()
        p = args.c()
        self.rt.check(self.rt.L.iqm_flip(self.rt.h, image.ctypes.data, ref.ctypes.data, w, h, w * 4,
                                         ctypes.byref(p), _fptr(m), ctypes.byref(out)))
        return FLIPResult(out.value, m)

    def compute_batch(self, pairs, args=None):
        args = args or FLIPArguments()
        keep = [(_img(a), _img(b)) for a, b in pairs]
        arr = _pairs([(a.ctypes.data, b.ctypes.data, a.shape[1], a.shape[0], a.shape[1] * 4) for a, b in keep])
        out = np.empty(len(keep), np.float64)
        p = args.c()
        self.rt.check(self.rt.L.iqm_flip_batch(self.rt.h, arr, len(keep), ctypes.byref(p),
                                               out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return out

    def compute_dev(self, dev_pairs, d_scores, args=None):
        args = args or FLIPArguments()
        arr = _pairs(dev_pairs)
        p = args.c()
        self.rt.check(self.rt.L.iqm_flip_dev(self.rt.h, arr, len(dev_pairs), ctypes.byref(p),
                                             ctypes.c_void_p(d_scores)))

    def ppd(self, args=None):
        args = args or FLIPArguments()
        p = args.c()
        return self.rt.L.iqm_flip_ppd(ctypes.byref(p))


class FSIM:
    """src/gpu/fsim/fsim.h:33-36.  energy_mode 0 pools the noise-energy estimates as the
    reference does (first ceil(N/2) pixels); 1 pools all N."""

    def __init__(self, runtime, precision=IQM_FP32, energy_mode=0):
        self.rt = runtime
        self.precision = precision
        self.energy_mode = energy_mode

    def compute_metric(self, image, ref):
        image, ref = _img(image), _img(ref)
        _check_same(image, ref)
        h, w = image.shape[:2]
        f, fc = ctypes.c_double(), ctypes.c_double()
        self.rt.check(self.rt.L.iqm_fsim(self.rt.h, image.ctypes.data, ref.ctypes.data, w, h, w * 4,
                                         self.precision, self.energy_mode, ctypes.byref(f), ctypes.byref(fc)))
        return FSIMResult(f.value, fc.value)

    def compute_batch(self, pairs):
        keep = [(_img(a), _img(b)) for a, b in pairs]
        arr = _pairs([(a.ctypes.data, b.ctypes.data, a.shape[1], a.shape[0], a.shape[1] * 4) for a, b in keep])
        out = np.empty(2 * len(keep), np.float64)
        self.rt.check(self.rt.L.iqm_fsim_batch(self.rt.h, arr, len(keep), self.precision, self.energy_mode,
                                               out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return out.reshape(-1, 2)

    def plan_constants(self, w2, h2):
        """(EM_n, EstSumAn2, EstSumAiAj) per orientation for a W'xH' plane."""
        em, an2, aiaj = np.empty(4), np.empty(4), np.empty(4)
        P = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        self.rt.check(self.rt.L.iqm_fsim_plan_constants(self.rt.h, w2, h2, self.energy_mode, P(em), P(an2), P(aiaj)))
        return em, an2, aiaj

    def compute_dev(self, dev_pairs, d_scores):
        arr = _pairs(dev_pairs)
        self.rt.check(self.rt.L.iqm_fsim_dev(self.rt.h, arr, len(dev_pairs), self.precision, self.energy_mode,
                                             ctypes.c_void_p(d_scores)))


# ---------------------------------------------------------------- batches over several metrics
def _split_scores(mask, n, flat):
    """Flat metric-by-metric score layout -> {"ssim": (n,), "fsim": (n, 2), "flip": (n,), "msvd": (n,)}."""
    out, off = {}, 0
    names = {METRIC_SSIM: "ssim", METRIC_FSIM: "fsim", METRIC_FLIP: "flip", METRIC_MSVD: "msvd"}
    for flag, k in _SCORES:
        if mask & flag:
            v = np.asarray(flat[off:off + k * n])
            out[names[flag]] = v.reshape(n, 2) if k == 2 else v
            off += k * n
    return out


def scores_per_pair(mask):
    return sum(k for flag, k in _SCORES if mask & flag)


def _ssim_params(rt, ssim):
    return ssim if isinstance(ssim, SSIMParams) else (ssim or SSIM(rt)).params()


def batch(rt, mask, pairs, ssim=None, flip=None, precision=IQM_FP32, energy_mode=0):
    """Evaluates host pairs [(image, ref), ...] (RGBA8 arrays, sizes may differ) with every metric in
    `mask` in one call; returns the per-metric score arrays."""
    imgs = [(_img(a), _img(b)) for a, b in pairs]
    for a, b in imgs:
        _check_same(a, b)
    items = [(a.ctypes.data, b.ctypes.data, a.shape[1], a.shape[0], a.shape[1] * 4) for a, b in imgs]
    arr = _pairs(items)
    n = len(items)
    out = np.empty(scores_per_pair(mask) * n, np.float64)
    sp = _ssim_params(rt, ssim)
    fp = (flip or FLIPArguments()).c()
    rt.check(rt.L.iqm_batch(rt.h, mask, arr, n, ctypes.byref(sp), ctypes.byref(fp), precision, energy_mode,
                            out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
    return _split_scores(mask, n, out)


class BatchPlan:
    """A fixed batch of device-resident pairs evaluated with several metrics by one CUDA-graph
    replay (iqm_batch_plan_*); FSIM launch shapes autotuned at creation."""

    def __init__(self, rt, mask, dev_pairs, d_scores, ssim=None, flip=None, precision=IQM_FP32, energy_mode=0,
                 autotune=True):
        self.rt, self.mask, self.n = rt, mask, len(dev_pairs)
        arr = _pairs(dev_pairs)
        sp = _ssim_params(rt, ssim)
        fp = (flip or FLIPArguments()).c()
        h = ctypes.c_void_p()
        rt.check(rt.L.iqm_batch_plan_create(rt.h, mask, arr, self.n, ctypes.byref(sp), ctypes.byref(fp), precision,
                                            energy_mode, 1 if autotune else 0, ctypes.c_void_p(d_scores),
                                            ctypes.byref(h)))
        self.h = h

    def run(self):
        self.rt.check(self.rt.L.iqm_batch_plan_run(self.h))

    def info(self):
        buf = ctypes.create_string_buffer(1024)
        launches = ctypes.c_int()
        self.rt.L.iqm_batch_plan_info(self.h, buf, len(buf), ctypes.byref(launches))
        return buf.value.decode(), launches.value

    def close(self):
        if getattr(self, "h", None):
            self.rt.L.iqm_batch_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

