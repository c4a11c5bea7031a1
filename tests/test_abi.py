"""CPU checks of the C-ABI boundary: the library loads and exports every symbol the public
header declares; argument validation that needs no device."""
import ctypes
import os
import re

import pytest

import iqm_b200

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "iqm_cuda.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(iqm_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_what_python_binds():
    assert set(declared_symbols()) == set(iqm_b200.EXPORTS)


def test_library_exports_every_declared_symbol():
    from iqm_b200 import build
    build.build()
    lib = ctypes.CDLL(iqm_b200.LIB_PATH)
    for name in declared_symbols():
        assert hasattr(lib, name), name


def test_default_params_without_device():
    L = iqm_b200.load_library()
    p = iqm_b200.SSIMParams()
    p.precision = 7
    L.iqm_ssim_default_params(ctypes.byref(p))
    assert (p.kernel_size, round(p.k1, 6), round(p.k2, 6), p.sigma) == (11, 0.01, 0.03, 1.5)
    assert p.precision == iqm_b200.IQM_FP32
    f = iqm_b200.FLIPParams()
    L.iqm_flip_default_params(ctypes.byref(f))
    assert (f.monitor_resolution_x, round(f.monitor_distance, 6), round(f.monitor_width, 6)) == (2560.0, 0.7, 0.6)


def test_null_context_is_rejected():
    L = iqm_b200.load_library()
    out = ctypes.c_double()
    assert L.iqm_ssim(None, None, None, 16, 16, 64, None, None, ctypes.byref(out)) == iqm_b200.IQM_EINVAL
    assert L.iqm_destroy(None) == iqm_b200.IQM_EINVAL
    h = ctypes.c_void_p()
    assert L.iqm_create(0, None) == iqm_b200.IQM_EINVAL
