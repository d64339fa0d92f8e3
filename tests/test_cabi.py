"""CPU-side checks of the C-ABI library: it loads, exports every declared symbol,
and rejects bad arguments before touching a device."""

import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "s2b.h")
LIB = os.path.join(ROOT, "s2fft_b200", "libs2b.so")


def declared_symbols():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"\b(s2b_[a-z_0-9]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(LIB):
        from s2fft_b200 import _build

        _build.build()
    return ctypes.CDLL(LIB)


def test_exports_every_declared_symbol(lib):
    syms = declared_symbols()
    assert "s2b_inverse" in syms and "s2b_forward" in syms
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_version_and_error_string(lib):
    lib.s2b_version.restype = ctypes.c_int
    assert lib.s2b_version() >= 100
    lib.s2b_last_error.restype = ctypes.c_char_p
    assert isinstance(lib.s2b_last_error(), bytes)


def test_invalid_descriptors_rejected_on_host(lib):
    from s2fft_b200._lib import Desc

    lib.s2b_plan_create.restype = ctypes.c_int
    lib.s2b_last_error.restype = ctypes.c_char_p
    base = dict(L=8, spin=0, nside=0, sampling=0, reality=0, L_lower=0, precision=0, batch=1,
                iter=0, N=0)
    bad = [dict(L=1), dict(sampling=9), dict(sampling=4, nside=0), dict(sampling=4, nside=8),
           dict(reality=1, spin=2), dict(spin=8), dict(L_lower=8), dict(batch=0),
           dict(precision=5), dict(iter=-1)]
    for b in bad:
        d = Desc(**{**base, **b})
        p = ctypes.c_void_p()
        rc = lib.s2b_plan_create(ctypes.byref(d), ctypes.byref(p))
        assert rc == 1, b
        assert lib.s2b_last_error()
    rc = lib.s2b_plan_create(None, None)
    assert rc == 1


def test_python_argument_errors():
    import s2fft_b200

    flm = np.zeros((8, 15), complex)
    with pytest.raises(ValueError, match="not recognised"):
        s2fft_b200.inverse(flm, 8, method="nope")
    with pytest.raises(Warning):
        s2fft_b200.inverse(flm, 8, spin=8)
    with pytest.raises(Warning):
        s2fft_b200.forward(np.zeros((8, 15), complex), 8, spin=9)
    with pytest.raises(AssertionError):
        s2fft_b200.inverse(flm, 8, nside=8, sampling="healpix")
    with pytest.raises(ValueError):
        s2fft_b200.inverse(flm, 8, sampling="xyz")


def test_no_cpu_fallback_without_gpu():
    import torch

    import s2fft_b200

    if torch.cuda.is_available():
        pytest.skip("GPU present")
    with pytest.raises(RuntimeError, match="CUDA"):
        s2fft_b200.inverse(np.zeros((8, 15), complex), 8)


def test_fourier_wigner_arguments_rejected_on_host(lib):
    """s2b_fw_plan_create validates L, sampling and precision before any CUDA call."""
    lib.s2b_fw_plan_create.restype = ctypes.c_int
    lib.s2b_fw_workspace_size.restype = ctypes.c_size_t
    lib.s2b_fw_workspace_size.argtypes = [ctypes.c_void_p] + [ctypes.c_int] * 4
    for L, N, sampling, precision in ((1, 1, 0, 0), (8, 2, 2, 0), (8, 2, 3, 0), (8, 2, 4, 0),
                                      (8, 2, 0, 2), (8, 2, 1, 7), (8, 0, 0, 0), (8, 9, 1, 0)):
        p = ctypes.c_void_p()
        assert lib.s2b_fw_plan_create(L, N, sampling, precision, ctypes.byref(p)) == 1
        assert not p.value
        assert lib.s2b_last_error()
    assert lib.s2b_fw_plan_create(8, 2, 0, 0, None) == 1
    assert lib.s2b_fw_workspace_size(None, 0, 1, 0, 1) == 0


def test_rotation_arguments_rejected_on_host(lib):
    """s2b_rotate_flms / s2b_rotate_dls check L, buffers, aliasing, precision and the
    workspace size before any CUDA call; the workspace size grows with L."""
    vp, sz = ctypes.c_void_p, ctypes.c_size_t
    lib.s2b_rotate_workspace_size.restype = sz
    lib.s2b_rotate_workspace_size.argtypes = [ctypes.c_int]
    lib.s2b_rotate_flms.restype = ctypes.c_int
    lib.s2b_rotate_flms.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int] + \
        [ctypes.c_double] * 3 + [vp, vp, vp, vp, sz, vp]
    lib.s2b_rotate_dls.restype = ctypes.c_int
    lib.s2b_rotate_dls.argtypes = [ctypes.c_int, ctypes.c_double, vp, vp, sz, vp]
    assert lib.s2b_rotate_workspace_size(0) == 0
    w8, w64 = lib.s2b_rotate_workspace_size(8), lib.s2b_rotate_workspace_size(64)
    assert 0 < w8 < w64
    a, b, ws = vp(16), vp(4096), vp(1 << 20)  # never dereferenced: rejected first
    cases = [
        (0, 1, 0, a, b, None, ws, w8),         # L < 1
        (8, 0, 0, a, b, None, ws, w8),         # batch < 1
        (8, 1, 0, None, b, None, ws, w8),      # no input
        (8, 1, 0, a, a, None, ws, w8),         # out aliases flm
        (8, 1, 5, a, b, None, ws, w8),         # precision
        (9000, 1, 0, a, b, None, ws, 1 << 62),  # L above the recurrence limit, no planes
    ]
    for L, B, prec, x, y, dl, w, wb in cases:
        assert lib.s2b_rotate_flms(L, B, prec, 0.1, 0.2, 0.3, x, y, dl, w, wb, None) == 1
        assert lib.s2b_last_error()
    assert lib.s2b_rotate_flms(8, 1, 0, 0.1, 0.2, 0.3, a, b, None, ws, w8 - 1, None) == 3
    assert lib.s2b_rotate_dls(9000, 0.2, b, ws, 1 << 62, None) == 1
    assert lib.s2b_rotate_dls(8, 0.2, b, ws, w8 - 1, None) == 3
    assert lib.s2b_rotate_dls(8, 0.2, None, ws, w8, None) == 1
