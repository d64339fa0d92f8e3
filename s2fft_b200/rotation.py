"""Rotation of spherical-harmonic coefficients on one B200 (drop-in for
``s2fft.utils.rotation``).

``rotate_flms(flm, L, rotation, dl_array=None)`` follows upstream
(s2fft/utils/rotation.py:9-64): for Euler angles ``rotation = (alpha, beta, gamma)``,

    flm'[l, m] = exp(-i m alpha) sum_n d^l_{m,n}(beta) exp(-i n gamma) flm[l, n].

Without ``dl_array`` the Wigner-d values at beta are generated on the device by the
three-term recurrence in the degree of every (m, n), fused with the contraction (upstream
builds the planes with Risbo's recursion, s2fft/recursions/risbo.py:4-120; the two agree
to rounding); with it (the layout of ``generate_rotate_dls``, rotation.py:75-96) only the
contraction runs. The arithmetic is double; complex64 inputs are returned as
complex64. A leading batch dimension is accepted (upstream takes one map).
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .spherical import _device, _ret, _to_device


def _workspace(dev, L):
    n = int(_lib.lib().s2b_rotate_workspace_size(L))
    return torch.empty(n, dtype=torch.uint8, device=dev)


def rotate_flms(flm, L: int, rotation, dl_array=None):
    """Rotate flm [..., L, 2L-1] by the Euler angles (alpha, beta, gamma)."""
    alpha, beta, gamma = (float(a) for a in rotation)
    single = (isinstance(flm, np.ndarray) and flm.dtype == np.complex64) or (
        isinstance(flm, torch.Tensor) and flm.dtype == torch.complex64)
    cdt = torch.complex64 if single else torch.complex128
    x, was_np, odev = _to_device(flm, cdt, _device())
    if tuple(x.shape[-2:]) != (L, 2 * L - 1):
        raise ValueError(f"flm must have trailing shape {(L, 2 * L - 1)}")
    bs = tuple(x.shape[:-2])
    B = int(np.prod(bs)) if bs else 1
    out = torch.empty_like(x)
    dl = None
    if dl_array is not None:
        dl, _, _ = _to_device(dl_array, torch.float64, x.device)
        if tuple(dl.shape) != (L, 2 * L - 1, 2 * L - 1):
            raise ValueError(f"dl_array must have shape {(L, 2 * L - 1, 2 * L - 1)}")
    ws = _workspace(x.device, L)
    _lib.check(_lib.lib().s2b_rotate_flms(
        L, B, _lib.PRECISION["f32" if single else "f64"], alpha, beta, gamma, x.data_ptr(),
        out.data_ptr(), dl.data_ptr() if dl is not None else None, ws.data_ptr(), ws.numel(),
        _lib.stream_handle(x.device)))
    return _ret(out, was_np, odev)


def generate_rotate_dls(L: int, beta: float):
    """The Wigner-d planes d^l_{m,n}(beta) as [L, 2L-1, 2L-1] float64 (upstream layout)."""
    dev = _device()
    out = torch.empty((L, 2 * L - 1, 2 * L - 1), dtype=torch.float64, device=dev)
    ws = _workspace(dev, L)
    _lib.check(_lib.lib().s2b_rotate_dls(L, float(beta), out.data_ptr(), ws.data_ptr(),
                                         ws.numel(), _lib.stream_handle(dev)))
    return out
