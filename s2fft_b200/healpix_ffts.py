"""HEALPix ring FFTs on one B200 (drop-in for ``s2fft.utils.healpix_ffts``).

``healpix_fft(f, L, nside, method, reality)`` and ``healpix_ifft(ftm, L, nside,
method, reality)`` follow upstream (s2fft/utils/healpix_ffts.py:187-423):
per-ring FFT with fftshift and periodic extension to ``(4 nside - 1, 2L)``
columns (column c holds m = c - L), and the inverse with spectral folding;
no ring phase shifts and no normalisation. The work runs in
``s2b_healpix_fft`` / ``s2b_healpix_ifft`` of ``libs2b.so``.

Difference from upstream: for ``reality=True`` the inverse returns a real map
(upstream's numpy variant returns the real values in a complex array).
"""

from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .spherical import _check_method, _device, _dtypes, _ret, _to_device


def _plan(dev, L, nside, reality, precision, B):
    assert L >= 2 * nside
    return _lib.get_plan(dev, L=L, spin=0, nside=nside, sampling=_lib.SAMPLING["healpix"],
                         reality=int(bool(reality)), L_lower=0,
                         precision=_lib.PRECISION[precision], batch=B, iter=0, N=0)


def healpix_fft(f, L: int, nside: int, method: str = "cuda", reality: bool = False,
                precision: str = "f64"):
    """HEALPix map [.., 12 nside^2] -> ring spectra [.., 4 nside - 1, 2L]."""
    _check_method(method)
    cdt, rdt = _dtypes(precision)
    if reality:
        if isinstance(f, torch.Tensor) and f.is_complex():
            f = f.real
        elif isinstance(f, np.ndarray) and np.iscomplexobj(f):
            f = np.real(f)
    x, was_np, odev = _to_device(f, rdt if reality else cdt, _device())
    npix = 12 * nside * nside
    if x.shape[-1] != npix:
        raise ValueError(f"f must have trailing size {npix}")
    bs = tuple(x.shape[:-1])
    B = int(np.prod(bs)) if bs else 1
    plan = _plan(x.device, L, nside, reality, precision, B)
    out = torch.empty(bs + (4 * nside - 1, 2 * L), dtype=cdt, device=x.device)
    _lib.check(_lib.lib().s2b_healpix_fft(plan.ptr, x.data_ptr(), out.data_ptr(),
                                          _lib.stream_handle(x.device)))
    return _ret(out, was_np, odev)


def healpix_ifft(ftm, L: int, nside: int, method: str = "cuda", reality: bool = False,
                 precision: str = "f64"):
    """Ring spectra [.., 4 nside - 1, 2L] -> HEALPix map [.., 12 nside^2]."""
    _check_method(method)
    cdt, rdt = _dtypes(precision)
    x, was_np, odev = _to_device(ftm, cdt, _device())
    if tuple(x.shape[-2:]) != (4 * nside - 1, 2 * L):
        raise ValueError(f"ftm must have trailing shape {(4 * nside - 1, 2 * L)}")
    bs = tuple(x.shape[:-2])
    B = int(np.prod(bs)) if bs else 1
    plan = _plan(x.device, L, nside, reality, precision, B)
    out = torch.empty(bs + (12 * nside * nside,), dtype=rdt if reality else cdt,
                      device=x.device)
    _lib.check(_lib.lib().s2b_healpix_ifft(plan.ptr, x.data_ptr(), out.data_ptr(),
                                           _lib.stream_handle(x.device)))
    return _ret(out, was_np, odev)
