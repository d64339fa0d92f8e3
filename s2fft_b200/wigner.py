"""Drop-in Wigner (SO(3)) transforms on one B200.

Same call surface as upstream ``s2fft.wigner.inverse`` / ``forward``
(s2fft/transforms/wigner.py:13-107, 346-439): ``(flmn|f, L, N, nside, sampling,
method, reality, precomps, L_lower)``. The transform is 2N-1 spin (-n)
transforms run by ``libs2b.so`` plus a DFT over gamma.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .spherical import _check_method, _device, _dtypes, _ret, _to_device, f_shape


def so3_f_shape(L, N, sampling="mw", nside=None):
    return (2 * N - 1,) + f_shape(L, sampling, nside)


def flmn_shape(L, N):
    return 2 * N - 1, L, 2 * L - 1


def _check(L, N, nside, sampling, L_lower):
    s = sampling.lower()
    if s not in _lib.SAMPLING:
        raise ValueError(f"Sampling scheme sampling={sampling} not supported")
    if N >= 8:
        # upstream raises Warning for the recursive methods (wigner.py:87-88, 419-420)
        raise Warning("Recursive transform may provide lower precision beyond N ~ 8")
    if N < 1 or N > L:
        raise ValueError("1 <= N <= L required")
    if s == "healpix":
        if nside is None:
            raise ValueError("healpix sampling needs nside")
        assert L >= 2 * nside
    if not 0 <= L_lower < L:
        raise ValueError("L_lower must satisfy 0 <= L_lower < L")
    return s


def _plan(dev, L, N, nside, s, reality, L_lower, precision, B):
    return _lib.get_plan(dev, L=L, spin=0, nside=nside or 0, sampling=_lib.SAMPLING[s],
                         reality=int(bool(reality)), L_lower=L_lower,
                         precision=_lib.PRECISION[precision], batch=B, iter=0, N=N)


def inverse(flmn, L: int, N: int, nside: int = None, sampling: str = "mw",
            method: str = "cuda", reality: bool = False, precomps=None, L_lower: int = 0,
            _ssht_backend: int = 1, precision: str = "f64"):
    """Inverse Wigner transform: flmn [.., 2N-1, L, 2L-1] -> f [.., 2N-1, (grid)]."""
    _check_method(method)
    s = _check(L, N, nside, sampling, L_lower)
    cdt, rdt = _dtypes(precision)
    x, was_np, odev = _to_device(flmn, cdt, _device())
    if tuple(x.shape[-3:]) != flmn_shape(L, N):
        raise ValueError(f"flmn must have trailing shape {flmn_shape(L, N)}")
    bs = tuple(x.shape[:-3])
    B = int(np.prod(bs)) if bs else 1
    plan = _plan(x.device, L, N, nside, s, reality, L_lower, precision, B)
    out = torch.empty(bs + so3_f_shape(L, N, s, nside), dtype=rdt if reality else cdt,
                      device=x.device)
    ws = plan.workspace(False)
    _lib.check(_lib.lib().s2b_wigner_inverse(plan.ptr, x.data_ptr(), out.data_ptr(),
                                             ws.data_ptr(), ws.numel(),
                                             _lib.stream_handle(x.device)))
    return _ret(out, was_np, odev)


def forward(f, L: int, N: int, nside: int = None, sampling: str = "mw", method: str = "cuda",
            reality: bool = False, precomps=None, L_lower: int = 0, _ssht_backend: int = 1,
            precision: str = "f64"):
    """Forward Wigner transform: f [.., 2N-1, (grid)] -> flmn [.., 2N-1, L, 2L-1]."""
    _check_method(method)
    s = _check(L, N, nside, sampling, L_lower)
    cdt, rdt = _dtypes(precision)
    if reality:
        if isinstance(f, torch.Tensor) and f.is_complex():
            f = f.real
        elif isinstance(f, np.ndarray) and np.iscomplexobj(f):
            f = np.real(f)
    x, was_np, odev = _to_device(f, rdt if reality else cdt, _device())
    fs = so3_f_shape(L, N, s, nside)
    if tuple(x.shape[-len(fs):]) != fs:
        raise ValueError(f"f must have trailing shape {fs}")
    bs = tuple(x.shape[:-len(fs)])
    B = int(np.prod(bs)) if bs else 1
    plan = _plan(x.device, L, N, nside, s, reality, L_lower, precision, B)
    out = torch.empty(bs + flmn_shape(L, N), dtype=cdt, device=x.device)
    ws = plan.workspace(True)
    _lib.check(_lib.lib().s2b_wigner_forward(plan.ptr, x.data_ptr(), out.data_ptr(),
                                             ws.data_ptr(), ws.numel(),
                                             _lib.stream_handle(x.device)))
    return _ret(out, was_np, odev)
