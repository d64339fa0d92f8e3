"""Drop-in Wigner (SO(3)) transforms on one B200.

Same call surface as upstream ``s2fft.wigner.inverse`` / ``forward``
(s2fft/transforms/wigner.py:13-107, 346-439): ``(flmn|f, L, N, nside, sampling,
method, reality, precomps, L_lower)``. The transform is 2N-1 spin (-n)
transforms run by ``libs2b.so`` plus a DFT over gamma.

When a torch input requires grad, the transform is composed from the
differentiable spin transforms (whose backward passes run the adjoint kernels)
and a gamma DFT written as a dense (2N-1) x (2N-1) product (complex signals) or
torch's real DFT over gamma (real signals, slices n >= 0 as upstream).

Difference from upstream: upstream's recursive methods raise ``Warning`` for
N >= 8 (wigner.py:87-88); here N = 8 is accepted and ``Warning`` is raised from
N = 9. The spin transforms stay accurate for any spin (orders m < |spin| run on
the degree recursion), so the limit only keeps the drop-in raising where upstream
would for larger N.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _lib
from . import spherical as _sph
from .spherical import _check_method, _device, _dtypes, _needs_grad, _ret, _to_device, f_shape


def so3_f_shape(L, N, sampling="mw", nside=None):
    return (2 * N - 1,) + f_shape(L, sampling, nside)


def flmn_shape(L, N):
    return 2 * N - 1, L, 2 * L - 1


def _check(L, N, nside, sampling, L_lower):
    s = sampling.lower()
    if s not in _lib.SAMPLING:
        raise ValueError(f"Sampling scheme sampling={sampling} not supported")
    if N > 8:
        # upstream warns from N = 8 (wigner.py:87-88); N = 8 is accepted here
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


def _gamma_phases(N, sign, device, dtype):
    """P[k, j] = exp(sign 2 pi i (j - (N-1)) k / (2N-1)), k, j < 2N-1."""
    G = 2 * N - 1
    k = np.arange(G)[:, None]
    n = np.arange(G)[None, :] - (N - 1)
    ph = np.exp(sign * 2j * np.pi * ((n * k) % G) / G)
    return torch.from_numpy(ph).to(device=device, dtype=dtype)


def _lnorm(L, n, L_lower, device, dtype, inverse):
    l = np.arange(L, dtype=np.float64)
    if inverse:
        v = (-1.0) ** n * np.sqrt((2 * l + 1) / (16 * np.pi ** 3))
    else:
        v = (-1.0) ** n * np.sqrt(4 * np.pi / (2 * l + 1))
        v[:L_lower] = 0.0
    return torch.from_numpy(v).to(device=device, dtype=dtype)[:, None]


def _inverse_composed(x, L, N, nside, s, L_lower, precision, reality=False):
    """Differentiable inverse: 2N-1 spin(-n) inverses and the gamma inverse DFT
    (s2fft/transforms/wigner.py:110-196). Real signals as upstream: slices n >= 0 only
    (n = 0 by the real spin-0 inverse) and an inverse real DFT over gamma."""
    rdt = x.real.dtype
    gdim = len(f_shape(L, s, nside))
    cdt = x.dtype
    fs = []
    for n in range(0 if reality else -(N - 1), N):
        j = N - 1 + n
        t = x[..., j, :, :] * _lnorm(L, n, L_lower, x.device, rdt, True)
        fs.append(_sph.inverse(t, L, -n, nside, s, L_lower=L_lower, precision=precision,
                               reality=reality and n == 0).to(cdt))
    fban = torch.stack(fs, dim=-gdim - 1)  # [.., n, grid]
    if reality:
        return torch.fft.irfft(fban, 2 * N - 1, dim=-gdim - 1, norm="forward")
    P = _gamma_phases(N, +1, x.device, x.dtype)
    return torch.movedim(torch.tensordot(fban, P, dims=([-gdim - 1], [1])), -1, -gdim - 1)


def _forward_composed(x, L, N, nside, s, L_lower, precision, reality=False):
    """Differentiable forward: gamma DFT times 2 pi/(2N-1), spin(-n) forwards
    (s2fft/transforms/wigner.py:442-533). Real signals as upstream: a real DFT over
    gamma, slices n >= 0 (n = 0 by the real spin-0 forward), and the slices n < 0
    mirrored, flmn[-n] = conj(flip(flmn[n] (-1)^|m| (-1)^n))."""
    rdt = x.real.dtype
    gdim = len(f_shape(L, s, nside))
    if reality:
        fban = torch.fft.rfft(x, dim=-gdim - 1, norm="backward") * (2 * np.pi / (2 * N - 1))
    else:
        P = _gamma_phases(N, -1, x.device, x.dtype) * (2 * np.pi / (2 * N - 1))
        # fban[.., j, grid] = sum_k P[k, j] f[.., k, grid]
        fban = torch.movedim(torch.tensordot(x, P, dims=([-gdim - 1], [0])), -1, -gdim - 1)
    n0 = 0 if reality else -(N - 1)
    out = {}
    for n in range(n0, N):
        fb = fban.select(-gdim - 1, n - n0)
        if reality and n == 0:
            fb = fb.real
        flm = _sph.forward(fb, L, -n, nside, s, L_lower=L_lower, precision=precision,
                           reality=reality and n == 0)
        out[n] = flm * _lnorm(L, n, L_lower, x.device, rdt, False)
    if reality:
        sgn = torch.from_numpy((-1.0) ** np.abs(np.arange(-L + 1, L))).to(x.device, rdt)
        for n in range(1, N):
            out[-n] = torch.conj(torch.flip(out[n] * sgn * (-1) ** n, dims=[-1]))
    return torch.stack([out[n] for n in range(-(N - 1), N)], dim=-3)


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
    if _needs_grad(x):
        return _ret(_inverse_composed(x, L, N, nside, s, L_lower, precision, reality),
                    was_np, odev)
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
    if _needs_grad(x):
        return _ret(_forward_composed(x, L, N, nside, s, L_lower, precision, reality),
                    was_np, odev)
    plan = _plan(x.device, L, N, nside, s, reality, L_lower, precision, B)
    out = torch.empty(bs + flmn_shape(L, N), dtype=cdt, device=x.device)
    ws = plan.workspace(True)
    _lib.check(_lib.lib().s2b_wigner_forward(plan.ptr, x.data_ptr(), out.data_ptr(),
                                             ws.data_ptr(), ws.numel(),
                                             _lib.stream_handle(x.device)))
    return _ret(out, was_np, odev)
