"""Wigner (SO(3)) transforms (float64). Restates s2fft/transforms/wigner.py numpy paths."""

import numpy as np

from . import samples, spherical


def inverse(flmn, L, N, nside=None, sampling="mw", reality=False, L_lower=0):
    """wigner.py:110-196: 2N-1 spin-(-n) SHTs then an inverse FFT over gamma."""
    fban = np.zeros(samples.so3_f_shape(L, N, sampling, nside), dtype=np.complex128)
    flmn = np.array(flmn, dtype=np.complex128, copy=True)
    flmn[:, L_lower:] *= np.sqrt((2 * np.arange(L_lower, L) + 1) / (16 * np.pi**3))[None, :, None]
    n0 = 0 if reality else -N + 1
    for n in range(n0, N):
        fban[N - 1 + n] = (-1) ** n * spherical.inverse(
            flmn[N - 1 + n], L, -n, nside, sampling, reality if n == 0 else False,
            None, L_lower)
    ax = -2 if sampling.lower() == "healpix" else -3
    if reality:
        return np.fft.irfft(fban[N - 1:], 2 * N - 1, axis=ax, norm="forward")
    return np.fft.ifft(np.fft.ifftshift(fban, axes=ax), axis=ax, norm="forward")


def forward(f, L, N, nside=None, sampling="mw", reality=False, L_lower=0):
    """wigner.py:442-533: FFT over gamma, 2N-1 spin-(-n) forward SHTs, reality fill."""
    flmn = np.zeros(samples.flmn_shape(L, N), dtype=np.complex128)
    ax = -2 if sampling.lower() == "healpix" else -3
    if reality:
        fban = np.fft.rfft(np.real(f), axis=ax, norm="backward")
    else:
        fban = np.fft.fftshift(np.fft.fft(f, axis=ax, norm="backward"), axes=ax)
    fban = fban * (2 * np.pi / (2 * N - 1))
    n0 = 0 if reality else -N + 1
    sgn = (-1.0) ** np.abs(np.arange(-L + 1, L))
    for n in range(n0, N):
        flmn[N - 1 + n] = (-1) ** n * spherical.forward(
            fban[n - n0], L, -n, nside, sampling, reality if n == 0 else False, None, L_lower)
        if reality and n != 0:
            flmn[N - 1 - n] = np.conj(np.flip(flmn[N - 1 + n] * sgn * (-1) ** n, axis=-1))
    flmn[:, L_lower:] *= np.sqrt(4 * np.pi / (2 * np.arange(L_lower, L) + 1))[None, :, None]
    return flmn
