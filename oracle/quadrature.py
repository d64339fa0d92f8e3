"""Quadrature weights (float64). Restates s2fft/utils/quadrature.py."""

import numpy as np

from . import samples


def _mw_weight(m):
    """Fourier weights of the MW quadrature. quadrature.py:291-320."""
    if m == 1:
        return 1j * np.pi / 2
    if m == -1:
        return -1j * np.pi / 2
    if m % 2 == 0:
        return 2.0 / (1 - m * m)
    return 0.0


def weights_mwss_theta_only(L, spin=0):
    """quadrature.py:238-262: FFT of the analytic weights on 2L points, folded to L+1 rings."""
    w = np.zeros(2 * L, dtype=np.complex128)
    for i in range(-(L - 1) + 1, L + 1):
        w[i + L - 1] = _mw_weight(i - 1)
    wr = np.real(np.fft.fft(np.fft.ifftshift(w), norm="backward")) / (2 * L)
    q = wr[: L + 1].copy()
    q[1:L] = q[1:L] + (-1) ** spin * wr[-1:L:-1]
    return q


def weights_mw_theta_only(L, spin=0):
    """quadrature.py:265-288."""
    w = np.zeros(2 * L - 1, dtype=np.complex128)
    for i in range(-(L - 1), L):
        w[i + L - 1] = _mw_weight(i)
    w *= np.exp(-1j * np.arange(-(L - 1), L) * np.pi / (2 * L - 1))
    wr = np.real(np.fft.fft(np.fft.ifftshift(w), norm="backward")) / (2 * L - 1)
    q = wr[:L].copy()
    q[: L - 1] = q[: L - 1] + (-1) ** spin * wr[-1 : L - 1 : -1]
    return q


def weights_gl(L):
    """Gauss-Legendre weights by Newton iteration, times 2pi/(2L-1). quadrature.py:125-161."""
    x1, x2 = -1.0, 1.0
    weights = np.zeros(L, dtype=np.float64)
    m = (L + 1) // 2
    xl = 0.5 * (x2 - x1)
    i = np.arange(1, m + 1)
    z = np.cos(np.pi * (i - 0.25) / (L + 0.5))
    z1 = 2.0
    while np.max(np.abs(z - z1)) > 1e-14:
        p1 = np.ones_like(z)
        p2 = np.zeros_like(z)
        for j in range(1, L + 1):
            p3 = p2
            p2 = p1
            p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j
        pp = L * (z * p1 - p2) / (z * z - 1.0)
        z1 = z
        z = z1 - p1 / pp
    weights[i - 1] = 2.0 * xl / ((1.0 - z**2) * pp * pp)
    weights[L - i] = weights[i - 1]
    return weights * 2 * np.pi / (2 * L - 1)


def weights_dh(L):
    """Driscoll-Healy weights, times 2pi/(2L-1). quadrature.py:164-201."""
    th = samples.thetas(L, "dh")
    k = np.arange(L)[:, None]
    w = np.sum(np.sin((2 * k + 1) * th[None, :]) / (2 * k + 1), axis=0)
    w *= 2.0 / L * np.sin(th)
    return w * 2 * np.pi / (2 * L - 1)


def weights_hp(nside):
    """Uniform HEALPix weights 4pi/Npix. quadrature.py:99-122."""
    return np.full(4 * nside - 1, 4 * np.pi / (12 * nside**2), dtype=np.float64)


def quad_weights_transform(L, sampling="mwss", spin=0, nside=0):
    """Transform weights with 2pi/nphi folded in. quadrature.py:7-50 (MW/MWSS use MWSS at 2L)."""
    s = sampling.lower()
    if s == "mwss":
        return weights_mwss_theta_only(2 * L, spin=0) * 2 * np.pi / (2 * L)
    if s == "dh":
        return weights_dh(L)
    if s == "gl":
        return weights_gl(L)
    if s == "healpix":
        return weights_hp(nside)
    raise ValueError(f"Sampling scheme sampling={sampling} not supported")


def quad_weights(L=None, sampling="mw", spin=0, nside=None):
    """Integration weights per scheme (quadrature.py:53-96)."""
    s = sampling.lower()
    if s == "mw":
        return weights_mw_theta_only(L, spin) * 2 * np.pi / (2 * L - 1)
    if s == "mwss":
        return weights_mwss_theta_only(L, spin) * 2 * np.pi / (2 * L)
    if s == "dh":
        return weights_dh(L)
    if s == "gl":
        return weights_gl(L)
    if s == "healpix":
        return weights_hp(nside)
    raise ValueError(f"Sampling scheme sampling={sampling} not implemented")
