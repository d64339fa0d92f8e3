"""Sampling geometry (float64). Restates s2fft/sampling/s2_samples.py and so3_samples.py."""

import numpy as np

SAMPLINGS = ("mw", "mwss", "dh", "gl", "healpix")


def ntheta(L=None, sampling="mw", nside=None):
    """Rings per scheme. s2fft/sampling/s2_samples.py:4-52."""
    s = sampling.lower()
    if s in ("mw", "gl"):
        return L
    if s == "mwss":
        return L + 1
    if s == "dh":
        return 2 * L
    if s == "healpix":
        if nside is None:
            raise ValueError("healpix sampling needs nside")
        return 4 * nside - 1
    raise ValueError(f"Sampling scheme sampling={sampling} not supported")


def nphi_equiang(L, sampling="mw"):
    """Samples per ring for the equiangular schemes. s2_samples.py:85-123."""
    s = sampling.lower()
    if s in ("mw", "gl", "dh"):
        return 2 * L - 1
    if s == "mwss":
        return 2 * L
    raise ValueError(f"Sampling scheme sampling={sampling} not supported")


def ftm_shape(L, sampling="mw", nside=None):
    """Shape of the ring-spectrum array. s2_samples.py:126-155 (2L columns for mwss/healpix)."""
    s = sampling.lower()
    if s in ("mwss", "healpix"):
        return ntheta(L, s, nside), 2 * L
    return ntheta(L, s, nside), 2 * L - 1


def f_shape(L=None, sampling="mw", nside=None):
    """Signal shape. s2_samples.py:446-478."""
    if sampling.lower() == "healpix":
        return (12 * nside**2,)
    return ntheta(L, sampling), nphi_equiang(L, sampling)


def flm_shape(L):
    """Harmonic array [l, L-1+m]. s2_samples.py:481-492."""
    return L, 2 * L - 1


def nphi_ring(t, nside):
    """HEALPix ring length. s2_samples.py:173-200."""
    if 0 <= t < nside - 1:
        return 4 * (t + 1)
    if nside - 1 <= t <= 3 * nside - 1:
        return 4 * nside
    if 3 * nside - 1 < t <= 4 * nside - 2:
        return 4 * (4 * nside - t - 1)
    raise ValueError(f"Ring t={t} not contained by nside={nside}")


def _healpix_theta(t, nside):
    """HEALPix ring colatitudes from z. s2_samples.py:284-308."""
    t = np.asarray(t, dtype=np.float64)
    z = np.zeros_like(t)
    north = t < nside - 1
    belt = (t >= nside - 1) & (t <= 3 * nside - 1)
    south = (t > 3 * nside - 1) & (t <= 4 * nside - 2)
    z[north] = 1 - (t[north] + 1) ** 2 / (3 * nside**2)
    z[belt] = 4 / 3 - 2 * (t[belt] + 1) / (3 * nside)
    z[south] = (4 * nside - 1 - t[south]) ** 2 / (3 * nside**2) - 1
    return np.arccos(z)


def thetas(L=None, sampling="mw", nside=None):
    """Ring colatitudes. s2_samples.py:203-281."""
    s = sampling.lower()
    if s == "gl":
        return np.flip(np.arccos(np.polynomial.legendre.leggauss(L)[0]))
    t = np.arange(ntheta(L, s, nside), dtype=np.float64)
    if s == "mw":
        return (2 * t + 1) * np.pi / (2 * L - 1)
    if s == "mwss":
        return 2 * t * np.pi / (2 * L)
    if s == "dh":
        return (2 * t + 1) * np.pi / (4 * L)
    if s == "healpix":
        return _healpix_theta(t, nside)
    raise ValueError(f"Sampling scheme sampling={sampling} not supported")


def phis_equiang(L, sampling="mw"):
    """Ring longitudes. s2_samples.py:356-409."""
    p = np.arange(nphi_equiang(L, sampling))
    n = 2 * L if sampling.lower() == "mwss" else 2 * L - 1
    return 2 * p * np.pi / n


def p2phi_ring(t, p, nside):
    """HEALPix pixel longitude within ring t. s2_samples.py:329-353."""
    shift = 0.5
    if nside <= t + 1 <= 3 * nside:
        shift *= (t - nside + 2) % 2
        return np.pi / (2 * nside) * (p + shift)
    if t + 1 > 3 * nside:
        return np.pi / (2 * (4 * nside - t - 1)) * (p + shift)
    return np.pi / (2 * (t + 1)) * (p + shift)


def hp_ring_offsets(nside):
    """Start pixel and length of every HEALPix ring (ring-ordered map)."""
    nth = 4 * nside - 1
    lens = np.array([nphi_ring(t, nside) for t in range(nth)], dtype=np.int64)
    offs = np.concatenate(([0], np.cumsum(lens)[:-1]))
    return offs, lens


# --- SO(3) sampling: s2fft/sampling/so3_samples.py ---------------------------------


def so3_f_shape(L, N, sampling="mw", nside=None):
    """so3_samples.py:6-47."""
    if sampling.lower() == "healpix":
        return 2 * N - 1, 12 * nside**2
    return (2 * N - 1,) + f_shape(L, sampling)


def flmn_shape(L, N):
    """so3_samples.py:50-65."""
    return 2 * N - 1, L, 2 * L - 1
