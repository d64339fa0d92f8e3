"""HEALPix ring FFTs (float64). Restates s2fft/utils/healpix_ffts.py (numpy variants)."""

import numpy as np

from . import samples


def spectral_folding(fm, nphi, L):
    """Alias a 2L-wide ring spectrum onto nphi bins. healpix_ffts.py:19-50."""
    start = L - nphi // 2
    out = fm[start : start + nphi].copy()
    for k in range(2 * L):
        if start <= k < start + nphi:
            continue
        out[(k - start) % nphi] += fm[k]
    return out


def spectral_periodic_extension(fm, nphi, L):
    """Periodically extend an nphi ring spectrum to 2L columns. healpix_ffts.py:85-117."""
    start = L - nphi // 2
    k = np.arange(2 * L)
    return fm[(k - start) % nphi]


def healpix_fft(f, L, nside, reality=False):
    """Per-ring FFT + fftshift + periodic extension to (4nside-1, 2L). healpix_ffts.py:187-226."""
    nth = 4 * nside - 1
    ftm = np.zeros((nth, 2 * L), dtype=np.complex128)
    offs, lens = samples.hp_ring_offsets(nside)
    for t in range(nth):
        n = int(lens[t])
        ring = f[offs[t] : offs[t] + n]
        if reality and n == 2 * L:
            chunk = np.zeros(n, dtype=np.complex128)
            chunk[n // 2 :] = np.fft.rfft(np.real(ring), norm="backward")[:-1]
        else:
            chunk = np.fft.fftshift(np.fft.fft(ring, norm="backward"))
        ftm[t] = chunk if n == 2 * L else spectral_periodic_extension(chunk, n, L)
    return ftm


def healpix_ifft(ftm, L, nside, reality=False):
    """Fold each row to its ring length and inverse FFT. healpix_ffts.py:297-371.

    The upstream numpy version returns complex128 even for real maps (healpix_ffts.py:356).
    """
    assert L >= 2 * nside
    f = np.zeros(12 * nside**2, dtype=np.complex128)
    offs, lens = samples.hp_ring_offsets(nside)
    for t in range(ftm.shape[0]):
        n = int(lens[t])
        chunk = ftm[t] if n == 2 * L else spectral_folding(ftm[t], n, L)
        if reality and n == 2 * L:
            f[offs[t] : offs[t] + n] = np.fft.irfft(chunk[n // 2 :], n, norm="forward")
        else:
            f[offs[t] : offs[t] + n] = np.fft.ifft(np.fft.ifftshift(chunk), norm="forward")
    return f


def ring_phi0(nside):
    """Longitude of the first pixel of each ring. healpix_ffts.py:429-452."""
    t = np.arange(4 * nside - 1)
    out = np.zeros(t.shape, dtype=np.float64)
    belt = (t + 1 >= nside) & (t + 1 <= 3 * nside)
    out = np.where(belt, 0.5 * ((t - nside + 2) % 2) * np.pi / (2 * nside), out)
    out = np.where(t + 1 > 3 * nside, 0.5 * np.pi / (2 * (4 * nside - t - 1)), out)
    out = np.where(t + 1 < nside, 0.5 * np.pi / (2 * (t + 1)), out)
    return out


def ring_phase_shifts_hp(L, nside, forward=False, reality=False):
    """exp(+-i m phi0(t)). healpix_ffts.py:482-509."""
    sign = -1 if forward else 1
    m0 = 0 if reality else -L + 1
    return np.exp(sign * 1j * np.outer(ring_phi0(nside), np.arange(m0, L)))
