"""MW -> MWSS resampling and x2 upsampling (float64). Restates s2fft/utils/resampling.py."""

import numpy as np

from . import samples


def periodic_extension(f, L, spin=0, sampling="mw"):
    """theta extension to [0, 2pi) in the phi-Fourier domain. resampling.py:6-61.

    f has shape (batch, ntheta, nphi); returns (batch, ntheta_ext, nphi).
    """
    nth = samples.ntheta(L, sampling)
    nph = samples.nphi_equiang(L, sampling)
    nth_ext = 2 * L - 1 if sampling == "mw" else 2 * L
    mo = 1 if sampling == "mwss" else 0
    fe = np.zeros((f.shape[0], nth_ext, nph), dtype=np.complex128)
    fe[:, :nth, :nph] = f[:, :nth, :nph]
    fe = np.fft.fftshift(np.fft.fft(fe, axis=-1, norm="backward"), axes=-1)
    lo, hi = L + mo, 2 * L - 1 + mo
    fe[:, lo:hi, mo:hi] = np.flip(fe[:, mo : L - 1 + mo, mo:hi], axis=-2)
    fe[:, lo:hi, mo:hi] *= (-1) ** np.abs(np.arange(-(L - 1), L))
    fe[:, lo:hi, mo:hi] *= (-1) ** abs(spin)
    return np.fft.ifft(np.fft.ifftshift(fe, axes=-1), axis=-1, norm="backward")


def periodic_extension_spatial_mwss(f, L, spin=0):
    """Spatial theta extension of an MWSS map to 2L rings. resampling.py:64-101."""
    nth, nph = L + 1, 2 * L
    fe = np.zeros((f.shape[0], 2 * L, nph), dtype=np.complex128)
    fe[:, :nth, :nph] = f[:, :nth, :nph]
    fe[:, nth:, :] = (-1) ** abs(spin) * np.fft.fftshift(
        np.flip(f[:, 1 : nth - 1, :], axis=-2), axes=-1
    )
    return fe


def upsample_by_two_mwss(f, L, spin=0):
    """MWSS(L) -> MWSS(2L) by zero-padding the theta spectrum. resampling.py:104-160."""
    squeeze = f.ndim == 2
    if squeeze:
        f = f[None]
    fe = periodic_extension_spatial_mwss(f, L, spin)
    fe = np.fft.fftshift(np.fft.fft(fe, axis=-2, norm="forward"), axes=-2)
    up = np.zeros((fe.shape[0], 4 * L, 2 * L), dtype=np.complex128)
    up[:, L : 3 * L, :] = fe
    up = np.fft.ifft(np.fft.ifftshift(up, axes=-2), axis=-2, norm="forward")
    out = up[:, : 2 * L + 1, :]
    return out[0] if squeeze else out


def mw_to_mwss_phi(f, L):
    """phi resampling 2L-1 -> 2L by spectral zero-padding. resampling.py:248-281."""
    out = np.zeros((f.shape[0], L + 1, 2 * L), dtype=np.complex128)
    out[:, :, 1:] = np.fft.fftshift(np.fft.fft(f, axis=-1, norm="forward"), axes=-1)
    return np.fft.ifft(np.fft.ifftshift(out, axes=-1), axis=-1, norm="forward")


def mw_to_mwss_theta(f, L, spin=0):
    """theta resampling MW -> MWSS with a half-sample shift. resampling.py:284-326."""
    fe = periodic_extension(f, L, spin=spin, sampling="mw")
    fm = np.zeros((fe.shape[0], 2 * L, 2 * L - 1), dtype=np.complex128)
    fm[:, 1:, :] = np.fft.fftshift(np.fft.fft(fe, axis=-2, norm="forward"), axes=-2)
    shift = np.exp(-1j * np.arange(-(L - 1), L) * np.pi / (2 * L - 1))
    fm[:, 1:, :] *= shift[None, :, None]
    out = np.fft.ifft(np.fft.ifftshift(fm, axes=-2), axis=-2, norm="forward")
    return out[:, : L + 1, :]


def mw_to_mwss(f, L, spin=0):
    """resampling.py:329-355."""
    if f.ndim == 2:
        return mw_to_mwss_phi(mw_to_mwss_theta(f[None], L, spin), L)[0]
    return mw_to_mwss_phi(mw_to_mwss_theta(f, L, spin), L)
