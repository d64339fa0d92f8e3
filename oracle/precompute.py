"""Precompute-kernel spherical transforms (float64).

Restates s2fft/precompute_transforms/construct.py:16-161 (kernel
K[t, l, m] = d^l_{m,-s}(theta_t) sqrt((2l+1)/4pi) [x w_t] [x HEALPix phase]) and
s2fft/precompute_transforms/spherical.py:87-149, 314-380 (the einsum transforms).
"""

import numpy as np

from . import healpix, quadrature, recursion, resampling, samples


def _dtable(L, spin, th):
    """d^l_{m,-spin}(theta) [t, l, L-1+m], with exact pole rows."""
    pole_n = np.isclose(th, 0.0, atol=1e-14)
    pole_s = np.isclose(th, np.pi, atol=1e-14)
    inner = ~(pole_n | pole_s)
    d = np.zeros((len(th), L, 2 * L - 1))
    if inner.any():
        d[inner] = recursion.wigner_d_slice(L, spin, th[inner])
    el = np.arange(L)
    ok = el >= abs(spin)
    for t in np.where(pole_n)[0]:
        d[t, ok, L - 1 - spin] = 1.0
    for t in np.where(pole_s)[0]:
        d[t, ok, L - 1 + spin] = (-1.0) ** ((el[ok] + spin) % 2)
    return d


def spin_spherical_kernel(L, spin=0, reality=False, sampling="mw", nside=None, forward=True):
    """construct.py:16-161 (values only; the recursion used to build them is irrelevant)."""
    sampling = sampling.lower()
    if reality and spin != 0:
        reality = False
    m0 = L - 1 if reality else 0
    if forward and sampling in ("mw", "mwss"):
        sampling = "mwss"
        th = samples.thetas(2 * L, "mwss")
    else:
        th = samples.thetas(L, sampling, nside)
    dl = _dtable(L, spin, th)[:, :, m0:]
    dl *= np.sqrt((2 * np.arange(L) + 1) / (4 * np.pi))[None, :, None]
    if forward:
        dl *= quadrature.quad_weights_transform(L, sampling, 0, nside)[:, None, None]
    if sampling == "healpix":
        ph = healpix.ring_phase_shifts_hp(L, nside, forward, False)[:, m0:]
        dl = dl * ph[:, None, :]
    return dl


def inverse_transform(flm, kernel, L, sampling, reality, spin, nside):
    """spherical.py:87-149 (precompute)."""
    sampling = sampling.lower()
    mo = 1 if sampling in ("mwss", "healpix") else 0
    m0 = L - 1 if reality else 0
    ftm = np.zeros(samples.ftm_shape(L, sampling, nside), dtype=np.complex128)
    ftm[:, m0 + mo:] = np.einsum("tlm,lm->tm", kernel, flm[:, m0:])
    ftm *= (-1) ** spin
    if sampling == "healpix":
        if reality:
            ftm[:, mo : m0 + mo] = np.flip(np.conj(ftm[:, m0 + mo + 1:]), axis=-1)
        return healpix.healpix_ifft(ftm, L, nside, reality)
    if reality:
        return np.fft.irfft(ftm[:, m0 + mo:], samples.nphi_equiang(L, sampling), axis=-1,
                            norm="forward")
    return np.fft.ifft(np.fft.ifftshift(ftm, axes=-1), axis=-1, norm="forward")


def forward_transform(f, kernel, L, sampling, reality, spin, nside):
    """spherical.py:314-380 (precompute)."""
    sampling = sampling.lower()
    if sampling == "mw":
        f = resampling.mw_to_mwss(f, L, spin)
    if sampling in ("mw", "mwss"):
        sampling = "mwss"
        f = resampling.upsample_by_two_mwss(f, L, spin)
    mo = 1 if sampling in ("mwss", "healpix") else 0
    m0 = L - 1 if reality else 0
    if sampling == "healpix":
        ftm = healpix.healpix_fft(f, L, nside, reality)[:, mo:]
        if reality:
            ftm = ftm[:, m0:]
    elif reality:
        ftm = np.fft.rfft(np.real(f), axis=-1, norm="backward")
        if mo:
            ftm = ftm[:, :-1]
    else:
        ftm = np.fft.fftshift(np.fft.fft(f, axis=-1, norm="backward"), axes=-1)[:, mo:]
    flm = np.zeros(samples.flm_shape(L), dtype=np.complex128)
    flm[:, m0:] = np.einsum("tlm,tm->lm", kernel, ftm)
    if reality:
        flm[:, :m0] = np.flip((-1.0) ** (np.arange(1, L) % 2) * np.conj(flm[:, m0 + 1:]),
                              axis=-1)
    return flm * (-1) ** spin
