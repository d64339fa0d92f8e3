"""Spin spherical-harmonic transforms (float64).

Restates s2fft/transforms/spherical.py: ``inverse_numpy`` (lines 112-208),
``forward_numpy`` (467-588) and the iterative-refinement wrapper used by
``forward`` (425-464 -> s2fft/utils/iterative_refinement.py:9-46).
"""

import numpy as np

from . import healpix, quadrature, recursion, resampling, samples


def _steps(backend):
    """The latitudinal steps: the numpy restatement, or its C port (oracle/csrc/otf.c)."""
    if backend == "c":
        from . import cport

        return cport
    return recursion


def _norm(L, L0):
    return np.sqrt((2 * np.arange(L0, L) + 1) / (4 * np.pi))


def inverse(flm, L, spin=0, nside=None, sampling="mw", reality=False, precomps=None,
            L_lower=0, max_steps=None, backend="numpy"):
    """spherical.py:112-208."""
    sampling = sampling.lower()
    th = samples.thetas(L, sampling, nside)
    mo = 1 if sampling in ("mwss", "healpix") else 0
    m0 = L - 1 if reality else 0
    flm = np.array(flm, dtype=np.complex128, copy=True)
    flm[L_lower:] *= _norm(L, L_lower)[:, None]
    ftm = _steps(backend).inverse_latitudinal_step(
        flm, th, L, spin, sampling, reality, precomps, L_lower, max_steps, nside)
    # pole rows carry only m = +-spin (176-184)
    if sampling in ("mw", "mwss"):
        ftm[-1] = 0
        ftm[-1, L - 1 + spin + mo] = np.nansum(
            (-1.0) ** np.abs(np.arange(L_lower, L) - spin) * flm[L_lower:, L - 1 + spin])
    if sampling == "mwss":
        ftm[0] = 0
        ftm[0, L - 1 - spin + mo] = np.nansum(flm[L_lower:, L - 1 - spin])
    if sampling == "healpix":
        ftm[:, m0 + mo:] *= healpix.ring_phase_shifts_hp(L, nside, False, reality)
    ftm *= (-1) ** spin
    if sampling == "healpix":
        if reality:
            ftm[:, mo : L - 1 + mo] = np.flip(np.conj(ftm[:, L - 1 + mo + 1:]), axis=-1)
        return healpix.healpix_ifft(ftm, L, nside, reality)
    if reality:
        return np.fft.irfft(ftm[:, L - 1 + mo:], samples.nphi_equiang(L, sampling), axis=1,
                            norm="forward")
    return np.fft.ifft(np.fft.ifftshift(ftm, axes=1), axis=1, norm="forward")


def _forward_once(f, L, spin=0, nside=None, sampling="mw", reality=False, precomps=None,
                  L_lower=0, max_steps=None, backend="numpy"):
    """spherical.py:467-588."""
    sampling = sampling.lower()
    if sampling == "mw":
        f = resampling.mw_to_mwss(f, L, spin)
    if sampling in ("mw", "mwss"):
        sampling = "mwss"
        f = resampling.upsample_by_two_mwss(f, L, spin)
        th = samples.thetas(2 * L, sampling)
    else:
        th = samples.thetas(L, sampling, nside)
    w = quadrature.quad_weights_transform(L, sampling, 0, nside)
    mo = 1 if sampling in ("mwss", "healpix") else 0
    m0 = L - 1 if reality else 0
    if sampling == "healpix":
        ftm = healpix.healpix_fft(f, L, nside, reality)
    elif reality:
        t = np.fft.rfft(np.real(f), axis=1, norm="backward")
        if mo:
            t = t[:, :-1]
        ftm = np.zeros(f.shape, dtype=np.complex128)
        ftm[:, L - 1 + mo:] = t
    else:
        ftm = np.fft.fftshift(np.fft.fft(f, axis=1, norm="backward"), axes=1)
    ftm = ftm * w[:, None]
    if sampling == "healpix":
        ftm[:, m0 + mo:] *= healpix.ring_phase_shifts_hp(L, nside, True, reality)
    if sampling == "mwss":
        flm = _steps(backend).forward_latitudinal_step(
            ftm[1:-1], th[1:-1], L, spin, sampling, reality, precomps, L_lower, max_steps)
        flm[L_lower:, L - 1 + spin] += (-1.0) ** np.abs(np.arange(L_lower, L) - spin) * \
            ftm[-1, L - 1 + spin + mo]
        flm[L_lower:, L - 1 - spin] += ftm[0, L - 1 - spin + mo]
    else:
        flm = _steps(backend).forward_latitudinal_step(
            ftm, th, L, spin, sampling, reality, precomps, L_lower, max_steps)
    flm[L_lower:] *= _norm(L, L_lower)[:, None]
    if reality:
        mc = (-1.0) ** (np.arange(1, L) % 2)
        flm[..., :m0] = np.flip(mc * np.conj(flm[..., m0 + 1:]), axis=-1)
    flm[: max(abs(spin), L_lower)] = 0.0
    return flm * (-1) ** spin


def forward(f, L, spin=0, nside=None, sampling="mw", reality=False, precomps=None,
            L_lower=0, iter=0, max_steps=None, backend="numpy"):
    """forward + Jacobi refinement: flm = F(f); repeat: flm += F(f - I(flm)).

    spherical.py:425-464 and iterative_refinement.py:9-46.
    """
    kw = dict(L=L, spin=spin, nside=nside, sampling=sampling, reality=reality, L_lower=L_lower)
    flm = _forward_once(f, precomps=precomps, max_steps=max_steps, backend=backend, **kw)
    for _ in range(iter or 0):
        err = f - inverse(flm, max_steps=max_steps, backend=backend, **kw)
        flm = flm + _forward_once(err, precomps=precomps, max_steps=max_steps, backend=backend,
                                  **kw)
    return flm
