"""Price-McEwen latitudinal recursion (float64).

Restates s2fft/recursions/price_mcewen.py (the O(L^2)-memory coefficient
generator, lines 118-255) and s2fft/transforms/otf_recursions.py (the numpy
inverse/forward latitudinal steps, lines 15-171 and 432-588).

The recursion runs over m for all (theta, l) at once, from |m| = l inward,
renormalising every step in log space, exactly as upstream. ``max_steps``
truncates the m loop; it exists only so that the CPU baseline can time a
bounded sample of the reference algorithm.
"""

import numpy as np

from . import samples


def precompute(L, spin, beta, L_lower=0):
    """[lrenorm, vsign, cpi, cp2] for spin and ring colatitudes beta.

    Follows price_mcewen.py:118-255 (generate_precomputes_jax), evaluated with numpy.
    """
    mm = -spin
    L0 = L_lower
    el = np.arange(L0, L)
    nth = len(beta)
    with np.errstate(divide="ignore"):
        lt = np.log(np.abs(np.tan(-beta / 2.0)))
        lc2 = np.log(np.abs(np.cos(beta / 2.0)))
    halves = [el + mm + 1, el - mm + 1]

    # cp(m) = cplus(l - m) coefficients, rolled so that row m-1 serves step m. 181-201
    cpi = np.zeros((L + 1, L - L0))
    cp2 = np.zeros((L + 1, L - L0))
    with np.errstate(divide="ignore", invalid="ignore"):
        cpi[0] = 2.0 / np.sqrt(2 * el)
        for m in range(2, L + 1):
            cpi[m - 1] = 2.0 / np.sqrt(m * (2 * el + 1 - m))
            cp2[m - 1] = cpi[m - 1] / cpi[m - 2]
    for k in range(L0, L):
        cpi[:, k - L0] = np.roll(cpi[:, k - L0], L - k - 1)
        cp2[:, k - L0] = np.roll(cp2[:, k - L0], L - k - 1)

    # sign table. 206-210
    msign = np.hstack(((-1.0) ** np.abs(np.arange(L - 1)), np.ones(L)))
    lsign = (-1.0) ** np.abs(mm + el)
    vsign = np.outer(msign, lsign)
    vsign[: L - 1] *= (-1.0) ** abs(mm + 1 + L)

    # log of the first-row seeds log|d^l_{-+l, mm}|. 212-243
    lrenorm = np.zeros((2, nth, L - L0))
    row = np.outer(lc2, 2.0 * el)  # log_first_row[0]
    for h in range(2):
        lrenorm[h] = np.where(halves[h][None, :] == 1, row, lrenorm[h])
    with np.errstate(divide="ignore", invalid="ignore"):
        for i in range(2, L + abs(mm) + 2):
            row = row + np.log((2 * el + 2 - i) / (i - 1))[None, :] / 2 + lt[:, None]
            for h in range(2):
                lrenorm[h] = np.where(halves[h][None, :] == i, row, lrenorm[h])
    # 251-253
    lrenorm = np.nan_to_num(lrenorm, nan=0.0, posinf=0.0, neginf=0.0)
    cpi = np.nan_to_num(cpi, nan=0.0, posinf=0.0, neginf=0.0)
    cp2 = np.nan_to_num(cp2, nan=0.0, posinf=0.0, neginf=0.0)
    return [lrenorm, vsign, cpi, cp2]


def _lambda(el, omc, c, s, col, half_slice):
    """lambda(theta, l) at step col. otf_recursions.py:104-109, 140-145."""
    lam = np.outer(omc, el + 1) + np.outer(c, col + el) - half_slice[None, :]
    return lam / s[:, None]


def inverse_latitudinal_step(flm, beta, L, spin, sampling="mw", reality=False,
                             precomps=None, L_lower=0, max_steps=None, nside=None):
    """ftm[theta, m] = sum_l d^l_{m,-s}(theta) flm[l, m]. otf_recursions.py:15-171."""
    mm = -spin
    nth = len(beta)
    ncol = samples.ftm_shape(L, sampling, nside)[1]
    ftm = np.zeros((nth, ncol), dtype=np.complex128)
    el = np.arange(L_lower, L)
    c, s = np.cos(beta), np.sin(beta)
    omc = 1.0 - c
    halves = [el + mm + 1, el - mm + 1]
    if precomps is None:
        precomps = precompute(L, -mm, beta, L_lower)
    lrenorm, vsign, cpi, cp2 = precomps[:4]
    lrenorm = lrenorm.copy()
    lidx = el[None, :]
    with np.errstate(all="ignore"):
        for i in range(2):
            if reality and i == 0:
                continue
            mo = 1 if sampling in ("mwss", "healpix") and i == 0 else 0
            lind = L - 1 - L_lower
            sind = (0, -1)[i]
            sgn = (-1) ** i
            d = np.ones((2, nth, L - L_lower))
            lam = _lambda(el, omc, c, s, 2 - L, halves[i])
            d[1, :, lind:] = cpi[0, lind:] * d[0, :, lind:] * lam[:, lind:]
            ftm[:, sind + mo] = np.nansum(
                d[0, :, lind:] * vsign[sind, lind:] * np.exp(lrenorm[i, :, lind:])
                * flm[lind + L_lower:, sind], axis=-1)
            ftm[:, sind + sgn + mo] = np.nansum(
                d[1, :, lind - 1:] * vsign[sind + sgn, lind - 1:]
                * np.exp(lrenorm[i, :, lind - 1:]) * flm[lind - 1 + L_lower:, sind + sgn],
                axis=-1)
            entry = np.zeros((nth, L))
            last = L - 1 + i if max_steps is None else min(L - 1 + i, 2 + max_steps)
            for m in range(2, last):
                act = lidx >= L - m - 1
                lam = _lambda(el, omc, c, s, m - L + 1, halves[i])
                entry[:, L_lower:] = np.where(
                    act, cpi[m - 1] * d[1] * lam - cp2[m - 1] * d[0], entry[:, L_lower:])
                entry[:, -(m + 1)] = 1
                col = sind + sgn * m
                ftm[:, col + mo] = np.nansum(
                    entry[:, L_lower:] * vsign[col] * np.exp(lrenorm[i]) * flm[L_lower:, col],
                    axis=-1)
                mag = np.abs(entry[:, L_lower:])
                d0 = np.where(act, d[1] / mag, d[0])
                d1 = np.where(act, entry[:, L_lower:] / mag, d[1])
                lrenorm[i] = np.where(act, lrenorm[i] + np.log(mag), lrenorm[i])
                d[0], d[1] = d0, d1
    return ftm


def forward_latitudinal_step(ftm, beta, L, spin, sampling="mw", reality=False,
                             precomps=None, L_lower=0, max_steps=None):
    """flm[l, m] = sum_theta d^l_{m,-s}(theta) ftm[theta, m]. otf_recursions.py:432-588."""
    mm = -spin
    nth = len(beta)
    flm = np.zeros(samples.flm_shape(L), dtype=np.complex128)
    el = np.arange(L_lower, L)
    c, s = np.cos(beta), np.sin(beta)
    omc = 1.0 - c
    halves = [el + mm + 1, el - mm + 1]
    if precomps is None:
        precomps = precompute(L, -mm, beta, L_lower)
    lrenorm, vsign, cpi, cp2 = precomps[:4]
    lrenorm = lrenorm.copy()
    lidx = el[None, :]
    with np.errstate(all="ignore"):
        for i in range(2):
            if reality and i == 0:
                continue
            mo = 1 if sampling in ("mwss", "healpix") and i == 0 else 0
            lind = L - 1 - L_lower
            sind = (0, -1)[i]
            sgn = (-1) ** i
            d = np.ones((2, nth, L - L_lower))
            lam = _lambda(el, omc, c, s, 2 - L, halves[i])
            d[1, :, lind:] = cpi[0, lind:] * d[0, :, lind:] * lam[:, lind:]
            flm[lind + L_lower:, sind] = np.nansum(
                d[0, :, lind:] * vsign[sind, lind:] * np.exp(lrenorm[i, :, lind:])
                * ftm[:, sind + mo][:, None], axis=-2)
            flm[lind - 1 + L_lower:, sind + sgn] = np.nansum(
                d[1, :, lind - 1:] * vsign[sind + sgn, lind - 1:]
                * np.exp(lrenorm[i, :, lind - 1:]) * ftm[:, sind + sgn + mo][:, None],
                axis=-2)
            entry = np.zeros((nth, L))
            last = L - 1 + i if max_steps is None else min(L - 1 + i, 2 + max_steps)
            for m in range(2, last):
                act = lidx >= L - m - 1
                lam = _lambda(el, omc, c, s, m - L + 1, halves[i])
                entry[:, L_lower:] = np.where(
                    act, cpi[m - 1] * d[1] * lam - cp2[m - 1] * d[0], entry[:, L_lower:])
                entry[:, -(m + 1)] = 1
                col = sind + sgn * m
                flm[L_lower:, col] = np.nansum(
                    entry[:, L_lower:] * vsign[col] * np.exp(lrenorm[i])
                    * ftm[:, col + mo][:, None], axis=-2)
                mag = np.abs(entry[:, L_lower:])
                d0 = np.where(act, d[1] / mag, d[0])
                d1 = np.where(act, entry[:, L_lower:] / mag, d[1])
                lrenorm[i] = np.where(act, lrenorm[i] + np.log(mag), lrenorm[i])
                d[0], d[1] = d0, d1
    return flm


def wigner_d_slice(L, spin, beta):
    """Dense d^l_{m,-spin}(beta) table [t, l, L-1+m] from the same recursion.

    Built by projecting unit coefficient columns; used only by small tests
    and by the precompute-kernel oracle. O(L^3) memory.
    """
    nth = len(beta)
    out = np.zeros((nth, L, 2 * L - 1))
    for el in range(abs(spin), L):
        flm = np.zeros((L, 2 * L - 1), dtype=np.complex128)
        flm[el, :] = 1.0
        ftm = inverse_latitudinal_step(flm, beta, L, spin, "mw")
        out[:, el, :] = np.real(ftm)
        out[:, el, : L - 1 - el] = 0
        out[:, el, L + el:] = 0
    return out
