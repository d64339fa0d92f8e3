"""Seeded test signals. Restates s2fft/utils/signal_generator.py:10-201."""

import numpy as np

DEFAULT_SEED = 8966433580120847635  # tests/conftest.py:15 upstream


def complex_normal(rng, size, var=1.0):
    """signal_generator.py:10-39."""
    return np.asarray((rng.standard_normal(size) + 1j * rng.standard_normal(size))
                      * (var / 2) ** 0.5).astype(np.complex128)


def _tri(L, min_el):
    """(l, m) index pairs with m >= 1, l >= max(m, min_el). signal_generator.py:42-73."""
    el, m = np.tril_indices(L, k=-1)
    m = m + 1
    keep = el >= min_el
    return el[keep], m[keep]


def generate_flm(rng, L, L_lower=0, spin=0, reality=False):
    """signal_generator.py:76-123 (m = 0 real; zeros below max(L_lower, |spin|))."""
    flm = np.zeros((L, 2 * L - 1), dtype=np.complex128)
    lo = max(L_lower, abs(spin))
    flm[lo:L, L - 1] = rng.standard_normal(L - lo)
    el, m = _tri(L, lo)
    flm[el, L - 1 + m] = complex_normal(rng, len(m), var=2)
    if reality:
        flm[el, L - 1 - m] = (-1) ** m * flm[el, L - 1 + m].conj()
    else:
        flm[el, L - 1 - m] = complex_normal(rng, len(m), var=2)
    return flm


def generate_flm_full_complex(rng, L, L_lower=0, spin=0):
    """Re and Im i.i.d. N(0,1) for every |m| <= l (including a complex m = 0)."""
    flm = np.zeros((L, 2 * L - 1), dtype=np.complex128)
    lo = max(L_lower, abs(spin))
    for el in range(lo, L):
        n = 2 * el + 1
        flm[el, L - 1 - el: L + el] = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    return flm


def generate_flmn(rng, L, N=1, L_lower=0, reality=False):
    """signal_generator.py:126-201."""
    flmn = np.zeros((2 * N - 1, L, 2 * L - 1), dtype=np.complex128)
    for n in range(-N + 1, N):
        lo = max(L_lower, abs(n))
        if reality:
            if n == 0:
                flmn[N - 1, lo:L, L - 1] = rng.standard_normal(L - lo)
            elif n > 0:
                flmn[N - 1 + n, lo:L, L - 1] = complex_normal(rng, L - lo, var=2)
                flmn[N - 1 - n, lo:L, L - 1] = (-1) ** n * flmn[N - 1 + n, lo:L, L - 1].conj()
        else:
            flmn[N - 1 + n, lo:L, L - 1] = complex_normal(rng, L - lo, var=2)
        el, m = _tri(L, lo)
        flmn[N - 1 + n, el, L - 1 + m] = complex_normal(rng, len(m), var=2)
        if reality:
            flmn[N - 1 - n, el, L - 1 - m] = (-1.0) ** (m + n) * \
                flmn[N - 1 + n, el, L - 1 + m].conj()
        else:
            flmn[N - 1 + n, el, L - 1 - m] = complex_normal(rng, len(m), var=2)
    return flmn
