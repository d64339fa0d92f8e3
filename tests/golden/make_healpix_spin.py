"""HEALPix spin transforms with exact Wigner-d values (fixture generator).

Upstream's recursive HEALPix transforms lose terms for spin != 0 where the
log-renormalised m-recursion (s2fft/transforms/otf_recursions.py:134-171) passes
through an exact zero of d^l_{m,-s} at one of HEALPix's rational cos(theta) rings:
log(0) = -inf turns the following values into NaN, which np.nansum drops. At
L=5 nside=2 spin 1, for example, d^3_{-1,-1}(arccos(1/3)) = 0.3317 comes out as 0 and
the map is off by 19 %. The float64 oracle restates that recursion, so it shares the
loss. This script therefore builds the reference values from exact d: the oracle's own
precompute-kernel path (construct.py:16-161, precompute spherical.py:87-149, 314-380)
with its d table replaced by Wigner's explicit sum in 40-digit arithmetic (mpmath).
The substitution is checked on MW first, where upstream's recursion is exact.

Writes ``healpix_spin.npz`` / ``healpix_spin.json``. Run from the repository root:
``python tests/golden/make_healpix_spin.py``.
"""

import json
import os
import sys

import mpmath as mp
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from oracle import precompute  # noqa: E402

mp.mp.dps = 40
SEED = 20261203


def wigner_d(l, m, n, theta):
    """d^l_{m,n}(theta), Wigner's explicit sum (first index m, second n)."""
    c, s = mp.cos(mp.mpf(theta) / 2), mp.sin(mp.mpf(theta) / 2)
    f = mp.factorial
    pre = mp.sqrt(f(l + m) * f(l - m) * f(l + n) * f(l - n))
    tot = mp.mpf(0)
    for k in range(0, 2 * l + 1):
        a = (l + n - k, k, m - n + k, l - m - k)
        if min(a) < 0:
            continue
        tot += (-1) ** (m - n + k) * pre / (f(a[0]) * f(a[1]) * f(a[2]) * f(a[3])) \
            * c ** (2 * l + n - m - 2 * k) * s ** (m - n + 2 * k)
    return tot


def exact_dtable(L, spin, th):
    """d^l_{m,-spin}(theta) [t, l, L-1+m] (the layout of oracle.precompute._dtable)."""
    d = np.zeros((len(th), L, 2 * L - 1))
    for t, theta in enumerate(th):
        for l in range(abs(spin), L):
            for m in range(-l, l + 1):
                d[t, l, L - 1 + m] = float(wigner_d(l, m, -spin, theta))
    return d


def transforms(flm, L, spin, sampling, nside):
    kin = precompute.spin_spherical_kernel(L, spin, False, sampling, nside, forward=False)
    f = precompute.inverse_transform(flm, kin, L, sampling, False, spin, nside)
    kfw = precompute.spin_spherical_kernel(L, spin, False, sampling, nside, forward=True)
    g = precompute.forward_transform(f, kfw, L, sampling, False, spin, nside)
    return f, g


def main():
    rng = np.random.default_rng(SEED)
    recursion_dtable = precompute._dtable

    # the exact-d substitution reproduces upstream where its recursion is exact (MW)
    L, spin = 9, 2
    flm = oracle.signal.generate_flm(rng, L, 0, spin, False)
    f_rec, g_rec = transforms(flm, L, spin, "mw", None)
    precompute._dtable = exact_dtable
    f_ex, g_ex = transforms(flm, L, spin, "mw", None)
    precompute._dtable = recursion_dtable
    assert np.abs(f_ex - f_rec).max() < 1e-12 * np.abs(f_rec).max()
    assert np.abs(g_ex - g_rec).max() < 1e-12 * np.abs(g_rec).max()

    out, index = {}, []
    precompute._dtable = exact_dtable
    for k, (L, nside, spin) in enumerate(((5, 2, 1), (5, 2, -1), (5, 2, 2), (9, 4, 2),
                                          (12, 4, -1))):
        flm = oracle.signal.generate_flm(rng, L, 0, spin, False)
        f, g = transforms(flm, L, spin, "healpix", nside)
        name = f"hp{k}"
        out[f"{name}/flm"] = flm
        out[f"{name}/f"] = f
        out[f"{name}/flm_fwd"] = g
        index.append(dict(name=name, L=L, nside=nside, spin=spin))
    precompute._dtable = recursion_dtable
    np.savez(os.path.join(HERE, "healpix_spin.npz"), **out)
    with open(os.path.join(HERE, "healpix_spin.json"), "w") as fh:
        json.dump(index, fh, indent=1)


if __name__ == "__main__":
    main()
