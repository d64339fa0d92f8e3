"""Exact spin spherical harmonics on the rings nearest the poles (fixture generator).

Writes ``high_spin.npz``: for MW sampling and a few (L, spin, l, m), the values
f(theta_t, phi) = c_t exp(i m phi) of the inverse transform of the unit coefficient
flm[l, m] = 1 on the rings t nearest the poles, with

    c_t = (-1)^s sqrt((2l + 1) / 4pi) d^l_{m,-s}(theta_t)

evaluated by Wigner's explicit sum in 60-digit arithmetic (mpmath). These are the
orders where the m-recursion of upstream's on-the-fly path (s2fft/transforms/
otf_recursions.py) runs through the decaying range below m = -s cos(theta) and loses
digits; the fixture pins the exact values there. The convention (sign, normalisation,
theta grid) is checked against the float64 oracle first, on a small band-limit where
the oracle is accurate.

Run from the repository root: ``python tests/golden/make_high_spin.py``.
"""

import json
import os
import sys

import mpmath as mp
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402

mp.mp.dps = 60


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


def ring_factor(l, m, spin, theta):
    return (-1) ** (spin % 2) * mp.sqrt((2 * l + 1) / (4 * mp.pi)) * wigner_d(l, m, -spin, theta)


def check_convention():
    L, spin = 12, -3
    th = oracle.samples.thetas(L, "mw")
    phi = oracle.samples.phis_equiang(L, "mw")
    for (l, m) in ((3, 0), (5, -2), (9, 4)):
        flm = np.zeros((L, 2 * L - 1), dtype=np.complex128)
        flm[l, L - 1 + m] = 1.0
        f = oracle.spherical.inverse(flm, L, spin, None, "mw")
        for t in (0, 4, L - 2):
            ref = float(ring_factor(l, m, spin, th[t])) * np.exp(1j * m * phi)
            assert np.max(np.abs(f[t] - ref)) < 1e-12, (l, m, t)


CASES = [
    # L, spin, [(l, m)], rings
    (256, -7, [(7, 0), (7, 3), (40, 1), (255, 0), (255, 6), (100, -3), (9, -5)]),
    (256, 7, [(7, 0), (7, -3), (40, -1), (255, 0), (255, -6), (100, 3), (9, 5)]),
    (128, -15, [(15, 0), (15, 7), (60, 2), (127, 14), (127, -9)]),
]


def main():
    check_convention()
    out, index = {}, []
    for k, (L, spin, lms) in enumerate(CASES):
        th = oracle.samples.thetas(L, "mw")
        rings = [0, 1, 2, L - 3, L - 2]
        vals = np.array([[float(ring_factor(l, m, spin, th[t])) for t in rings] for (l, m) in lms])
        out[f"c{k}/values"] = vals
        index.append(dict(name=f"c{k}", L=L, spin=spin, lm=[list(x) for x in lms], rings=rings))
    np.savez(os.path.join(HERE, "high_spin.npz"), **out)
    with open(os.path.join(HERE, "high_spin.json"), "w") as fh:
        json.dump(index, fh, indent=1)


if __name__ == "__main__":
    main()
