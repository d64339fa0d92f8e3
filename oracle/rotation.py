"""Rotation of spherical-harmonic coefficients (float64, numpy).

Restates s2fft/utils/rotation.py:9-96 (rotate_flms, generate_rotate_dls) with the
Wigner-d planes from Risbo's recursion (s2fft/recursions/risbo.py:4-120: two
half-degree steps per degree), written here as a vectorised gather over the new plane.
"""

import numpy as np


def _half_step(S, j, c, s):
    """Plane S (j x j) -> D ((j+1) x (j+1)) for the half-degree step with 2l = j."""
    n = j + 1
    I = np.arange(n)[:, None]
    K = np.arange(n)[None, :]
    P = np.zeros((j + 2, j + 2))  # S padded with a zero border on both sides
    P[1:j + 1, 1:j + 1] = S
    sjI, sI = np.sqrt(np.maximum(j - I, 0)), np.sqrt(I)
    sjK, sK = np.sqrt(np.maximum(j - K, 0)), np.sqrt(K)
    D = (c * sjI * sjK * P[I + 1, K + 1] - s * sI * sjK * P[I, K + 1]
         + s * sjI * sK * P[I + 1, K] + c * sI * sK * P[I, K])
    return D / j


def dl_planes(L, beta):
    """[d^l(beta)] for 0 <= l < L; plane l is (2l+1)^2 with d^l_{m,n} at [l+m, l+n]."""
    c, s = np.cos(beta / 2), np.sin(beta / 2)
    P = np.ones((1, 1))
    out = [P]
    for l in range(1, L):
        P = _half_step(_half_step(P, 2 * l - 1, c, s), 2 * l, c, s)
        out.append(P)
    return out


def generate_rotate_dls(L, beta):
    """rotation.py:75-96: [L, 2L-1, 2L-1] with d^l_{m,n}(beta) at [l, L-1+m, L-1+n]."""
    dl = np.zeros((L, 2 * L - 1, 2 * L - 1))
    for l, P in enumerate(dl_planes(L, beta)):
        dl[l, L - 1 - l:L + l, L - 1 - l:L + l] = P
    return dl


def rotate_flms(flm, L, rotation, dl_array=None):
    """rotation.py:9-64: flm'[l, m] = e^{-i m alpha} sum_n d^l_{m,n}(beta) e^{-i n gamma} flm[l, n]."""
    alpha, beta, gamma = rotation
    ea = np.exp(-1j * np.arange(-L + 1, L) * alpha)
    eg = np.exp(-1j * np.arange(-L + 1, L) * gamma)
    dl = dl_array if dl_array is not None else generate_rotate_dls(L, beta)
    return np.einsum("lmn,m,n,ln->lm", dl, ea, eg, flm)
