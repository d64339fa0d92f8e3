"""Fourier-Wigner SO(3) transforms and the spin-subset lifting ops (float64, numpy).

TEST INFRASTRUCTURE ONLY (see the package docstring).

Restates
  s2fft/precompute_transforms/fourier_wigner.py:13-88   inverse_transform (precomps path)
  s2fft/precompute_transforms/fourier_wigner.py:177-333 forward_transform (precomps path)
  s2fft/precompute_transforms/construct.py:614-639      fourier_wigner_kernel
  s2fft/precompute_transforms/custom_ops.py:5-83        wigner_subset_to_s2
  s2fft/precompute_transforms/custom_ops.py:168-205     so3_to_wigner_subset
  s2fft/precompute_transforms/custom_ops.py:251-333     s2_to_wigner_subset

The transforms factor through the planes Delta^l = d^l(pi/2) (Risbo's recursion,
``rotation.generate_rotate_dls``): with c_l = (2l+1)/(8 pi^2),

  inverse  Y_n[a, m] = i^(n-m) e^{i a theta0} sum_l c_l Delta^l_{a,m} Delta^l_{a,n} flmn[n,l,m],
           then a DFT over a (beta, keep the sampled rings) and over m (alpha);
  forward  alpha DFT, periodic extension of beta to [0, 2pi) with the sign
           (-1)^(|m|+|n|), beta DFT, the quadrature applied as a product in the
           4L-3 upsampled beta domain, then
           flmn[n,l,m] = (2 pi)^2 i^(m-n) sum_b G_n[b, m] Delta^l_{b,m} Delta^l_{b,n}.

Frequency indices are stored "value mod length" (what fftshift / ifftshift do
upstream); i^k is taken from an exact table.
"""

import numpy as np

from . import quadrature, rotation

_IPOW = np.array([1.0, 1.0j, -1.0, -1.0j])


def _ipow(k):
    return _IPOW[np.mod(k, 4)]


def _geometry(L, sampling):
    s = sampling.lower()
    if s not in ("mw", "mwss"):
        raise ValueError(f"Fourier-Wigner algorithm does not support {sampling} sampling.")
    mwss = s == "mwss"
    ntheta = L + 1 if mwss else L
    nphi = 2 * L if mwss else 2 * L - 1
    theta0 = 0.0 if mwss else np.pi / (2 * L - 1)
    return mwss, ntheta, nphi, theta0


def upsampled_quads(L):
    """construct.py:629-634: the MW weights w(-mm), |mm| <= 2L-2, summed on 4L-3 points."""
    P = 4 * L - 3
    W = np.zeros(P, dtype=np.complex128)
    for mm in range(-2 * (L - 1), 2 * (L - 1) + 1):
        W[mm % P] = quadrature._mw_weight(-mm)
    return np.fft.ifft(W) * P


def fourier_wigner_kernel(L):
    """construct.py:614-639: (Delta [L, 2L-1, 2L-1] at beta = pi/2, quads [4L-3])."""
    return rotation.generate_rotate_dls(L, np.pi / 2), upsampled_quads(L)


def inverse_core(F, nvals, delta, L, sampling="mw"):
    """Spin slices F[e] ([E, L, 2L-1], slice e has azimuthal index n = nvals[e]) to
    sphere maps [E, ntheta, nphi] (fourier_wigner.py:59-87 without the gamma DFT;
    custom_ops.py:57-83)."""
    mwss, ntheta, nphi, theta0 = _geometry(L, sampling)
    v = np.arange(-(L - 1), L)
    c = (2 * np.arange(L) + 1) / (8 * np.pi ** 2)
    out = np.zeros((len(nvals), ntheta, nphi), dtype=np.complex128)
    for e, n in enumerate(nvals):
        Y = np.einsum("l,lam,la,lm->am", c, delta, delta[:, :, L - 1 + n], F[e])
        Y = Y * _ipow(n - v)[None, :] * np.exp(1j * v * theta0)[:, None]
        X = np.zeros((nphi, nphi), dtype=np.complex128)
        X[np.ix_(v % nphi, v % nphi)] = Y
        T = (np.fft.ifft(X, axis=0) * nphi)[:ntheta]
        out[e] = np.fft.ifft(T, axis=1) * nphi
    return out


def forward_core(fs, nvals, delta, quads, L, sampling="mw"):
    """Sphere maps fs[e] ([E, ntheta, nphi]) to spin slices [E, L, 2L-1] with azimuthal
    index n = nvals[e] (fourier_wigner.py:239-316 after the gamma DFT;
    custom_ops.py:281-333)."""
    mwss, ntheta, nphi, _ = _geometry(L, sampling)
    v = np.arange(-(L - 1), L)
    P = 4 * L - 3
    nx = ntheta + L - 1  # periodically extended beta samples: 2L-1 (mw) or 2L (mwss)
    bvals = np.arange(-L, L) if mwss else v
    out = np.zeros((len(nvals), L, 2 * L - 1), dtype=np.complex128)
    for e, n in enumerate(nvals):
        S = (np.fft.fft(fs[e], axis=1) / nphi)[:, v % nphi]  # [t, m]
        sgn = np.where((np.abs(v) + abs(n)) % 2 == 1, -1.0, 1.0)
        ext = np.concatenate((S, (S[::-1] * sgn[None, :])[1:L]), axis=0)
        Bh = np.fft.fft(ext, axis=0) / nx
        B = Bh[bvals % nx]
        if not mwss:
            B = B * np.exp(-1j * bvals * np.pi / (2 * L - 1))[:, None]
        U = np.zeros((P, 2 * L - 1), dtype=np.complex128)
        U[bvals % P] = B
        u = np.fft.ifft(U, axis=0) * P * quads[:, None]
        G = (np.fft.fft(u, axis=0) / P)[v % P]  # [b, m]
        H = np.einsum("bm,lbm,lb->lm", G, delta, delta[:, :, L - 1 + n])
        out[e] = H * _ipow(v - n)[None, :] * (2 * np.pi) ** 2
    return out


def inverse_transform(flmn, L, N, precomps=None, reality=False, sampling="mw"):
    """fourier_wigner.py:13-88: flmn [2N-1, L, 2L-1] -> f [2N-1, ntheta, nphi]."""
    delta = (precomps if precomps is not None else fourier_wigner_kernel(L))[0]
    nvals = np.arange(0 if reality else -(N - 1), N)
    maps = inverse_core(flmn[N - 1 + nvals], nvals, delta, L, sampling)
    G = 2 * N - 1
    if reality:
        return np.fft.irfft(maps, G, axis=0) * G
    X = np.zeros((G,) + maps.shape[1:], dtype=np.complex128)
    X[nvals % G] = maps
    return np.fft.ifft(X, axis=0) * G


def forward_transform(f, L, N, precomps=None, reality=False, sampling="mw"):
    """fourier_wigner.py:177-333: f [2N-1, ntheta, nphi] -> flmn [2N-1, L, 2L-1]."""
    delta, quads = precomps if precomps is not None else fourier_wigner_kernel(L)
    G = 2 * N - 1
    if reality:
        nvals = np.arange(0, N)
        fs = np.fft.rfft(np.real(f), axis=0) / G
    else:
        nvals = np.arange(-(N - 1), N)
        fs = (np.fft.fft(f, axis=0) / G)[nvals % G]
    x = forward_core(fs, nvals, delta, quads, L, sampling)
    out = np.zeros((G, L, 2 * L - 1), dtype=np.complex128)
    out[N - 1 + nvals] = x
    if reality:
        v = np.arange(-(L - 1), L)
        for n in range(1, N):
            sgn = np.where((np.abs(v) + n) % 2 == 1, -1.0, 1.0)
            out[N - 1 - n] = np.conj(out[N - 1 + n][:, ::-1]) * sgn[None, :]
    return out


def _channels_first(x):
    # [batch, s, ..., channels] -> [batch, channels, s, ...]
    return np.moveaxis(x, -1, 1)


def _channels_last(x):
    return np.moveaxis(x, 1, -1)


def wigner_subset_to_s2(flmn, spins, DW, L, sampling="mw"):
    """custom_ops.py:5-83: flmn [batch, n_s, L, 2L-1, ch] -> [batch, n_s, ntheta, nphi, ch]."""
    _geometry(L, sampling)
    spins = np.asarray(spins)
    if flmn.shape[1] != spins.shape[0]:
        raise ValueError(
            f"Number of spins specified {spins.shape[0]} does not match the number of "
            f"Wigner coefficients {flmn.shape[1]}")
    x = _channels_first(flmn)
    Bt, C, S = x.shape[:3]
    nv = np.tile(-spins, Bt * C)
    maps = inverse_core(x.reshape((-1,) + x.shape[3:]), nv, DW[0], L, sampling)
    return _channels_last(maps.reshape((Bt, C, S) + maps.shape[1:]))


def s2_to_wigner_subset(fs, spins, DW, L, sampling="mw"):
    """custom_ops.py:251-333: fs [batch, n_s, ntheta, nphi, ch] -> [batch, n_s, L, 2L-1, ch]."""
    _geometry(L, sampling)
    spins = np.asarray(spins)
    x = _channels_first(fs)
    Bt, C, S = x.shape[:3]
    nv = np.tile(-spins, Bt * C)
    out = forward_core(x.reshape((-1,) + x.shape[3:]), nv, DW[0], DW[1], L, sampling)
    return _channels_last(out.reshape((Bt, C, S) + out.shape[1:]))


def so3_to_wigner_subset(f, spins, DW, L, N, sampling="mw"):
    """custom_ops.py:168-205: DFT over gamma at the requested spins, then
    s2_to_wigner_subset. f [batch, n_gamma, ntheta, nphi, ch]."""
    spins = np.asarray(spins)
    G = f.shape[1]
    e = np.exp(2j * np.pi * np.outer(np.arange(G), spins) / G)  # exp(-2 pi i g (-s) / G)
    x = np.einsum("bgtpc,gn->bntpc", f, e) / G
    return s2_to_wigner_subset(x, spins, DW, L, sampling)
