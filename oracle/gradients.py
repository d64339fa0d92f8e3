"""Gradients of the spin transforms as upstream computes them (float64).

TEST INFRASTRUCTURE ONLY (see the package docstring).

Upstream differentiates its transforms with two custom VJP rules and JAX's
autodiff for everything around them:

* inverse: the latitudinal step's cotangent map is the forward latitudinal
  step applied to the ring-spectrum cotangent, without quadrature weights
  (``flm_to_ftm`` in s2fft/transforms/spherical.py:291-325);
* forward: the latitudinal step's cotangent map is the inverse latitudinal
  step applied to the coefficient cotangent (``ftm_to_flm``,
  spherical.py:695-730).

Its torch wrapper conjugates cotangents on the way into and out of ``jax.vjp``
(s2fft/utils/torch_wrapper.py:219-228), so the gradient a torch caller sees for
a real loss is the conjugate transpose A^H g of each complex-linear stage (for
the real-coefficient latitudinal steps, A^H = A^T: exactly the two rules
above). This module restates that chain in torch's convention: the latitudinal
steps by the two rules (``oracle.recursion``), the pole rows, ring phases,
signs, normalisation and the real-signal mirror by their conjugate transposes
written out, and the stages that JAX differentiates as plain linear code (ring
FFTs, HEALPix ring FFTs, the MW -> MWSS resampling) by the exact
vector-Jacobian product of this package's restatement of them
(``linear_vjp``).

Convention: for a real loss L and an array x, the gradient is
dL/dRe(x) + i dL/dIm(x) (complex x) or dL/dx (real x), as torch reports it.
"""

import numpy as np

from . import healpix, quadrature, recursion, resampling, samples
from .spherical import _norm, forward, inverse


def linear_vjp(fn, x, g):
    """Gradient with respect to x of the real loss whose gradient with respect to
    y = fn(x) is g, for an R-linear fn: over the 2n real directions e of x, the
    derivative Re(<g, fn(e)>). Exact to rounding; 2n calls of fn (n = x.size), so for
    small cases only. This is what JAX's autodiff returns for linear numpy code."""
    x = np.asarray(x)
    g = np.asarray(g)
    cplx = np.iscomplexobj(x)
    out = np.zeros(x.shape, dtype=np.complex128 if cplx else np.float64)
    flat = out.reshape(-1)
    e = np.zeros(x.shape, dtype=np.complex128 if cplx else np.float64)
    ef = e.reshape(-1)
    for k in range(ef.size):
        for part in ((1.0, 1j) if cplx else (1.0,)):
            ef[k] = part
            d = np.real(np.vdot(g, np.asarray(fn(e))))  # Re(sum conj(g) y)
            ef[k] = 0
            flat[k] += d if part == 1.0 else 1j * d
    return out


def inverse_vjp(g_f, L, spin=0, nside=None, sampling="mw", reality=False, L_lower=0):
    """Gradient w.r.t. flm of a real loss with gradient g_f w.r.t. f = inverse(flm).

    Reverse of oracle.spherical.inverse (upstream spherical.py:112-208 and the
    JAX version 211-346 with its custom VJP 291-325)."""
    sampling = sampling.lower()
    th = samples.thetas(L, sampling, nside)
    mo = 1 if sampling in ("mwss", "healpix") else 0
    m0 = L - 1 if reality else 0
    nth, ncol = samples.ftm_shape(L, sampling, nside)

    # longitudinal stage (JAX autodiff of the ring IFFTs): exact VJP of the restated code
    def post(ftm):
        ftm = np.array(ftm, dtype=np.complex128)
        if sampling == "healpix":
            if reality:
                ftm[:, mo:L - 1 + mo] = np.flip(np.conj(ftm[:, L - 1 + mo + 1:]), axis=-1)
            return healpix.healpix_ifft(ftm, L, nside, reality)
        if reality:
            return np.fft.irfft(ftm[:, L - 1 + mo:], samples.nphi_equiang(L, sampling),
                                axis=1, norm="forward")
        return np.fft.ifft(np.fft.ifftshift(ftm, axes=1), axis=1, norm="forward")

    gt = linear_vjp(post, np.zeros((nth, ncol), np.complex128), g_f)
    gt = gt * (-1) ** spin
    if sampling == "healpix":
        gt[:, m0 + mo:] *= np.conj(healpix.ring_phase_shifts_hp(L, nside, False, reality))
    glm = np.zeros((L, 2 * L - 1), dtype=np.complex128)
    el = np.arange(L_lower, L)
    if sampling in ("mw", "mwss"):  # ftm[-1] = 0; ftm[-1, L-1+s+mo] = sum (-1)^|l-s| flm
        glm[L_lower:, L - 1 + spin] += (-1.0) ** np.abs(el - spin) * gt[-1, L - 1 + spin + mo]
        gt[-1] = 0
    if sampling == "mwss":  # ftm[0] = 0; ftm[0, L-1-s+mo] = sum flm[l, L-1-s]
        glm[L_lower:, L - 1 - spin] += gt[0, L - 1 - spin + mo]
        gt[0] = 0
    # upstream's custom VJP of the latitudinal step: the forward step, no weights
    glm += recursion.forward_latitudinal_step(gt, th, L, spin, sampling, reality, None, L_lower)
    glm[:L_lower] = 0
    glm[L_lower:] *= _norm(L, L_lower)[:, None]
    return glm


def _forward_once_vjp(g_flm, L, spin, nside, sampling, reality, L_lower):
    """Reverse of oracle.spherical._forward_once (upstream spherical.py:467-588, JAX
    591-755 with its custom VJP 695-730)."""
    sampling0 = sampling.lower()
    mo = 1 if sampling0 in ("mwss", "mw", "healpix") else 0
    m0 = L - 1 if reality else 0
    g = np.array(g_flm, dtype=np.complex128) * (-1) ** spin
    g[: max(abs(spin), L_lower)] = 0
    if reality:  # flm[:, :m0] = flip(mc conj(flm[:, m0 + 1:])) overwrote the m < 0 half
        mc = (-1.0) ** (np.arange(1, L) % 2)
        g[:, m0 + 1:] += mc * np.conj(np.flip(g[:, :m0], axis=-1))
        g[:, :m0] = 0
    g[:L_lower] = 0
    g[L_lower:] *= _norm(L, L_lower)[:, None]
    if sampling0 in ("mw", "mwss"):
        sam = "mwss"
        th = samples.thetas(2 * L, sam)
        nth, ncol = 2 * L + 1, 2 * L
    else:
        sam = sampling0
        th = samples.thetas(L, sam, nside)
        nth, ncol = samples.ftm_shape(L, sam, nside)
    gt = np.zeros((nth, ncol), dtype=np.complex128)
    el = np.arange(L_lower, L)
    if sam == "mwss":
        # flm[l, L-1+s] += (-1)^|l-s| ftm[-1, L-1+s+mo]; flm[l, L-1-s] += ftm[0, L-1-s+mo]
        gt[-1, L - 1 + spin + mo] += np.sum((-1.0) ** np.abs(el - spin) * g[L_lower:, L - 1 + spin])
        gt[0, L - 1 - spin + mo] += np.sum(g[L_lower:, L - 1 - spin])
        # upstream's custom VJP of the latitudinal step: the inverse step
        gt[1:-1] += recursion.inverse_latitudinal_step(g, th[1:-1], L, spin, sam, reality,
                                                       None, L_lower, None, nside)
    else:
        gt += recursion.inverse_latitudinal_step(g, th, L, spin, sam, reality, None, L_lower,
                                                 None, nside)
    if sam == "healpix":
        gt[:, m0 + mo:] *= np.conj(healpix.ring_phase_shifts_hp(L, nside, True, reality))
    gt *= quadrature.quad_weights_transform(L, sam, 0, nside)[:, None]

    # resampling and ring FFTs (JAX autodiff): exact VJP of the restated code
    def pre(f):
        if sampling0 == "mw":
            f = resampling.mw_to_mwss(f, L, spin)
        if sampling0 in ("mw", "mwss"):
            f = resampling.upsample_by_two_mwss(f, L, spin)
        if sam == "healpix":
            return healpix.healpix_fft(f, L, nside, reality)
        if reality:
            t = np.fft.rfft(np.real(f), axis=1, norm="backward")
            if mo:
                t = t[:, :-1]
            ftm = np.zeros(np.shape(f), dtype=np.complex128)
            ftm[:, L - 1 + mo:] = t
            return ftm
        return np.fft.fftshift(np.fft.fft(f, axis=1, norm="backward"), axes=1)

    fshape = samples.f_shape(L, sampling0, nside)
    x0 = np.zeros(fshape, dtype=np.float64 if reality else np.complex128)
    return linear_vjp(pre, x0, gt)


def forward_vjp(g_flm, L, spin=0, nside=None, sampling="mw", reality=False, L_lower=0,
                iter=0):
    """Gradient w.r.t. f of a real loss with gradient g_flm w.r.t. flm = forward(f, iter).

    The refinement flm_{k+1} = flm_k + F(f - I(flm_k)) (upstream
    s2fft/utils/iterative_refinement.py:9-46) is reversed step by step."""
    kw = dict(L=L, spin=spin, nside=nside, sampling=sampling, reality=reality,
              L_lower=L_lower)
    gy = np.array(g_flm, dtype=np.complex128)
    gf = 0
    for _ in range(iter or 0):
        gr = _forward_once_vjp(gy, **kw)
        gf = gf + gr
        gy = gy - inverse_vjp(gr, **kw)
    return gf + _forward_once_vjp(gy, **kw)


def loss_inverse(flm, f_target, **kw):
    """sum |inverse(flm) - f_target|^2 (the loss of upstream's gradient tests)."""
    return float(np.sum(np.abs(inverse(flm, **kw) - f_target) ** 2))


def loss_forward(f, flm_target, **kw):
    """sum |forward(f) - flm_target|^2."""
    return float(np.sum(np.abs(forward(f, **kw) - flm_target) ** 2))
