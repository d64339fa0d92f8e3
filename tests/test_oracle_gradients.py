"""The gradient oracle (oracle.gradients) pinned on the CPU.

oracle.gradients restates upstream's differentiation of the spin transforms:
its two custom VJP rules for the latitudinal steps (s2fft/transforms/
spherical.py:291-325, 695-730) with the conjugate transposes of the stages
around them, in torch's gradient convention (s2fft/utils/torch_wrapper.py:
219-228). Here it is checked against (i) the exact vector-Jacobian product of
the whole float64 transform, formed column by column, and (ii) central finite
differences of the loss used by upstream's gradient tests
(tests/test_spherical_custom_grads.py: sum |T(x) - target|^2), for every
sampling, spins -2, 0, 1 and reality (spin 0, as upstream tests it).
"""

import numpy as np
import pytest

import oracle
from oracle import gradients as G

CASES = [(s, spin, reality) for s in ("mw", "mwss", "dh", "gl", "healpix")
         for spin in (-2, 0, 1) for reality in (False, True) if not (reality and spin != 0)]


def _kw(sampling, spin, reality, L=8, L_lower=2):
    nside = 4 if sampling == "healpix" else None
    return dict(L=L, spin=spin, nside=nside, sampling=sampling, reality=reality,
                L_lower=L_lower)


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("sampling,spin,reality", CASES)
def test_inverse_vjp_is_the_exact_gradient(rng, sampling, spin, reality):
    kw = _kw(sampling, spin, reality)
    flm = oracle.signal.generate_flm(rng, kw["L"], kw["L_lower"], spin, reality)
    f_t = oracle.spherical.inverse(
        oracle.signal.generate_flm(rng, kw["L"], kw["L_lower"], spin, reality), **kw)
    g_f = 2 * (oracle.spherical.inverse(flm, **kw) - f_t)  # gradient of sum |f - f_t|^2
    got = G.inverse_vjp(g_f, **kw)
    exact = G.linear_vjp(lambda x: oracle.spherical.inverse(x, **kw), flm, g_f)
    assert _rel(got, exact) < 1e-10


@pytest.mark.parametrize("sampling,spin,reality", CASES)
def test_forward_vjp_is_the_exact_gradient(rng, sampling, spin, reality):
    kw = _kw(sampling, spin, reality)
    L = kw["L"]
    f = oracle.spherical.inverse(oracle.signal.generate_flm(rng, L, kw["L_lower"], spin,
                                                            reality), **kw)
    f = (np.real(f) + 0.1 * rng.standard_normal(f.shape) if reality else
         f + 0.1 * oracle.signal.complex_normal(rng, f.shape))
    flm_t = oracle.signal.generate_flm(rng, L, kw["L_lower"], spin, reality)
    g = 2 * (oracle.spherical.forward(f, **kw) - flm_t)
    got = G.forward_vjp(g, **kw)
    exact = G.linear_vjp(lambda x: oracle.spherical.forward(x, **kw), f, g)
    assert _rel(got, exact) < 1e-10


@pytest.mark.parametrize("sampling,spin,reality", [("mw", 0, False), ("gl", -2, False),
                                                   ("mwss", 0, True), ("healpix", 0, True)])
def test_gradients_match_central_differences(rng, sampling, spin, reality):
    kw = _kw(sampling, spin, reality)
    L = kw["L"]
    flm = oracle.signal.generate_flm(rng, L, kw["L_lower"], spin, reality)
    f_t = oracle.spherical.inverse(oracle.signal.generate_flm(rng, L, kw["L_lower"], spin,
                                                              reality), **kw)
    grad = G.inverse_vjp(2 * (oracle.spherical.inverse(flm, **kw) - f_t), **kw)
    h = 1e-5
    for _ in range(6):
        l = int(rng.integers(max(kw["L_lower"], abs(spin)), L))
        m = int(rng.integers(0 if reality else -l, l + 1))
        for part in (1.0, 1j):
            e = np.zeros_like(flm)
            e[l, L - 1 + m] = part * h
            fd = (G.loss_inverse(flm + e, f_t, **kw) - G.loss_inverse(flm - e, f_t, **kw)) / (2 * h)
            an = grad[l, L - 1 + m].real if part == 1.0 else grad[l, L - 1 + m].imag
            assert abs(fd - an) <= 1e-6 * max(1.0, abs(an)), (l, m, part, fd, an)
    # forward transform, gradient w.r.t. the map, with refinement iterations on healpix
    iters = 2 if sampling == "healpix" else 0
    f = oracle.spherical.inverse(flm, **kw)
    if reality:
        f = np.real(f)
    flm_t = oracle.signal.generate_flm(rng, L, kw["L_lower"], spin, reality)
    g = 2 * (oracle.spherical.forward(f, iter=iters, **kw) - flm_t)
    gf = G.forward_vjp(g, iter=iters, **kw)
    for _ in range(6):
        idx = tuple(int(rng.integers(n)) for n in f.shape)
        for part in ((1.0,) if reality else (1.0, 1j)):
            e = np.zeros_like(f)
            e[idx] = part * h
            fd = (G.loss_forward(f + e, flm_t, iter=iters, **kw)
                  - G.loss_forward(f - e, flm_t, iter=iters, **kw)) / (2 * h)
            an = gf[idx].real if part == 1.0 else gf[idx].imag
            assert abs(fd - an) <= 1e-6 * max(1.0, abs(an)), (idx, part, fd, an)
