"""Gradients through the adjoint kernels (s2b_inverse_adjoint / s2b_forward_adjoint).

For a complex-linear map y = A x, torch's backward returns A^H applied to the
gradient of y; the adjoint kernels implement A^H directly (the d-recursion is
recomputed, never stored). Checked three ways:
  * dot-product identities <A x, y> = <x, A^H y> for every sampling and spins 0, 2, -1;
  * central finite differences of a real loss on 32 random coefficients
    (S2: MW L=1024 spin 0, loss ||inverse(flm) - g||^2;
     SO(3): MW L=128 N=8, loss ||forward(inverse(flmn)) - target||^2);
  * the float32 gradients against the float64 ones.
The loss is quadratic in the coefficients, so a central difference with step 1 is
exact up to rounding. Upstream's JAX gradients cannot run here (JAX is absent).
"""

import numpy as np
import pytest

import oracle
from tests.conftest import relerr

pytestmark = pytest.mark.gpu

TOL = {"f64": 1e-10, "f32": 1e-5}


@pytest.fixture(scope="module")
def s2b():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import s2fft_b200

    return s2fft_b200


def _vdot(a, b):
    return complex((a.conj() * b).sum().item())


@pytest.mark.parametrize("precision", ["f64", "f32"])
@pytest.mark.parametrize("sampling", ["mw", "mwss", "dh", "gl", "healpix"])
@pytest.mark.parametrize("spin", [0, 2, -1])
def test_adjoint_dot_products(s2b, rng, sampling, spin, precision):
    import torch

    L, nside = (16, 8) if sampling == "healpix" else (24, None)
    cdt = torch.complex128 if precision == "f64" else torch.complex64
    shape = s2b.f_shape(L, sampling, nside)
    x = torch.tensor(oracle.signal.generate_flm(rng, L, 0, spin), dtype=cdt, device="cuda",
                     requires_grad=True)
    y = torch.tensor(rng.normal(size=shape) + 1j * rng.normal(size=shape), dtype=cdt,
                     device="cuda")
    f = s2b.inverse(x, L, spin, nside, sampling, precision=precision)
    (gx,) = torch.autograd.grad(f, x, grad_outputs=y)
    lhs, rhs = _vdot(f.detach(), y), _vdot(x.detach(), gx)
    assert abs(lhs - rhs) <= TOL[precision] * max(abs(lhs), 1e-30) * 10, (lhs, rhs)

    fin = torch.tensor(rng.normal(size=shape) + 1j * rng.normal(size=shape), dtype=cdt,
                       device="cuda", requires_grad=True)
    h = torch.tensor(oracle.signal.generate_flm(rng, L, 0, spin), dtype=cdt, device="cuda")
    flm = s2b.forward(fin, L, spin, nside, sampling, precision=precision)
    (gf,) = torch.autograd.grad(flm, fin, grad_outputs=h)
    lhs, rhs = _vdot(flm.detach(), h), _vdot(fin.detach(), gf)
    assert abs(lhs - rhs) <= TOL[precision] * max(abs(lhs), 1e-30) * 10, (lhs, rhs)


@pytest.mark.parametrize("sampling", ["mw", "dh"])
@pytest.mark.parametrize("spin", [-7, 6])
def test_adjoint_dot_products_high_spin(s2b, rng, sampling, spin):
    """The adjoints at L=256 and |spin| > 4, where orders m < |spin| run on the degree
    recursion (both directions and both halves)."""
    import torch

    L = 256
    shape = s2b.f_shape(L, sampling)
    x = torch.tensor(oracle.signal.generate_flm(rng, L, 0, spin), device="cuda",
                     requires_grad=True)
    y = torch.tensor(rng.normal(size=shape) + 1j * rng.normal(size=shape), device="cuda")
    f = s2b.inverse(x, L, spin, None, sampling)
    (gx,) = torch.autograd.grad(f, x, grad_outputs=y)
    lhs, rhs = _vdot(f.detach(), y), _vdot(x.detach(), gx)
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs), (lhs, rhs)
    fin = torch.tensor(rng.normal(size=shape) + 1j * rng.normal(size=shape), device="cuda",
                       requires_grad=True)
    h = torch.tensor(oracle.signal.generate_flm(rng, L, 0, spin), device="cuda")
    flm = s2b.forward(fin, L, spin, None, sampling)
    (gf,) = torch.autograd.grad(flm, fin, grad_outputs=h)
    lhs, rhs = _vdot(flm.detach(), h), _vdot(fin.detach(), gf)
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs), (lhs, rhs)


def _fd_check(loss_fn, x, grad, coords, tol):
    """Central differences on the real and imaginary part of each coordinate."""
    import torch

    worst = 0.0
    scale = float(grad.abs().max())
    for c in coords:
        for unit in (1.0, 1j):
            e = torch.zeros_like(x)
            e[c] = unit
            with torch.no_grad():
                d = (loss_fn(x + e) - loss_fn(x - e)) / 2.0
            g = grad[c].real if unit == 1.0 else grad[c].imag
            worst = max(worst, abs(float(d) - float(g)) / scale)
    assert worst < tol, worst
    return worst


def _valid_coords(rng, L, n, lmin=0):
    out = []
    while len(out) < n:
        l = int(rng.integers(lmin, L))
        m = int(rng.integers(-l, l + 1))
        out.append((l, L - 1 + m))
    return out


def test_fd_inverse_mw_L1024(s2b, rng):
    """S2: MW L=1024 spin 0, loss = ||inverse(flm) - g||^2."""
    import torch

    L = 1024
    flm0 = oracle.signal.generate_flm_full_complex(rng, L)
    g = rng.normal(size=(L, 2 * L - 1)) + 1j * rng.normal(size=(L, 2 * L - 1))
    grads = {}
    for prec, cdt in (("f64", torch.complex128), ("f32", torch.complex64)):
        x = torch.tensor(flm0, dtype=cdt, device="cuda", requires_grad=True)
        gt = torch.tensor(g, dtype=cdt, device="cuda")

        def loss(z):
            return (s2b.inverse(z, L, precision=prec) - gt).abs().pow(2).sum()

        (gx,) = torch.autograd.grad(loss(x), x)
        grads[prec] = gx.to(torch.complex128)
        if prec == "f64":
            _fd_check(loss, x.detach(), gx, [tuple(c) for c in _valid_coords(rng, L, 32)], 1e-9)
    err = relerr(grads["f32"].cpu().numpy(), grads["f64"].cpu().numpy())
    assert err < 1e-5, err


def test_fd_wigner_L128_N8(s2b, rng):
    """SO(3): MW L=128 N=8, loss = ||forward(inverse(flmn)) - target||^2."""
    import torch

    L, N = 128, 8
    flmn0 = oracle.signal.generate_flmn(rng, L, N)
    target = oracle.signal.generate_flmn(rng, L, N)
    grads = {}
    for prec, cdt in (("f64", torch.complex128), ("f32", torch.complex64)):
        x = torch.tensor(flmn0, dtype=cdt, device="cuda", requires_grad=True)
        tt = torch.tensor(target, dtype=cdt, device="cuda")

        def loss(z):
            f = s2b.wigner.inverse(z, L, N, precision=prec)
            return (s2b.wigner.forward(f, L, N, precision=prec) - tt).abs().pow(2).sum()

        (gx,) = torch.autograd.grad(loss(x), x)
        grads[prec] = gx.to(torch.complex128)
        if prec == "f64":
            coords = []
            while len(coords) < 32:
                n = int(rng.integers(-(N - 1), N))
                l = int(rng.integers(abs(n), L))
                m = int(rng.integers(-l, l + 1))
                coords.append((N - 1 + n, l, L - 1 + m))
            _fd_check(loss, x.detach(), gx, coords, 1e-9)
    err = relerr(grads["f32"].cpu().numpy(), grads["f64"].cpu().numpy())
    assert err < 1e-5, err


def test_composed_wigner_matches_cabi(s2b, rng):
    """The differentiable Wigner composition gives the C-ABI transform's values."""
    import torch

    L, N = 32, 4
    flmn = oracle.signal.generate_flmn(rng, L, N)
    ref = s2b.wigner.inverse(flmn, L, N)
    x = torch.tensor(flmn, device="cuda", requires_grad=True)
    f = s2b.wigner.inverse(x, L, N)
    assert relerr(f.detach().cpu().numpy(), ref) < 1e-12
    g = s2b.wigner.forward(f, L, N)
    assert relerr(g.detach().cpu().numpy(), flmn) < 1e-10


def test_refinement_gradient_is_adjoint(s2b, rng):
    """HEALPix forward with iter=2: <F_iter f, h> = <f, F_iter^H h> through autograd."""
    import torch

    L, nside = 16, 8
    npix = 12 * nside * nside
    fin = torch.tensor(rng.normal(size=npix) + 1j * rng.normal(size=npix), device="cuda",
                       requires_grad=True)
    h = torch.tensor(oracle.signal.generate_flm(rng, L, 0, 0), device="cuda")
    flm = s2b.forward(fin, L, 0, nside, "healpix", iter=2)
    ref = s2b.forward(fin.detach(), L, 0, nside, "healpix", iter=2)
    assert relerr(flm.detach().cpu().numpy(), ref.cpu().numpy()) < 1e-12
    (gf,) = torch.autograd.grad(flm, fin, grad_outputs=h)
    lhs, rhs = _vdot(flm.detach(), h), _vdot(fin.detach(), gf)
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs), (lhs, rhs)


@pytest.mark.parametrize("precision", ["f64", "f32"])
@pytest.mark.parametrize("sampling", ["mw", "mwss", "dh", "gl", "healpix"])
@pytest.mark.parametrize("spin", [0, -2])
def test_precompute_adjoint_dot_products(s2b, rng, sampling, spin, precision):
    """Precompute transforms (kernel tables) through s2b_precompute_inverse_adjoint /
    s2b_precompute_forward_adjoint: <A x, y> = <x, A^H y> for a batch of 3 maps (small
    batches use the register-tiled contraction) and of 20 maps (the shared-memory one)."""
    import torch

    L, nside = (16, 8) if sampling == "healpix" else (20, None)
    cdt = torch.complex128 if precision == "f64" else torch.complex64
    shape = s2b.f_shape(L, sampling, nside)
    kin = s2b.precompute.spin_spherical_kernel(L, spin, False, sampling, nside, False,
                                               precision=precision)
    kfw = s2b.precompute.spin_spherical_kernel(L, spin, False, sampling, nside, True,
                                               precision=precision)
    for B in (3, 20):
        x = torch.tensor(np.stack([oracle.signal.generate_flm(rng, L, 0, spin) for _ in range(B)]),
                         dtype=cdt, device="cuda", requires_grad=True)
        y = torch.tensor(rng.normal(size=(B,) + shape) + 1j * rng.normal(size=(B,) + shape),
                         dtype=cdt, device="cuda")
        f = s2b.precompute.inverse(x, L, spin, kin, sampling, nside=nside, precision=precision)
        (gx,) = torch.autograd.grad(f, x, grad_outputs=y)
        lhs, rhs = _vdot(f.detach(), y), _vdot(x.detach(), gx)
        assert abs(lhs - rhs) <= TOL[precision] * max(abs(lhs), 1e-30) * 10, (B, lhs, rhs)

        fin = torch.tensor(rng.normal(size=(B,) + shape) + 1j * rng.normal(size=(B,) + shape),
                           dtype=cdt, device="cuda", requires_grad=True)
        h = torch.tensor(np.stack([oracle.signal.generate_flm(rng, L, 0, spin) for _ in range(B)]),
                         dtype=cdt, device="cuda")
        flm = s2b.precompute.forward(fin, L, spin, kfw, sampling, nside=nside,
                                     precision=precision)
        (gf,) = torch.autograd.grad(flm, fin, grad_outputs=h)
        lhs, rhs = _vdot(flm.detach(), h), _vdot(fin.detach(), gf)
        assert abs(lhs - rhs) <= TOL[precision] * max(abs(lhs), 1e-30) * 10, (B, lhs, rhs)


def test_precompute_gradient_matches_otf(s2b, rng):
    """The precompute inverse's gradient equals the on-the-fly transform's (same map)."""
    import torch

    L = 24
    x = torch.tensor(oracle.signal.generate_flm(rng, L, 0, 1), device="cuda",
                     requires_grad=True)
    g = torch.tensor(rng.normal(size=(L, 2 * L - 1)), device="cuda")
    loss = (s2b.precompute.inverse(x, L, 1, None, "gl").real - g).pow(2).sum()
    (g1,) = torch.autograd.grad(loss, x)
    x2 = x.detach().clone().requires_grad_(True)
    loss2 = (s2b.inverse(x2, L, 1, None, "gl").real - g).pow(2).sum()
    (g2,) = torch.autograd.grad(loss2, x2)
    assert relerr(g1.cpu().numpy(), g2.cpu().numpy()) < 1e-10
