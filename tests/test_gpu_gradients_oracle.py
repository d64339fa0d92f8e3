"""Device gradients against upstream's own gradient rules (oracle.gradients).

The cases follow upstream's gradient tests (tests/test_spherical_custom_grads.py):
L = 16, L_lower = 2, spins -2, 0, 1, samplings mw, mwss, dh, gl (plus healpix,
nside 8, here), reality for spin 0, loss sum |T(x) - target|^2. torch's backward
through s2fft_b200 (the adjoint kernels; real signals through the exact
complex rewrites described in s2fft_b200.spherical) is compared with the float64
restatement of upstream's custom-VJP chain, itself pinned to exact
vector-Jacobian products and finite differences on the CPU
(tests/test_oracle_gradients.py). Tolerances relative to the largest gradient
entry: 1e-10 for float64, 1e-5 for float32. The forward transforms are
differentiated at maps that are not band-limited (band-limited part plus noise).
"""

import numpy as np
import pytest

import oracle
from oracle import gradients as G
from tests.conftest import relerr

pytestmark = pytest.mark.gpu

TOL = {"f64": 1e-10, "f32": 1e-5}
# HEALPix with spin != 0 is left out: there upstream's log-renormalised recursion drops
# terms at exact zeros of d on HEALPix's rational rings (the device is held to exact
# values instead, tests/test_gpu_spherical.py::test_healpix_spin_exact)
CASES = [(s, spin, reality) for s in ("mw", "mwss", "dh", "gl", "healpix")
         for spin in (-2, 0, 1) for reality in (False, True)
         if not (reality and spin != 0) and not (s == "healpix" and spin != 0)]


@pytest.fixture(scope="module")
def s2b():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import s2fft_b200

    return s2fft_b200


def _kw(sampling, spin, reality):
    return dict(L=16, spin=spin, nside=8 if sampling == "healpix" else None,
                sampling=sampling, reality=reality, L_lower=2)


@pytest.mark.parametrize("precision", ["f64", "f32"])
@pytest.mark.parametrize("sampling,spin,reality", CASES)
def test_inverse_gradient_matches_upstream_rules(s2b, rng, sampling, spin, reality, precision):
    import torch

    kw = _kw(sampling, spin, reality)
    L = kw["L"]
    cdt = torch.complex128 if precision == "f64" else torch.complex64
    flm = oracle.signal.generate_flm(rng, L, 2, spin, reality)
    f_t = oracle.spherical.inverse(oracle.signal.generate_flm(rng, L, 2, spin, reality), **kw)
    if reality:
        f_t = np.real(f_t)
    ref = G.inverse_vjp(2 * (oracle.spherical.inverse(flm, **kw) - f_t), **kw)

    x = torch.tensor(flm, dtype=cdt, device="cuda", requires_grad=True)
    f = s2b.inverse(x, L, spin, kw["nside"], sampling, reality=reality, L_lower=2,
                    precision=precision)
    assert f.is_complex() != reality
    loss = (torch.abs(f - torch.as_tensor(f_t, device="cuda")) ** 2).sum()
    loss.backward()
    assert relerr(x.grad.cpu().numpy(), ref) < TOL[precision]


@pytest.mark.parametrize("precision", ["f64", "f32"])
@pytest.mark.parametrize("sampling,spin,reality", CASES)
def test_forward_gradient_matches_upstream_rules(s2b, rng, sampling, spin, reality, precision):
    import torch

    kw = _kw(sampling, spin, reality)
    L = kw["L"]
    iters = 1 if sampling == "healpix" else 0
    f = oracle.spherical.inverse(oracle.signal.generate_flm(rng, L, 2, spin, reality), **kw)
    f = (np.real(f) + 0.05 * rng.standard_normal(f.shape) if reality else
         f + 0.05 * oracle.signal.complex_normal(rng, f.shape))
    flm_t = oracle.signal.generate_flm(rng, L, 2, spin, reality)
    ref = G.forward_vjp(2 * (oracle.spherical.forward(f, iter=iters, **kw) - flm_t),
                        iter=iters, **kw)

    rdt = torch.float64 if precision == "f64" else torch.float32
    cdt = torch.complex128 if precision == "f64" else torch.complex64
    x = torch.tensor(f, dtype=rdt if reality else cdt, device="cuda", requires_grad=True)
    y = s2b.forward(x, L, spin, kw["nside"], sampling, reality=reality, L_lower=2, iter=iters,
                    precision=precision)
    loss = (torch.abs(y - torch.as_tensor(flm_t, device="cuda")) ** 2).sum()
    loss.backward()
    assert relerr(x.grad.cpu().numpy(), ref) < TOL[precision]


@pytest.mark.parametrize("sampling", ["mw", "mwss", "gl"])
@pytest.mark.parametrize("spin", [1, -2])
def test_real_signals_with_spin_match_upstream(s2b, rng, sampling, spin):
    """reality=True with spin != 0: upstream's on-the-fly path accepts it, keeps the
    orders m >= 0 and returns a real map (inverse) / mirrored coefficients (forward)."""
    kw = _kw(sampling, spin, True)
    L = kw["L"]
    flm = oracle.signal.generate_flm(rng, L, 2, spin, False)
    ref = oracle.spherical.inverse(flm, **kw)
    got = s2b.inverse(flm, L, spin, kw["nside"], sampling, reality=True, L_lower=2)
    assert np.isrealobj(got)
    assert relerr(got, np.real(ref)) < 1e-10
    f = np.real(ref) + 0.1 * rng.standard_normal(np.shape(ref))
    ref_f = oracle.spherical.forward(f, iter=1, **kw)
    got_f = s2b.forward(f, L, spin, kw["nside"], sampling, reality=True, L_lower=2, iter=1)
    assert relerr(got_f, ref_f) < 1e-10


@pytest.mark.parametrize("sampling", ["mw", "gl"])
def test_wigner_real_signal_gradients(s2b, rng, sampling):
    """Real SO(3) signals: gradients of sum |f - target|^2 (inverse) and
    sum |flmn - target|^2 (forward) against central differences (float64)."""
    import torch

    L, N = 8, 3
    flmn = oracle.signal.generate_flmn(rng, L, N, 0, True)
    f_t = s2b.wigner.inverse(flmn * 0.5 + 0.1, L, N, sampling=sampling, reality=True)
    x = torch.tensor(flmn, device="cuda", requires_grad=True)

    def loss_inv(v):
        f = s2b.wigner.inverse(v, L, N, sampling=sampling, reality=True)
        return (torch.abs(f - torch.as_tensor(f_t, device="cuda")) ** 2).sum()

    loss_inv(x).backward()
    g = x.grad.cpu().numpy()
    h = 1e-4
    for _ in range(6):
        n = int(rng.integers(N))
        l = int(rng.integers(abs(n), L))
        m = int(rng.integers(0, l + 1))
        for part in (1.0, 1j):
            e = np.zeros_like(flmn)
            e[N - 1 + n, l, L - 1 + m] = part * h
            with torch.no_grad():
                fd = (loss_inv(torch.tensor(flmn + e, device="cuda"))
                      - loss_inv(torch.tensor(flmn - e, device="cuda"))).item() / (2 * h)
            an = g[N - 1 + n, l, L - 1 + m]
            an = an.real if part == 1.0 else an.imag
            assert abs(fd - an) <= 1e-7 * max(1.0, abs(an)), (n, l, m, part, fd, an)

    fmap = np.real(f_t) + 0.05 * rng.standard_normal(np.shape(f_t))
    flmn_t = oracle.signal.generate_flmn(rng, L, N, 0, True)
    z = torch.tensor(fmap, device="cuda", requires_grad=True)

    def loss_fwd(v):
        y = s2b.wigner.forward(v, L, N, sampling=sampling, reality=True)
        return (torch.abs(y - torch.as_tensor(flmn_t, device="cuda")) ** 2).sum()

    loss_fwd(z).backward()
    gz = z.grad.cpu().numpy()
    for _ in range(6):
        idx = tuple(int(rng.integers(k)) for k in fmap.shape)
        e = np.zeros_like(fmap)
        e[idx] = h
        with torch.no_grad():
            fd = (loss_fwd(torch.tensor(fmap + e, device="cuda"))
                  - loss_fwd(torch.tensor(fmap - e, device="cuda"))).item() / (2 * h)
        assert abs(fd - gz[idx]) <= 1e-7 * max(1.0, abs(gz[idx])), (idx, fd, gz[idx])
