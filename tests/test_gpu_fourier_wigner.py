"""Fourier-Wigner transforms and spin-subset ops on the GPU against upstream's numpy code
(tests/golden/fourier_wigner.npz, made by tests/golden/make_fourier_wigner.py) and the
oracle. Tolerances: float64 atol 1e-12 (upstream's own tests/test_fourier_wigner.py),
float32 relative 1e-5."""

import json
import os

import numpy as np
import pytest
import torch

import oracle
from tests.conftest import GOLDEN_DIR, relerr

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fwg():
    d = np.load(os.path.join(GOLDEN_DIR, "fourier_wigner.npz"))
    with open(os.path.join(GOLDEN_DIR, "fourier_wigner.json")) as fh:
        return d, json.load(fh)["cases"]


@pytest.fixture(scope="module")
def s2b():
    import s2fft_b200

    return s2fft_b200


def test_kernel_matches_upstream(fwg, s2b):
    d, _ = fwg
    for L in (8, 16):
        delta, quads = s2b.fourier_wigner.fourier_wigner_kernel(L)
        assert np.abs(delta.cpu().numpy() - d[f"kernel_L{L}/delta"]).max() < 1e-13
        assert np.abs(quads.cpu().numpy() - d[f"kernel_L{L}/quads"]).max() < 1e-13


@pytest.mark.parametrize("use_upstream_precomps", [False, True])
def test_transforms_match_upstream_f64(fwg, s2b, use_upstream_precomps):
    d, cases = fwg
    fw = s2b.fourier_wigner
    seen = 0
    for c in cases:
        if c["kind"] != "fourier_wigner":
            continue
        n, L, N, s, r = c["name"], c["L"], c["N"], c["sampling"], c["reality"]
        pre = (d[f"kernel_L{L}/delta"], d[f"kernel_L{L}/quads"]) if (
            use_upstream_precomps and L in (8, 16)) else None
        f = fw.inverse_transform(d[f"{n}/flmn"], L, N, pre, r, s)
        np.testing.assert_allclose(f, d[f"{n}/f"], atol=1e-12, err_msg=n)
        assert (f.dtype == np.float64) if r else (f.dtype == np.complex128)
        g = fw.forward_transform(d[f"{n}/f"], L, N, pre, r, s)
        np.testing.assert_allclose(g, d[f"{n}/flmn_fwd"], atol=1e-12, err_msg=n)
        seen += 1
    assert seen == 10


def test_transforms_f32(fwg, s2b):
    d, cases = fwg
    fw = s2b.fourier_wigner
    for c in cases:
        if c["kind"] != "fourier_wigner":
            continue
        n, L, N, s, r = c["name"], c["L"], c["N"], c["sampling"], c["reality"]
        f = fw.inverse_transform(d[f"{n}/flmn"], L, N, None, r, s, precision="f32")
        assert f.dtype == (np.float32 if r else np.complex64)
        assert relerr(f, d[f"{n}/f"]) < 1e-5, n
        g = fw.forward_transform(d[f"{n}/f"], L, N, None, r, s, precision="f32")
        assert relerr(g, d[f"{n}/flmn_fwd"]) < 1e-5, n


def test_subset_ops_match_upstream(fwg, s2b):
    d, cases = fwg
    ops = s2b.custom_ops
    for c in cases:
        if c["kind"] != "subset_ops":
            continue
        n, L, N, s, sp = c["name"], c["L"], c["N"], c["sampling"], np.array(c["spins"])
        DW = s2b.fourier_wigner.fourier_wigner_kernel(L)
        np.testing.assert_allclose(ops.wigner_subset_to_s2(d[f"{n}/flmn"], sp, DW, L, s),
                                   d[f"{n}/fs"], atol=1e-12)
        np.testing.assert_allclose(ops.s2_to_wigner_subset(d[f"{n}/fs"], sp, DW, L, s),
                                   d[f"{n}/back"], atol=1e-12)
        np.testing.assert_allclose(ops.so3_to_wigner_subset(d[f"{n}/fso3"], sp, DW, L, N, s),
                                   d[f"{n}/sub"], atol=1e-12)
        for fn, x, ref in ((ops.wigner_subset_to_s2, d[f"{n}/flmn"], d[f"{n}/fs"]),
                           (ops.s2_to_wigner_subset, d[f"{n}/fs"], d[f"{n}/back"])):
            y = fn(x, sp, DW, L, s, precision="f32")
            assert relerr(y, ref) < 1e-5, n
        # device tensors in, device tensors out
        t = torch.as_tensor(d[f"{n}/flmn"]).cuda()
        y = ops.wigner_subset_to_s2(t, torch.as_tensor(sp), DW, L, s)
        assert y.is_cuda and relerr(y.cpu().numpy(), d[f"{n}/fs"]) < 1e-12


def test_errors(fwg, s2b):
    d, _ = fwg
    with pytest.raises(ValueError):
        s2b.fourier_wigner.inverse_transform(d["fw0/flmn"], 8, 2, None, False, "gl")
    with pytest.raises(ValueError):
        s2b.fourier_wigner.forward_transform(d["fw0/f"], 8, 2, None, False, "healpix")
    DW = s2b.fourier_wigner.fourier_wigner_kernel(8)
    with pytest.raises(ValueError):
        s2b.custom_ops.wigner_subset_to_s2(d["ops0/flmn"], np.array([0, 1]), DW, 8, "mw")
    with pytest.raises(ValueError):
        s2b.custom_ops.s2_to_wigner_subset(d["ops0/fs"], np.array([0, -2, 3]), DW, 8, "dh")


@pytest.mark.parametrize("sampling,reality", [("mw", False), ("mwss", True)])
def test_oracle_L40_and_batch(s2b, sampling, reality):
    """L=40, N=6 against the oracle; a batch of three maps equals three single calls."""
    L, N = 40, 6
    rng = np.random.default_rng(5)
    flmn = np.stack([oracle.signal.generate_flmn(rng, L, N, 0, reality) for _ in range(3)])
    fw = s2b.fourier_wigner
    f = fw.inverse_transform(flmn, L, N, None, reality, sampling)
    ref = oracle.fourier_wigner.inverse_transform(flmn[1], L, N, None, reality, sampling)
    assert relerr(f[1], ref) < 1e-12
    for k in range(3):
        fk = fw.inverse_transform(flmn[k], L, N, None, reality, sampling)
        assert np.array_equal(fk, f[k])
    g = fw.forward_transform(f, L, N, None, reality, sampling)
    assert relerr(g, flmn) < 1e-11
    gref = oracle.fourier_wigner.forward_transform(f[2], L, N, None, reality, sampling)
    assert relerr(g[2], gref) < 1e-12


def test_round_trip_L128_N8_and_recursion_agreement(s2b):
    """MW L=128, N=8: forward(inverse(flmn)) = flmn, and the Fourier-Wigner inverse agrees
    with the recursion-based Wigner inverse of this library."""
    L, N = 128, 8
    rng = np.random.default_rng(11)
    flmn = oracle.signal.generate_flmn(rng, L, N, 0, False)
    fw = s2b.fourier_wigner
    f = fw.inverse_transform(flmn, L, N)
    g = fw.forward_transform(f, L, N)
    assert relerr(g, flmn) < 1e-10
    f_rec = s2b.wigner.inverse(flmn, L, N, sampling="mw")
    assert relerr(f, f_rec) < 1e-9
    f32 = fw.inverse_transform(flmn, L, N, precision="f32")
    assert relerr(f32, f) < 1e-5


@pytest.mark.parametrize("L,N,sampling,reality", [(2, 1, "mw", False), (2, 2, "mwss", True),
                                                  (3, 1, "mwss", False), (5, 5, "mw", True),
                                                  (7, 3, "mwss", False)])
def test_small_band_limits(s2b, L, N, sampling, reality):
    """Tiny band-limits and N = 1 / N = L against the oracle (which is pinned to upstream)."""
    rng = np.random.default_rng(L * 10 + N)
    flmn = oracle.signal.generate_flmn(rng, L, N, 0, reality)
    fw = s2b.fourier_wigner
    f = fw.inverse_transform(flmn, L, N, None, reality, sampling)
    ref = oracle.fourier_wigner.inverse_transform(flmn, L, N, None, reality, sampling)
    np.testing.assert_allclose(f, ref, atol=1e-12)
    g = fw.forward_transform(ref, L, N, None, reality, sampling)
    gref = oracle.fourier_wigner.forward_transform(ref, L, N, None, reality, sampling)
    np.testing.assert_allclose(g, gref, atol=1e-12)
    np.testing.assert_allclose(g, flmn, atol=1e-12)


def test_subset_ops_single_slice_and_f32_batches(s2b):
    """One spin, one map, one channel; and a larger float32 batch against the float64 call."""
    L = 12
    rng = np.random.default_rng(3)
    DW = s2b.fourier_wigner.fourier_wigner_kernel(L)
    ops = s2b.custom_ops
    for sampling in ("mw", "mwss"):
        full = oracle.signal.generate_flmn(rng, L, 4, 0, False)
        flmn = full[3 + 2][None, None, :, :, None]  # n = 2 -> spin -2
        sp = np.array([-2])
        fs = ops.wigner_subset_to_s2(flmn, sp, DW, L, sampling)
        ref = oracle.fourier_wigner.wigner_subset_to_s2(
            flmn, sp, oracle.fourier_wigner.fourier_wigner_kernel(L), L, sampling)
        np.testing.assert_allclose(fs, ref, atol=1e-12)
        back = ops.s2_to_wigner_subset(fs, sp, DW, L, sampling)
        np.testing.assert_allclose(back, flmn, atol=1e-12)
    x = (rng.standard_normal((5, 3, L, 2 * L - 1, 4))
         + 1j * rng.standard_normal((5, 3, L, 2 * L - 1, 4)))
    sp = np.array([0, 3, -5])
    y64 = ops.wigner_subset_to_s2(x, sp, DW, L, "mw")
    y32 = ops.wigner_subset_to_s2(x, sp, DW, L, "mw", precision="f32")
    assert relerr(y32, y64) < 1e-5


def test_c_abi_errors(s2b):
    """The Fourier-Wigner entry points reject a short workspace, NULL or misaligned pointers
    and too many slices with a status code (no launch)."""
    import ctypes

    from s2fft_b200 import _lib
    from s2fft_b200 import fourier_wigner as fw

    L, N = 8, 3
    lib = fw._fwlib()
    plan = fw.get_plan(torch.device("cuda", 0), L, "mw", "f64", N)
    delta, quads = fw.fourier_wigner_kernel(L)
    flmn = torch.zeros((2 * N - 1, L, 2 * L - 1), dtype=torch.complex128, device="cuda")
    f = torch.empty((2 * N - 1, L, 2 * L - 1), dtype=torch.complex128, device="cuda")
    need = int(lib.s2b_fw_workspace_size(plan.ptr, fw.OP_INVERSE, 1, 0, 1))
    ws = torch.empty(need, dtype=torch.uint8, device="cuda")
    st = _lib.stream_handle(torch.device("cuda", 0))
    assert lib.s2b_fw_inverse(plan.ptr, 1, 0, delta.data_ptr(), flmn.data_ptr(), f.data_ptr(),
                              ws.data_ptr(), need, st) == 0
    assert lib.s2b_fw_inverse(plan.ptr, 1, 0, delta.data_ptr(), flmn.data_ptr(), f.data_ptr(),
                              ws.data_ptr(), need - 1, st) == 3
    assert lib.s2b_fw_inverse(plan.ptr, 1, 0, None, flmn.data_ptr(), f.data_ptr(),
                              ws.data_ptr(), need, st) == 4
    assert lib.s2b_fw_inverse(plan.ptr, 1, 0, delta.data_ptr(), flmn.data_ptr() + 8,
                              f.data_ptr(), ws.data_ptr(), need, st) == 4
    assert lib.s2b_fw_inverse(plan.ptr, 70000, 0, delta.data_ptr(), flmn.data_ptr(),
                              f.data_ptr(), ws.data_ptr(), need, st) == 1
    spins = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert lib.s2b_fw_subset_to_s2(plan.ptr, 1, 0, spins.data_ptr(), delta.data_ptr(),
                                   flmn.data_ptr(), f.data_ptr(), ws.data_ptr(), need, st) == 1
    assert lib.s2b_last_error()
    torch.cuda.synchronize()


def _vdot(a, b):
    return complex((a.conj() * b).sum().item())


@pytest.mark.parametrize("sampling", ["mw", "mwss"])
@pytest.mark.parametrize("L,N", [(12, 3), (10, 10), (16, 13)])
@pytest.mark.parametrize("precision,tol", [("f64", 1e-10), ("f32", 1e-5)])
def test_adjoint_dot_products(s2b, sampling, L, N, precision, tol):
    """Gradients through s2b_fw_inverse_adjoint / s2b_fw_forward_adjoint: for y = A x,
    <A x, y> = <x, A^H y>, with two signals per call (N = 13 takes the gamma FFT)."""
    rng = np.random.default_rng(L + 100 * N)
    fw = s2b.fourier_wigner
    cdt = torch.complex128 if precision == "f64" else torch.complex64
    nth, nph = (L + 1, 2 * L) if sampling == "mwss" else (L, 2 * L - 1)
    G = 2 * N - 1
    x = torch.tensor(np.stack([oracle.signal.generate_flmn(rng, L, N, 0, False)
                               for _ in range(2)]), dtype=cdt, device="cuda",
                     requires_grad=True)
    y = torch.tensor(rng.normal(size=(2, G, nth, nph)) + 1j * rng.normal(size=(2, G, nth, nph)),
                     dtype=cdt, device="cuda")
    f = fw.inverse_transform(x, L, N, None, False, sampling, precision=precision)
    (gx,) = torch.autograd.grad(f, x, grad_outputs=y)
    lhs, rhs = _vdot(f.detach(), y), _vdot(x.detach(), gx)
    assert abs(lhs - rhs) <= tol * max(abs(lhs), 1e-30) * 10, (lhs, rhs)

    fin = torch.tensor(rng.normal(size=(2, G, nth, nph)) + 1j * rng.normal(size=(2, G, nth, nph)),
                       dtype=cdt, device="cuda", requires_grad=True)
    h = torch.tensor(rng.normal(size=(2, G, L, 2 * L - 1))
                     + 1j * rng.normal(size=(2, G, L, 2 * L - 1)), dtype=cdt, device="cuda")
    flmn = fw.forward_transform(fin, L, N, None, False, sampling, precision=precision)
    (gf,) = torch.autograd.grad(flmn, fin, grad_outputs=h)
    lhs, rhs = _vdot(flmn.detach(), h), _vdot(fin.detach(), gf)
    assert abs(lhs - rhs) <= tol * max(abs(lhs), 1e-30) * 10, (lhs, rhs)


def test_gradient_matches_recursion_wigner(s2b):
    """MW L=32 N=4: the gradient of ||inverse(flmn) - g||^2 by the Fourier-Wigner adjoint equals
    the recursion-based Wigner transform's (its own adjoint kernels)."""
    L, N = 32, 4
    rng = np.random.default_rng(9)
    x = torch.tensor(oracle.signal.generate_flmn(rng, L, N, 0, False), device="cuda",
                     requires_grad=True)
    g = torch.tensor(rng.normal(size=(2 * N - 1, L, 2 * L - 1)), device="cuda")
    loss = (s2b.fourier_wigner.inverse_transform(x, L, N).real - g).pow(2).sum()
    (g1,) = torch.autograd.grad(loss, x)
    x2 = x.detach().clone().requires_grad_(True)
    loss2 = (s2b.wigner.inverse(x2, L, N, sampling="mw").real - g).pow(2).sum()
    (g2,) = torch.autograd.grad(loss2, x2)
    assert relerr(g1.cpu().numpy(), g2.cpu().numpy()) < 1e-9


@pytest.mark.parametrize("sampling", ["mw", "mwss"])
@pytest.mark.parametrize("precision,tol", [("f64", 1e-10), ("f32", 1e-5)])
def test_subset_ops_adjoint_dot_products(s2b, sampling, precision, tol):
    """Gradients of the three spin-subset ops (batch 2, 3 channels, spins {0, 3, -2}):
    <A x, y> = <x, A^H y> through the s2b_fw_*_adjoint entry points."""
    L, N = 10, 4
    rng = np.random.default_rng(21)
    ops = s2b.custom_ops
    DW = s2b.fourier_wigner.fourier_wigner_kernel(L)
    cdt = torch.complex128 if precision == "f64" else torch.complex64
    nth, nph = (L + 1, 2 * L) if sampling == "mwss" else (L, 2 * L - 1)
    sp = np.array([0, 3, -2])

    def rnd(shape):
        return torch.tensor(rng.normal(size=shape) + 1j * rng.normal(size=shape), dtype=cdt,
                            device="cuda")

    cases = [
        (lambda x: ops.wigner_subset_to_s2(x, sp, DW, L, sampling, precision=precision),
         (2, 3, L, 2 * L - 1, 3), (2, 3, nth, nph, 3)),
        (lambda x: ops.s2_to_wigner_subset(x, sp, DW, L, sampling, precision=precision),
         (2, 3, nth, nph, 3), (2, 3, L, 2 * L - 1, 3)),
        (lambda x: ops.so3_to_wigner_subset(x, sp, DW, L, N, sampling, precision=precision),
         (2, 2 * N - 1, nth, nph, 3), (2, 3, L, 2 * L - 1, 3)),
    ]
    for fn, ishape, oshape in cases:
        x = rnd(ishape).requires_grad_(True)
        y = rnd(oshape)
        out = fn(x)
        (gx,) = torch.autograd.grad(out, x, grad_outputs=y)
        lhs, rhs = _vdot(out.detach(), y), _vdot(x.detach(), gx)
        assert abs(lhs - rhs) <= tol * max(abs(lhs), 1e-30) * 10, (ishape, lhs, rhs)
