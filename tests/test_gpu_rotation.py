"""Rotation of coefficients on the device (s2b_rotate_flms / s2b_rotate_dls) against
upstream's Risbo-based rotation (tests/golden/rotation.npz) and size-independent
properties at larger band-limits."""

import os

import numpy as np
import pytest

import oracle
from tests.conftest import GOLDEN_DIR, relerr

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def s2b():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import s2fft_b200

    return s2fft_b200


@pytest.fixture(scope="module")
def fixture():
    return np.load(os.path.join(GOLDEN_DIR, "rotation.npz"))


@pytest.mark.parametrize("k", [0, 1, 2])
def test_rotation_golden(s2b, fixture, k):
    L = int(fixture[f"r{k}/L"])
    rot = tuple(fixture[f"r{k}/rotation"])
    flm, ref = fixture[f"r{k}/flm"], fixture[f"r{k}/rotated"]
    # Wigner-d values by the degree recurrence on the device
    r = s2b.rotation.rotate_flms(flm, L, rot)
    assert relerr(r, ref) < 1e-12, relerr(r, ref)
    # float32 in and out (double arithmetic inside)
    r32 = s2b.rotation.rotate_flms(flm.astype(np.complex64), L, rot)
    assert r32.dtype == np.complex64 and relerr(r32, ref) < 1e-6
    # planes generated on the device, then passed back in (upstream's dl_array route)
    dl = s2b.rotation.generate_rotate_dls(L, rot[1]).cpu().numpy()
    assert np.abs(dl - fixture[f"r{k}/dls"]).max() < 1e-13
    r2 = s2b.rotation.rotate_flms(flm, L, rot, dl_array=dl)
    assert relerr(r2, ref) < 1e-12, relerr(r2, ref)


def test_rotation_inverse_and_batch(s2b, rng):
    """Rotating by (alpha, beta, gamma) and then by (-gamma, -beta, -alpha) gives flm back
    (L=512, a batch of 2), and each map of the batch equals its single rotation."""
    L = 512
    flm = np.stack([oracle.signal.generate_flm(rng, L, 0, 0, False) for _ in range(2)])
    rot = (0.7, 1.9, -2.4)
    r = s2b.rotation.rotate_flms(flm, L, rot)
    back = s2b.rotation.rotate_flms(r, L, (-rot[2], -rot[1], -rot[0]))
    assert relerr(back, flm) < 1e-10, relerr(back, flm)
    single = s2b.rotation.rotate_flms(flm[1], L, rot)
    assert relerr(single, r[1]) < 1e-13


@pytest.mark.parametrize("L,beta", [(48, 0.05), (48, np.pi / 2), (37, 3.1), (20, 0.0)])
def test_rotation_planes_against_risbo(s2b, L, beta):
    """generate_rotate_dls against the oracle's Risbo planes, including betas whose start
    values underflow (0.05, 3.1: the scaled path) and an odd band-limit."""
    dl = s2b.rotation.generate_rotate_dls(L, beta).cpu().numpy()
    ref = oracle.rotation.generate_rotate_dls(L, beta)
    assert np.abs(dl - ref).max() < 1e-12, np.abs(dl - ref).max()


@pytest.mark.parametrize("L,rot", [(1024, (0.3, 0.05, -1.2)), (600, (2.0, 3.05, 0.4)),
                                   (1500, (0.3, 2.9, 1.0)), (2049, (0.5, 1.1, 2.5))])
def test_rotation_unitary_large(s2b, rng, L, rot):
    """Rotation keeps the power of every degree, sum_m |flm'[l, m]|^2 = sum_m |flm[l, m]|^2,
    and rotating back restores flm: at L = 1024 and 600 with betas near 0 and pi (start
    values below 2^-960, renormalised recurrences), at L = 1500 (clusters of 12 CTAs on
    the tensor-core path) and at L = 2049 (four n per lane)."""
    import torch

    flm = torch.from_numpy(oracle.signal.generate_flm(rng, L, 0, 0, False)).cuda()
    r = s2b.rotation.rotate_flms(flm, L, rot)
    p0 = (flm.abs() ** 2).sum(-1)
    p1 = (r.abs() ** 2).sum(-1)
    assert float(((p1 - p0).abs() / p0.clamp_min(1e-300)).max()) < 1e-11
    back = s2b.rotation.rotate_flms(r, L, (-rot[2], -rot[1], -rot[0]))
    assert float((back - flm).abs().max() / flm.abs().max()) < 1e-10


@pytest.mark.parametrize("L", [1, 2, 3, 9])
def test_rotation_small_band_limits(s2b, rng, L):
    """The smallest band-limits (one warp, one CTA per cluster, partial order tiles)."""
    rot = (0.4, 2.2, -0.9)
    flm = oracle.signal.generate_flm(rng, L, 0, 0, False)
    r = s2b.rotation.rotate_flms(flm, L, rot)
    ref = oracle.rotation.rotate_flms(flm, L, rot)
    assert relerr(r, ref) < 1e-13, relerr(r, ref)
    dl = s2b.rotation.generate_rotate_dls(L, rot[1]).cpu().numpy()
    assert np.abs(dl - oracle.rotation.generate_rotate_dls(L, rot[1])).max() < 1e-14


def test_rotation_f32_batch(s2b, rng):
    """complex64 maps (float in and out, double inside) in a batch of three at L = 300
    against the float64 rotation of the same maps, and each map against its own call."""
    L = 300
    rot = (1.2, 0.8, -0.3)
    flm = np.stack([oracle.signal.generate_flm(rng, L, 0, 0, False) for _ in range(3)])
    r64 = s2b.rotation.rotate_flms(flm, L, rot)
    r32 = s2b.rotation.rotate_flms(flm.astype(np.complex64), L, rot)
    assert r32.dtype == np.complex64 and relerr(r32, r64) < 1e-6, relerr(r32, r64)
    one = s2b.rotation.rotate_flms(flm[2].astype(np.complex64), L, rot)
    assert np.array_equal(one, r32[2])


@pytest.mark.parametrize("L", [512, 1040])
def test_rotation_planes_passed_back(s2b, rng, L):
    """Planes passed back as dl_array give the rotation computed without them: L = 512 (four
    orders per tile in CTAs of four warps) and L = 1040 (36 GB; two n per lane)."""
    import torch

    rot = (0.9, 1.3, -0.6)
    flm = torch.from_numpy(oracle.signal.generate_flm(rng, L, 0, 0, False)).cuda()
    dl = s2b.rotation.generate_rotate_dls(L, rot[1])
    r1 = s2b.rotation.rotate_flms(flm, L, rot, dl_array=dl)
    del dl
    torch.cuda.empty_cache()
    r0 = s2b.rotation.rotate_flms(flm, L, rot)
    assert float((r1 - r0).abs().max() / r0.abs().max()) < 1e-12


def test_rotation_batch_tensor_core_path(s2b, rng):
    """A batch of two maps at L = 1024 (the tensor-core kernel walks the maps one after the
    other, continuing its chunk sequence): each map equals its own call."""
    import torch

    L = 1024
    rot = (2.1, 0.6, 1.4)
    flm = torch.from_numpy(np.stack([oracle.signal.generate_flm(rng, L, 0, 0, False)
                                     for _ in range(2)])).cuda()
    r = s2b.rotation.rotate_flms(flm, L, rot)
    for k in range(2):
        one = s2b.rotation.rotate_flms(flm[k], L, rot)
        assert torch.equal(one, r[k])


def test_rotation_f32_tensor_core_path(s2b, rng):
    """complex64 maps on the tensor-core kernel (L = 1024) against the float64 rotation."""
    import torch

    L = 1024
    rot = (0.2, 2.4, -1.7)
    flm = torch.from_numpy(oracle.signal.generate_flm(rng, L, 0, 0, False)).cuda()
    r64 = s2b.rotation.rotate_flms(flm, L, rot)
    r32 = s2b.rotation.rotate_flms(flm.to(torch.complex64), L, rot)
    assert r32.dtype == torch.complex64
    err = float((r32.to(torch.complex128) - r64).abs().max() / r64.abs().max())
    assert err < 1e-6, err


def test_rotation_against_oracle_L256(s2b, rng):
    """The device rotation at L = 256 (shuffle kernel, two orders per tile) against the
    oracle's Risbo-based rotation of the same map."""
    L = 256
    rot = (1.1, 2.3, -0.4)
    flm = oracle.signal.generate_flm(rng, L, 0, 0, False)
    ref = oracle.rotation.rotate_flms(flm, L, rot)
    r = s2b.rotation.rotate_flms(flm, L, rot)
    assert relerr(r, ref) < 1e-12, relerr(r, ref)
