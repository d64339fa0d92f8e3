"""The C restatement of the latitudinal steps (oracle/csrc/otf.c, the timed CPU
baseline) against the numpy oracle and the upstream golden vectors."""

import numpy as np
import pytest

import oracle
from oracle import cport, recursion
from tests.conftest import relerr


@pytest.fixture(scope="module", autouse=True)
def built():
    cport.build()


@pytest.mark.parametrize("L,spin,sampling,reality,L0,nside", [
    (16, 0, "mw", False, 0, None), (16, 2, "mwss", False, 2, None), (12, -1, "dh", False, 0, None),
    (16, 0, "gl", True, 0, None), (8, 0, "healpix", False, 0, 4), (8, 0, "healpix", True, 1, 4),
    (20, -3, "mw", False, 3, None)])
def test_steps_match_numpy_restatement(rng, L, spin, sampling, reality, L0, nside):
    th = oracle.samples.thetas(L, sampling, nside)
    p_np = recursion.precompute(L, spin, th, L0)
    p_c = cport.precompute(L, spin, th, L0)
    for a, b in zip(p_np, p_c):
        assert np.array_equal(a, b) or relerr(b, a) < 1e-14
    flm = oracle.signal.generate_flm(rng, L, L0, spin, reality)
    a = recursion.inverse_latitudinal_step(flm, th, L, spin, sampling, reality, p_np, L0, None,
                                           nside)
    b = cport.inverse_latitudinal_step(flm, th, L, spin, sampling, reality, p_c, L0, None, nside)
    fin = np.isfinite(a)  # rings at the poles (mwss) overflow in both, identically
    assert np.array_equal(fin, np.isfinite(b))
    assert relerr(b[fin], a[fin]) < 1e-13
    ftm = rng.standard_normal(a.shape) + 1j * rng.standard_normal(a.shape)
    c = recursion.forward_latitudinal_step(ftm, th, L, spin, sampling, reality, p_np, L0)
    d = cport.forward_latitudinal_step(ftm, th, L, spin, sampling, reality, p_c, L0)
    fin = np.isfinite(c)
    assert np.array_equal(fin, np.isfinite(d))
    assert relerr(d[fin], c[fin]) < 1e-13


def test_transforms_match_golden(golden):
    data, index = golden
    n = 0
    for case in index["cases"]:
        if case["kind"] != "spherical" or case["L"] > 16:
            continue
        kw = dict(L=case["L"], spin=case["spin"], nside=case["nside"],
                  sampling=case["sampling"], reality=case["reality"], L_lower=case["L_lower"])
        name = case["name"]
        f = oracle.spherical.inverse(data[f"{name}/flm"], backend="c", **kw)
        assert relerr(f, data[f"{name}/f"]) < 1e-12, name
        g = oracle.spherical.forward(data[f"{name}/f"], backend="c", **kw)
        assert relerr(g, data[f"{name}/flm_fwd"]) < 1e-12, name
        n += 1
    assert n >= 20
