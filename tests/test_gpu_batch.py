"""Batched transforms of maps of uneven size (s2fft_b200.batch.BatchedSHT): grouping,
concurrent streams, CUDA-graph replay and the tile autotuner must leave every map's
result equal to the unbatched call on that map."""

import numpy as np
import pytest

import oracle
from tests.conftest import relerr

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def s2b():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import s2fft_b200

    return s2fft_b200


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_batched_uneven_matches_unbatched(s2b, rng, precision):
    Ls = [16, 32, 48]
    samplings = ["mw", "mwss", "dh", "gl"]
    specs = [(int(rng.choice(Ls)), int(rng.integers(0, 4)), str(rng.choice(samplings)))
             for _ in range(24)]
    flms = [oracle.signal.generate_flm(rng, L, 0, s) for L, s, _ in specs]
    b = s2b.batch.BatchedSHT(specs, precision=precision)
    b.load(flms)
    for rep in range(2):  # replay twice: the graph is reusable
        b.run()
    tol = 1e-5 if precision == "f32" else 1e-10
    for i, (L, s, smp) in enumerate(specs):
        f_ref = s2b.inverse(flms[i], L, s, None, smp, precision=precision)
        assert relerr(b.maps(i).cpu().numpy(), f_ref) < tol, (i, specs[i])
        g_ref = s2b.forward(f_ref, L, s, None, smp, precision=precision)
        assert relerr(b.coefficients(i).cpu().numpy(), g_ref) < tol, (i, specs[i])
        assert relerr(b.coefficients(i).cpu().numpy(), flms[i]) < tol * 10
    assert len(b.summary()) == len({(L, s, smp) for L, s, smp in specs})


def test_tile_variants_agree(s2b, rng):
    """Both tile variants of each latitudinal kernel give the same transform."""
    import ctypes

    import torch
    from s2fft_b200 import _lib

    L = 40
    flm = oracle.signal.generate_flm(rng, L, 0, 2)
    out = []
    for v in (0, 1):
        for smp in ("mw", "gl"):
            plan = _lib.get_plan(torch.device("cuda", 0), L=L, spin=2, nside=0,
                                 sampling=_lib.SAMPLING[smp], reality=0, L_lower=0,
                                 precision=_lib.PRECISION["f32"], batch=1, iter=0, N=0)
            _lib.check(_lib.lib().s2b_plan_set_tuning(plan.ptr, 0, v))
            _lib.check(_lib.lib().s2b_plan_set_tuning(plan.ptr, 1, v))
            f = s2b.inverse(flm, L, 2, None, smp, precision="f32")
            out.append((f, s2b.forward(f, L, 2, None, smp, precision="f32")))
    for (fa, ga), (fb, gb) in zip(out[:2], out[2:]):
        assert relerr(fa, fb) < 1e-6 and relerr(ga, gb) < 1e-6
