"""Batched transforms of maps of uneven size (s2fft_b200.batch.BatchedSHT and the
s2b_batch_* entry points): grouping, the persistent latitudinal launches over all
groups, concurrent streams, CUDA-graph replay and the tile autotuner must leave every
map's result equal to the unbatched call on that map."""

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


@pytest.mark.parametrize("persistent", [True, False, None])
@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_batched_uneven_matches_unbatched(s2b, rng, precision, persistent):
    Ls = [16, 32, 48]
    samplings = ["mw", "mwss", "dh", "gl"]
    specs = [(int(rng.choice(Ls)), int(rng.integers(0, 4)), str(rng.choice(samplings)))
             for _ in range(24)]
    flms = [oracle.signal.generate_flm(rng, L, 0, s) for L, s, _ in specs]
    b = s2b.batch.BatchedSHT(specs, precision=precision, persistent=persistent)
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
    assert b.schedule == {True: "persistent", False: "streams"}.get(persistent, b.schedule)


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


def _entry_plan(desc):
    import torch
    from s2fft_b200 import _lib

    full = dict(nside=0, reality=0, L_lower=0, batch=1, iter=0, N=0)
    full.update(desc)
    full["sampling"] = _lib.SAMPLING[full["sampling"]]
    full["precision"] = _lib.PRECISION[full["precision"]]
    return _lib.get_plan(torch.device("cuda", 0), **full)


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_batch_entry_points_mixed_entries(s2b, rng, precision):
    """s2b_batch_inverse / s2b_batch_forward over 54 entries, more than one persistent
    launch holds (48 plans): every sampling, spins -2..3, reality, L_lower, maps per entry,
    HEALPix with refinement iterations, an entry too small for the latitudinal kernels
    (L = 2), the same plan in several entries, and tile shapes that differ between plans
    (several launches per kernel variant). Each entry must equal the single-plan call."""
    import torch

    from s2fft_b200 import _lib
    from s2fft_b200.spherical import f_shape

    fixed = [dict(L=16, spin=0, sampling="healpix", nside=8, reality=1, iter=2),
             dict(L=24, spin=-2, sampling="mw", batch=3),
             dict(L=40, spin=0, sampling="gl", reality=1, L_lower=3),
             dict(L=2, spin=0, sampling="mw"),
             dict(L=20, spin=1, sampling="mwss"),
             dict(L=8, spin=0, sampling="dh"),
             dict(L=12, spin=2, sampling="healpix", nside=4, iter=1)]
    descs = fixed + [dict(L=int(rng.choice([8, 16, 24, 32])), spin=int(rng.integers(-2, 4)),
                          sampling=str(rng.choice(["mw", "mwss", "dh", "gl"])))
                     for _ in range(47)]
    for d in descs:
        d["precision"] = precision
    plans = [_entry_plan(d) for d in descs]
    for k, p in enumerate(plans):  # mixed tile shapes across plans
        _lib.check(_lib.lib().s2b_plan_set_tuning(p.ptr, 1, 2 + (k % 2)))
        _lib.check(_lib.lib().s2b_plan_set_tuning(p.ptr, 0, (k // 2) % 2))
    cdt = torch.complex64 if precision == "f32" else torch.complex128
    rdt = torch.float32 if precision == "f32" else torch.float64
    flms, fs, outs, ws_i, ws_f = [], [], [], [], []
    for d, p in zip(descs, plans):
        B, L = d.get("batch", 1), d["L"]
        x = np.stack([oracle.signal.generate_flm(rng, L, d.get("L_lower", 0), d["spin"],
                                                 bool(d.get("reality", 0)))
                      for _ in range(B)])
        flms.append(torch.as_tensor(x).to("cuda", cdt))
        fs.append(torch.empty((B,) + f_shape(L, d["sampling"], d.get("nside")),
                              dtype=rdt if d.get("reality") else cdt, device="cuda"))
        outs.append(torch.empty_like(flms[-1]))
        ws_i.append(torch.empty_like(p.workspace(0)))  # own workspaces: plans repeat
        ws_f.append(torch.empty_like(p.workspace(1)))
    batch = _lib.Batch(plans)
    stream = torch.cuda.current_stream()
    batch.inverse(flms, fs, ws_i, stream)
    batch.forward(fs, outs, ws_f, stream)
    torch.cuda.synchronize()
    # other schedules (waves, CTAs per SM of the persistent launches): the same results, up
    # to the order of the forward's atomic accumulation
    same = 1e-6 if precision == "f32" else 1e-13
    for waves, per_sm in ((2, 0), (3, 1), (4, 2)):
        batch.set_schedule(waves, per_sm)
        f2 = [torch.empty_like(x) for x in fs]
        o2 = [torch.empty_like(x) for x in outs]
        batch.inverse(flms, f2, ws_i, stream)
        batch.forward(f2, o2, ws_f, stream)
        torch.cuda.synchronize()
        for k in range(len(descs)):
            assert relerr(f2[k].cpu().numpy(), fs[k].cpu().numpy()) < same, (waves, per_sm, k)
            assert relerr(o2[k].cpu().numpy(), outs[k].cpu().numpy()) < same, (waves, per_sm, k)
    tol = 1e-5 if precision == "f32" else 1e-10
    for k, d in enumerate(descs):
        kw = dict(reality=bool(d.get("reality", 0)), L_lower=d.get("L_lower", 0),
                  precision=precision)
        for b in range(d.get("batch", 1)):
            f_ref = s2b.inverse(flms[k][b], d["L"], d["spin"], d.get("nside"), d["sampling"],
                                **kw)
            assert relerr(fs[k][b].cpu().numpy(), f_ref.cpu().numpy()) < tol, (k, d)
            g_ref = s2b.forward(fs[k][b], d["L"], d["spin"], d.get("nside"), d["sampling"],
                                iter=d.get("iter", 0), **kw)
            assert relerr(outs[k][b].cpu().numpy(), g_ref.cpu().numpy()) < tol, (k, d)


def test_batch_rejects_mixed_precision(s2b):
    from s2fft_b200 import _lib

    a = _entry_plan(dict(L=8, spin=0, sampling="mw", precision="f32"))
    b = _entry_plan(dict(L=8, spin=0, sampling="mw", precision="f64"))
    with pytest.raises(_lib.S2BError, match="precision"):
        _lib.Batch([a, b])
