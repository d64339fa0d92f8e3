"""Golden subsets at the benchmark configurations, from the upstream numpy code.

The benchmark sizes are too large to store whole (an L=1024 MW map is 33 MB), so
this script runs upstream's numpy transforms (imported through ``_refstub``,
unmodified) once on the seeded inputs that ``bench.py`` uses and stores, per case,
the seed and recipe of the input plus a few thousand sampled output entries:

* ``mw_L1024``: MW, L=1024, spin 0, complex; ``inverse_numpy`` then
  ``forward_numpy`` of that map (s2fft/transforms/spherical.py:112-208, 467-588).
* ``hp_L512``: HEALPix nside=256, L=512, spin 0, real signal; ``inverse_numpy`` and
  ``forward(..., method="numpy", iter=3)`` (spherical.py:352-464,
  s2fft/utils/iterative_refinement.py:9-46).
* ``gl_L512_s{+2,-2}_map{0,1}``: Gauss-Legendre, L=512, spin +-2, the first two maps
  of the 64-map batch; inverse and forward.
* ``mix_{i}``: the first eight maps with L <= 512 of the uneven 256-map mix (L in
  {64..1024}, spin 0..3, mw/mwss/dh/gl); inverse and forward.

Inputs: Re and Im of flm i.i.d. N(0,1) for every |m| <= l with |spin| <= l < L
(with reality: m = 0 real and the conjugate symmetry), drawn from
``numpy.random.default_rng(seed)`` exactly as ``bench.py`` draws them. Writes
``large.npz`` / ``large.json``. Needs about 20 GB of host memory and 20-30 minutes
(the L=1024 forward alone takes five). Run from the repository root:
``python tests/golden/make_large.py upstream_root``.
"""

import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
NSAMP = 2048
HEADLINE_SEED = 8966433580120847635   # bench.py: rank 0 of the headline workload
HEALPIX_SEED = 7
GL_SEED = 1000                        # + spin
MIX_SEED = 4242
MIX_LS = [64, 128, 256, 512, 1024]
MIX_SAMPLINGS = ["mw", "mwss", "dh", "gl"]


def seeded_flm(rng, L, spin=0, reality=False):
    """The benchmark's input draw (bench.py seeded_flm)."""
    flm = np.zeros((L, 2 * L - 1), dtype=np.complex128)
    for el in range(abs(spin), L):
        n = 2 * el + 1
        flm[el, L - 1 - el: L + el] = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        if reality:
            flm[el, L - 1] = flm[el, L - 1].real
            m = np.arange(1, el + 1)
            flm[el, L - 1 - m] = (-1.0) ** m * np.conj(flm[el, L - 1 + m])
    return flm


def headline_input():
    return seeded_flm(np.random.default_rng(HEADLINE_SEED), 1024)


def healpix_input():
    return seeded_flm(np.random.default_rng(HEALPIX_SEED), 512, 0, True)


def gl_inputs(spin, count):
    rng = np.random.default_rng(GL_SEED + spin)
    return [seeded_flm(rng, 512, spin) for _ in range(count)]


def mix_specs_and_inputs(nmaps=256):
    rng = np.random.default_rng(MIX_SEED)
    specs = [(int(rng.choice(MIX_LS)), int(rng.integers(0, 4)), str(rng.choice(MIX_SAMPLINGS)))
             for _ in range(nmaps)]
    flms = [seeded_flm(rng, L, sp) for L, sp, _ in specs]
    return specs, flms


def mix_selection(specs, count=8, Lmax=512):
    return [i for i, (L, _, _) in enumerate(specs) if L <= Lmax][:count]


def flm_mask(L, spin):
    m = np.arange(-(L - 1), L)[None, :]
    el = np.arange(L)[:, None]
    return (np.abs(m) <= el) & (el >= abs(spin))


def sample(rng, arr, mask=None):
    flat = np.flatnonzero(mask) if mask is not None else np.arange(arr.size)
    idx = np.sort(rng.choice(flat, size=min(NSAMP, flat.size), replace=False))
    return idx.astype(np.int64), arr.reshape(-1)[idx]


def main(ref_root):
    sys.path.insert(0, HERE)
    import _refstub

    _refstub.install(ref_root)
    import s2fft
    from s2fft.transforms import spherical as sph

    srng = np.random.default_rng(12345)  # sampled indices
    cases, index = {}, []

    def put(name, meta, f, g, flm, spin):
        fi, fv = sample(srng, f)
        gi, gv = sample(srng, g, flm_mask(meta["L"], spin))
        cases[f"{name}/f_idx"], cases[f"{name}/f_val"] = fi, fv
        cases[f"{name}/flm_idx"], cases[f"{name}/flm_val"] = gi, gv
        # the input's first entries, so that a consumer can check it drew the same flm
        cases[f"{name}/flm_head"] = flm[abs(spin):abs(spin) + 2].copy()
        rt = float(np.abs(g - flm).max() / np.abs(flm).max())
        index.append(dict(name=name, roundtrip_max_rel=rt, **meta))
        print(f"{name}: round trip {rt:.2e}", flush=True)

    t0 = time.time()
    flm = healpix_input()
    f = np.real(sph.inverse_numpy(flm, 512, 0, 256, "healpix", True))
    g = s2fft.forward(f, 512, 0, 256, "healpix", "numpy", True, iter=3)
    put("hp_L512", dict(L=512, spin=0, nside=256, sampling="healpix", reality=True, iter=3,
                        seed=HEALPIX_SEED), f, g, flm, 0)
    print(f"  {time.time() - t0:.0f} s", flush=True)

    for spin in (2, -2):
        for k, flm in enumerate(gl_inputs(spin, 2)):
            f = sph.inverse_numpy(flm, 512, spin, None, "gl", False)
            g = sph.forward_numpy(f, 512, spin, None, "gl", False)
            put(f"gl_L512_s{spin:+d}_map{k}", dict(L=512, spin=spin, nside=None, sampling="gl",
                                                   reality=False, iter=0, seed=GL_SEED + spin,
                                                   map=k), f, g, flm, spin)
        print(f"  {time.time() - t0:.0f} s", flush=True)

    specs, flms = mix_specs_and_inputs()
    for i in mix_selection(specs):
        L, spin, smp = specs[i]
        f = sph.inverse_numpy(flms[i], L, spin, None, smp, False)
        g = sph.forward_numpy(f, L, spin, None, smp, False)
        put(f"mix_{i}", dict(L=L, spin=spin, nside=None, sampling=smp, reality=False, iter=0,
                             seed=MIX_SEED, map=i), f, g, flms[i], spin)
    print(f"  {time.time() - t0:.0f} s", flush=True)

    flm = headline_input()
    f = sph.inverse_numpy(flm, 1024, 0, None, "mw", False)
    g = sph.forward_numpy(f, 1024, 0, None, "mw", False)
    put("mw_L1024", dict(L=1024, spin=0, nside=None, sampling="mw", reality=False, iter=0,
                         seed=HEADLINE_SEED), f, g, flm, 0)
    print(f"  {time.time() - t0:.0f} s", flush=True)

    np.savez_compressed(os.path.join(HERE, "large.npz"), **cases)
    with open(os.path.join(HERE, "large.json"), "w") as fh:
        json.dump(dict(upstream="astro-informatics/s2fft numpy paths", samples=NSAMP,
                       index_seed=12345, cases=index), fh, indent=1)
    print(f"wrote {len(index)} cases")


if __name__ == "__main__":
    sys.path.insert(0, HERE)
    import _refstub

    main(_refstub.upstream_root(sys.argv))
