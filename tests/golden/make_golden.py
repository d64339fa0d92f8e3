"""Generate golden input/output vectors from the upstream s2fft numpy code.

Run in a container where the upstream source tree is mounted (its path is the
first argument, or ``S2FFT_UPSTREAM``); the fixtures it writes (``tests/golden/*.npz``) travel
with the repository, the upstream tree does not. JAX is absent there, so the
upstream package is imported through ``_refstub`` and only its numpy paths run:

* ``s2fft.transforms.spherical.inverse_numpy`` / ``forward_numpy`` / ``forward``
  (with ``iter``) for every sampling, spin in {-2, -1, 0, 2}, reality and L_lower;
* ``s2fft.transforms.wigner.inverse_numpy`` / ``forward_numpy``;
* ``s2fft.precompute_transforms.construct.spin_spherical_kernel`` and the
  precompute ``inverse_transform`` / ``forward_transform``;
* ``s2fft.utils.quadrature.quad_weights_transform`` and ``quad_weights``;
* the signal generator itself (``generate_flm`` / ``generate_flmn``), so the
  seeded inputs are pinned too.

Usage: ``python tests/golden/make_golden.py upstream_root``.
"""

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SEED = 8966433580120847635


def main(ref_root):
    sys.path.insert(0, HERE)
    import _refstub

    _refstub.install(ref_root)
    import s2fft
    from s2fft.precompute_transforms import construct
    from s2fft.precompute_transforms import spherical as pcs
    from s2fft.utils import quadrature
    from s2fft.utils import signal_generator as sg

    rng = np.random.default_rng(SEED)
    cases = {}
    index = []

    def put(name, meta, **arrays):
        for k, v in arrays.items():
            cases[f"{name}/{k}"] = v
        index.append(dict(name=name, **meta))

    # spherical transforms, small L, every sampling / spin / reality / L_lower
    for sampling in ["mw", "mwss", "dh", "gl", "healpix"]:
        for spin in [0, 2, -1, -2]:
            for reality in [False, True]:
                for L0 in [0, 2]:
                    if reality and spin != 0:
                        continue
                    if sampling == "healpix" and spin != 0:
                        continue
                    L, nside = (8, 4) if sampling == "healpix" else (11, None)
                    flm = sg.generate_flm(rng, L, L0, spin, reality)
                    f = s2fft.transforms.spherical.inverse_numpy(
                        flm, L, spin, nside, sampling, reality, None, L0)
                    g = s2fft.transforms.spherical.forward_numpy(
                        f, L, spin, nside, sampling, reality, None, L0)
                    name = f"sph_{sampling}_s{spin}_r{int(reality)}_l{L0}"
                    put(name, dict(kind="spherical", L=L, spin=spin, nside=nside,
                                   sampling=sampling, reality=reality, L_lower=L0),
                        flm=flm, f=f, flm_fwd=g)

    # HEALPix forward with Jacobi refinement (upstream forward(..., iter=n))
    for it in [0, 1, 3]:
        L, nside = 16, 8
        flm = sg.generate_flm(rng, L, 0, 0, True)
        f = np.real(s2fft.transforms.spherical.inverse_numpy(flm, L, 0, nside, "healpix", True))
        g = s2fft.forward(f, L, 0, nside, "healpix", "numpy", True, iter=it)
        put(f"hp_iter{it}", dict(kind="healpix_iter", L=L, nside=nside, iter=it),
            flm=flm, f=f, flm_fwd=g)

    # the small plain-method configuration: MW, L=128, spin 0, complex128
    L = 128
    flm = sg.generate_flm(rng, L, 0, 0, False)
    f = s2fft.transforms.spherical.inverse_numpy(flm, L, 0, None, "mw", False)
    g = s2fft.transforms.spherical.forward_numpy(f, L, 0, None, "mw", False)
    put("mw_L128", dict(kind="spherical", L=L, spin=0, nside=None, sampling="mw",
                        reality=False, L_lower=0), flm=flm, f=f, flm_fwd=g)

    # Wigner transforms
    for sampling in ["mw", "mwss", "dh", "gl"]:
        for reality in [False, True]:
            L, N = 7, 3
            flmn = sg.generate_flmn(rng, L, N, 0, reality)
            f = s2fft.wigner.inverse_numpy(flmn, L, N, None, sampling, reality)
            g = s2fft.wigner.forward_numpy(f, L, N, None, sampling, reality)
            put(f"wig_{sampling}_r{int(reality)}", dict(kind="wigner", L=L, N=N,
                                                        sampling=sampling, reality=reality),
                flmn=flmn, f=f, flmn_fwd=g)

    # precompute kernels and transforms
    for sampling in ["mw", "mwss", "dh", "gl", "healpix"]:
        for spin in [0, 2]:
            if sampling == "healpix" and spin != 0:
                continue
            L, nside = (8, 4) if sampling == "healpix" else (8, None)
            kin = construct.spin_spherical_kernel(L, spin, False, sampling, nside, False)
            kfw = construct.spin_spherical_kernel(L, spin, False, sampling, nside, True)
            flm = sg.generate_flm(rng, L, 0, spin, False)
            f = pcs.inverse_transform(flm, kin, L, sampling, False, spin, nside)
            g = pcs.forward_transform(f, kfw, L, sampling, False, spin, nside)
            put(f"pre_{sampling}_s{spin}", dict(kind="precompute", L=L, spin=spin, nside=nside,
                                                 sampling=sampling),
                kernel_inv=kin, kernel_fwd=kfw, flm=flm, f=f, flm_fwd=g)

    # quadrature
    for s in ["mwss", "dh", "gl", "healpix"]:
        cases[f"quad/transform_{s}"] = quadrature.quad_weights_transform(12, s, 0, 4)
    for s in ["mw", "mwss"]:
        for spin in [0, 1]:
            cases[f"quad/weights_{s}_s{spin}"] = quadrature.quad_weights(12, s, spin)

    # signal generator
    r2 = np.random.default_rng(SEED)
    cases["gen/flm_L9_s1"] = sg.generate_flm(r2, 9, 0, 1, False)
    cases["gen/flm_L9_real"] = sg.generate_flm(r2, 9, 2, 0, True)
    cases["gen/flmn_L6_N3"] = sg.generate_flmn(r2, 6, 3, 0, False)
    cases["gen/flmn_L6_N3_real"] = sg.generate_flmn(r2, 6, 3, 0, True)

    np.savez_compressed(os.path.join(HERE, "golden.npz"), **cases)
    with open(os.path.join(HERE, "golden_index.json"), "w") as fh:
        json.dump(dict(seed=SEED, upstream="astro-informatics/s2fft numpy paths",
                       cases=index), fh, indent=1)
    print(f"wrote {len(index)} cases, {len(cases)} arrays")


if __name__ == "__main__":
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    import _refstub

    main(_refstub.upstream_root(sys.argv))
