"""Fourier-Wigner and spin-subset fixtures from the upstream numpy code (fixture generator).

Imports upstream s2fft through ``_refstub`` (JAX is absent) and runs, unmodified:

* ``s2fft.precompute_transforms.construct.fourier_wigner_kernel`` (Delta planes at
  pi/2 by Risbo's recursion and the upsampled quadrature weights);
* ``s2fft.precompute_transforms.fourier_wigner.inverse_transform`` /
  ``forward_transform`` with and without precomputes, mw and mwss, complex and real;
* ``s2fft.precompute_transforms.custom_ops.wigner_subset_to_s2``,
  ``s2_to_wigner_subset`` and ``so3_to_wigner_subset`` (numpy versions).

Inputs come from upstream's own ``signal_generator.generate_flmn``. Writes
``fourier_wigner.npz`` and ``fourier_wigner.json``. Run from the repository root:
``python tests/golden/make_fourier_wigner.py upstream_root``.
"""

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref_root):
    sys.path.insert(0, HERE)
    import _refstub

    _refstub.install(ref_root)
    from s2fft.precompute_transforms import construct, custom_ops
    from s2fft.precompute_transforms import fourier_wigner as fw
    from s2fft.utils import signal_generator as sg

    rng = np.random.default_rng(20261203)
    arrays, index = {}, []

    for L in (8, 16):
        d, w = construct.fourier_wigner_kernel(L)
        arrays[f"kernel_L{L}/delta"] = d
        arrays[f"kernel_L{L}/quads"] = w

    cases = [(8, 2, "mw", False), (8, 2, "mwss", True), (8, 8, "mw", True),
             (8, 8, "mwss", False), (16, 8, "mw", False), (16, 8, "mwss", True),
             (16, 16, "mw", False), (16, 16, "mwss", True), (12, 5, "mw", True),
             (12, 5, "mwss", False)]
    for k, (L, N, sampling, reality) in enumerate(cases):
        pre = construct.fourier_wigner_kernel(L)
        flmn = sg.generate_flmn(rng, L, N, 0, reality)
        f = fw.inverse_transform(flmn, L, N, pre, reality, sampling)
        f_otf = fw.inverse_transform(flmn, L, N, None, reality, sampling)
        g = fw.forward_transform(f, L, N, pre, reality, sampling)
        name = f"fw{k}"
        arrays[f"{name}/flmn"] = flmn
        arrays[f"{name}/f"] = f
        arrays[f"{name}/flmn_fwd"] = g
        index.append(dict(name=name, kind="fourier_wigner", L=L, N=N, sampling=sampling,
                          reality=reality, otf_vs_precomp=float(np.abs(f_otf - f).max())))

    # spin-subset lifting ops: batch 2, channels 3, arbitrary spins (|s| < N <= L)
    for k, (L, N, sampling, spins) in enumerate(((8, 4, "mw", [0, -2, 3]),
                                                 (10, 6, "mwss", [1, 5, -4, 0]))):
        DW = construct.fourier_wigner_kernel(L)
        S = len(spins)
        flmn = np.zeros((2, S, L, 2 * L - 1, 3), dtype=np.complex128)
        for b in range(2):
            for c in range(3):
                full = sg.generate_flmn(rng, L, N, 0, False)
                flmn[b, :, :, :, c] = full[N - 1 - np.asarray(spins)]
        sp = np.asarray(spins)
        fs = custom_ops.wigner_subset_to_s2(flmn, sp, DW, L, sampling)
        back = custom_ops.s2_to_wigner_subset(fs, sp, DW, L, sampling)
        nth = L + 1 if sampling == "mwss" else L
        nph = 2 * L if sampling == "mwss" else 2 * L - 1
        fso3 = rng.standard_normal((2, 2 * N - 1, nth, nph, 3)) + 1j * rng.standard_normal(
            (2, 2 * N - 1, nth, nph, 3))
        sub = custom_ops.so3_to_wigner_subset(fso3, sp, DW, L, N, sampling)
        name = f"ops{k}"
        arrays[f"{name}/flmn"] = flmn
        arrays[f"{name}/fs"] = fs
        arrays[f"{name}/back"] = back
        arrays[f"{name}/fso3"] = fso3
        arrays[f"{name}/sub"] = sub
        index.append(dict(name=name, kind="subset_ops", L=L, N=N, sampling=sampling,
                          spins=spins))

    np.savez_compressed(os.path.join(HERE, "fourier_wigner.npz"), **arrays)
    with open(os.path.join(HERE, "fourier_wigner.json"), "w") as fh:
        json.dump({"cases": index}, fh, indent=1)


if __name__ == "__main__":
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    import _refstub

    main(_refstub.upstream_root(sys.argv))
