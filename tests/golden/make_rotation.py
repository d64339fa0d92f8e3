"""Rotation fixtures from upstream's own Risbo recursion (fixture generator).

Upstream's rotate_flms (s2fft/utils/rotation.py:9-64) is jitted JAX, which is absent
here; its planes come from s2fft/recursions/risbo.py (numpy only), which this script
imports directly from the upstream tree and steps degree by degree exactly as
rotate_flms does. The contraction is upstream's einsum written out in numpy.
Writes ``rotation.npz``. Run from the repository root:
``python tests/golden/make_rotation.py upstream_root``.
"""

import importlib.util
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402


def main(ref_root):
    spec = importlib.util.spec_from_file_location(
        "risbo", os.path.join(ref_root, "s2fft", "recursions", "risbo.py"))
    risbo = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(risbo)
    rng = np.random.default_rng(7)
    out = {}
    for k, (L, rot) in enumerate(((8, (0.3, 1.1, -0.7)), (12, (-2.0, 2.9, 0.4)),
                                  (5, (0.0, 0.0, 1.3)))):
        flm = oracle.signal.generate_flm(rng, L, 0, 0, False)
        alpha = np.exp(-1j * np.arange(-L + 1, L) * rot[0])
        gamma = np.exp(-1j * np.arange(-L + 1, L) * rot[2])
        dl = np.zeros((2 * L - 1, 2 * L - 1))
        planes = np.zeros((L, 2 * L - 1, 2 * L - 1))
        rotated = np.zeros_like(flm)
        for el in range(L):
            dl = risbo.compute_full(dl, rot[1], L, el)
            planes[el] = dl
            m = np.arange(-el, el + 1)
            rotated[el, L - 1 + m] = np.einsum(
                "mn,n->m", dl[np.ix_(m + L - 1, m + L - 1)] * alpha[m + L - 1][:, None],
                gamma[m + L - 1] * flm[el, m + L - 1])
        out[f"r{k}/L"] = np.array(L)
        out[f"r{k}/rotation"] = np.array(rot)
        out[f"r{k}/flm"] = flm
        out[f"r{k}/rotated"] = rotated
        out[f"r{k}/dls"] = planes
    np.savez(os.path.join(HERE, "rotation.npz"), **out)


if __name__ == "__main__":
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    import _refstub

    main(_refstub.upstream_root(sys.argv))
