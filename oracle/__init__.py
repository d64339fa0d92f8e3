"""CPU oracle for the spin spherical-harmonic / Wigner transform path.

TEST INFRASTRUCTURE ONLY. This package is a float64 numpy restatement of the
upstream s2fft algorithm for the transform path (sampling geometry, quadrature,
resampling, HEALPix ring FFTs, the Price-McEwen latitudinal recursion, the
spherical and Wigner front-ends, the precompute-kernel transforms and the rotation of
coefficients). Each
function cites the upstream file:line it follows.

It is imported only by ``tests/``, by ``__graft_entry__.smoke()`` and by the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py``, and only as the
checker or as the timed CPU baseline. The product (``s2fft_b200``) never
imports it; a missing CUDA extension is an error there, not a fallback.

Parity pin: ``tests/test_oracle_golden.py`` checks every function here against
golden vectors produced by the upstream numpy code itself
(``tests/golden/make_golden.py``, run where the upstream tree is available).
"""

from . import (  # noqa: F401
    fourier_wigner,
    healpix,
    precompute,
    quadrature,
    recursion,
    resampling,
    rotation,
    samples,
    signal,
    spherical,
    wigner,
)
