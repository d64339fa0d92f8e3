"""s2fft_b200: spin spherical-harmonic and Wigner transforms on NVIDIA B200.

Drop-in for the transform calls of upstream ``s2fft`` (``forward``,
``inverse``, ``wigner.forward``, ``wigner.inverse``) with the kernels written
for sm_100a and exposed through the C ABI of ``libs2b.so`` (``include/s2b.h``).
"""

from . import _lib  # noqa: F401
from . import (batch, custom_ops, fourier_wigner, healpix_ffts, precompute,  # noqa: F401
               rotation, wigner)
from .spherical import f_shape, flm_shape, forward, inverse  # noqa: F401

__all__ = ["forward", "inverse", "f_shape", "flm_shape", "wigner", "precompute", "batch",
           "healpix_ffts", "rotation", "fourier_wigner", "custom_ops"]
