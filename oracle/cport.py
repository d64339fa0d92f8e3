"""ctypes front-end of the C restatement of the latitudinal steps (oracle/csrc/otf.c).

TEST INFRASTRUCTURE ONLY (see the package docstring): the timed CPU baseline of
``bench.py`` and a checker in ``tests/``. Same signatures and results (to summation
order) as ``oracle.recursion.precompute`` / ``inverse_latitudinal_step`` /
``forward_latitudinal_step``, which restate s2fft/recursions/price_mcewen.py:118-255
and s2fft/transforms/otf_recursions.py:15-171, 432-588; the rings run on all host
threads (OpenMP).
"""

import ctypes
import os
import subprocess

import numpy as np

from . import samples

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc", "otf.c")
LIB = os.path.join(HERE, "libotf.so")
_lib = None


def build(force=False):
    """Compile libotf.so next to this file (gcc, OpenMP, a baseline x86-64 ISA so that the
    library runs on any host of the same architecture)."""
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    cmd = ["gcc", "-O3", "-fopenmp", "-fPIC", "-shared", "-march=x86-64-v2", "-o", LIB + ".tmp",
           SRC, "-lm"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"gcc failed:\n{r.stderr}")
    os.replace(LIB + ".tmp", LIB)
    return LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        h = ctypes.CDLL(LIB)
        dp = ctypes.POINTER(ctypes.c_double)
        h.s2o_precompute.argtypes = [ctypes.c_int] * 3 + [dp, ctypes.c_int] + [dp] * 4
        h.s2o_precompute.restype = None
        lat = [ctypes.c_int] * 6 + [dp] * 6 + [ctypes.c_int, dp, ctypes.c_int]
        h.s2o_inverse_lat.argtypes = lat
        h.s2o_inverse_lat.restype = None
        h.s2o_forward_lat.argtypes = lat
        h.s2o_forward_lat.restype = None
        h.s2o_max_threads.restype = ctypes.c_int
        _lib = h
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def max_threads():
    return lib().s2o_max_threads()


def precompute(L, spin, beta, L_lower=0):
    """[lrenorm, vsign, cpi, cp2] in the layout of oracle.recursion.precompute."""
    beta = np.ascontiguousarray(beta, dtype=np.float64)
    n = L - L_lower
    lr = np.zeros((2, len(beta), n))
    vs = np.zeros((2 * L - 1, n))
    cpi = np.zeros((L + 1, n))
    cp2 = np.zeros((L + 1, n))
    lib().s2o_precompute(L, spin, len(beta), _p(beta), L_lower, _p(lr), _p(vs), _p(cpi), _p(cp2))
    return [lr, vs, cpi, cp2]


def _prep(precomps, L, spin, beta, L_lower):
    if precomps is None:
        precomps = precompute(L, spin, beta, L_lower)
    return [np.ascontiguousarray(a, dtype=np.float64) for a in precomps[:4]]


def inverse_latitudinal_step(flm, beta, L, spin, sampling="mw", reality=False, precomps=None,
                             L_lower=0, max_steps=None, nside=None, threads=0):
    """ftm[theta, m] = sum_l d^l_{m,-s}(theta) flm[l, m] (otf_recursions.py:15-171)."""
    if max_steps is not None:
        raise ValueError("the C port runs whole transforms")
    beta = np.ascontiguousarray(beta, dtype=np.float64)
    lr, vs, cpi, cp2 = _prep(precomps, L, spin, beta, L_lower)
    ncol = samples.ftm_shape(L, sampling, nside)[1]
    flm = np.ascontiguousarray(flm, dtype=np.complex128)
    ftm = np.zeros((len(beta), ncol), dtype=np.complex128)
    mo = 1 if sampling in ("mwss", "healpix") else 0
    lib().s2o_inverse_lat(L, spin, L_lower, int(bool(reality)), mo, len(beta), _p(beta), _p(lr),
                          _p(vs), _p(cpi), _p(cp2), _p(flm.view(np.float64)), ncol,
                          _p(ftm.view(np.float64)), int(threads))
    return ftm


def forward_latitudinal_step(ftm, beta, L, spin, sampling="mw", reality=False, precomps=None,
                             L_lower=0, max_steps=None, threads=0):
    """flm[l, m] = sum_theta d^l_{m,-s}(theta) ftm[theta, m] (otf_recursions.py:432-588)."""
    if max_steps is not None:
        raise ValueError("the C port runs whole transforms")
    beta = np.ascontiguousarray(beta, dtype=np.float64)
    lr, vs, cpi, cp2 = _prep(precomps, L, spin, beta, L_lower)
    ftm = np.ascontiguousarray(ftm, dtype=np.complex128)
    flm = np.zeros((L, 2 * L - 1), dtype=np.complex128)
    mo = 1 if sampling in ("mwss", "healpix") else 0
    lib().s2o_forward_lat(L, spin, L_lower, int(bool(reality)), mo, len(beta), _p(beta), _p(lr),
                          _p(vs), _p(cpi), _p(cp2), _p(ftm.view(np.float64)), ftm.shape[1],
                          _p(flm.view(np.float64)), int(threads))
    return flm
