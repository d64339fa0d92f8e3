"""Import the upstream s2fft numpy code paths without JAX.

Used only by ``make_golden.py`` in a container where the upstream source tree
is mounted. JAX, jaxlib and the compiled ``s2fft_lib`` extension are replaced
by stand-ins: ``jit``/``custom_vjp`` become identity decorators and
``jax.numpy`` maps onto numpy, which is enough for every ``*_numpy`` function
(and ``base_transforms``) to import and run unmodified.
"""

import sys
import types
from unittest import mock

import numpy as np


def upstream_root(argv) -> str:
    """The upstream s2fft source tree: the first command-line argument, else the
    ``S2FFT_UPSTREAM`` environment variable. There is no default location."""
    import os

    root = argv[1] if len(argv) > 1 else os.environ.get("S2FFT_UPSTREAM")
    if not root:
        raise SystemExit("give the upstream s2fft source tree as the first argument "
                         "or in S2FFT_UPSTREAM")
    if not os.path.isdir(os.path.join(root, "s2fft")):
        raise SystemExit(f"{root} does not hold the upstream s2fft package")
    return root


def install(ref_root: str) -> None:
    if "s2fft" in sys.modules:
        return

    def _identity_decorator(*args, **kwargs):
        if len(args) == 1 and callable(args[0]) and not kwargs:
            return args[0]

        def wrap(fn):
            return fn

        return wrap

    class _CustomVJP:
        def __init__(self, fn, *a, **k):
            self.fn = fn

        def __call__(self, *a, **k):
            return self.fn(*a, **k)

        def defvjp(self, *a, **k):
            return None

    jax = types.ModuleType("jax")
    jax.jit = _identity_decorator
    jax.custom_vjp = lambda fn=None, **k: (_CustomVJP(fn) if fn else (lambda f: _CustomVJP(f)))
    jax.vmap = lambda f, *a, **k: f
    jax.pmap = lambda f, *a, **k: f
    jax.local_device_count = lambda: 1
    jax.config = mock.MagicMock()
    jax.config.read = lambda name: True
    jax.numpy = np
    jax.Array = np.ndarray
    jax.typing = mock.MagicMock()
    jax.lax = mock.MagicMock()
    jax.scipy = mock.MagicMock()
    for name in [
        "jax", "jax.numpy", "jax.lax", "jax.scipy", "jax.scipy.special",
        "jax.core", "jax.interpreters", "jax.interpreters.mlir",
        "jax.interpreters.ad", "jax.interpreters.batching", "jax.lib",
        "jax.dlpack", "jax.tree_util", "jax._src", "jax._src.numpy",
        "jax._src.numpy.util", "jax.extend", "jax.extend.core", "jax.test_util",
        "jaxlib", "jaxlib.mlir", "jaxlib.mlir.ir", "jaxlib.hlo_helpers",
        "jaxlib.mlir.dialects", "s2fft_lib", "s2fft_lib._s2fft",
        "pyssht", "healpy", "so3", "ducc0",
    ]:
        if name == "jax":
            sys.modules[name] = jax
        elif name == "jax.numpy":
            sys.modules[name] = np
        else:
            sys.modules[name] = mock.MagicMock()
    sys.modules["jax.lax"] = jax.lax
    # healpix_ffts.py iterates over _s2fft.registration().items() at import time
    sys.modules["s2fft_lib"]._s2fft.registration.return_value = {}
    sys.path.insert(0, ref_root)
