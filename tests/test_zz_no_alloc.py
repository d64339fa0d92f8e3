"""s2b_inverse_noalloc: the spin inverse transform without any allocation.

Some callers of this library cannot allocate device memory: a plugin inside a
host program that owns every device allocation and hands over only the input
and output buffers, or code on a path where an allocation would stall the
device. For them the library keeps one fixed scratch array per GPU
(S2B_NOALLOC_SCRATCH_BYTES, 32 MiB) and this entry point uses it in place of
a caller-provided workspace. These tests call it through the C ABI and check
it against s2b_inverse, which takes the caller's workspace, on two calls in a
row (the second call finds the first call's leftovers in the shared array).

The file name makes pytest collect it last.
"""

import ctypes

import numpy as np
import pytest

import oracle
from tests.conftest import relerr

pytestmark = pytest.mark.gpu

TOL = {"f64": 1e-10, "f32": 1e-5}
SCRATCH_BYTES = 32 << 20


@pytest.fixture(scope="module")
def cabi():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from s2fft_b200 import _lib

    return _lib


def _plan(_lib, **kw):
    import torch

    desc = dict(L=8, spin=0, nside=0, sampling=0, reality=0, L_lower=0, precision=0, batch=1,
                iter=0, N=0)
    desc.update(kw)
    return _lib.Plan(torch.device("cuda", torch.cuda.current_device()), **desc)


@pytest.mark.parametrize("L,spin,sampling,precision,batch", [
    (64, 0, "mw", "f64", 1),
    (48, 2, "gl", "f32", 2),
    (40, -1, "dh", "f64", 3),
])
def test_noalloc_matches_workspace_inverse(cabi, rng, L, spin, sampling, precision, batch):
    import torch

    _lib = cabi
    cdt = torch.complex128 if precision == "f64" else torch.complex64
    plan = _plan(_lib, L=L, spin=spin, sampling=_lib.SAMPLING[sampling],
                 precision=_lib.PRECISION[precision], batch=batch)
    nth = {"mw": L, "gl": L, "dh": 2 * L}[sampling]
    shape = (batch, nth, 2 * L - 1)
    flms = [torch.from_numpy(np.stack([oracle.signal.generate_flm(rng, L, 0, spin)
                                       for _ in range(batch)])).to("cuda", cdt)
            for _ in range(2)]
    stream = _lib.stream_handle(flms[0].device)
    lib = _lib.lib()

    ws = plan.workspace(False)
    refs = []
    for x in flms:
        out = torch.empty(shape, dtype=cdt, device="cuda")
        _lib.check(lib.s2b_inverse(plan.ptr, x.data_ptr(), out.data_ptr(), ws.data_ptr(),
                                   ws.numel(), stream))
        refs.append(out)
    torch.cuda.synchronize()

    outs = [torch.full(shape, float("nan"), dtype=cdt, device="cuda") for _ in flms]
    allocated = torch.cuda.memory_allocated()
    lib_allocs = lib.s2b_device_alloc_count()  # every cudaMalloc the library makes
    for x, out in zip(flms, outs):  # two calls in a row, sharing the scratch array
        _lib.check(lib.s2b_inverse_noalloc(plan.ptr, x.data_ptr(), out.data_ptr(), stream))
    torch.cuda.synchronize()
    assert torch.cuda.memory_allocated() == allocated
    assert lib.s2b_device_alloc_count() == lib_allocs
    for out, ref in zip(outs, refs):
        err = relerr(out.cpu().numpy(), ref.cpu().numpy())
        assert err < TOL[precision], err
    assert plan.status() == 0


def test_noalloc_rejects_plans_beyond_the_scratch_array(cabi):
    import torch

    _lib = cabi
    plan = _plan(_lib, L=64, batch=256)  # float64, about 75 MB of inverse workspace
    need = ctypes.c_size_t()
    _lib.check(_lib.lib().s2b_workspace_size(plan.ptr, 0, ctypes.byref(need)))
    assert need.value > SCRATCH_BYTES
    flm = torch.zeros((256, 64, 127), dtype=torch.complex128, device="cuda")
    f = torch.empty((256, 64, 127), dtype=torch.complex128, device="cuda")
    rc = _lib.lib().s2b_inverse_noalloc(plan.ptr, flm.data_ptr(), f.data_ptr(),
                                        _lib.stream_handle(flm.device))
    assert rc == 3  # S2B_ERR_WORKSPACE
    msg = _lib.lib().s2b_last_error().decode()
    assert "S2B_NOALLOC_SCRATCH_BYTES" in msg and str(need.value) in msg
    rc = _lib.lib().s2b_inverse_noalloc(None, flm.data_ptr(), f.data_ptr(), None)
    assert rc == 1  # S2B_ERR_INVALID: NULL plan
