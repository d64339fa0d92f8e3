"""Plans are bound to the device they were created on.

A plan's tables live on one GPU; an execute call launches on the current
device. Every execute entry point compares the two and returns
S2B_ERR_INVALID, before launching anything, when they differ. With one GPU the
mismatch is produced by overwriting the plan's recorded ordinal through the
testing hook s2b_debug_set_plan_device, so no kernel ever sees another
device's pointers.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cabi():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from s2fft_b200 import _lib

    return _lib


def _plan(_lib, **kw):
    import torch

    desc = dict(L=16, spin=0, nside=0, sampling=0, reality=0, L_lower=0, precision=0, batch=1,
                iter=0, N=0)
    desc.update(kw)
    return _lib.Plan(torch.device("cuda", torch.cuda.current_device()), **desc)


def _expect_wrong_device(_lib, rc):
    assert rc == 1, rc  # S2B_ERR_INVALID
    msg = _lib.lib().s2b_last_error().decode()
    assert "not the plan's device" in msg, msg


def test_plan_records_its_device(cabi):
    import torch

    plan = _plan(cabi)
    dev = ctypes.c_int(-7)
    cabi.check(cabi.lib().s2b_plan_device(plan.ptr, ctypes.byref(dev)))
    assert dev.value == torch.cuda.current_device()


def test_execute_calls_reject_another_device(cabi):
    import torch

    _lib = cabi
    lib = _lib.lib()
    L = 16
    me = torch.cuda.current_device()
    plan = _plan(_lib, L=L)
    flm = torch.zeros((L, 2 * L - 1), dtype=torch.complex128, device="cuda")
    f = torch.zeros((L, 2 * L - 1), dtype=torch.complex128, device="cuda")
    stream = _lib.stream_handle(flm.device)
    ws = [plan.workspace(k) for k in range(4)]
    ksz = ctypes.c_size_t()
    _lib.check(lib.s2b_kernel_size(plan.ptr, 0, ctypes.byref(ksz)))
    K = torch.zeros(max(int(ksz.value), 256), dtype=torch.uint8, device="cuda")

    _lib.check(lib.s2b_debug_set_plan_device(plan.ptr, me + 1))
    try:
        calls = [
            lambda: lib.s2b_inverse(plan.ptr, flm.data_ptr(), f.data_ptr(), ws[0].data_ptr(),
                                    ws[0].numel(), stream),
            lambda: lib.s2b_forward(plan.ptr, f.data_ptr(), flm.data_ptr(), ws[1].data_ptr(),
                                    ws[1].numel(), stream),
            lambda: lib.s2b_inverse_adjoint(plan.ptr, f.data_ptr(), flm.data_ptr(),
                                            ws[2].data_ptr(), ws[2].numel(), stream),
            lambda: lib.s2b_forward_adjoint(plan.ptr, flm.data_ptr(), f.data_ptr(),
                                            ws[3].data_ptr(), ws[3].numel(), stream),
            lambda: lib.s2b_inverse_noalloc(plan.ptr, flm.data_ptr(), f.data_ptr(), stream),
            lambda: lib.s2b_kernel_build(plan.ptr, 0, K.data_ptr(), stream),
            lambda: lib.s2b_precompute_inverse(plan.ptr, K.data_ptr(), flm.data_ptr(),
                                               f.data_ptr(), ws[0].data_ptr(), ws[0].numel(),
                                               stream),
        ]
        for call in calls:
            _expect_wrong_device(_lib, call())
    finally:
        _lib.check(lib.s2b_debug_set_plan_device(plan.ptr, me))
    torch.cuda.synchronize()
    # the rejected calls launched nothing; with the ordinal restored the plan works again
    x = torch.from_numpy(np.random.default_rng(3).standard_normal((L, 2 * L - 1)) + 0j).to("cuda")
    _lib.check(lib.s2b_inverse(plan.ptr, x.data_ptr(), f.data_ptr(), ws[0].data_ptr(),
                               ws[0].numel(), stream))
    torch.cuda.synchronize()
    assert torch.isfinite(torch.view_as_real(f)).all()
    assert plan.status() == 0


def test_wigner_and_healpix_plans_reject_another_device(cabi):
    import torch

    _lib = cabi
    lib = _lib.lib()
    me = torch.cuda.current_device()
    L, N = 8, 2
    wplan = _plan(_lib, L=L, N=N)
    flmn = torch.zeros((2 * N - 1, L, 2 * L - 1), dtype=torch.complex128, device="cuda")
    fso3 = torch.zeros((2 * N - 1, L, 2 * L - 1), dtype=torch.complex128, device="cuda")
    ws = wplan.workspace(0)
    stream = _lib.stream_handle(flmn.device)
    hplan = _plan(_lib, L=8, sampling=4, nside=4)
    fmap = torch.zeros(12 * 16, dtype=torch.complex128, device="cuda")
    ftm = torch.zeros((15, 16), dtype=torch.complex128, device="cuda")
    for plan in (wplan, hplan):
        _lib.check(lib.s2b_debug_set_plan_device(plan.ptr, me + 3))
    try:
        _expect_wrong_device(_lib, lib.s2b_wigner_inverse(
            wplan.ptr, flmn.data_ptr(), fso3.data_ptr(), ws.data_ptr(), ws.numel(), stream))
        _expect_wrong_device(_lib, lib.s2b_wigner_forward(
            wplan.ptr, fso3.data_ptr(), flmn.data_ptr(), ws.data_ptr(), ws.numel(), stream))
        _expect_wrong_device(_lib, lib.s2b_healpix_fft(hplan.ptr, fmap.data_ptr(),
                                                       ftm.data_ptr(), stream))
        _expect_wrong_device(_lib, lib.s2b_healpix_ifft(hplan.ptr, ftm.data_ptr(),
                                                        fmap.data_ptr(), stream))
    finally:
        for plan in (wplan, hplan):
            _lib.check(lib.s2b_debug_set_plan_device(plan.ptr, me))
    torch.cuda.synchronize()
    assert wplan.status() == 0 and hplan.status() == 0
