"""Fourier-Wigner SO(3) transforms on one B200 (drop-in for
``s2fft.precompute_transforms.fourier_wigner`` and ``construct.fourier_wigner_kernel``).

``inverse_transform(flmn, L, N, precomps=None, reality=False, sampling="mw")`` and
``forward_transform(f, L, N, precomps=None, reality=False, sampling="mw")`` follow upstream
(s2fft/precompute_transforms/fourier_wigner.py:13-88, 177-333): the Wigner transform is
factored through the planes Delta^l = d^l(pi/2) and FFTs over (alpha, beta, gamma).
``precomps`` is ``(delta, quads)`` as returned by ``fourier_wigner_kernel(L)``
(construct.py:614-639); without it the kernel is built on the device for the call (and
cached per device and L while the planes take at most 2 GiB). Unlike upstream a leading
batch dimension is accepted, and ``precision="f32"`` runs the transform in float (the planes
stay float64). Complex transforms are differentiable in their input through the adjoint
entry points ``s2b_fw_inverse_adjoint`` / ``s2b_fw_forward_adjoint`` (upstream differentiates
its JAX version by autodiff).
"""

from __future__ import annotations

import ctypes
import math
import threading

import numpy as np
import torch

from . import _lib
from .spherical import _device, _ret, _to_device, _dense, _aligned

_SAMPLINGS = ("mw", "mwss")

_fw_sigs_done = False
_fw_lock = threading.Lock()


def _fwlib():
    """The library with the Fourier-Wigner entry points typed."""
    global _fw_sigs_done
    h = _lib.lib()
    with _fw_lock:
        if not _fw_sigs_done:
            vp, ci, sz = ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t
            sigs = {
                "s2b_fw_plan_create": [ci, ci, ci, ci, ctypes.POINTER(vp)],
                "s2b_fw_plan_destroy": [vp],
                "s2b_fw_quads": [vp, vp, vp],
                "s2b_fw_inverse": [vp, ci, ci, vp, vp, vp, vp, sz, vp],
                "s2b_fw_forward": [vp, ci, ci, vp, vp, vp, vp, vp, sz, vp],
                "s2b_fw_subset_to_s2": [vp, ci, ci, vp, vp, vp, vp, vp, sz, vp],
                "s2b_fw_s2_to_subset": [vp, ci, ci, vp, vp, vp, vp, vp, vp, sz, vp],
                "s2b_fw_so3_to_subset": [vp, ci, ci, ci, vp, vp, vp, vp, vp, vp, sz, vp],
                "s2b_fw_subset_to_s2_adjoint": [vp, ci, ci, vp, vp, vp, vp, vp, sz, vp],
                "s2b_fw_s2_to_subset_adjoint": [vp, ci, ci, vp, vp, vp, vp, vp, vp, sz, vp],
                "s2b_fw_so3_to_subset_adjoint": [vp, ci, ci, ci, vp, vp, vp, vp, vp, vp, sz,
                                                 vp],
                "s2b_fw_inverse_adjoint": [vp, ci, vp, vp, vp, vp, sz, vp],
                "s2b_fw_forward_adjoint": [vp, ci, vp, vp, vp, vp, vp, sz, vp],
            }
            for name, argt in sigs.items():
                fn = getattr(h, name)
                fn.argtypes = argt
                fn.restype = ci
            h.s2b_fw_workspace_size.argtypes = [vp, ci, ci, ci, ci]
            h.s2b_fw_workspace_size.restype = sz
            _fw_sigs_done = True
    return h


OP_INVERSE, OP_FORWARD, OP_SUBSET_TO_S2, OP_S2_TO_SUBSET, OP_SO3_TO_SUBSET = range(5)


class FWPlan:
    """FFT tables of one (L, N, sampling, precision) on one device."""

    def __init__(self, device, L, N, sampling, precision):
        self.device, self.L, self.N = device, L, N
        self.sampling, self.precision = sampling, precision
        ptr = ctypes.c_void_p()
        with torch.cuda.device(device):
            _lib.check(_fwlib().s2b_fw_plan_create(L, N, _lib.SAMPLING[sampling],
                                                   _lib.PRECISION[precision], ctypes.byref(ptr)))
        self.ptr = ptr
        self._ws = {}

    def workspace(self, op, batch, reality=False, nspins=1):
        n = int(_fwlib().s2b_fw_workspace_size(self.ptr, op, batch, int(bool(reality)),
                                                nspins))
        cur = self._ws.get("ws")
        if cur is None or cur.numel() < n:
            cur = torch.empty(max(n, 256), dtype=torch.uint8, device=self.device)
            self._ws["ws"] = cur
        return cur

    def __del__(self):
        try:
            if getattr(self, "ptr", None) and self.ptr.value:
                _fwlib().s2b_fw_plan_destroy(self.ptr)
        except Exception:
            pass


_plans: dict = {}
_kernels: dict = {}
_plans_lock = threading.Lock()


def get_plan(device, L, sampling, precision, N=1) -> FWPlan:
    key = (str(device), L, N, sampling, precision)
    with _plans_lock:
        p = _plans.get(key)
        if p is None:
            p = FWPlan(device, L, N, sampling, precision)
            _plans[key] = p
    return p


def _check_sampling(sampling):
    s = sampling.lower()
    if s not in _SAMPLINGS:
        raise ValueError(f"Fourier-Wigner algorithm does not support {sampling} sampling.")
    return s


def _geometry(L, s):
    return (L + 1, 2 * L) if s == "mwss" else (L, 2 * L - 1)


def fourier_wigner_kernel(L: int):
    """(delta [L, 2L-1, 2L-1] float64, quads [4L-3] complex128), on the current device.

    delta holds d^l_{a,b}(pi/2) (Risbo's recursion on the device, as upstream's
    construct.fourier_wigner_kernel, construct.py:614-639); quads the MW quadrature weights
    upsampled to 4L-3 points."""
    from .rotation import generate_rotate_dls

    dev = _device()
    delta = generate_rotate_dls(L, math.pi / 2)
    quads = torch.empty(4 * L - 3, dtype=torch.complex128, device=dev)
    plan = get_plan(dev, L, "mw", "f64")
    _lib.check(_fwlib().s2b_fw_quads(plan.ptr, quads.data_ptr(), _lib.stream_handle(dev)))
    return delta, quads


# planes built for calls without precomps are kept per (device, L) up to this size; larger
# ones (L (2L-1)^2 float64: 2.1 GB at L=512, 34 GB at L=1024) are rebuilt on every call
_KERNEL_CACHE_BYTES = 1 << 31


def _precomps(precomps, L, dev):
    if precomps is None:
        key = (str(dev), L)
        with _plans_lock:
            k = _kernels.get(key)
        if k is None:
            k = fourier_wigner_kernel(L)
            if k[0].numel() * 8 <= _KERNEL_CACHE_BYTES:
                with _plans_lock:
                    _kernels[key] = k
        return k
    delta, quads = precomps
    delta, _, _ = _to_device(delta, torch.float64, dev)
    quads, _, _ = _to_device(quads, torch.complex128, dev)
    if tuple(delta.shape) != (L, 2 * L - 1, 2 * L - 1):
        raise ValueError(f"delta must have shape {(L, 2 * L - 1, 2 * L - 1)}")
    if tuple(quads.shape) != (4 * L - 3,):
        raise ValueError(f"quads must have shape {(4 * L - 3,)}")
    return delta, quads


def _cdt(precision):
    if precision not in ("f64", "f32"):
        raise ValueError("precision must be 'f64' or 'f32'")
    return torch.complex128 if precision == "f64" else torch.complex64


class _FWInverseFn(torch.autograd.Function):
    """f = inverse_transform(flmn) (complex); backward: s2b_fw_inverse_adjoint."""

    @staticmethod
    def forward(ctx, x, plan, B, delta, out_shape, cdt):
        x = _aligned(_dense(x))
        ctx.plan, ctx.B, ctx.delta, ctx.in_shape = plan, B, delta, x.shape
        out = torch.empty(out_shape, dtype=cdt, device=x.device)
        ws = plan.workspace(OP_INVERSE, B, False)
        _lib.check(_fwlib().s2b_fw_inverse(plan.ptr, B, 0, delta.data_ptr(), x.data_ptr(),
                                           out.data_ptr(), ws.data_ptr(), ws.numel(),
                                           _lib.stream_handle(x.device)))
        return out

    @staticmethod
    def backward(ctx, g):
        g = _aligned(_dense(g))
        gx = torch.empty(ctx.in_shape, dtype=g.dtype, device=g.device)
        ws = ctx.plan.workspace(OP_INVERSE, ctx.B, False)
        _lib.check(_fwlib().s2b_fw_inverse_adjoint(ctx.plan.ptr, ctx.B, ctx.delta.data_ptr(),
                                                   g.data_ptr(), gx.data_ptr(), ws.data_ptr(),
                                                   ws.numel(), _lib.stream_handle(g.device)))
        return gx, None, None, None, None, None


class _FWForwardFn(torch.autograd.Function):
    """flmn = forward_transform(f) (complex); backward: s2b_fw_forward_adjoint."""

    @staticmethod
    def forward(ctx, x, plan, B, delta, quads, out_shape, cdt):
        x = _aligned(_dense(x))
        ctx.plan, ctx.B, ctx.delta, ctx.quads, ctx.in_shape = plan, B, delta, quads, x.shape
        out = torch.empty(out_shape, dtype=cdt, device=x.device)
        ws = plan.workspace(OP_FORWARD, B, False)
        _lib.check(_fwlib().s2b_fw_forward(plan.ptr, B, 0, delta.data_ptr(), quads.data_ptr(),
                                           x.data_ptr(), out.data_ptr(), ws.data_ptr(),
                                           ws.numel(), _lib.stream_handle(x.device)))
        return out

    @staticmethod
    def backward(ctx, g):
        g = _aligned(_dense(g))
        gx = torch.empty(ctx.in_shape, dtype=g.dtype, device=g.device)
        ws = ctx.plan.workspace(OP_FORWARD, ctx.B, False)
        _lib.check(_fwlib().s2b_fw_forward_adjoint(
            ctx.plan.ptr, ctx.B, ctx.delta.data_ptr(), ctx.quads.data_ptr(), g.data_ptr(),
            gx.data_ptr(), ws.data_ptr(), ws.numel(), _lib.stream_handle(g.device)))
        return gx, None, None, None, None, None, None


def _needs_grad(x, reality):
    if not (isinstance(x, torch.Tensor) and x.requires_grad and torch.is_grad_enabled()):
        return False
    if reality:
        raise NotImplementedError("gradients are available for complex transforms (reality=False)")
    return True


def inverse_transform(flmn, L: int, N: int, precomps=None, reality: bool = False,
                      sampling: str = "mw", precision: str = "f64"):
    """flmn [..., 2N-1, L, 2L-1] -> f [..., 2N-1, ntheta, nphi] (real when reality)."""
    s = _check_sampling(sampling)
    cdt = _cdt(precision)
    dev = _device()
    x, was_np, odev = _to_device(flmn, cdt, dev)
    if tuple(x.shape[-3:]) != (2 * N - 1, L, 2 * L - 1):
        raise ValueError(f"flmn must have trailing shape {(2 * N - 1, L, 2 * L - 1)}")
    bs = tuple(x.shape[:-3])
    B = int(np.prod(bs)) if bs else 1
    delta, _ = _precomps(precomps, L, x.device)
    nth, nph = _geometry(L, s)
    rdt = torch.float64 if precision == "f64" else torch.float32
    out = torch.empty(bs + (2 * N - 1, nth, nph), dtype=rdt if reality else cdt,
                      device=x.device)
    plan = get_plan(x.device, L, s, precision, N)
    if _needs_grad(x, reality):
        return _ret(_FWInverseFn.apply(x, plan, B, delta, out.shape, cdt), was_np, odev)
    ws = plan.workspace(OP_INVERSE, B, reality)
    _lib.check(_fwlib().s2b_fw_inverse(plan.ptr, B, int(bool(reality)), delta.data_ptr(),
                                       x.data_ptr(), out.data_ptr(), ws.data_ptr(), ws.numel(),
                                       _lib.stream_handle(x.device)))
    return _ret(out, was_np, odev)


def forward_transform(f, L: int, N: int, precomps=None, reality: bool = False,
                      sampling: str = "mw", precision: str = "f64"):
    """f [..., 2N-1, ntheta, nphi] -> flmn [..., 2N-1, L, 2L-1]."""
    s = _check_sampling(sampling)
    cdt = _cdt(precision)
    rdt = torch.float64 if precision == "f64" else torch.float32
    dev = _device()
    if reality:
        # upstream takes np.real(f) before the real FFT over gamma
        if isinstance(f, torch.Tensor) and f.is_complex():
            f = f.real
        elif isinstance(f, np.ndarray) and np.iscomplexobj(f):
            f = np.real(f)
    x, was_np, odev = _to_device(f, rdt if reality else cdt, dev)
    nth, nph = _geometry(L, s)
    if tuple(x.shape[-3:]) != (2 * N - 1, nth, nph):
        raise ValueError(f"f must have trailing shape {(2 * N - 1, nth, nph)}")
    bs = tuple(x.shape[:-3])
    B = int(np.prod(bs)) if bs else 1
    delta, quads = _precomps(precomps, L, x.device)
    out = torch.empty(bs + (2 * N - 1, L, 2 * L - 1), dtype=cdt, device=x.device)
    plan = get_plan(x.device, L, s, precision, N)
    if _needs_grad(x, reality):
        return _ret(_FWForwardFn.apply(x, plan, B, delta, quads, out.shape, cdt), was_np, odev)
    ws = plan.workspace(OP_FORWARD, B, reality)
    _lib.check(_fwlib().s2b_fw_forward(plan.ptr, B, int(bool(reality)), delta.data_ptr(),
                                       quads.data_ptr(), x.data_ptr(), out.data_ptr(),
                                       ws.data_ptr(), ws.numel(), _lib.stream_handle(x.device)))
    return _ret(out, was_np, odev)
