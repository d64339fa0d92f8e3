"""Spin-subset lifting ops on one B200 (drop-in for
``s2fft.precompute_transforms.custom_ops``).

Mirrors upstream (s2fft/precompute_transforms/custom_ops.py):
  ``wigner_subset_to_s2(flmn, spins, DW, L, sampling)``     (5-83)
  ``so3_to_wigner_subset(f, spins, DW, L, N, sampling)``    (168-205)
  ``s2_to_wigner_subset(fs, spins, DW, L, sampling)``       (251-333)
Arrays carry upstream's layout ``[batch, n_s, ..., channels]``; ``DW`` is
``fourier_wigner.fourier_wigner_kernel(L)`` (or upstream's numpy pair). The work runs in
the Fourier-Wigner kernels of ``libs2b.so`` with (batch x channels) maps per spin; the
channel axis is moved next to the batch axis on the device around each call. The ops are
differentiable in their array input (adjoint entry points ``s2b_fw_*_adjoint``), as
upstream's JAX versions are by autodiff.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .fourier_wigner import (OP_S2_TO_SUBSET, OP_SO3_TO_SUBSET, OP_SUBSET_TO_S2, _cdt,
                             _check_sampling, _fwlib, _geometry, _precomps, get_plan)
from .spherical import _device, _ret, _to_device, _dense, _aligned


def _spins(spins, dev, L):
    sp = np.asarray(spins.cpu() if isinstance(spins, torch.Tensor) else spins).astype(np.int64)
    if sp.ndim != 1 or sp.size == 0:
        raise ValueError("spins must be a non-empty 1-d array")
    if np.abs(sp).max() > L - 1:
        raise ValueError(f"|spin| must be <= L-1 = {L - 1}")
    return sp, torch.as_tensor(sp.astype(np.int32), device=dev)


def _channels_first(x):
    # [batch, s, a, b, ch] -> [batch, ch, s, a, b] contiguous
    return x.permute(0, 4, 1, 2, 3).contiguous()


def _channels_last(x):
    return x.permute(0, 2, 3, 4, 1).contiguous()


class _OpFn(torch.autograd.Function):
    """A linear op on channel-first device arrays: forward call(x, out), backward
    adjoint(g, gx)."""

    @staticmethod
    def forward(ctx, xc, call, adjoint, out_shape):
        xc = _aligned(_dense(xc))
        ctx.adjoint, ctx.in_shape = adjoint, xc.shape
        out = torch.empty(out_shape, dtype=xc.dtype, device=xc.device)
        call(xc, out)
        return out

    @staticmethod
    def backward(ctx, g):
        g = _aligned(_dense(g))
        gx = torch.empty(ctx.in_shape, dtype=g.dtype, device=g.device)
        ctx.adjoint(g, gx)
        return gx, None, None, None


def _apply(xc, call, adjoint, out_shape):
    if xc.requires_grad and torch.is_grad_enabled():
        return _OpFn.apply(xc, call, adjoint, out_shape)
    out = torch.empty(out_shape, dtype=xc.dtype, device=xc.device)
    call(xc, out)
    return out


def wigner_subset_to_s2(flmn, spins, DW, L: int, sampling: str = "mw",
                        precision: str = "f64"):
    """flmn [batch, n_s, L, 2L-1, ch] -> spin maps [batch, n_s, ntheta, nphi, ch]."""
    s = _check_sampling(sampling)
    cdt = _cdt(precision)
    dev = _device()
    x, was_np, odev = _to_device(flmn, cdt, dev)
    sp, spd = _spins(spins, x.device, L)
    if x.shape[1] != sp.shape[0]:
        raise ValueError(
            f"Number of spins specified {sp.shape[0]} does not match the number of Wigner "
            f"coefficients {x.shape[1]}")
    if x.dim() != 5 or tuple(x.shape[2:4]) != (L, 2 * L - 1):
        raise ValueError(f"flmn must have shape [batch, n_s, {L}, {2 * L - 1}, channels]")
    delta, _ = _precomps(DW, L, x.device)
    Bt, S, _, _, C = x.shape
    xc = _channels_first(x)
    nth, nph = _geometry(L, s)
    plan = get_plan(x.device, L, s, precision)

    def run(name):
        def call(a, b):
            ws = plan.workspace(OP_SUBSET_TO_S2, Bt * C, nspins=S)
            _lib.check(getattr(_fwlib(), name)(plan.ptr, Bt * C, S, spd.data_ptr(),
                                               delta.data_ptr(), a.data_ptr(), b.data_ptr(),
                                               ws.data_ptr(), ws.numel(),
                                               _lib.stream_handle(a.device)))
        return call

    out = _apply(xc, run("s2b_fw_subset_to_s2"), run("s2b_fw_subset_to_s2_adjoint"),
                 (Bt, C, S, nth, nph))
    return _ret(_channels_last(out), was_np, odev)


def s2_to_wigner_subset(fs, spins, DW, L: int, sampling: str = "mw", precision: str = "f64"):
    """spin maps fs [batch, n_s, ntheta, nphi, ch] -> [batch, n_s, L, 2L-1, ch]."""
    s = _check_sampling(sampling)
    cdt = _cdt(precision)
    dev = _device()
    x, was_np, odev = _to_device(fs, cdt, dev)
    sp, spd = _spins(spins, x.device, L)
    nth, nph = _geometry(L, s)
    if x.dim() != 5 or x.shape[1] != sp.shape[0] or tuple(x.shape[2:4]) != (nth, nph):
        raise ValueError(f"fs must have shape [batch, {sp.shape[0]}, {nth}, {nph}, channels]")
    delta, quads = _precomps(DW, L, x.device)
    Bt, S, _, _, C = x.shape
    xc = _channels_first(x)
    plan = get_plan(x.device, L, s, precision)

    def run(name):
        def call(a, b):
            ws = plan.workspace(OP_S2_TO_SUBSET, Bt * C, nspins=S)
            _lib.check(getattr(_fwlib(), name)(plan.ptr, Bt * C, S, spd.data_ptr(),
                                               delta.data_ptr(), quads.data_ptr(), a.data_ptr(),
                                               b.data_ptr(), ws.data_ptr(), ws.numel(),
                                               _lib.stream_handle(a.device)))
        return call

    out = _apply(xc, run("s2b_fw_s2_to_subset"), run("s2b_fw_s2_to_subset_adjoint"),
                 (Bt, C, S, L, 2 * L - 1))
    return _ret(_channels_last(out), was_np, odev)


def so3_to_wigner_subset(f, spins, DW, L: int, N: int, sampling: str = "mw",
                         precision: str = "f64"):
    """SO(3) signal f [batch, n_gamma, ntheta, nphi, ch] -> [batch, n_s, L, 2L-1, ch]: the
    gamma DFT at the requested spins, then s2_to_wigner_subset."""
    s = _check_sampling(sampling)
    cdt = _cdt(precision)
    dev = _device()
    x, was_np, odev = _to_device(f, cdt, dev)
    sp, spd = _spins(spins, x.device, L)
    nth, nph = _geometry(L, s)
    if x.dim() != 5 or tuple(x.shape[2:4]) != (nth, nph):
        raise ValueError(f"f must have shape [batch, n_gamma, {nth}, {nph}, channels]")
    delta, quads = _precomps(DW, L, x.device)
    Bt, G, _, _, C = x.shape
    S = sp.shape[0]
    xc = _channels_first(x)
    plan = get_plan(x.device, L, s, precision)

    def run(name):
        def call(a, b):
            ws = plan.workspace(OP_SO3_TO_SUBSET, Bt * C, nspins=S)
            _lib.check(getattr(_fwlib(), name)(plan.ptr, Bt * C, G, S, spd.data_ptr(),
                                               delta.data_ptr(), quads.data_ptr(), a.data_ptr(),
                                               b.data_ptr(), ws.data_ptr(), ws.numel(),
                                               _lib.stream_handle(a.device)))
        return call

    out = _apply(xc, run("s2b_fw_so3_to_subset"), run("s2b_fw_so3_to_subset_adjoint"),
                 (Bt, C, S, L, 2 * L - 1))
    return _ret(_channels_last(out), was_np, odev)
