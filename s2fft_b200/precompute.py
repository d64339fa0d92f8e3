"""Drop-in precompute-kernel transforms on one B200.

Precision "bf16x3" runs the contractions (forward and inverse) on the tcgen05 tensor
cores with 3-term bf16 split operands (its kernels are opaque packed buffers).

Mirrors upstream ``s2fft.precompute_transforms.spherical.inverse`` / ``forward``
(s2fft/precompute_transforms/spherical.py:19-84, 226-311) and
``construct.spin_spherical_kernel`` (construct.py:16-161). The kernel table
K[t, l, m] has the upstream layout and meaning; here it is built on the device
and returned as a torch tensor (an upstream numpy kernel is accepted too).
"""

from __future__ import annotations

import ctypes
from warnings import warn

import numpy as np
import torch

from . import _lib
from .spherical import _check_method, _device, _dtypes, _ret, _to_device, f_shape, _dense


def _plan(dev, L, spin, nside, s, reality, precision, B):
    return _lib.get_plan(dev, L=L, spin=spin, nside=nside or 0, sampling=_lib.SAMPLING[s],
                         reality=int(bool(reality)), L_lower=0,
                         precision=_lib.PRECISION[precision], batch=B, iter=0, N=0)


def _kernel_shape(L, s, nside, reality, forward):
    M = L if reality else 2 * L - 1
    if forward and s in ("mw", "mwss"):
        nth = 2 * L + 1
    else:
        nth = f_shape(L, s, nside)[0] if s != "healpix" else 4 * nside - 1
    return nth, L, M


def _reality(reality, spin):
    if reality and spin != 0:
        warn("Reality acceleration only supports spin 0 fields. Defering to complex transform.",
             stacklevel=3)
        return False
    return reality


def spin_spherical_kernel(L: int, spin: int = 0, reality: bool = False, sampling: str = "mw",
                          nside: int = None, forward: bool = True, recursion: str = "auto",
                          precision: str = "f64"):
    """Kernel K[t, l, m] built on the device (torch tensor on the current CUDA device)."""
    s = sampling.lower()
    reality = _reality(reality, spin)
    _, rdt = _dtypes(precision)
    cdt = _dtypes(precision)[0]
    dev = _device()
    plan = _plan(dev, L, spin, nside, s, reality, precision, 1)
    n = ctypes.c_size_t()
    _lib.check(_lib.lib().s2b_kernel_size(plan.ptr, int(forward), ctypes.byref(n)))
    if precision == "bf16x3":
        # packed bf16 hi/lo operand tiles for the tensor-core contraction (opaque)
        K = torch.empty(n.value, dtype=torch.uint8, device=dev)
    else:
        shape = _kernel_shape(L, s, nside, reality, forward)
        K = torch.empty(shape, dtype=cdt if s == "healpix" else rdt, device=dev)
        assert n.value == K.numel() * K.element_size()
    _lib.check(_lib.lib().s2b_kernel_build(plan.ptr, int(forward), K.data_ptr(),
                                           _lib.stream_handle(dev)))
    return K


def _kernel_tensor(kernel, L, s, nside, reality, forward, precision, spin, dev):
    cdt, rdt = _dtypes(precision)
    if kernel is None:
        return spin_spherical_kernel(L, spin, reality, s, nside, forward, precision=precision)
    if precision == "bf16x3":
        if not (isinstance(kernel, torch.Tensor) and kernel.dtype == torch.uint8):
            raise ValueError("bf16x3 needs the packed kernel from spin_spherical_kernel")
        return kernel.to(dev)
    want = cdt if s == "healpix" else rdt
    if isinstance(kernel, np.ndarray):
        kernel = torch.from_numpy(np.ascontiguousarray(kernel))
    return _aligned(kernel.to(device=dev, dtype=want).contiguous())


def _aligned(t):
    # the C ABI takes 16-byte aligned operands (a slice of a stacked kernel may not be)
    return t if t.data_ptr() % 16 == 0 else t.clone()


def _pre_call(name, plan, K, x, out, forward):
    ws = plan.workspace(forward)
    _lib.check(getattr(_lib.lib(), name)(plan.ptr, K.data_ptr(), x.data_ptr(), out.data_ptr(),
                                         ws.data_ptr(), ws.numel(),
                                         _lib.stream_handle(x.device)))
    return out


class _PreInverseFn(torch.autograd.Function):
    """f = precompute inverse(flm); backward: s2b_precompute_inverse_adjoint."""

    @staticmethod
    def forward(ctx, x, plan, K, out_shape, cdt):
        x = _aligned(_dense(x))
        ctx.plan, ctx.K, ctx.in_shape = plan, K, x.shape
        out = torch.empty(out_shape, dtype=cdt, device=x.device)
        return _pre_call("s2b_precompute_inverse", plan, K, x, out, False)

    @staticmethod
    def backward(ctx, g):
        g = _aligned(_dense(g))
        gx = torch.empty(ctx.in_shape, dtype=g.dtype, device=g.device)
        _pre_call("s2b_precompute_inverse_adjoint", ctx.plan, ctx.K, g, gx, False)
        return gx, None, None, None, None


class _PreForwardFn(torch.autograd.Function):
    """flm = precompute forward(f) (one pass); backward: s2b_precompute_forward_adjoint."""

    @staticmethod
    def forward(ctx, x, plan, K, out_shape, cdt):
        x = _aligned(_dense(x))
        ctx.plan, ctx.K, ctx.in_shape = plan, K, x.shape
        out = torch.empty(out_shape, dtype=cdt, device=x.device)
        return _pre_call("s2b_precompute_forward", plan, K, x, out, True)

    @staticmethod
    def backward(ctx, g):
        g = _aligned(_dense(g))
        gx = torch.empty(ctx.in_shape, dtype=g.dtype, device=g.device)
        _pre_call("s2b_precompute_forward_adjoint", ctx.plan, ctx.K, g, gx, True)
        return gx, None, None, None, None


def _needs_grad(x, reality, precision):
    if not (isinstance(x, torch.Tensor) and x.requires_grad and torch.is_grad_enabled()):
        return False
    if reality or precision == "bf16x3":
        raise NotImplementedError("precompute gradients need complex transforms "
                                  "(reality=False) with f64 or f32 kernels")
    return True


def inverse(flm, L: int, spin: int = 0, kernel=None, sampling: str = "mw",
            reality: bool = False, method: str = "cuda", nside: int = None,
            precision: str = "f64"):
    """Inverse spin SHT through a precomputed kernel (upstream spherical.py:19-84).
    Differentiable in flm (complex transforms, f64 / f32 kernels)."""
    _check_method(method)
    s = sampling.lower()
    reality = _reality(reality, spin)
    cdt, rdt = _dtypes(precision)
    x, was_np, odev = _to_device(flm, cdt, _device())
    bs = tuple(x.shape[:-2])
    B = int(np.prod(bs)) if bs else 1
    K = _kernel_tensor(kernel, L, s, nside, reality, False, precision, spin, x.device)
    plan = _plan(x.device, L, spin, nside, s, reality, precision, B)
    if _needs_grad(x, reality, precision):
        return _ret(_PreInverseFn.apply(x, plan, K, bs + f_shape(L, s, nside), cdt), was_np,
                    odev)
    out = torch.empty(bs + f_shape(L, s, nside), dtype=rdt if reality else cdt, device=x.device)
    return _ret(_pre_call("s2b_precompute_inverse", plan, K, x, out, False), was_np, odev)


def _forward_once(x, K, L, spin, s, nside, reality, precision):
    cdt, _ = _dtypes(precision)
    nd = len(f_shape(L, s, nside))
    bs = tuple(x.shape[:-nd])
    B = int(np.prod(bs)) if bs else 1
    plan = _plan(x.device, L, spin, nside, s, reality, precision, B)
    if _needs_grad(x, reality, precision):
        return _PreForwardFn.apply(x, plan, K, bs + (L, 2 * L - 1), cdt)
    out = torch.empty(bs + (L, 2 * L - 1), dtype=cdt, device=x.device)
    return _pre_call("s2b_precompute_forward", plan, K, x, out, True)


def forward(f, L: int, spin: int = 0, kernel=None, sampling: str = "mw",
            reality: bool = False, method: str = "cuda", nside: int = None, iter: int = 0,
            precision: str = "f64"):
    """Forward spin SHT through a precomputed kernel (upstream spherical.py:226-311)."""
    _check_method(method)
    s = sampling.lower()
    reality = _reality(reality, spin)
    cdt, rdt = _dtypes(precision)
    if reality:
        if isinstance(f, torch.Tensor) and f.is_complex():
            f = f.real
        elif isinstance(f, np.ndarray) and np.iscomplexobj(f):
            f = np.real(f)
    x, was_np, odev = _to_device(f, rdt if reality else cdt, _device())
    K = _kernel_tensor(kernel, L, s, nside, reality, True, precision, spin, x.device)
    flm = _forward_once(x, K, L, spin, s, nside, reality, precision)
    if iter:
        Ki = spin_spherical_kernel(L, spin, reality, s, nside, False, precision=precision)
        for _ in range(iter):
            fr = inverse(flm, L, spin, Ki, s, reality, method, nside, precision)
            flm = flm + _forward_once(x - fr, K, L, spin, s, nside, reality, precision)
    return _ret(flm, was_np, odev)


# ---------------------------------------------------------------------------------------
# Precompute-kernel Wigner (SO(3)) transforms
# (s2fft/precompute_transforms/wigner.py:13-467, construct.py:332-470)
# ---------------------------------------------------------------------------------------
def _wigner_ns(N, reality):
    return range(0 if reality else -(N - 1), N)


def _wigner_l_factor(L, N, n, forward, dev, dtype):
    l = np.arange(L, dtype=np.float64)
    if forward:
        v = (-1.0) ** n * (2 * np.pi / (2 * N - 1)) / np.sqrt((2 * l + 1) / (4 * np.pi))
    else:
        v = (-1.0) ** n * np.sqrt((2 * l + 1) / (16 * np.pi ** 3))
    return torch.from_numpy(v).to(device=dev, dtype=dtype)[None, :, None]


def wigner_kernel(L: int, N: int, reality: bool = False, sampling: str = "mw",
                  nside: int = None, forward: bool = False, mode: str = "auto",
                  precision: str = "f64"):
    """Wigner-d kernel K[n, t, l, m] in the upstream layout (construct.py:332-470):
    d^l_{m,n}(theta_t) (2l+1)/(8 pi^2) for the inverse, d^l_{m,n}(theta_t) w_t 2pi/(2N-1)
    for the forward (MWSS(2L) rings for mw / mwss), HEALPix ring phases folded in;
    n >= 0 only when ``reality``. Built on the device from the spin kernels of spin -n
    (``mode`` is accepted for signature compatibility: the recursion is always the
    on-device one)."""
    s = sampling.lower()
    if precision == "bf16x3":
        raise ValueError("Wigner kernels are built in f64 or f32")
    dev = _device()
    slabs = []
    for n in _wigner_ns(N, reality):
        K = spin_spherical_kernel(L, -n, False, s, nside, forward, precision=precision)
        slabs.append(K * _wigner_l_factor(L, N, n, forward, dev, K.real.dtype))
    return torch.stack(slabs)


def _wigner_kernel_tensor(kernel, L, N, s, nside, reality, forward, precision, dev):
    if kernel is None:
        return wigner_kernel(L, N, reality, s, nside, forward, precision=precision)
    cdt, rdt = _dtypes(precision)
    want = cdt if s == "healpix" else rdt
    if isinstance(kernel, np.ndarray):
        kernel = torch.from_numpy(np.ascontiguousarray(kernel))
    return kernel.to(device=dev, dtype=want).contiguous()


def wigner_inverse(flmn, L: int, N: int, kernel=None, sampling: str = "mw",
                   reality: bool = False, method: str = "cuda", nside: int = None,
                   precision: str = "f64"):
    """Inverse Wigner transform through a precomputed kernel
    (upstream precompute_transforms/wigner.py:13-221): per n the contraction with the
    kernel slice and the phi FFT (the spin precompute inverse of spin -n), then the
    unnormalised inverse DFT over gamma."""
    _check_method(method)
    s = sampling.lower()
    cdt, rdt = _dtypes(precision)
    x, was_np, odev = _to_device(flmn, cdt, _device())
    K = _wigner_kernel_tensor(kernel, L, N, s, nside, reality, False, precision, x.device)
    G = 2 * N - 1
    fs = []
    for j, n in enumerate(_wigner_ns(N, reality)):
        fs.append(inverse(x[..., N - 1 + n, :, :], L, -n, K[j], s, False, method, nside,
                          precision))
    gdim = len(f_shape(L, s, nside))
    fban = torch.stack(fs, dim=-gdim - 1)
    ns = np.array(list(_wigner_ns(N, reality)))
    k = np.arange(G)
    P = np.exp(2j * np.pi * np.outer(ns, k) / G)  # [n, k]
    if reality:
        P[ns > 0] *= 2.0
    Pt = torch.from_numpy(P).to(device=x.device, dtype=cdt)
    f = torch.movedim(torch.tensordot(fban, Pt, dims=([-gdim - 1], [0])), -1, -gdim - 1)
    if reality:
        f = f.real.contiguous()
    return _ret(f, was_np, odev)


def wigner_forward(f, L: int, N: int, kernel=None, sampling: str = "mw",
                   reality: bool = False, method: str = "cuda", nside: int = None,
                   precision: str = "f64"):
    """Forward Wigner transform through a precomputed kernel
    (upstream precompute_transforms/wigner.py:224-371): unnormalised DFT over gamma, then
    per n the spin precompute forward of spin -n (MW / MWSS resampling, phi FFT and the
    contraction with the kernel slice); n < 0 from the conjugate symmetry when ``reality``."""
    _check_method(method)
    s = sampling.lower()
    cdt, rdt = _dtypes(precision)
    x, was_np, odev = _to_device(f, cdt, _device())
    K = _wigner_kernel_tensor(kernel, L, N, s, nside, reality, True, precision, x.device)
    G = 2 * N - 1
    gdim = len(f_shape(L, s, nside))
    ns = np.array(list(_wigner_ns(N, reality)))
    P = np.exp(-2j * np.pi * np.outer(np.arange(G), ns) / G)  # [k, n]
    Pt = torch.from_numpy(P).to(device=x.device, dtype=cdt)
    fin = x.real.to(cdt) if reality else x
    fban = torch.movedim(torch.tensordot(fin, Pt, dims=([-gdim - 1], [0])), -1, -gdim - 1)
    bs = tuple(x.shape[:-gdim - 1])
    out = torch.zeros(bs + (G, L, 2 * L - 1), dtype=cdt, device=x.device)
    for j, n in enumerate(ns):
        fb = fban.select(-gdim - 1, j).contiguous()
        out[..., N - 1 + n, :, :] = forward(fb, L, int(-n), K[j], s, False, method, nside,
                                            0, precision)
    if reality:
        m = torch.arange(-(L - 1), L, device=x.device)
        sm = ((-1.0) ** m.abs()).to(cdt)
        for n in range(1, N):
            out[..., N - 1 - n, :, :] = (-1.0) ** n * torch.flip(
                out[..., N - 1 + n, :, :].conj(), dims=(-1,)) * sm
    return _ret(out, was_np, odev)
