"""Drop-in spin spherical-harmonic transforms on one B200.

Same call surface as upstream ``s2fft.forward`` / ``s2fft.inverse``
(s2fft/transforms/spherical.py:21-109 and 352-464): positional order
``(flm|f, L, spin, nside, sampling, method, reality, precomps, spmd, L_lower)``
plus ``iter`` for the forward transform. The method string selects the
implementation; ``"cuda"`` (the default here) runs the sm_100a kernels of
``libs2b.so``. Upstream method names that need JAX or CPU libraries raise.

Extra keyword ``precision``: ``"f64"`` (default, complex128 in and out) or
``"f32"`` (float32 recursion and projection with double seeds, exponent
bookkeeping and weights; complex64 arrays).

Inputs may be numpy arrays (returned as numpy) or torch tensors (returned as
torch tensors on the same device). A leading batch dimension is accepted.

Differentiation: when a torch input requires grad, the transforms run as
``torch.autograd.Function``s whose backward passes call the adjoint kernels
(``s2b_inverse_adjoint`` / ``s2b_forward_adjoint``, recomputing the Wigner-d
recursion instead of storing it); refinement iterations are composed from the
single passes. Complex transforms only (``reality=False``).
"""

from __future__ import annotations

import numpy as np
import torch

from . import _lib

_METHODS = ("cuda",)
_UPSTREAM_ONLY = ("numpy", "jax", "jax_cuda", "jax_ssht", "jax_healpy", "torch")


def _check_method(method):
    if method in _UPSTREAM_ONLY:
        raise ValueError(
            f"Method {method} is provided by upstream s2fft; this package implements 'cuda'.")
    if method not in _METHODS:
        raise ValueError(f"Method {method} not recognised.")


def _check_args(L, spin, nside, sampling, reality, L_lower):
    s = sampling.lower()
    if s not in _lib.SAMPLING:
        raise ValueError(f"Sampling scheme sampling={sampling} not supported")
    if spin >= 8:
        # upstream raises Warning for the recursive methods (spherical.py:88-89)
        raise Warning("Recursive transform may provide lower precision beyond spin ~ 8")
    if s == "healpix":
        if nside is None:
            raise ValueError(f"Sampling scheme sampling={sampling} with nside={nside} not supported")
        assert L >= 2 * nside
    if reality and spin != 0:
        raise ValueError("reality=True requires spin 0")
    if not 0 <= L_lower < L:
        raise ValueError("L_lower must satisfy 0 <= L_lower < L")
    return s


def f_shape(L, sampling="mw", nside=None):
    s = sampling.lower()
    if s == "healpix":
        return (12 * nside**2,)
    nth = {"mw": L, "gl": L, "mwss": L + 1, "dh": 2 * L}[s]
    nph = 2 * L if s == "mwss" else 2 * L - 1
    return nth, nph


def flm_shape(L):
    return L, 2 * L - 1


def _device():
    if not torch.cuda.is_available():
        raise RuntimeError("s2fft_b200 needs a CUDA device (no CPU fallback)")
    return torch.device("cuda", torch.cuda.current_device())


def _aligned(t):
    # the C ABI takes 16-byte aligned operands; a view into a larger tensor may not be
    return t if t.data_ptr() % 16 == 0 else t.clone()


def _to_device(x, dtype, device):
    """(contiguous, 16-byte aligned tensor on device, was_numpy, original device)."""
    if isinstance(x, np.ndarray):
        t = torch.from_numpy(np.ascontiguousarray(x))
        return _aligned(t.to(device=device, dtype=dtype).contiguous()), True, None
    if isinstance(x, torch.Tensor):
        dev = x.device
        t = x.to(device=device if dev.type != "cuda" else dev, dtype=dtype).contiguous()
        return _aligned(t), False, dev
    t = torch.as_tensor(np.asarray(x))
    return _aligned(t.to(device=device, dtype=dtype).contiguous()), True, None


def _ret(t, was_numpy, dev):
    if was_numpy:
        return t.cpu().numpy()
    if dev is not None and dev.type != "cuda":
        return t.to(dev)
    return t


def _dtypes(precision):
    if precision not in _lib.PRECISION:
        raise ValueError("precision must be 'f64', 'f32' or 'bf16x3'")
    return (torch.complex128, torch.float64) if precision == "f64" else (torch.complex64,
                                                                          torch.float32)


class _InverseFn(torch.autograd.Function):
    """f = inverse(flm); backward applies the adjoint kernel (s2b_inverse_adjoint)."""

    @staticmethod
    def forward(ctx, flm, plan, f_shape_full, out_dtype):
        out = torch.empty(f_shape_full, dtype=out_dtype, device=flm.device)
        ws = plan.workspace(0)
        _lib.check(_lib.lib().s2b_inverse(plan.ptr, flm.data_ptr(), out.data_ptr(),
                                          ws.data_ptr(), ws.numel(),
                                          _lib.stream_handle(flm.device)))
        ctx.plan = plan
        ctx.in_shape = flm.shape
        return out

    @staticmethod
    def backward(ctx, g):
        g = g.contiguous()
        gflm = torch.empty(ctx.in_shape, dtype=g.dtype, device=g.device)
        ws = ctx.plan.workspace(2)
        _lib.check(_lib.lib().s2b_inverse_adjoint(ctx.plan.ptr, g.data_ptr(), gflm.data_ptr(),
                                                  ws.data_ptr(), ws.numel(),
                                                  _lib.stream_handle(g.device)))
        return gflm, None, None, None


class _ForwardFn(torch.autograd.Function):
    """flm = forward(f) (single pass); backward applies s2b_forward_adjoint."""

    @staticmethod
    def forward(ctx, f, plan, flm_shape_full, out_dtype):
        out = torch.empty(flm_shape_full, dtype=out_dtype, device=f.device)
        ws = plan.workspace(1)
        _lib.check(_lib.lib().s2b_forward(plan.ptr, f.data_ptr(), out.data_ptr(),
                                          ws.data_ptr(), ws.numel(),
                                          _lib.stream_handle(f.device)))
        ctx.plan = plan
        ctx.in_shape = f.shape
        return out

    @staticmethod
    def backward(ctx, g):
        g = g.contiguous()
        gf = torch.empty(ctx.in_shape, dtype=g.dtype, device=g.device)
        ws = ctx.plan.workspace(3)
        _lib.check(_lib.lib().s2b_forward_adjoint(ctx.plan.ptr, g.data_ptr(), gf.data_ptr(),
                                                  ws.data_ptr(), ws.numel(),
                                                  _lib.stream_handle(g.device)))
        return gf, None, None, None


def _needs_grad(x):
    return isinstance(x, torch.Tensor) and x.requires_grad and torch.is_grad_enabled()


def inverse(flm, L: int, spin: int = 0, nside: int = None, sampling: str = "mw",
            method: str = "cuda", reality: bool = False, precomps=None, spmd: bool = False,
            L_lower: int = 0, _ssht_backend: int = 1, precision: str = "f64"):
    """Inverse spin-SHT: flm [.., L, 2L-1] -> f on the sampling grid."""
    _check_method(method)
    s = _check_args(L, spin, nside, sampling, reality, L_lower)
    cdt, rdt = _dtypes(precision)
    dev = _device()
    x, was_np, odev = _to_device(flm, cdt, dev)
    batch_shape = tuple(x.shape[:-2])
    if tuple(x.shape[-2:]) != (L, 2 * L - 1):
        raise ValueError(f"flm must have trailing shape {(L, 2 * L - 1)}, got {tuple(x.shape)}")
    B = int(np.prod(batch_shape)) if batch_shape else 1
    plan = _lib.get_plan(x.device, L=L, spin=spin, nside=nside or 0, sampling=_lib.SAMPLING[s],
                         reality=int(bool(reality)), L_lower=L_lower,
                         precision=_lib.PRECISION[precision], batch=B, iter=0, N=0)
    if _needs_grad(x):
        if reality:
            raise NotImplementedError("gradients are available for complex transforms (reality=False)")
        return _ret(_InverseFn.apply(x, plan, batch_shape + f_shape(L, s, nside), cdt),
                    was_np, odev)
    out = torch.empty(batch_shape + f_shape(L, s, nside), dtype=rdt if reality else cdt,
                      device=x.device)
    ws = plan.workspace(False)
    _lib.check(_lib.lib().s2b_inverse(plan.ptr, x.data_ptr(), out.data_ptr(), ws.data_ptr(),
                                      ws.numel(), _lib.stream_handle(x.device)))
    return _ret(out, was_np, odev)


def forward(f, L: int, spin: int = 0, nside: int = None, sampling: str = "mw",
            method: str = "cuda", reality: bool = False, precomps=None, spmd: bool = False,
            L_lower: int = 0, iter: int = None, _ssht_backend: int = 1,
            precision: str = "f64"):
    """Forward spin-SHT: f on the sampling grid -> flm [.., L, 2L-1].

    ``iter`` Jacobi refinement iterations (upstream default: 0 except for the
    healpy backend; spherical.py:431-432).
    """
    _check_method(method)
    s = _check_args(L, spin, nside, sampling, reality, L_lower)
    if iter is None:
        iter = 0
    cdt, rdt = _dtypes(precision)
    dev = _device()
    if reality:
        if isinstance(f, torch.Tensor) and f.is_complex():
            f = f.real
        elif isinstance(f, np.ndarray) and np.iscomplexobj(f):
            f = np.real(f)
    x, was_np, odev = _to_device(f, rdt if reality else cdt, dev)
    fs = f_shape(L, s, nside)
    nd = len(fs)
    if tuple(x.shape[-nd:]) != fs:
        raise ValueError(f"f must have trailing shape {fs}, got {tuple(x.shape)}")
    batch_shape = tuple(x.shape[:-nd])
    B = int(np.prod(batch_shape)) if batch_shape else 1
    if _needs_grad(x):
        if reality:
            raise NotImplementedError("gradients are available for complex transforms (reality=False)")
        # refinement flm <- flm + F(f - I(flm)) composed from the differentiable single passes
        kw = dict(L=L, spin=spin, nside=nside or 0, sampling=_lib.SAMPLING[s], reality=0,
                  L_lower=L_lower, precision=_lib.PRECISION[precision], batch=B, N=0)
        p0 = _lib.get_plan(x.device, iter=0, **kw)
        flm_shape = batch_shape + (L, 2 * L - 1)
        y = _ForwardFn.apply(x, p0, flm_shape, cdt)
        for _ in range(int(iter)):
            r = x - _InverseFn.apply(y, p0, batch_shape + fs, cdt)
            y = y + _ForwardFn.apply(r, p0, flm_shape, cdt)
        return _ret(y, was_np, odev)
    plan = _lib.get_plan(x.device, L=L, spin=spin, nside=nside or 0, sampling=_lib.SAMPLING[s],
                         reality=int(bool(reality)), L_lower=L_lower,
                         precision=_lib.PRECISION[precision], batch=B, iter=int(iter), N=0)
    out = torch.empty(batch_shape + (L, 2 * L - 1), dtype=cdt, device=x.device)
    ws = plan.workspace(True)
    _lib.check(_lib.lib().s2b_forward(plan.ptr, x.data_ptr(), out.data_ptr(), ws.data_ptr(),
                                      ws.numel(), _lib.stream_handle(x.device)))
    return _ret(out, was_np, odev)
