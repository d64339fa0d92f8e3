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
single passes. Real signals (``reality=True``) are differentiated through
exact rewrites on the complex kernels: upstream's real inverse keeps the orders
m >= 0 and reads the map off the Hermitian extension of the ring spectra, which
is ``Re(inverse(D flm))`` with D = 1 at m = 0, 2 at m > 0 and 0 at m < 0; its
real forward takes the real part of the (upsampled) map before the ring FFTs and
mirrors the m < 0 half from m >= 0 (s2fft/transforms/spherical.py:176-208,
526-588), which is the complex forward averaged with the conjugate of the
complex forward of the phi-reflected map (MW / MWSS) and then mirrored. The same
rewrites serve ``reality=True`` with spin != 0, which upstream's on-the-fly
methods accept and treat the same way.

``precomps`` and ``spmd`` are accepted for signature compatibility: the
recursion tables are built on the device per plan, and one GPU runs each call,
so a supplied value is ignored (with a ``UserWarning``).
"""

from __future__ import annotations

import warnings

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


def _dense(t):
    """A tensor whose memory holds its values: conjugate and negative views (lazy bits that
    torch sets, e.g. on gradients flowing through torch.conj) are materialised, since the
    C ABI reads raw memory."""
    return t.resolve_conj().resolve_neg().contiguous()


def _aligned(t):
    # the C ABI takes 16-byte aligned operands; a view into a larger tensor may not be
    return t if t.data_ptr() % 16 == 0 else t.clone()


def _to_device(x, dtype, device):
    """(contiguous, 16-byte aligned tensor on device, was_numpy, original device)."""
    if isinstance(x, np.ndarray):
        t = torch.from_numpy(np.ascontiguousarray(x))
        return _aligned(_dense(t.to(device=device, dtype=dtype))), True, None
    if isinstance(x, torch.Tensor):
        dev = x.device
        t = _dense(x.to(device=device if dev.type != "cuda" else dev, dtype=dtype))
        return _aligned(t), False, dev
    t = torch.as_tensor(np.asarray(x))
    return _aligned(_dense(t.to(device=device, dtype=dtype))), True, None


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
        flm = _aligned(_dense(flm))
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
        g = _aligned(_dense(g))
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
        f = _aligned(_dense(f))
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
        g = _aligned(_dense(g))
        gf = torch.empty(ctx.in_shape, dtype=g.dtype, device=g.device)
        ws = ctx.plan.workspace(3)
        _lib.check(_lib.lib().s2b_forward_adjoint(ctx.plan.ptr, g.data_ptr(), gf.data_ptr(),
                                                  ws.data_ptr(), ws.numel(),
                                                  _lib.stream_handle(g.device)))
        return gf, None, None, None


def _needs_grad(x):
    return isinstance(x, torch.Tensor) and x.requires_grad and torch.is_grad_enabled()


def _warn_unused(precomps, spmd):
    if precomps is not None:
        warnings.warn("precomps is ignored: the recursion tables are built on the device "
                      "per plan", UserWarning, stacklevel=3)
    if spmd:
        warnings.warn("spmd is ignored: each call runs on the current GPU", UserWarning,
                      stacklevel=3)


def _real_orders(L, device, dtype):
    """D[L-1+m] = 1 at m = 0, 2 at m > 0, 0 at m < 0 (the Hermitian extension's weights)."""
    d = torch.zeros(2 * L - 1, dtype=dtype, device=device)
    d[L - 1] = 1
    d[L:] = 2
    return d


def _mirror_real(y, L):
    """Upstream's completion of a real signal's coefficients from the m >= 0 half:
    flm[l, -m] = (-1)^m conj(flm[l, m]) (s2fft/transforms/spherical.py:577-582)."""
    mc = torch.from_numpy((-1.0) ** (np.arange(1, L) % 2)).to(device=y.device,
                                                              dtype=y.real.dtype)
    neg = torch.flip(torch.conj(y[..., L:]) * mc, dims=[-1])
    return torch.cat([neg, y[..., L - 1:]], dim=-1)


def inverse(flm, L: int, spin: int = 0, nside: int = None, sampling: str = "mw",
            method: str = "cuda", reality: bool = False, precomps=None, spmd: bool = False,
            L_lower: int = 0, _ssht_backend: int = 1, precision: str = "f64"):
    """Inverse spin-SHT: flm [.., L, 2L-1] -> f on the sampling grid."""
    _check_method(method)
    s = _check_args(L, spin, nside, sampling, reality, L_lower)
    _warn_unused(precomps, spmd)
    cdt, rdt = _dtypes(precision)
    dev = _device()
    x, was_np, odev = _to_device(flm, cdt, dev)
    batch_shape = tuple(x.shape[:-2])
    if tuple(x.shape[-2:]) != (L, 2 * L - 1):
        raise ValueError(f"flm must have trailing shape {(L, 2 * L - 1)}, got {tuple(x.shape)}")
    B = int(np.prod(batch_shape)) if batch_shape else 1
    kw = dict(L=L, spin=spin, nside=nside or 0, sampling=_lib.SAMPLING[s], L_lower=L_lower,
              precision=_lib.PRECISION[precision], batch=B, iter=0, N=0)
    fs = batch_shape + f_shape(L, s, nside)
    if reality and (spin != 0 or _needs_grad(x)):
        # f = Re(I(D flm)) on the complex kernels: exactly upstream's real inverse (orders
        # m >= 0 on the Hermitian extension), differentiable and valid for any spin
        pc = _lib.get_plan(x.device, reality=0, **kw)
        xd = x * _real_orders(L, x.device, rdt)
        return _ret(_InverseFn.apply(xd, pc, fs, cdt).real.contiguous(), was_np, odev)
    plan = _lib.get_plan(x.device, reality=int(bool(reality)), **kw)
    if _needs_grad(x):
        return _ret(_InverseFn.apply(x, plan, fs, cdt), was_np, odev)
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
    _warn_unused(precomps, spmd)
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
    if _needs_grad(x) or (reality and spin != 0):
        # refinement flm <- flm + F(f - I(flm)) composed from the differentiable single
        # passes on the complex kernels; real signals as upstream (module docstring)
        kw = dict(L=L, spin=spin, nside=nside or 0, sampling=_lib.SAMPLING[s], reality=0,
                  L_lower=L_lower, precision=_lib.PRECISION[precision], batch=B, N=0)
        p0 = _lib.get_plan(x.device, iter=0, **kw)
        flm_shape = batch_shape + (L, 2 * L - 1)
        if reality:
            dord = _real_orders(L, x.device, rdt)
            reflect = s in ("mw", "mwss")
            if reflect:  # phi -> -phi on the ring grid
                nph = fs[-1]
                ridx = torch.from_numpy((-np.arange(nph)) % nph).to(x.device)

            def fwd1(r):
                y = _ForwardFn.apply(r.to(cdt), p0, flm_shape, cdt)
                if reflect:
                    # upstream takes the real part of the upsampled MW / MWSS map, which
                    # averages each order m with the conjugate of the transform of the
                    # phi-reflected map (s2fft/transforms/spherical.py:526-534)
                    yr = _ForwardFn.apply(r.index_select(-1, ridx).to(cdt), p0, flm_shape,
                                          cdt)
                    y = 0.5 * (y + torch.conj(yr))
                return _mirror_real(y, L)

            def inv1(y):
                return _InverseFn.apply(y * dord, p0, batch_shape + fs, cdt).real
        else:
            def fwd1(r):
                return _ForwardFn.apply(r, p0, flm_shape, cdt)

            def inv1(y):
                return _InverseFn.apply(y, p0, batch_shape + fs, cdt)
        y = fwd1(x)
        for _ in range(int(iter)):
            y = y + fwd1(x - inv1(y))
        return _ret(y, was_np, odev)
    plan = _lib.get_plan(x.device, L=L, spin=spin, nside=nside or 0, sampling=_lib.SAMPLING[s],
                         reality=int(bool(reality)), L_lower=L_lower,
                         precision=_lib.PRECISION[precision], batch=B, iter=int(iter), N=0)
    out = torch.empty(batch_shape + (L, 2 * L - 1), dtype=cdt, device=x.device)
    ws = plan.workspace(True)
    _lib.check(_lib.lib().s2b_forward(plan.ptr, x.data_ptr(), out.data_ptr(), ws.data_ptr(),
                                      ws.numel(), _lib.stream_handle(x.device)))
    return _ret(out, was_np, odev)
