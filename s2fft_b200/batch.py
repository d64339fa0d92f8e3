"""Batched spin transforms over many maps of uneven size.

A workload mixes band-limits, spins and samplings. Maps that share
``(L, spin, sampling, nside)`` form a group: one plan with ``batch`` equal to
the group size, so each kernel of the chain processes the whole group in one
launch. Groups run concurrently on several CUDA streams (largest first), the
whole inverse + forward of all groups is captured once in a CUDA graph and
replayed on every call, and an autotuner picks each group's latitudinal launch
shapes (``s2b_plan_set_tuning``: tiles, inverse segments along m) by timing them
on the group itself.

Only the host-side scheduling is new here; every transform runs the same
kernels as :func:`s2fft_b200.inverse` / :func:`s2fft_b200.forward`, so each
map's result equals the unbatched call on that map.

Example::

    specs = [(L, spin, "mw") for ...]
    b = BatchedSHT(specs, precision="f32")
    b.load(flms)               # list of [L, 2L-1] coefficient arrays
    b.run()                    # inverse then forward of every map (one graph replay)
    f_i, flm_i = b.maps(i), b.coefficients(i)
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from .spherical import _device, _dtypes, f_shape


@dataclass
class _Group:
    L: int
    spin: int
    sampling: str
    nside: int
    members: list = field(default_factory=list)  # map indices, in batch order
    plan: object = None
    flm_in: torch.Tensor = None
    f: torch.Tensor = None
    flm_out: torch.Tensor = None
    ws_inv: torch.Tensor = None
    ws_fwd: torch.Tensor = None
    tiles: tuple = (0, 0, 1)  # (forward tile, inverse tile, inverse segments along m)

    def work(self):
        nth = f_shape(self.L, self.sampling, self.nside)[0] if self.sampling != "healpix" \
            else 4 * self.nside - 1
        return len(self.members) * nth * self.L * self.L


class BatchedSHT:
    """Inverse followed by forward spin transform of many maps of uneven size."""

    def __init__(self, specs, precision="f32", streams=4, tune=True, graph=True):
        self.device = _device()
        self.precision = precision
        self.cdt, _ = _dtypes(precision)
        self.n = len(specs)
        groups = {}
        self.where = []
        for i, sp in enumerate(specs):
            if isinstance(sp, dict):
                L, spin, sampling, nside = sp["L"], sp.get("spin", 0), sp.get("sampling", "mw"), \
                    sp.get("nside", 0)
            else:
                L, spin, sampling = sp[:3]
                nside = sp[3] if len(sp) > 3 else 0
            key = (int(L), int(spin), sampling.lower(), int(nside or 0))
            g = groups.setdefault(key, _Group(*key))
            self.where.append((key, len(g.members)))
            g.members.append(i)
        # largest groups first, so that they start before the small ones fill the GPU
        self.groups = sorted(groups.values(), key=lambda g: -g.work())
        self.by_key = {(g.L, g.spin, g.sampling, g.nside): g for g in self.groups}
        for g in self.groups:
            B = len(g.members)
            g.plan = _lib.get_plan(self.device, L=g.L, spin=g.spin, nside=g.nside,
                                   sampling=_lib.SAMPLING[g.sampling], reality=0, L_lower=0,
                                   precision=_lib.PRECISION[precision], batch=B, iter=0, N=0)
            g.flm_in = torch.zeros((B, g.L, 2 * g.L - 1), dtype=self.cdt, device=self.device)
            g.f = torch.empty((B,) + f_shape(g.L, g.sampling, g.nside or None), dtype=self.cdt,
                              device=self.device)
            g.flm_out = torch.empty_like(g.flm_in)
            g.ws_inv = g.plan.workspace(0)
            g.ws_fwd = g.plan.workspace(1)
        self.streams = [torch.cuda.Stream(self.device) for _ in range(max(1, streams))]
        self.graph = None
        if tune:
            self.tune()
        if graph:
            self.capture()

    # -- data -------------------------------------------------------------------------
    def load(self, flms):
        """Copy map i's coefficients [L, 2L-1] into the batch (numpy or torch)."""
        for i, x in enumerate(flms):
            key, pos = self.where[i]
            t = torch.as_tensor(np.asarray(x) if not isinstance(x, torch.Tensor) else x)
            self.by_key[key].flm_in[pos].copy_(t.to(self.cdt), non_blocking=True)

    def maps(self, i):
        key, pos = self.where[i]
        return self.by_key[key].f[pos]

    def coefficients(self, i):
        key, pos = self.where[i]
        return self.by_key[key].flm_out[pos]

    # -- execution --------------------------------------------------------------------
    def _launch(self, g, stream):
        lib = _lib.lib()
        h = ctypes.c_void_p(stream.cuda_stream)
        _lib.check(lib.s2b_inverse(g.plan.ptr, g.flm_in.data_ptr(), g.f.data_ptr(),
                                   g.ws_inv.data_ptr(), g.ws_inv.numel(), h))
        _lib.check(lib.s2b_forward(g.plan.ptr, g.f.data_ptr(), g.flm_out.data_ptr(),
                                   g.ws_fwd.data_ptr(), g.ws_fwd.numel(), h))

    def _run_all(self):
        main = torch.cuda.current_stream(self.device)
        for s in self.streams:
            s.wait_stream(main)
        for k, g in enumerate(self.groups):
            self._launch(g, self.streams[k % len(self.streams)])
        for s in self.streams:
            main.wait_stream(s)

    def run(self):
        """Inverse then forward transform of every map (graph replay when captured)."""
        if self.graph is not None:
            self.graph.replay()
        else:
            self._run_all()

    def capture(self):
        """Capture the launches of all groups in one CUDA graph (after one eager warm-up)."""
        self._run_all()
        torch.cuda.synchronize(self.device)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph, capture_error_mode="relaxed"):
            self._run_all()
        torch.cuda.synchronize(self.device)

    # -- autotuner --------------------------------------------------------------------
    def tune(self, reps=3):
        """Per group, time the launch shapes of the inverse and the forward latitudinal
        kernels (tile x segments along m; forward segments apply to the equator-symmetric
        forward) on the group itself and keep the fastest."""
        lib = _lib.lib()
        stream = torch.cuda.current_stream(self.device)
        h = ctypes.c_void_p(stream.cuda_stream)

        def timed(fn):
            fn()
            e0, e1 = torch.cuda.Event(True), torch.cuda.Event(True)
            e0.record(stream)
            for _ in range(reps):
                fn()
            e1.record(stream)
            e1.synchronize()
            return e0.elapsed_time(e1)

        inv = [(t, n) for t in (2, 3) for n in (2, 4)]  # (tile, segments along m)
        for g in self.groups:
            def call_inv():
                _lib.check(lib.s2b_inverse(g.plan.ptr, g.flm_in.data_ptr(), g.f.data_ptr(),
                                           g.ws_inv.data_ptr(), g.ws_inv.numel(), h))

            def call_fwd():
                _lib.check(lib.s2b_forward(g.plan.ptr, g.f.data_ptr(), g.flm_out.data_ptr(),
                                           g.ws_fwd.data_ptr(), g.ws_fwd.numel(), h))

            t = []
            for tile, nseg in inv:
                _lib.check(lib.s2b_plan_set_tuning(g.plan.ptr, 1, tile))
                _lib.check(lib.s2b_plan_set_tuning(g.plan.ptr, 2, nseg))
                t.append(timed(call_inv))
            tile_inv, nseg = inv[int(np.argmin(t))]
            _lib.check(lib.s2b_plan_set_tuning(g.plan.ptr, 1, tile_inv))
            _lib.check(lib.s2b_plan_set_tuning(g.plan.ptr, 2, nseg))
            t = []
            fwd = [(v, n) for v in (0, 1) for n in (2, 4)]  # (tile, segments along m)
            for v, n in fwd:
                _lib.check(lib.s2b_plan_set_tuning(g.plan.ptr, 0, v))
                _lib.check(lib.s2b_plan_set_tuning(g.plan.ptr, 3, n))
                t.append(timed(call_fwd))
            tile_fwd, nseg_fwd = fwd[int(np.argmin(t))]
            _lib.check(lib.s2b_plan_set_tuning(g.plan.ptr, 0, tile_fwd))
            _lib.check(lib.s2b_plan_set_tuning(g.plan.ptr, 3, nseg_fwd))
            g.tiles = (tile_fwd, tile_inv, nseg)
        torch.cuda.synchronize(self.device)

    def summary(self):
        return [dict(L=g.L, spin=g.spin, sampling=g.sampling, maps=len(g.members),
                     forward_tile=g.tiles[0], inverse_tile=g.tiles[1], inverse_segments=g.tiles[2])
                for g in self.groups]
