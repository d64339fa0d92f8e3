"""Batched spin transforms over many maps of uneven size.

A workload mixes band-limits, spins and samplings. Maps that share
``(L, spin, sampling, nside)`` form a group: one plan with ``batch`` equal to
the group size, so each kernel of the chain processes the whole group in one
launch. Two schedules:

* ``persistent=True``: all groups form one uneven batch
  (``s2b_batch_inverse`` / ``s2b_batch_forward``). The ring FFTs and the other
  per-group stages run on the batch's streams, and the latitudinal kernels of
  all groups -- the O(L^3) part -- run as persistent launches, one per kernel
  variant (spin 0 or not, tile shape), whose CTAs pull (group, tile) items
  from a device work counter, so small groups fill the SMs that the large
  ones leave idle in their tails. Waves (``s2b_batch_set_option``) let the
  ring FFTs of one part of the batch overlap the persistent launches of the
  next. The autotuner picks tile shapes and segment counts per class of
  groups (spin 0, spin != 0) and the waves / CTAs per SM, by timing the whole
  batch.
* ``persistent=False``: every group runs its own chain of launches; groups run
  concurrently on several CUDA streams (largest first), and the autotuner
  picks each group's launch shapes (``s2b_plan_set_tuning``: tiles, inverse
  segments along m) by timing them on the group itself.
* ``persistent=None`` (default): the autotuner times both and keeps the
  faster schedule (``self.schedule``, ``self.timings``).

Either way the whole inverse + forward of all groups is captured once in a
CUDA graph and replayed on every call.

Only the scheduling is new here: every transform runs the same stages as
:func:`s2fft_b200.inverse` / :func:`s2fft_b200.forward` (the persistent launches
run the same per-tile code as the per-plan latitudinal kernels), so each map's
result equals the unbatched call on that map.

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
    # s2b_plan_set_tuning values (forward tile, inverse tile, inverse segments, forward
    # segments) in force, and the tuned ones per schedule
    tuning: tuple = None
    tuned: dict = field(default_factory=dict)

    def work(self):
        nth = f_shape(self.L, self.sampling, self.nside)[0] if self.sampling != "healpix" \
            else 4 * self.nside - 1
        return len(self.members) * nth * self.L * self.L


class BatchedSHT:
    """Inverse followed by forward spin transform of many maps of uneven size."""

    def __init__(self, specs, precision="f32", streams=4, tune=True, graph=True, persistent=None):
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
        # persistent: True / False force a schedule, None lets the autotuner pick one
        self.requested = persistent
        self.batch = _lib.Batch([g.plan for g in self.groups]) if persistent is not False else None
        self.schedule = "persistent" if self.batch is not None else "streams"
        self.batch_schedule = (1, 0)
        self.timings = {}
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

    def _batch_inverse(self, stream):
        gs = self.groups
        self.batch.inverse([g.flm_in for g in gs], [g.f for g in gs], [g.ws_inv for g in gs],
                           stream)

    def _batch_forward(self, stream):
        gs = self.groups
        self.batch.forward([g.f for g in gs], [g.flm_out for g in gs], [g.ws_fwd for g in gs],
                           stream)

    def _run_streams(self):
        main = torch.cuda.current_stream(self.device)
        for s in self.streams:
            s.wait_stream(main)
        for k, g in enumerate(self.groups):
            self._launch(g, self.streams[k % len(self.streams)])
        for s in self.streams:
            main.wait_stream(s)

    def _run_all(self):
        if self.schedule == "persistent":
            main = torch.cuda.current_stream(self.device)
            self._batch_inverse(main)
            self._batch_forward(main)
        else:
            self._run_streams()

    def run(self):
        """Inverse then forward transform of every map (graph replay when captured)."""
        if self.graph is not None:
            self.graph.replay()
        else:
            self._run_all()

    def capture(self):
        """Capture the launches of all groups in one CUDA graph (after one eager warm-up)."""
        self.graph = None
        self._run_all()
        torch.cuda.synchronize(self.device)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph, capture_error_mode="relaxed"):
            self._run_all()
        torch.cuda.synchronize(self.device)

    # -- autotuner --------------------------------------------------------------------
    # s2b_plan_set_tuning keys: 0 forward tile, 1 inverse tile, 2 inverse segments along m,
    # 3 forward segments along m (equator-symmetric forward)
    _INV = [(t, n) for t in (2, 3) for n in (4, 8)]  # (inverse tile, segments)
    _FWD = [(v, n) for v in (0, 1) for n in (4, 8)]  # (forward tile, segments)
    _SCHED = [(1, 0), (2, 0), (2, 2), (3, 2)]  # (waves, CTAs per SM) of the persistent batch

    def _timed(self, fn, reps):
        stream = torch.cuda.current_stream(self.device)
        fn()
        e0, e1 = torch.cuda.Event(True), torch.cuda.Event(True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / reps

    @staticmethod
    def _set(g, tuning):
        lib = _lib.lib()
        for key, v in enumerate(tuning):
            _lib.check(lib.s2b_plan_set_tuning(g.plan.ptr, key, v))
        g.tuning = tuple(tuning)

    def _tune_streams(self, reps):
        """Per group, the inverse and forward shapes timed on the group itself."""
        lib = _lib.lib()
        h = ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)
        for g in self.groups:
            def call_inv():
                _lib.check(lib.s2b_inverse(g.plan.ptr, g.flm_in.data_ptr(), g.f.data_ptr(),
                                           g.ws_inv.data_ptr(), g.ws_inv.numel(), h))

            def call_fwd():
                _lib.check(lib.s2b_forward(g.plan.ptr, g.f.data_ptr(), g.flm_out.data_ptr(),
                                           g.ws_fwd.data_ptr(), g.ws_fwd.numel(), h))

            cur = list(g.tuning)
            t = []
            for tile, nseg in self._INV:
                cur[1], cur[2] = tile, nseg
                self._set(g, cur)
                t.append(self._timed(call_inv, reps))
            cur[1], cur[2] = self._INV[int(np.argmin(t))]
            t = []
            for v, n in self._FWD:
                cur[0], cur[3] = v, n
                self._set(g, cur)
                t.append(self._timed(call_fwd, reps))
            cur[0], cur[3] = self._FWD[int(np.argmin(t))]
            self._set(g, cur)
            g.tuned["streams"] = tuple(cur)

    def _tune_persistent(self, reps):
        """Shapes for the persistent schedule, then its waves and CTAs per SM, all timed on
        the whole batch. Two candidates for the shapes: each group's own (from the
        per-group tuner; a persistent launch then serves the groups that share a shape),
        and shapes shared by each class of groups (spin 0, spin != 0), tuned on the batch."""
        stream = torch.cuda.current_stream(self.device)

        def run_both():
            self._batch_inverse(stream)
            self._batch_forward(stream)

        self.batch.set_schedule(1, 0)
        cands = []
        if all("streams" in g.tuned for g in self.groups):
            for g in self.groups:
                self._set(g, g.tuned["streams"])
            cands.append((self._timed(run_both, reps), [g.tuning for g in self.groups]))
        for cls in (True, False):
            members = [g for g in self.groups if (g.spin == 0) == cls]
            if not members:
                continue
            for (kt, ks), opts, fn in (((1, 2), self._INV, lambda: self._batch_inverse(stream)),
                                       ((0, 3), self._FWD, lambda: self._batch_forward(stream))):
                def apply(c):
                    for g in members:
                        cur = list(g.tuning)
                        cur[kt], cur[ks] = c
                        self._set(g, cur)

                t = []
                for c in opts:
                    apply(c)
                    t.append(self._timed(fn, reps))
                apply(opts[int(np.argmin(t))])
        cands.append((self._timed(run_both, reps), [g.tuning for g in self.groups]))
        best = min(cands, key=lambda c: c[0])[1]
        for g, tu in zip(self.groups, best):
            self._set(g, tu)
        t = []
        for waves, per_sm in self._SCHED:
            self.batch.set_schedule(waves, per_sm)
            t.append(self._timed(run_both, reps))
        self.batch_schedule = self._SCHED[int(np.argmin(t))]
        self.batch.set_schedule(*self.batch_schedule)
        for g in self.groups:
            g.tuned["persistent"] = g.tuning
        return min(t)

    def tune(self, reps=3):
        """Pick launch shapes (and, with persistent=None, the schedule) by timing them."""
        with torch.no_grad():
            for g in self.groups:
                self._set(g, (0, 3, 8, 8))
            self._tune_streams(reps)  # per-group shapes: used by both schedules
            t_str = None
            if self.requested is not True:
                t_str = self._timed(self._run_streams, reps)
            t_pers = self._tune_persistent(reps) if self.batch is not None else None
            if t_pers is not None and (t_str is None or t_pers <= t_str):
                self.schedule = "persistent"
            else:
                self.schedule = "streams"
                for g in self.groups:
                    self._set(g, g.tuned["streams"])
            self.timings = {"persistent_ms": t_pers, "streams_ms": t_str}
        torch.cuda.synchronize(self.device)

    def summary(self):
        keys = ("forward_tile", "inverse_tile", "inverse_segments", "forward_segments")
        return [dict(L=g.L, spin=g.spin, sampling=g.sampling, maps=len(g.members),
                     **dict(zip(keys, g.tuning or (None,) * 4)))
                for g in self.groups]
