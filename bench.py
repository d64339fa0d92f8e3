#!/usr/bin/env python
"""Benchmark of the spin spherical-harmonic transform on B200.

Workload (the headline configuration): MW sampling, L = 1024, spin 0, complex
signal; one step = one inverse transform followed by one forward transform of
a seeded band-limited map (flm with Re, Im ~ N(0,1) for every |m| <= l), in the
mixed precision path (float32 recursion/projection, double seeds, exponent
bookkeeping and weights). The same step on the float64 path is timed too.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs as N independent replicas (one process per GPU, torchrun), the
transform does not shard across GPUs; value = total transforms of all ranks
divided by the slowest rank's time. Rank 0 prints one JSON line.
"""

import argparse
import ctypes
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "L=1024 SHT fwd+inv/s & batched maps/s, mixed vs FP64 GPU path at <=1e-5 err"
UNIT = "fwd+inv/s"
FLOPS_PER_TRIPLE = 9  # recursion (5) + complex-by-real projection (4) per (theta, l, m)


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--L", type=int, default=1024)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the secondary configurations (batched tensor-core, HEALPix)")
    ap.add_argument("--tc-profile", action="store_true",
                    help="small tensor-core case for ncu (GL L=256, 64 maps)")
    ap.add_argument("--cpu-budget", type=float, default=25.0,
                    help="seconds of host work for the CPU baseline sample")
    ap.add_argument("--profile-case", action="store_true",
                    help="small case for ncu: 2 steps, no baseline, no clocks")
    ap.add_argument("--healpix-profile", action="store_true",
                    help="HEALPix nside=256 L=512 real float32: one inverse and one forward "
                         "with 3 iterations between cudaProfilerStart/Stop")
    ap.add_argument("--rotate-profile", action="store_true",
                    help="rotate_flms at --L (float64, one map): warm-up, five timed calls, "
                         "then one call between cudaProfilerStart/Stop")
    ap.add_argument("--planes-profile", action="store_true",
                    help="generate_rotate_dls at --L and beta = pi/2: warm-up, three timed "
                         "calls, then one call between cudaProfilerStart/Stop")
    ap.add_argument("--fw-profile", action="store_true",
                    help="Fourier-Wigner SO(3) transforms at --L (N=8, MW, float32): warm-up, "
                         "five timed inverse and forward calls, then one of each between "
                         "cudaProfilerStart/Stop")
    ap.add_argument("--batch-profile", choices=["persistent", "streams"], default=None,
                    help="the 256-map uneven batch, one eager inverse + forward of the given "
                         "schedule between cudaProfilerStart/Stop (ncu --profile-from-start "
                         "off)")
    return ap.parse_args()


def seeded_flm(rng, L, spin=0, reality=False):
    """Band-limited synthetic coefficients flm[l, L-1+m]: Re and Im ~ N(0,1) for every
    |m| <= l with max(|spin|) <= l < L; with reality, m = 0 real and
    flm[l, -m] = (-1)^m conj(flm[l, m])."""
    flm = np.zeros((L, 2 * L - 1), dtype=np.complex128)
    for el in range(abs(spin), L):
        n = 2 * el + 1
        flm[el, L - 1 - el: L + el] = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        if reality:
            flm[el, L - 1] = flm[el, L - 1].real
            m = np.arange(1, el + 1)
            flm[el, L - 1 - m] = (-1.0) ** m * np.conj(flm[el, L - 1 + m])
    return flm


_GOLDEN = None


def golden_err(name, key, arr):
    """Max relative error of arr at the entries that upstream's float64 numpy transforms
    produced for the same seeded input (tests/golden/large.npz, written by
    tests/golden/make_large.py); None when the fixture is absent."""
    global _GOLDEN
    if _GOLDEN is None:
        path = os.path.join(ROOT, "tests", "golden", "large.npz")
        _GOLDEN = np.load(path) if os.path.exists(path) else False
    if _GOLDEN is False or f"{name}/{key}_idx" not in _GOLDEN:
        return None
    idx, ref = _GOLDEN[f"{name}/{key}_idx"], _GOLDEN[f"{name}/{key}_val"]
    got = np.asarray(arr).reshape(-1)[idx]
    return float(np.abs(got - ref).max() / np.abs(ref).max())


def triples(L, nrings, spin=0, reality=False):
    """(theta, l, m) terms with max(|m|, |s|) <= l < L, summed over rings."""
    ms = np.arange(0 if reality else -(L - 1), L)
    return nrings * int(np.sum(L - np.maximum(np.abs(ms), abs(spin))))


# ---------------------------------------------------------------------------
# clocks sampled with nvidia-smi during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(smax)),
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            return json.load(fh), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def simt_peak_tflops(torch, fp64):
    """FP32 / FP64 FMA rate measured with the library's FMA-chain probe (fp64 = 2: FP32 by
    packed-pair FMAs, fma.rn.f32x2)."""
    from s2fft_b200 import _lib

    lib = _lib.lib()
    lib.s2b_fma_probe.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                  ctypes.c_void_p]
    lib.s2b_fma_probe.restype = ctypes.c_int
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    blocks, iters = sms * 8, 4000 if not fp64 else 2000
    out = torch.empty(blocks * 256, dtype=torch.float64 if fp64 == 1 else torch.float32,
                      device="cuda")
    st = _lib.stream_handle(out.device)
    best = 0.0
    for rep in range(4):
        e0, e1 = torch.cuda.Event(True), torch.cuda.Event(True)
        e0.record()
        _lib.check(lib.s2b_fma_probe(int(fp64), blocks, iters, out.data_ptr(), st))
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        flops = blocks * 256.0 * iters * 16 * 8 * 2 * (2 if fp64 == 2 else 1)
        if rep > 0:
            best = max(best, flops / (ms * 1e-3) / 1e12)
    return best


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def job_rates(torch, ms, counts, world, dist=None, device="cpu"):
    """Whole-job rates of the replicas: every timed leg i takes the slowest rank's time
    (max over ranks, one all-reduce) and rate_i = world * counts_i / time_i. Returns
    (max times in ms, rates per second)."""
    t = torch.tensor([float(x) for x in ms], dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    mx = t.tolist()
    return mx, [world * c / (m * 1e-3) for c, m in zip(counts, mx)]


def run_ours(args, rank, world, torch, dist):
    import s2fft_b200
    from s2fft_b200 import _lib

    L = args.L
    dev = torch.device("cuda", torch.cuda.current_device())
    rng = np.random.default_rng(8966433580120847635 + rank)
    flm_np = seeded_flm(rng, L)
    nrings_inv, nrings_fwd = L, 2 * L - 1
    T_inv, T_fwd = triples(L, nrings_inv), triples(L, nrings_fwd)
    # executed: the forward's 2L-1 rings run as L ring pairs (the equator pairs with itself)
    T_fwd_exec = triples(L, (nrings_fwd + 1) // 2)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)  # > 126 MB L2

    def plans(precision):
        kw = dict(L=L, spin=0, nside=0, sampling=0, reality=0, L_lower=0,
                  precision=_lib.PRECISION[precision], batch=1, N=0)
        return _lib.get_plan(dev, iter=0, **kw), _lib.get_plan(dev, iter=0, **kw)

    def timed(precision, steps, warmup, lat_events):
        cdt = torch.complex64 if precision == "f32" else torch.complex128
        x = torch.from_numpy(flm_np).to(dev, cdt)
        f = s2fft_b200.inverse(x, L, precision=precision)
        y = s2fft_b200.forward(f, L, precision=precision)
        torch.cuda.synchronize()
        plan = plans(precision)[0]
        lib = _lib.lib()
        lib.s2b_plan_set_events.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                            ctypes.c_void_p]
        lib.s2b_plan_set_events.restype = ctypes.c_int
        for _ in range(warmup):
            flush.zero_()
            f = s2fft_b200.inverse(x, L, precision=precision)
            y = s2fft_b200.forward(f, L, precision=precision)
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        step_ev, lat_ev = [], []
        for _ in range(steps):
            flush.zero_()  # L2 flush between timed steps, outside the events
            e = [torch.cuda.Event(True) for _ in range(2)]
            le = [torch.cuda.Event(True) for _ in range(4)] if lat_events else None
            if le:
                for ev in le:
                    ev.record()  # materialise the handles before passing them to the library
                _lib.check(lib.s2b_plan_set_events(plan.ptr, 0, le[0].cuda_event,
                                                   le[1].cuda_event))
                _lib.check(lib.s2b_plan_set_events(plan.ptr, 1, le[2].cuda_event,
                                                   le[3].cuda_event))
            e[0].record()
            f = s2fft_b200.inverse(x, L, precision=precision)
            y = s2fft_b200.forward(f, L, precision=precision)
            e[1].record()
            step_ev.append(e)
            lat_ev.append(le)
        torch.cuda.synchronize()
        _lib.check(lib.s2b_plan_set_events(plan.ptr, 0, None, None))
        _lib.check(lib.s2b_plan_set_events(plan.ptr, 1, None, None))
        total_ms = sum(a.elapsed_time(b) for a, b in step_ev)
        lat = None
        if lat_events:
            li = [le[0].elapsed_time(le[1]) for le in lat_ev]
            lf = [le[2].elapsed_time(le[3]) for le in lat_ev]
            lat = (float(np.mean(li)), float(np.mean(lf)))
        err = float((y - x).abs().max().item() / x.abs().max().item())
        if rank == 0 and L == 1024:  # the seeded input of the golden subsets
            err_oracle = {"inverse": golden_err("mw_L1024", "f", f.cpu().numpy()),
                          "forward_of_inverse": golden_err("mw_L1024", "flm", y.cpu().numpy())}
        else:
            err_oracle = None
        return total_ms, lat, err, y, err_oracle

    steps, warmup = args.steps, args.warmup
    clocks = ClockSampler(dev.index if dev.index is not None else 0)
    clocks.start()
    ms32, lat32, err32, y32, orc32 = timed("f32", steps, warmup, True)
    clk = clocks.stop()
    ms64, lat64, err64, y64, orc64 = timed("f64", max(3, steps // 4), 2, True)
    # mixed-path coefficient error against the float64 path (itself <= 1e-10 of the oracle)
    err_mixed = float((y32.to(torch.complex128) - y64).abs().max().item()
                      / y64.abs().max().item())
    # a throughput number is only meaningful for a correct transform
    if not (np.isfinite(err_mixed) and np.isfinite(err32) and err_mixed < 1e-4 and err64 < 1e-9):
        raise RuntimeError(f"transform error out of bounds: mixed {err_mixed}, f32 round trip "
                           f"{err32}, f64 round trip {err64}")

    # end to end through the public API with pinned host buffers: each step copies its
    # coefficients host -> device, runs inverse + forward and copies the result back. The
    # copies run on their own streams with double-buffered pinned memory, so step i's
    # transfers overlap the compute of its neighbours (as a pipelined user would do); the
    # timed region spans the whole job, first upload and last download included, with an L2
    # flush on the compute stream before every step.
    nb = 2
    host_in = [torch.from_numpy(flm_np.astype(np.complex64)).pin_memory() for _ in range(nb)]
    host_out = [torch.empty_like(host_in[0]).pin_memory() for _ in range(nb)]
    dev_in = [torch.empty(host_in[0].shape, dtype=torch.complex64, device=dev) for _ in range(nb)]
    comp = torch.cuda.current_stream(dev)
    up, down = torch.cuda.Stream(dev), torch.cuda.Stream(dev)

    def e2e_job(nsteps):
        ev_up = [torch.cuda.Event() for _ in range(nb)]
        ev_done = [torch.cuda.Event() for _ in range(nb)]
        ev_read = [torch.cuda.Event() for _ in range(nb)]
        start, end = torch.cuda.Event(True), torch.cuda.Event(True)
        start.record(comp)
        up.wait_stream(comp)
        down.wait_stream(comp)
        for i in range(nsteps):
            j = i % nb
            if i >= nb:
                up.wait_event(ev_read[j])  # compute of step i-nb has consumed dev_in[j]
            with torch.cuda.stream(up):
                dev_in[j].copy_(host_in[j], non_blocking=True)
                ev_up[j].record(up)
            comp.wait_event(ev_up[j])
            flush.zero_()
            yd = s2fft_b200.forward(s2fft_b200.inverse(dev_in[j], L, precision="f32"), L,
                                    precision="f32")
            ev_read[j].record(comp)
            ev_done[j].record(comp)
            down.wait_event(ev_done[j])
            with torch.cuda.stream(down):
                host_out[j].copy_(yd, non_blocking=True)
            yd.record_stream(down)
        comp.wait_stream(up)
        comp.wait_stream(down)
        end.record(comp)
        torch.cuda.synchronize()
        return start.elapsed_time(end), yd

    # warm-up long enough for the copy/compute pipeline and the caching allocator's
    # cross-stream blocks to reach their steady state before the timed steps
    e2e_job(max(warmup, 4 * nb))
    e_steps = max(8, steps)
    e2e_ms, y_last = e2e_job(e_steps)
    j_last = (e_steps - 1) % nb
    if not torch.equal(host_out[j_last], y_last.cpu()):
        raise RuntimeError("pipelined end-to-end result differs from the device result")

    (ms32, ms64, e2e_ms), (value, value64, e2e) = job_rates(
        torch, [ms32, ms64, e2e_ms], [steps, max(3, steps // 4), e_steps], world, dist, dev)
    return dict(value=value, value64=value64, e2e=e2e, ms32=ms32 / steps, lat32=lat32,
                lat64=lat64, err32=err32, err64=err64, err_mixed=err_mixed, clocks=clk,
                err_oracle={"f32": orc32, "f64": orc64},
                T_inv=T_inv, T_fwd=T_fwd, T_fwd_exec=T_fwd_exec, h2d=host_in[0].numel() * 8, d2h=host_out[0].numel() * 8)


# ---------------------------------------------------------------------------
# secondary configurations (extra fields of the JSON line)
# ---------------------------------------------------------------------------
def _time(torch, fn, steps, warmup, flush):
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    tot = 0.0
    for _ in range(steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(True), torch.cuda.Event(True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        tot += e0.elapsed_time(e1)
    return tot / steps


def run_batched_precompute(torch, L=512, B=64, steps=5, warmup=2):
    """GL sampling, spin +-2, 64 maps: precompute forward and inverse, FP32 SIMT vs BF16x3
    tcgen05."""
    import s2fft_b200
    from s2fft_b200 import _lib

    dev = torch.device("cuda", torch.cuda.current_device())
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    out = {"workload": f"precompute forward (and inverse), GL, L={L}, {B} maps, spin +-2",
           "maps": B}
    for spin in (2, -2):
        rng = np.random.default_rng(1000 + spin)
        flm = np.stack([seeded_flm(rng, L, spin) for _ in range(B)])
        x64 = torch.from_numpy(flm).to(dev)
        f64 = s2fft_b200.inverse(x64, L, spin, None, "gl")  # seeded maps from the inverse
        K64 = s2fft_b200.precompute.spin_spherical_kernel(L, spin, False, "gl", None, True)
        ref = s2fft_b200.precompute.forward(f64, L, spin, K64, "gl")
        del K64
        torch.cuda.empty_cache()
        res = {}
        for prec in ("f32", "bf16x3"):
            K = s2fft_b200.precompute.spin_spherical_kernel(L, spin, False, "gl", None, True,
                                                            precision=prec)
            f32 = f64.to(torch.complex64)
            plan = _lib.get_plan(dev, L=L, spin=spin, nside=0, sampling=_lib.SAMPLING["gl"],
                                 reality=0, L_lower=0, precision=_lib.PRECISION[prec],
                                 batch=B, iter=0, N=0)
            ev = [torch.cuda.Event(True), torch.cuda.Event(True)]
            for e in ev:
                e.record()
            ms = _time(torch, lambda: s2fft_b200.precompute.forward(f32, L, spin, K, "gl",
                                                                    precision=prec),
                       steps, warmup, flush)
            _lib.check(_lib.lib().s2b_plan_set_events(plan.ptr, 1, ev[0].cuda_event,
                                                      ev[1].cuda_event))
            g = s2fft_b200.precompute.forward(f32, L, spin, K, "gl", precision=prec)
            torch.cuda.synchronize()
            _lib.check(_lib.lib().s2b_plan_set_events(plan.ptr, 1, None, None))
            kern_ms = ev[0].elapsed_time(ev[1]) if prec == "bf16x3" else None
            gh = g[:2].cpu().numpy()
            orc = [golden_err(f"gl_L512_s{spin:+d}_map{k}", "flm", gh[k]) for k in range(2)]
            d = (g.to(torch.complex128) - ref).abs()
            mx = ref.abs().max().item()
            res[prec] = {"maps_per_s": B / (ms * 1e-3), "ms_per_batch": ms,
                         "max_rel_err_vs_fp64_oracle_maps01": (max(orc) if None not in orc
                                                               else None),
                         "max_rel_err": d.max().item() / mx,
                         "rms_rel_err": (d.pow(2).mean().sqrt() / ref.abs().pow(2).mean().sqrt()).item()}
            if kern_ms:
                res[prec]["contraction_ms"] = kern_ms
                nth = L
                flops = 2.0 * L * nth * (2 * L - 1) * 2 * B  # algorithmic (one product per term)
                res[prec]["contraction_tflops_algorithmic"] = flops / (kern_ms * 1e-3) / 1e12
                kbytes = L * nth * (2 * L - 1) * 4.0
                res[prec]["kernel_table_gbs"] = kbytes / (kern_ms * 1e-3) / 1e9
            del K
            torch.cuda.empty_cache()
            # the inverse (flm -> maps) through the precomputed inverse kernel
            Ki = s2fft_b200.precompute.spin_spherical_kernel(L, spin, False, "gl", None, False,
                                                             precision=prec)
            x32 = x64.to(torch.complex64)
            ms_i = _time(torch, lambda: s2fft_b200.precompute.inverse(x32, L, spin, Ki, "gl",
                                                                      precision=prec),
                         steps, warmup, flush)
            fi = s2fft_b200.precompute.inverse(x32, L, spin, Ki, "gl", precision=prec)
            di = (fi.to(torch.complex128) - f64).abs()
            res[prec]["inverse"] = {
                "maps_per_s": B / (ms_i * 1e-3), "ms_per_batch": ms_i,
                "max_rel_err": di.max().item() / f64.abs().max().item(),
                "rms_rel_err": (di.pow(2).mean().sqrt() / f64.abs().pow(2).mean().sqrt()).item()}
            del Ki
            torch.cuda.empty_cache()
        out[f"spin{spin:+d}"] = res
    return out


def run_batched_uneven(torch, nmaps=256, steps=3, warmup=1, seed=4242):
    """256 maps, L uniform in {64..1024}, spin 0..3, sampling in {mw, mwss, dh, gl}, float32:
    inverse + forward of every map, grouped, autotuned and replayed as one CUDA graph: the
    latitudinal kernels of all groups in persistent launches, or every group's own chain of
    launches on concurrent streams (each timed; the headline is the autotuner's pick),
    against the same maps run one call at a time."""
    import s2fft_b200
    from s2fft_b200.batch import BatchedSHT

    Ls = [64, 128, 256, 512, 1024]
    smps = ["mw", "mwss", "dh", "gl"]
    specs, flms = uneven_specs(nmaps, seed)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    ms_sched = {}
    for sched in (True, False):  # each schedule forced, tuned and timed as a graph
        bs = BatchedSHT(specs, precision="f32", persistent=sched)
        bs.load(flms)
        ms_sched["persistent" if sched else "streams"] = _time(torch, bs.run, steps, warmup,
                                                               flush)
        if sched:
            waves = bs.batch_schedule
        del bs
    b = BatchedSHT(specs, precision="f32")  # the autotuner's pick
    b.load(flms)
    ms_graph = _time(torch, b.run, steps, warmup, flush)
    xs = [torch.as_tensor(x).to("cuda", torch.complex64) for x in flms]

    def sequential():
        for (L, sp, smp), x in zip(specs, xs):
            s2fft_b200.forward(s2fft_b200.inverse(x, L, sp, None, smp, precision="f32"), L, sp,
                               None, smp, precision="f32")

    ms_seq = _time(torch, sequential, steps, warmup, flush)
    # per-map parity of the batched path against the unbatched call (every 16th map)
    worst = 0.0
    for i in range(0, nmaps, 16):
        L, sp, smp = specs[i]
        ref = s2fft_b200.forward(s2fft_b200.inverse(xs[i], L, sp, None, smp, precision="f32"),
                                 L, sp, None, smp, precision="f32")
        got = b.coefficients(i)
        worst = max(worst, float((got - ref).abs().max() / ref.abs().max()))
    rt = max(float((b.coefficients(i) - xs[i]).abs().max() / xs[i].abs().max())
             for i in range(0, nmaps, 16))
    return {"workload": f"{nmaps} maps, L in {Ls}, spin 0..3, sampling in {smps}, float32, "
                        "inverse + forward",
            "groups": len(b.groups),
            "graph_maps_per_s": nmaps / (ms_graph * 1e-3), "graph_ms": ms_graph,
            "schedule": b.schedule,
            "schedule_maps_per_s": {k: nmaps / (v * 1e-3) for k, v in ms_sched.items()},
            "persistent_waves_ctas_per_sm": list(waves),
            "autotuner_ms": b.timings,
            "sequential_maps_per_s": nmaps / (ms_seq * 1e-3), "sequential_ms": ms_seq,
            "max_rel_err_vs_unbatched": worst, "max_rel_roundtrip_err": rt,
            "tiles": {"forward_half": sum(g.tuning[0] for g in b.groups),
                      "inverse_one_ring": sum(g.tuning[1] & 1 for g in b.groups),
                      "inverse_segments": {str(n): sum(g.tuning[2] == n for g in b.groups)
                                           for n in (1, 2, 4, 8)}}}


def uneven_specs(nmaps=256, seed=4242):
    """The uneven 256-map mix: L uniform in {64..1024}, spin 0..3, four samplings."""
    rng = np.random.default_rng(seed)
    Ls = [64, 128, 256, 512, 1024]
    smps = ["mw", "mwss", "dh", "gl"]
    specs = [(int(rng.choice(Ls)), int(rng.integers(0, 4)), str(rng.choice(smps)))
             for _ in range(nmaps)]
    return specs, [seeded_flm(rng, L, sp) for L, sp, _ in specs]


def profile_batched_uneven(torch, schedule):
    """One eager inverse + forward of the uneven mix under the given schedule (tuned),
    bracketed by cudaProfilerStart/Stop for a launch list of that call alone."""
    from s2fft_b200.batch import BatchedSHT

    specs, flms = uneven_specs()
    b = BatchedSHT(specs, precision="f32", persistent=schedule == "persistent", graph=False)
    b.load(flms)
    b.run()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(True), torch.cuda.Event(True)
    torch.cuda.profiler.start()
    e0.record()
    b.run()
    e1.record()
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    return {"schedule": schedule, "eager_ms": e0.elapsed_time(e1), "groups": len(b.groups)}


def profile_rotation(torch, L=1024, rot=(0.7, 1.9, -2.4), profile=True):
    """rotate_flms of one float64 map (Euler angles rot): CUDA-event times of five calls
    after a warm-up, the largest change of a degree's power and the round-trip error, then
    (profile) one call between cudaProfilerStart/Stop."""
    from s2fft_b200 import rotation

    dev = torch.device("cuda", torch.cuda.current_device())
    flm = torch.from_numpy(seeded_flm(np.random.default_rng(11), L, 0, False)).to(dev)
    r = rotation.rotate_flms(flm, L, rot)
    back = rotation.rotate_flms(r, L, (-rot[2], -rot[1], -rot[0]))
    torch.cuda.synchronize()
    ts = []
    for _ in range(5):
        e0, e1 = torch.cuda.Event(True), torch.cuda.Event(True)
        e0.record()
        rotation.rotate_flms(flm, L, rot)
        e1.record()
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    if profile:
        torch.cuda.profiler.start()
        rotation.rotate_flms(flm, L, rot)
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
    p0, p1 = (flm.abs() ** 2).sum(-1), (r.abs() ** 2).sum(-1)
    return {"workload": f"rotate_flms L={L} f64, one map, rotation {rot}",
            "ms_min": min(ts), "ms_median": float(np.median(ts)),
            "power_max_rel_change": float(((p1 - p0).abs() / p0.clamp_min(1e-300)).max()),
            "roundtrip_max_rel_err": float((back - flm).abs().max() / flm.abs().max())}


def profile_planes(torch, L=256, beta=np.pi / 2):
    """generate_rotate_dls(L, beta) (the Fourier-Wigner Delta planes at pi/2): CUDA-event
    times of three calls after a warm-up, the write rate of the [L][2L-1][2L-1] float64
    output, then one call between cudaProfilerStart/Stop."""
    from s2fft_b200 import rotation

    out = rotation.generate_rotate_dls(L, beta)
    torch.cuda.synchronize()
    ts = []
    for _ in range(3):
        e0, e1 = torch.cuda.Event(True), torch.cuda.Event(True)
        e0.record()
        out = rotation.generate_rotate_dls(L, beta)
        e1.record()
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    torch.cuda.profiler.start()
    out = rotation.generate_rotate_dls(L, beta)
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    nbytes = out.numel() * 8
    return {"workload": f"generate_rotate_dls L={L} beta={beta:.6f}", "ms_min": min(ts),
            "output_bytes": nbytes, "write_gbs": nbytes / (min(ts) * 1e6)}


def profile_fourier_wigner(torch, L=256, N=8, prec="f32"):
    """Fourier-Wigner inverse and forward of one seeded MW signal: CUDA-event minimum of five
    calls each after a warm-up, the round-trip error, then one inverse and one forward
    between cudaProfilerStart/Stop."""
    from s2fft_b200 import fourier_wigner as fw

    dev = torch.device("cuda", torch.cuda.current_device())
    rng = np.random.default_rng(8)
    flmn = np.stack([seeded_flm(rng, L, n) for n in range(-(N - 1), N)])
    x = torch.from_numpy(flmn).to(dev).to(torch.complex64 if prec == "f32" else torch.complex128)
    pre = fw.fourier_wigner_kernel(L)
    f = fw.inverse_transform(x, L, N, pre, precision=prec)
    g = fw.forward_transform(f, L, N, pre, precision=prec)
    torch.cuda.synchronize()
    out = {"workload": f"Fourier-Wigner mw L={L} N={N} {prec}, one signal"}
    for name, fn in (("inverse", lambda: fw.inverse_transform(x, L, N, pre, precision=prec)),
                     ("forward", lambda: fw.forward_transform(f, L, N, pre, precision=prec))):
        ts = []
        for _ in range(5):
            e0, e1 = torch.cuda.Event(True), torch.cuda.Event(True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        out[name + "_ms"] = min(ts)
    torch.cuda.profiler.start()
    f = fw.inverse_transform(x, L, N, pre, precision=prec)
    fw.forward_transform(f, L, N, pre, precision=prec)
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    out["roundtrip_max_rel_err"] = float((g.to(torch.complex128) - x.to(torch.complex128)).abs()
                                         .max() / x.abs().max())
    return out


def profile_healpix(torch, nside=256, L=512):
    """One float32 HEALPix inverse and forward (3 iterations) after a warm-up call, between
    cudaProfilerStart/Stop."""
    import s2fft_b200

    dev = torch.device("cuda", torch.cuda.current_device())
    flm = torch.from_numpy(seeded_flm(np.random.default_rng(7), L, 0, True)).to(dev,
                                                                                 torch.complex64)

    def call():
        f = s2fft_b200.inverse(flm, L, 0, nside, "healpix", reality=True, precision="f32")
        return s2fft_b200.forward(f, L, 0, nside, "healpix", reality=True, iter=3,
                                  precision="f32")

    call()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(True), torch.cuda.Event(True)
    torch.cuda.profiler.start()
    e0.record()
    g = call()
    e1.record()
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    err = ((g - flm).abs().max() / flm.abs().max()).item()
    return {"workload": f"healpix nside={nside} L={L} reality f32, inverse + forward iter=3",
            "eager_ms": e0.elapsed_time(e1), "roundtrip_max_rel_err": err}


def run_healpix_iter(torch, nside=256, L=512, steps=5, warmup=2):
    """HEALPix nside=256, L=512, real signal: inverse + forward with 3 refinement iterations."""
    import s2fft_b200

    dev = torch.device("cuda", torch.cuda.current_device())
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    rng = np.random.default_rng(7)
    flm = torch.from_numpy(seeded_flm(rng, L, 0, True)).to(dev)
    out = {"workload": f"healpix nside={nside} L={L} reality, forward iter=3"}
    for prec in ("f32", "f64"):
        x = flm.to(torch.complex64 if prec == "f32" else torch.complex128)
        f = s2fft_b200.inverse(x, L, 0, nside, "healpix", reality=True, precision=prec)
        ms_inv = _time(torch, lambda: s2fft_b200.inverse(x, L, 0, nside, "healpix", reality=True,
                                                         precision=prec), steps, warmup, flush)
        ms_fwd = _time(torch, lambda: s2fft_b200.forward(f, L, 0, nside, "healpix", reality=True,
                                                         iter=3, precision=prec),
                       steps, warmup, flush)
        g = s2fft_b200.forward(f, L, 0, nside, "healpix", reality=True, iter=3, precision=prec)
        err = ((g.to(torch.complex128) - flm).abs().max() / flm.abs().max()).item()
        out[prec] = {"inverse_ms": ms_inv, "forward_iter3_ms": ms_fwd,
                     "roundtrip_max_rel_err": err}
    return out


def run_so3(torch, L=128, N=8, steps=10, warmup=3):
    """SO(3), MW, L=128, N=8, one complex signal: inverse + forward by the Fourier-Wigner
    transforms (Delta-plane contraction + FFTs) and by the recursion-based Wigner
    transforms (2N-1 spin transforms + gamma DFT), float32 and float64."""
    import s2fft_b200
    from s2fft_b200 import fourier_wigner as fw

    dev = torch.device("cuda", torch.cuda.current_device())
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    rng = np.random.default_rng(8)
    # slice n holds a spin -n field: zero below l = |n|
    flmn = np.stack([seeded_flm(rng, L, n) for n in range(-(N - 1), N)])
    flmn64 = torch.from_numpy(flmn).to(dev)
    pre = fw.fourier_wigner_kernel(L)
    ref_f = fw.inverse_transform(flmn64, L, N, pre)
    out = {"workload": f"SO(3) mw L={L} N={N}, complex, inverse + forward, one signal"}
    for prec in ("f32", "f64"):
        x = flmn64.to(torch.complex64 if prec == "f32" else torch.complex128)
        f = fw.inverse_transform(x, L, N, pre, precision=prec)
        ms_fw = _time(torch, lambda: fw.forward_transform(
            fw.inverse_transform(x, L, N, pre, precision=prec), L, N, pre, precision=prec),
            steps, warmup, flush)
        fr = s2fft_b200.wigner.inverse(x, L, N, sampling="mw", precision=prec)
        ms_rec = _time(torch, lambda: s2fft_b200.wigner.forward(
            s2fft_b200.wigner.inverse(x, L, N, sampling="mw", precision=prec), L, N,
            sampling="mw", precision=prec), steps, warmup, flush)
        g = fw.forward_transform(f, L, N, pre, precision=prec)
        err_inv = ((f.to(torch.complex128) - ref_f).abs().max() / ref_f.abs().max()).item()
        err_rt = ((g.to(torch.complex128) - flmn64).abs().max() / flmn64.abs().max()).item()
        err_rec = ((fr.to(torch.complex128) - ref_f).abs().max() / ref_f.abs().max()).item()
        out[prec] = {"fourier_wigner_ms": ms_fw, "fourier_wigner_per_s": 1e3 / ms_fw,
                     "recursion_ms": ms_rec, "recursion_per_s": 1e3 / ms_rec,
                     "inverse_max_rel_err_vs_fw_f64": err_inv,
                     "roundtrip_max_rel_err": err_rt,
                     "recursion_vs_fw_f64_max_rel": err_rec}
    return out


# ---------------------------------------------------------------------------
# CPU reference: the float64 restatement of the upstream algorithm (oracle/):
# upstream's log-renormalised Price-McEwen latitudinal steps in C (oracle/csrc/otf.c,
# OpenMP over the rings on every host thread) with the resampling and ring FFT
# stages in numpy, as upstream runs them. Every step is one whole L=1024 MW
# inverse + forward; the recursion precomputes are built once, before timing (as
# the GPU plan is).
# ---------------------------------------------------------------------------
def jax_cpu_status():
    try:
        import jax  # noqa: F401
    except Exception:
        return "unavailable (jax not installed)"
    return "installed but not timed (the reference's JAX path is not part of this port)"


class CpuReference:
    def __init__(self, L):
        import oracle
        from oracle import cport

        cport.build()
        self.oracle, self.L = oracle, L
        rng = np.random.default_rng(0)
        self.flm = oracle.signal.generate_flm_full_complex(rng, L)
        t0 = time.perf_counter()
        self.pre_inv = cport.precompute(L, 0, oracle.samples.thetas(L, "mw"), 0)
        self.pre_fwd = cport.precompute(L, 0, oracle.samples.thetas(2 * L, "mwss")[1:-1], 0)
        self.precompute_s = time.perf_counter() - t0
        self.threads = cport.max_threads()

    def step(self):
        """One inverse + forward; returns (seconds, round-trip max relative error)."""
        o, L = self.oracle, self.L
        t0 = time.perf_counter()
        f = o.spherical.inverse(self.flm, L, 0, None, "mw", precomps=self.pre_inv, backend="c")
        g = o.spherical.forward(f, L, 0, None, "mw", precomps=self.pre_fwd, backend="c")
        dt = time.perf_counter() - t0
        return dt, float(np.abs(g - self.flm).max() / np.abs(self.flm).max())

    def sample(self, steps):
        return (f"oracle: C restatement of upstream's numpy latitudinal steps "
                f"(log-renormalised Price-McEwen recursion, exp/log per term; OpenMP over "
                f"rings, {self.threads} host threads) + numpy resampling/ring FFTs; {steps} "
                f"whole L={self.L} MW inverse+forward pairs, each timed in full (no "
                f"extrapolation); recursion precompute ({self.precompute_s:.2f} s) built once "
                f"before timing")


# ---------------------------------------------------------------------------
# main
# ---------------------------------------------------------------------------
def main():
    args = parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    config = {"workload": "spin SHT inverse+forward, MW sampling, L=1024, spin 0, complex, "
                          "float32 recursion/projection with float64 seeds/exponents/weights",
              "L": args.L, "sampling": "mw", "spin": 0, "maps_per_step": 1,
              "l2": "flushed between timed steps (256 MB write)",
              "parallelism": f"replicas x{world}"}

    if args.impl == "reference":
        if rank != 0:
            return
        ref = CpuReference(args.L)
        for _ in range(args.warmup):
            ref.step()
        times, rts = [], []
        t0 = time.perf_counter()
        for _ in range(args.steps):
            dt, rt = ref.step()
            times.append(dt)
            rts.append(rt)
        total = time.perf_counter() - t0
        v = args.steps / total
        line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT,
                "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded N(0,1) flm)", "config": config,
                "cpu_baseline": {"value": v, "unit": UNIT, "cores": ref.threads, "kind": "port",
                                 "sample": ref.sample(args.steps),
                                 "step_s_min": min(times), "step_s_max": max(times),
                                 "roundtrip_max_rel_err": max(rts),
                                 "precompute_s": ref.precompute_s},
                "jax_cpu": jax_cpu_status(),
                "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    import torch

    dist = None
    if world > 1:
        import datetime

        import torch.distributed as tdist

        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = tdist
    else:
        torch.cuda.set_device(0)
    if args.tc_profile:
        print(json.dumps(run_batched_precompute(torch, L=args.L if args.L != 1024 else 256, B=64,
                                                steps=1, warmup=1)))
        return
    if args.healpix_profile:
        print(json.dumps(profile_healpix(torch)))
        return
    if args.batch_profile:
        print(json.dumps(profile_batched_uneven(torch, args.batch_profile)))
        return
    if args.rotate_profile:
        print(json.dumps(profile_rotation(torch, args.L)))
        return
    if args.planes_profile:
        print(json.dumps(profile_planes(torch, args.L)))
        return
    if args.fw_profile:
        print(json.dumps(profile_fourier_wigner(torch, args.L)))
        return
    if args.profile_case:
        args.steps, args.warmup = 2, 1
    r = run_ours(args, rank, world, torch, dist)
    if dist is not None:
        dist.barrier()
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    peaks, kind = measured_peaks()
    fp32_peak = simt_peak_tflops(torch, False)
    fp64_peak = simt_peak_tflops(torch, True)
    lat_inv_ms, lat_fwd_ms = r["lat32"]
    ach_fwd = FLOPS_PER_TRIPLE * r["T_fwd"] / (lat_fwd_ms * 1e-3) / 1e12
    ach_inv = FLOPS_PER_TRIPLE * r["T_inv"] / (lat_inv_ms * 1e-3) / 1e12
    traffic = {"inverse": None, "forward": None}
    tpath = os.path.join(ROOT, "profiles", "latitudinal_traffic.txt")
    if os.path.exists(tpath):
        for ln in open(tpath):
            for k in traffic:
                if ln.startswith(f"L={args.L} {k}_f32 bytes_per_launch="):
                    traffic[k] = float(ln.split("=")[-1])
    line = {"metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms32"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded N(0,1) flm, all |m| <= l)", "config": config,
            "max_rel_err_vs_fp64": r["err_mixed"], "roundtrip_rel_err_f32": r["err32"],
            # against upstream's float64 numpy transforms of the same seeded input, at the
            # 2048 entries of each result stored in tests/golden/large.npz
            "max_rel_err_vs_fp64_oracle": r["err_oracle"],
            "roundtrip_rel_err_f64": r["err64"],
            "fp64_path": {"value": r["value64"], "unit": UNIT,
                          "speedup_mixed_over_fp64": r["value"] / r["value64"]},
            # the dominant kernel of the step: the inverse latitudinal (recursion + synthesis);
            # the forward one is reported beside it
            "roofline": {"bound": "fp32", "kernel": "latitudinal inverse (recursion+synthesis)",
                         "achieved": ach_inv, "peak": fp32_peak, "unit": "TFLOP/s",
                         "frac": ach_inv / fp32_peak, "traffic": traffic["inverse"],
                         "traffic_source": "dram bytes per launch from an ncu capture, "
                                           "profiles/latitudinal_traffic.txt (not measured "
                                           "in this run)",
                         "peak_source": "measured FMA-chain probe (MEASURED_PEAKS.json has no "
                                        "FP32-SIMT figure)",
                         "flops_per_launch": FLOPS_PER_TRIPLE * r["T_inv"],
                         "launch_ms": lat_inv_ms,
                         "forward": {
                             "kernel": "latitudinal forward (recursion+projection)",
                             "achieved": ach_fwd, "frac": ach_fwd / fp32_peak,
                             "traffic": traffic["forward"],
                             "flops_per_launch": FLOPS_PER_TRIPLE * r["T_fwd"],
                             "launch_ms": lat_fwd_ms,
                             # the spin-0 forward runs on the equator-symmetric MWSS(2L) rings:
                             # one recursion and one projection per ring pair (theta, pi -
                             # theta) serve both rings (d(pi - theta) = (-1)^(l+m) d(theta)),
                             # so it executes about half the algorithmic flops; its frac above
                             # 1 comes from that
                             "symmetric_ring_pairs": True,
                             "executed_flops_per_launch": FLOPS_PER_TRIPLE * r["T_fwd_exec"],
                             "executed_frac": FLOPS_PER_TRIPLE * r["T_fwd_exec"]
                             / (lat_fwd_ms * 1e-3) / 1e12 / fp32_peak}},
            "fp64_roofline": {"kernel": "latitudinal inverse",
                              "achieved": FLOPS_PER_TRIPLE * r["T_inv"] / (r["lat64"][0] * 1e-3)
                              / 1e12, "peak": fp64_peak, "unit": "TFLOP/s"},
            "hbm_peak_gbs": peaks.get("hbm_gbs"), "peaks_source": kind,
            "clocks": r["clocks"],
            "e2e": {"value": r["e2e"], "unit": UNIT, "h2d_bytes_per_step": r["h2d"],
                    "d2h_bytes_per_step": r["d2h"]},
            # per step: prologue (with the pole rows), inverse latitudinal, inverse ring FFTs,
            # forward ring FFTs, column chain, forward latitudinal, epilogue
            "gpu_launches": 7 * args.steps}
    if not args.profile_case and not args.no_extra and world == 1:
        line["batched_precompute"] = run_batched_precompute(torch)
        line["healpix_iter3"] = run_healpix_iter(torch)
        line["batched_uneven"] = run_batched_uneven(torch)
        line["so3_fourier_wigner"] = run_so3(torch)
        line["rotation"] = profile_rotation(torch, 1024, profile=False)
    if not args.no_cpu_baseline and not args.profile_case and world == 1:
        ref = CpuReference(args.L)
        ref.step()  # warm-up (thread pool, page faults)
        n, t = 0, 0.0
        while n < 1 or (t < args.cpu_budget and n < 5):
            t += ref.step()[0]
            n += 1
        line["cpu_baseline"] = {"value": n / t, "unit": UNIT, "cores": ref.threads,
                                "kind": "port", "sample": ref.sample(n),
                                "precompute_s": ref.precompute_s}
    line["jax_cpu"] = jax_cpu_status()
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
