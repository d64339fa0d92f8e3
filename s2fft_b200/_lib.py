"""ctypes binding of ``libs2b.so`` and the plan cache.

The library is the product: there is no CPU fallback. If the shared library
is missing, or no CUDA device is present, every transform raises.
"""

from __future__ import annotations

import ctypes
import os
import threading

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libs2b.so")

SAMPLING = {"mw": 0, "mwss": 1, "dh": 2, "gl": 3, "healpix": 4}
PRECISION = {"f64": 0, "f32": 1, "bf16x3": 2}

S2B_OK = 0
STATUS = {1: "invalid argument", 2: "CUDA error", 3: "workspace too small",
          4: "NULL or misaligned pointer", 5: "device wait timed out", 6: "internal error"}


class S2BError(RuntimeError):
    """A C-ABI call returned a non-zero status."""


class Desc(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in
                ("L", "spin", "nside", "sampling", "reality", "L_lower", "precision",
                 "batch", "iter", "N")]


_lib = None
_lib_lock = threading.Lock()

# name -> (argtypes); every entry point returns int
_SIGS = {
    "s2b_version": [],
    "s2b_plan_create": [ctypes.POINTER(Desc), ctypes.POINTER(ctypes.c_void_p)],
    "s2b_plan_destroy": [ctypes.c_void_p],
    "s2b_workspace_size": [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_size_t)],
    "s2b_inverse": [ctypes.c_void_p] * 4 + [ctypes.c_size_t, ctypes.c_void_p],
    "s2b_forward": [ctypes.c_void_p] * 4 + [ctypes.c_size_t, ctypes.c_void_p],
    "s2b_wigner_inverse": [ctypes.c_void_p] * 4 + [ctypes.c_size_t, ctypes.c_void_p],
    "s2b_wigner_forward": [ctypes.c_void_p] * 4 + [ctypes.c_size_t, ctypes.c_void_p],
    "s2b_plan_status": [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)],
    "s2b_kernel_size": [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_size_t)],
    "s2b_kernel_build": [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p],
    "s2b_precompute_inverse": [ctypes.c_void_p] * 5 + [ctypes.c_size_t, ctypes.c_void_p],
    "s2b_precompute_forward": [ctypes.c_void_p] * 5 + [ctypes.c_size_t, ctypes.c_void_p],
    "s2b_plan_set_events": [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p],
    "s2b_fma_probe": [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p],
    "s2b_inverse_noalloc": [ctypes.c_void_p] * 4,
    "s2b_healpix_fft": [ctypes.c_void_p] * 4,
    "s2b_healpix_ifft": [ctypes.c_void_p] * 4,
    "s2b_plan_set_tuning": [ctypes.c_void_p, ctypes.c_int, ctypes.c_int],
    "s2b_inverse_adjoint": [ctypes.c_void_p] * 4 + [ctypes.c_size_t, ctypes.c_void_p],
    "s2b_forward_adjoint": [ctypes.c_void_p] * 4 + [ctypes.c_size_t, ctypes.c_void_p],
    "s2b_precompute_inverse_adjoint": [ctypes.c_void_p] * 5 + [ctypes.c_size_t, ctypes.c_void_p],
    "s2b_precompute_forward_adjoint": [ctypes.c_void_p] * 5 + [ctypes.c_size_t, ctypes.c_void_p],
    "s2b_rotate_flms": [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                        ctypes.c_double, ctypes.c_double] + [ctypes.c_void_p] * 4
                       + [ctypes.c_size_t, ctypes.c_void_p],
    "s2b_rotate_dls": [ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p,
                       ctypes.c_size_t, ctypes.c_void_p],
    "s2b_plan_device": [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)],
    "s2b_debug_set_plan_device": [ctypes.c_void_p, ctypes.c_int],
    "s2b_batch_create": [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)],
    "s2b_batch_destroy": [ctypes.c_void_p],
    "s2b_batch_inverse": [ctypes.c_void_p] * 5 + [ctypes.c_void_p],
    "s2b_batch_forward": [ctypes.c_void_p] * 5 + [ctypes.c_void_p],
    "s2b_batch_set_option": [ctypes.c_void_p, ctypes.c_int, ctypes.c_int],
}


def lib():
    """Load the shared library (raises if it is absent)."""
    global _lib
    with _lib_lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(
                    f"{LIB_PATH} not found: build it with `python -m s2fft_b200._build`")
            handle = ctypes.CDLL(LIB_PATH)
            for name, argt in _SIGS.items():
                fn = getattr(handle, name)
                fn.argtypes = argt
                fn.restype = ctypes.c_int
            handle.s2b_last_error.argtypes = []
            handle.s2b_last_error.restype = ctypes.c_char_p
            handle.s2b_rotate_workspace_size.argtypes = [ctypes.c_int]
            handle.s2b_rotate_workspace_size.restype = ctypes.c_size_t
            handle.s2b_device_alloc_count.argtypes = []
            handle.s2b_device_alloc_count.restype = ctypes.c_longlong
            _lib = handle
    return _lib


def check(rc):
    if rc != S2B_OK:
        msg = lib().s2b_last_error().decode()
        raise S2BError(f"s2b status {rc} ({STATUS.get(rc, '?')}): {msg}")


class Plan:
    """A device plan plus its cached workspaces (one per direction)."""

    def __init__(self, device, **desc):
        self.device = device
        self.desc = dict(desc)
        d = Desc(**desc)
        ptr = ctypes.c_void_p()
        with torch.cuda.device(device):
            check(lib().s2b_plan_create(ctypes.byref(d), ctypes.byref(ptr)))
        self.ptr = ptr
        self._ws = {}

    def workspace(self, forward):
        """Workspace of a call: 0 inverse, 1 forward, 2 inverse adjoint, 3 forward adjoint."""
        key = int(forward)
        if key not in self._ws:
            n = ctypes.c_size_t()
            check(lib().s2b_workspace_size(self.ptr, key, ctypes.byref(n)))
            self._ws[key] = torch.empty(max(int(n.value), 256), dtype=torch.uint8,
                                        device=self.device)
        return self._ws[key]

    def status(self):
        """Device status word (synchronous); raises if a bounded device wait gave up."""
        st = ctypes.c_int()
        check(lib().s2b_plan_status(self.ptr, ctypes.byref(st)))
        return st.value

    def __del__(self):
        try:
            if getattr(self, "ptr", None) and self.ptr.value:
                lib().s2b_plan_destroy(self.ptr)
        except Exception:
            pass


class Batch:
    """An uneven batch of spin plans (s2b_batch_*): entry k transforms with plans[k]."""

    def __init__(self, plans):
        self.plans = list(plans)  # the plans must outlive the batch
        arr = (ctypes.c_void_p * len(self.plans))(*[p.ptr.value for p in self.plans])
        ptr = ctypes.c_void_p()
        with torch.cuda.device(self.plans[0].device):
            check(lib().s2b_batch_create(arr, len(self.plans), ctypes.byref(ptr)))
        self.ptr = ptr

    @staticmethod
    def _ptrs(tensors):
        return (ctypes.c_void_p * len(tensors))(*[t.data_ptr() for t in tensors])

    def _call(self, fn, ins, outs, ws, stream):
        n = len(self.plans)
        if not (len(ins) == len(outs) == len(ws) == n):
            raise ValueError(f"a batch of {n} entries needs {n} inputs, outputs and workspaces")
        sizes = (ctypes.c_size_t * n)(*[w.numel() for w in ws])
        check(fn(self.ptr, self._ptrs(ins), self._ptrs(outs), self._ptrs(ws), sizes,
                 ctypes.c_void_p(stream.cuda_stream)))

    def set_schedule(self, waves=1, ctas_per_sm=0):
        """Waves of the staged execution and CTAs per SM of the persistent launches."""
        check(lib().s2b_batch_set_option(self.ptr, 0, int(waves)))
        check(lib().s2b_batch_set_option(self.ptr, 1, int(ctas_per_sm)))

    def inverse(self, flms, fs, ws, stream):
        self._call(lib().s2b_batch_inverse, flms, fs, ws, stream)

    def forward(self, fs, flms, ws, stream):
        self._call(lib().s2b_batch_forward, fs, flms, ws, stream)

    def __del__(self):
        try:
            if getattr(self, "ptr", None) and self.ptr.value:
                lib().s2b_batch_destroy(self.ptr)
        except Exception:
            pass


_plans: dict = {}
_plans_lock = threading.Lock()


def get_plan(device, **desc) -> Plan:
    key = (str(device),) + tuple(sorted(desc.items()))
    with _plans_lock:
        plan = _plans.get(key)
        if plan is None:
            plan = Plan(device, **desc)
            _plans[key] = plan
    return plan


def clear_plans():
    with _plans_lock:
        _plans.clear()


def stream_handle(device):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)
