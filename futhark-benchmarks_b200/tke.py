"""Python host mirror of libtke.so (include/tke.h): the ocean model's
turbulent-kinetic-energy step, misc/ocean-sim/tke.fut's entry ``main`` (f32).

    ctx = TkeContext()                       # futhark_context_config_new + futhark_context_new
    outs = ctx.main(*inputs)                 # 25 host arrays in the entry's order -> 7 outputs

``main`` has the generated API's names and argument order (INPUT_NAMES,
OUTPUT_NAMES); ``step`` is the engine extension on device pointers (no
allocation, asynchronous on the context's stream).  There is no CPU fallback:
a missing libtke.so fails the construction loudly.
"""
from __future__ import annotations

import ctypes
import os
from typing import Dict, Sequence, Tuple

import numpy as np

from . import FUTHARK_OUT_OF_MEMORY, FUTHARK_PROGRAM_ERROR, FutharkError

TKE_LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libtke.so")

# tke.fut:64-95, the entry point's parameters in order
INPUT_NAMES = ("tketau", "tketaup1", "tketaum1", "dtketau", "dtketaup1", "dtketaum1", "utau", "vtau", "wtau",
               "maskU", "maskV", "maskW", "dxt", "dxu", "dyt", "dyu", "dzt", "dzw", "cost", "cosu", "kbot",
               "kappaM", "mxl", "forc", "forc_tke_surface")
# tke.fut:348
OUTPUT_NAMES = ("tketau", "tketaup1", "tketaum1", "dtketau", "dtketaup1", "dtketaum1", "tke_surf_corr")
# array kind of each input: (element type, rank)
_KIND = {name: ("f32", 3) for name in INPUT_NAMES}
_KIND.update({name: ("f32", 1) for name in ("dxt", "dxu", "dyt", "dyu", "dzt", "dzw", "cost", "cosu")})
_KIND["kbot"] = ("i32", 2)
_KIND["forc_tke_surface"] = ("f32", 2)
# the fields of struct tke_step_args after the three dimensions
STEP_INPUTS = ("tketau", "tketaup1", "dtketau", "dtketaum1", "utau", "vtau", "wtau", "maskU", "maskV", "maskW",
               "dxt", "dxu", "dyt", "dyu", "dzt", "dzw", "cost", "cosu", "kbot", "kappaM", "mxl", "forc",
               "forc_tke_surface")
STEP_OUTPUTS = ("tketaup1_out", "dtketau_out", "tke_surf_corr_out")


class _StepArgs(ctypes.Structure):
    _fields_ = ([("xdim", ctypes.c_int64), ("ydim", ctypes.c_int64), ("zdim", ctypes.c_int64)]
                + [(n, ctypes.c_void_p) for n in STEP_INPUTS + STEP_OUTPUTS] + [("scratch", ctypes.c_void_p)])


_lib = None


def load_library(path: str = TKE_LIB_PATH):
    """Load libtke.so and declare its C signatures."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing; build it with `python futhark-benchmarks_b200/build.py`")
    L = ctypes.CDLL(path)
    vp, i64, c_int = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int
    sig = {
        "futhark_context_config_new": (vp, []),
        "futhark_context_config_free": (None, [vp]),
        "futhark_context_config_set_device": (None, [vp, ctypes.c_char_p]),
        "futhark_context_config_set_debugging": (None, [vp, c_int]),
        "futhark_context_config_set_profiling": (None, [vp, c_int]),
        "futhark_context_config_set_logging": (None, [vp, c_int]),
        "futhark_context_new": (vp, [vp]),
        "futhark_context_free": (None, [vp]),
        "futhark_context_sync": (c_int, [vp]),
        "futhark_context_get_error": (ctypes.POINTER(ctypes.c_char), [vp]),
        "futhark_context_clear_caches": (c_int, [vp]),
        "futhark_new_f32_1d": (vp, [vp, vp, i64]),
        "futhark_new_f32_2d": (vp, [vp, vp, i64, i64]),
        "futhark_new_f32_3d": (vp, [vp, vp, i64, i64, i64]),
        "futhark_new_i32_2d": (vp, [vp, vp, i64, i64]),
        "futhark_entry_main": (c_int, [vp] + [ctypes.POINTER(vp)] * 7 + [vp] * 25),
        "tke_scratch_bytes": (ctypes.c_size_t, [i64, i64, i64]),
        "tke_step_f32": (c_int, [vp, ctypes.POINTER(_StepArgs)]),
        "tke_check": (c_int, [vp]),
        "tke_context_stream": (vp, [vp]),
        "tke_launches_per_step": (c_int, []),
    }
    for kind in ("f32_1d", "f32_2d", "f32_3d", "i32_2d"):
        sig[f"futhark_free_{kind}"] = (c_int, [vp, vp])
        sig[f"futhark_values_{kind}"] = (c_int, [vp, vp, vp])
        sig[f"futhark_shape_{kind}"] = (ctypes.POINTER(i64), [vp, vp])
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    L.free_str = ctypes.CDLL(None).free
    L.free_str.argtypes = [vp]
    L.free_str.restype = None
    _lib = L
    return L


class TkeContext:
    """A libtke.so context on one CUDA device ("#k" selects device k)."""

    def __init__(self, device: str | None = None):
        self.lib = load_library()
        cfg = self.lib.futhark_context_config_new()
        if device is not None:
            self.lib.futhark_context_config_set_device(cfg, device.encode())
        self._ctx = self.lib.futhark_context_new(cfg)
        self.lib.futhark_context_config_free(cfg)
        if not self._ctx:
            raise FutharkError(FUTHARK_OUT_OF_MEMORY, "futhark_context_new failed")
        err = self._take_error()
        if err:
            self.lib.futhark_context_free(self._ctx)
            self._ctx = None
            raise FutharkError(FUTHARK_PROGRAM_ERROR, err)

    def _take_error(self) -> str:
        p = self.lib.futhark_context_get_error(self._ctx)
        if not p:
            return ""
        msg = ctypes.cast(p, ctypes.c_char_p).value.decode(errors="replace")
        self.lib.free_str(ctypes.cast(p, ctypes.c_void_p))
        return msg

    def _check(self, rc: int):
        if rc != 0:
            raise FutharkError(rc, self._take_error() or "unknown error")

    def close(self):
        if getattr(self, "_ctx", None):
            self.lib.futhark_context_free(self._ctx)
            self._ctx = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _new(self, name: str, v: np.ndarray):
        etype, rank = _KIND[name]
        v = np.ascontiguousarray(v, dtype=np.int32 if etype == "i32" else np.float32)
        if v.ndim != rank:
            raise ValueError(f"tke main: {name} must have rank {rank}")
        h = getattr(self.lib, f"futhark_new_{etype}_{rank}d")(self._ctx, v.ctypes.data, *v.shape)
        if not h:
            raise FutharkError(FUTHARK_OUT_OF_MEMORY, self._take_error() or "array allocation failed")
        return h, f"{etype}_{rank}d"

    def _fetch(self, kind: str, h) -> np.ndarray:
        shape = getattr(self.lib, f"futhark_shape_{kind}")(self._ctx, h)
        rank = int(kind[4])
        res = np.empty(tuple(shape[r] for r in range(rank)), dtype=np.float32)
        self._check(getattr(self.lib, f"futhark_values_{kind}")(self._ctx, h, res.ctypes.data))
        return res

    def main(self, *inputs) -> Tuple[np.ndarray, ...]:
        """futhark_entry_main on 25 host arrays in INPUT_NAMES order; returns the
        7 outputs in OUTPUT_NAMES order as numpy arrays."""
        if len(inputs) != len(INPUT_NAMES):
            raise ValueError(f"tke main takes {len(INPUT_NAMES)} inputs")
        ins = []
        outs = [ctypes.c_void_p() for _ in OUTPUT_NAMES]
        try:
            for name, v in zip(INPUT_NAMES, inputs):
                ins.append(self._new(name, v))
            self._check(self.lib.futhark_entry_main(self._ctx, *[ctypes.byref(o) for o in outs],
                                                    *[h for h, _ in ins]))
            kinds = ["f32_3d"] * 6 + ["f32_2d"]
            return tuple(self._fetch(k, o) for k, o in zip(kinds, outs))
        finally:
            for k, o in zip(["f32_3d"] * 6 + ["f32_2d"], outs):
                if o.value:
                    getattr(self.lib, f"futhark_free_{k}")(self._ctx, o)
            for h, k in ins:
                getattr(self.lib, f"futhark_free_{k}")(self._ctx, h)

    def scratch_bytes(self, xdim: int, ydim: int, zdim: int) -> int:
        return int(self.lib.tke_scratch_bytes(xdim, ydim, zdim))

    def step(self, dims: Sequence[int], ptrs: Dict[str, int]):
        """tke_step_f32: one step on device pointers (ptrs maps STEP_INPUTS,
        STEP_OUTPUTS and "scratch" to addresses), asynchronous on this
        context's stream."""
        args = _StepArgs(*dims, *[ptrs[n] for n in STEP_INPUTS + STEP_OUTPUTS], ptrs["scratch"])
        self._check(self.lib.tke_step_f32(self._ctx, ctypes.byref(args)))

    def check(self):
        """Synchronises; raises if a step's vertical solve gave up on a copy."""
        self._check(self.lib.tke_check(self._ctx))

    def sync(self):
        self._check(self.lib.futhark_context_sync(self._ctx))

    @property
    def stream(self) -> int:
        return self.lib.tke_context_stream(self._ctx) or 0

    @property
    def launches_per_step(self) -> int:
        return int(self.lib.tke_launches_per_step())
