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

from .program_lib import ProgramContext, load_program_library

TKE_LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libtke.so")

# tke.fut:64-95, the entry point's parameters in order
INPUT_NAMES = ("tketau", "tketaup1", "tketaum1", "dtketau", "dtketaup1", "dtketaum1", "utau", "vtau", "wtau",
               "maskU", "maskV", "maskW", "dxt", "dxu", "dyt", "dyu", "dzt", "dzw", "cost", "cosu", "kbot",
               "kappaM", "mxl", "forc", "forc_tke_surface")
# tke.fut:348
OUTPUT_NAMES = ("tketau", "tketaup1", "tketaum1", "dtketau", "dtketaup1", "dtketaum1", "tke_surf_corr")
# array kind of each input
_KIND = {name: "f32_3d" for name in INPUT_NAMES}
_KIND.update({name: "f32_1d" for name in ("dxt", "dxu", "dyt", "dyu", "dzt", "dzw", "cost", "cosu")})
_KIND["kbot"] = "i32_2d"
_KIND["forc_tke_surface"] = "f32_2d"
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
    if _lib is None:
        vp, i64, c_int = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int
        _lib = load_program_library(path, ("f32_1d", "f32_2d", "f32_3d", "i32_2d"), {
            "futhark_entry_main": (c_int, [vp] + [ctypes.POINTER(vp)] * 7 + [vp] * 25),
            "tke_scratch_bytes": (ctypes.c_size_t, [i64, i64, i64]),
            "tke_step_f32": (c_int, [vp, ctypes.POINTER(_StepArgs)]),
            "tke_check": (c_int, [vp]),
            "tke_context_stream": (vp, [vp]),
            "tke_launches_per_step": (c_int, []),
        })
    return _lib


class TkeContext(ProgramContext):
    """A libtke.so context on one CUDA device ("#k" selects device k)."""

    def __init__(self, device: str | None = None):
        super().__init__(load_library(), device)

    def main(self, *inputs) -> Tuple[np.ndarray, ...]:
        """futhark_entry_main on 25 host arrays in INPUT_NAMES order; returns the
        7 outputs in OUTPUT_NAMES order as numpy arrays."""
        if len(inputs) != len(INPUT_NAMES):
            raise ValueError(f"tke main takes {len(INPUT_NAMES)} inputs")
        kinds = ["f32_3d"] * 6 + ["f32_2d"]
        ins = []
        outs = [ctypes.c_void_p() for _ in OUTPUT_NAMES]
        try:
            for name, v in zip(INPUT_NAMES, inputs):
                ins.append(self.new_array(_KIND[name], v))
            self._check(self.lib.futhark_entry_main(self._ctx, *[ctypes.byref(o) for o in outs],
                                                    *[h for h, _ in ins]))
            return tuple(self.fetch(k, o) for k, o in zip(kinds, outs))
        finally:
            for k, o in zip(kinds, outs):
                self.free(k, o.value)
            for h, k in ins:
                self.free(k, h)

    def scratch_bytes(self, xdim: int, ydim: int, zdim: int) -> int:
        return int(self.lib.tke_scratch_bytes(xdim, ydim, zdim))

    def step(self, dims: Sequence[int], ptrs: Dict[str, int]):
        """tke_step_f32: one step on device pointers (ptrs maps STEP_INPUTS,
        STEP_OUTPUTS and "scratch" to addresses), asynchronous on this
        context's stream."""
        args = _StepArgs(*dims, *[ptrs[n] for n in STEP_INPUTS + STEP_OUTPUTS], ptrs["scratch"])
        self._check(self.lib.tke_step_f32(self._ctx, ctypes.byref(args)))

    def check(self):
        """Synchronises the context's stream; raises if a step failed."""
        self._check(self.lib.tke_check(self._ctx))

    @property
    def stream(self) -> int:
        return self.lib.tke_context_stream(self._ctx) or 0

    @property
    def launches_per_step(self) -> int:
        return int(self.lib.tke_launches_per_step())
