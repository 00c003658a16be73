"""Python host mirror of libop.so (include/op.h): finpar/OptionPricing.fut's
entry ``main`` (f32), a Sobol / Brownian-bridge Monte-Carlo pricer.

    ctx = OpContext()                        # futhark_context_config_new + futhark_context_new
    prices = ctx.main(*inputs)               # the 11 inputs in the entry's order -> [num_models] f32

``price`` is the engine extension on device pointers (asynchronous on the
context's stream).  There is no CPU fallback: a missing libop.so fails the
construction loudly.
"""
from __future__ import annotations

import ctypes
import os
from typing import Dict

import numpy as np

from .program_lib import ProgramContext, load_program_library

OP_LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libop.so")

# OptionPricing.fut:304-314, the entry point's parameters in order
INPUT_NAMES = ("contract_number", "num_mc_it", "dir_vs", "md_cs", "md_vols", "md_drifts", "md_sts", "md_detvals",
               "md_discts", "bb_inds", "bb_data")
_KIND = {"dir_vs": "i32_2d", "md_cs": "f32_3d", "md_vols": "f32_3d", "md_drifts": "f32_3d", "md_sts": "f32_2d",
         "md_detvals": "f32_2d", "md_discts": "f32_2d", "bb_inds": "i32_2d", "bb_data": "f32_2d"}
ARRAY_NAMES = INPUT_NAMES[2:]


class _OpArgs(ctypes.Structure):
    _fields_ = ([(n, ctypes.c_int32) for n in ("contract_number", "num_mc_it", "num_bits", "num_models",
                                                "num_und", "num_dates", "num_discts")]
                + [(n, ctypes.c_void_p) for n in ARRAY_NAMES])


_lib = None


def load_library(path: str = OP_LIB_PATH):
    """Load libop.so and declare its C signatures."""
    global _lib
    if _lib is None:
        vp, i32, c_int = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int
        _lib = load_program_library(path, ("f32_1d", "f32_2d", "f32_3d", "i32_2d"), {
            "futhark_entry_main": (c_int, [vp, ctypes.POINTER(vp), i32, i32] + [vp] * 9),
            "op_scratch_bytes": (ctypes.c_size_t, [vp, ctypes.POINTER(_OpArgs)]),
            "op_price_f32": (c_int, [vp, ctypes.POINTER(_OpArgs), vp, vp]),
            "op_check": (c_int, [vp]),
            "op_context_stream": (vp, [vp]),
            "op_context_set_reduction_order": (c_int, [vp, i32]),
        })
    return _lib


def dims_of(inputs) -> Dict[str, int]:
    """The size parameters of main (num_bits, num_models, num_und, num_dates,
    num_discts) read off the inputs' shapes."""
    v = dict(zip(INPUT_NAMES, inputs))
    m, d, u = np.shape(v["md_vols"])
    return {"num_bits": int(np.shape(v["dir_vs"])[1]), "num_models": int(m), "num_und": int(u),
            "num_dates": int(d), "num_discts": int(np.shape(v["md_discts"])[1])}


class OpContext(ProgramContext):
    """A libop.so context on one CUDA device ("#k" selects device k)."""

    def __init__(self, device: str | None = None):
        super().__init__(load_library(), device)

    def main(self, *inputs) -> np.ndarray:
        """futhark_entry_main on the 11 inputs in INPUT_NAMES order; returns the
        [num_models] f32 mean payoffs."""
        if len(inputs) != len(INPUT_NAMES):
            raise ValueError(f"OptionPricing main takes {len(INPUT_NAMES)} inputs")
        ins = []
        out = ctypes.c_void_p()
        try:
            for name, v in zip(ARRAY_NAMES, inputs[2:]):
                ins.append(self.new_array(_KIND[name], v))
            self._check(self.lib.futhark_entry_main(self._ctx, ctypes.byref(out), int(inputs[0]), int(inputs[1]),
                                                    *[h for h, _ in ins]))
            return self.fetch("f32_1d", out)
        finally:
            self.free("f32_1d", out.value)
            for h, k in ins:
                self.free(k, h)

    def _args(self, contract: int, num_mc_it: int, dims: Dict[str, int], ptrs: Dict[str, int]) -> _OpArgs:
        return _OpArgs(contract, num_mc_it, dims["num_bits"], dims["num_models"], dims["num_und"],
                       dims["num_dates"], dims["num_discts"], *[ptrs[n] for n in ARRAY_NAMES])

    def scratch_bytes(self, contract: int, num_mc_it: int, dims: Dict[str, int]) -> int:
        a = self._args(contract, num_mc_it, dims, {n: 0 for n in ARRAY_NAMES})
        return int(self.lib.op_scratch_bytes(self._ctx, ctypes.byref(a)))

    def price(self, contract: int, num_mc_it: int, dims: Dict[str, int], ptrs: Dict[str, int], out: int,
              scratch: int):
        """op_price_f32 on device pointers (ptrs maps ARRAY_NAMES to addresses),
        asynchronous on this context's stream."""
        a = self._args(contract, num_mc_it, dims, ptrs)
        self._check(self.lib.op_price_f32(self._ctx, ctypes.byref(a), out, scratch))

    ORDER_F64 = 0
    ORDER_SEQUENTIAL_F32 = 1

    def set_reduction_order(self, order: int):
        """Order of the sum over paths for the calls that follow: ORDER_F64
        (default, f64 accumulation) or ORDER_SEQUENTIAL_F32 (an f32 running sum
        in path order -- the order of the reference's golden outputs)."""
        self._check(self.lib.op_context_set_reduction_order(self._ctx, order))

    def check(self):
        """Synchronises the context's stream; raises if a launch failed."""
        self._check(self.lib.op_check(self._ctx))

    @property
    def stream(self) -> int:
        return self.lib.op_context_stream(self._ctx) or 0
