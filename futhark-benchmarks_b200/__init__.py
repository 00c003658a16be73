"""B200-native engine for the finpar LocVolCalib benchmark (diku-dk/futhark-benchmarks).

The product is the C-ABI library ``liblvc.so`` (declared in
``include/LocVolCalib.h``): the Futhark-generated C API of
finpar/LocVolCalib.fut's entry point ``main`` plus batched and serving forms,
all running hand-written sm_100a kernels.  This module is the Python host
mirror of that API (ctypes), with the same names, argument meaning and error
behaviour as the generated library:

    ctx = Context()                       # futhark_context_config_new + futhark_context_new
    prices = ctx.main(16, 32, 256, 256, 0.03, 5.0, 0.2, 0.6, 0.5)        # f32, futhark_entry_main
    prices = ctx.main_f64(16, 32, 256, 256, 0.03, 5.0, 0.2, 0.6, 0.5)    # f64 twin
    plan = ctx.plan([Calibration(...), ...], precision=F64)              # batched form
    plan.run(); plan.prices()

A failing call raises ``FutharkError`` carrying futhark_context_get_error's
message and the non-zero return code.  There is no CPU fallback: if the
library is missing the import of this module fails loudly.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, astuple
from typing import Iterable, List, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liblvc.so")

FUTHARK_SUCCESS = 0
FUTHARK_PROGRAM_ERROR = 2
FUTHARK_OUT_OF_MEMORY = 3
F64 = 0
F32_STATE = 1

_lib = None


class FutharkError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code
        self.msg = msg


class _Calib(ctypes.Structure):
    _fields_ = [("outer", ctypes.c_int32), ("numX", ctypes.c_int32), ("numY", ctypes.c_int32),
                ("numT", ctypes.c_int32), ("s0", ctypes.c_double), ("t", ctypes.c_double),
                ("alpha", ctypes.c_double), ("nu", ctypes.c_double), ("beta", ctypes.c_double)]


@dataclass(frozen=True)
class Calibration:
    """The nine scalar inputs of `main` (finpar/LocVolCalib.fut:238-246)."""
    outer: int
    numX: int
    numY: int
    numT: int
    s0: float
    t: float
    alpha: float
    nu: float
    beta: float

    def work(self) -> int:
        """Option-cell-steps: outer * numX * numY * (numT - 1)."""
        return self.outer * self.numX * self.numY * max(self.numT - 1, 0)


class Shape(ctypes.Structure):
    """struct lvc_shape: kernel family x cluster size of a grid class."""
    _fields_ = [("family", ctypes.c_int32), ("cluster", ctypes.c_int32), ("threads", ctypes.c_int32),
                ("rows_per_cta", ctypes.c_int32), ("smem_bytes", ctypes.c_int32), ("hbm_state", ctypes.c_int32)]

    FAMILIES = {0: "chunk", 1: "line", 2: "line_full", 3: "line_pair", 4: "line_pair1"}

    def __repr__(self):
        fam = self.FAMILIES.get(self.family, "?") + ("_hbm" if self.hbm_state else "")
        return (f"Shape({fam}, cluster={self.cluster}, threads={self.threads}, "
                f"rows_per_cta={self.rows_per_cta}, smem={self.smem_bytes})")

    def key(self):
        return (self.family, self.cluster, self.hbm_state)


class LaunchInfo(ctypes.Structure):
    """struct lvc_launch_info: one rollback launch class of a plan."""
    _fields_ = [("family", ctypes.c_int32), ("cluster", ctypes.c_int32), ("threads", ctypes.c_int32),
                ("items", ctypes.c_int32), ("cell_steps", ctypes.c_int64), ("ms", ctypes.c_double)]

    def as_dict(self) -> dict:
        return {"family": Shape.FAMILIES.get(self.family, "?"), "cluster": self.cluster,
                "threads": self.threads, "items": self.items, "cell_steps": self.cell_steps, "ms": self.ms}


class TuningEntry(ctypes.Structure):
    """struct lvc_tuning_entry."""
    _fields_ = [("numX", ctypes.c_int32), ("numY", ctypes.c_int32), ("precision", ctypes.c_int32),
                ("tuned", ctypes.c_int32), ("shape", Shape), ("us_per_step_default", ctypes.c_double),
                ("us_per_step_best", ctypes.c_double)]


class _ServerConfig(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int32), ("max_inflight_requests", ctypes.c_int32),
                ("max_batch_requests", ctypes.c_int32), ("num_streams", ctypes.c_int32),
                ("hbm_budget_bytes", ctypes.c_int64)]


class _ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_int64), ("completed", ctypes.c_int64), ("failed", ctypes.c_int64),
                ("options", ctypes.c_int64), ("batches", ctypes.c_int64), ("hbm_reserved_bytes", ctypes.c_int64),
                ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double), ("mean_ms", ctypes.c_double),
                ("max_ms", ctypes.c_double), ("throughput_options_per_s", ctypes.c_double),
                ("span_s", ctypes.c_double)]


def load_library(path: str = LIB_PATH):
    """Load liblvc.so and declare its C signatures."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing; build it with `python futhark-benchmarks_b200/build.py`")
    L = ctypes.CDLL(path)
    vp, i32, i64, f32, f64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_float, ctypes.c_double
    sig = {
        "futhark_context_config_new": (vp, []),
        "futhark_context_config_free": (None, [vp]),
        "futhark_context_config_set_device": (None, [vp, ctypes.c_char_p]),
        "futhark_context_config_set_debugging": (None, [vp, ctypes.c_int]),
        "futhark_context_config_set_profiling": (None, [vp, ctypes.c_int]),
        "futhark_context_config_set_logging": (None, [vp, ctypes.c_int]),
        "futhark_context_config_set_cache_file": (None, [vp, ctypes.c_char_p]),
        "futhark_context_config_set_tuning_param": (ctypes.c_int, [vp, ctypes.c_char_p, ctypes.c_size_t]),
        "futhark_get_tuning_param_count": (ctypes.c_int, []),
        "futhark_get_tuning_param_name": (ctypes.c_char_p, [ctypes.c_int]),
        "futhark_get_tuning_param_class": (ctypes.c_char_p, [ctypes.c_int]),
        "lvc_context_set_tuning_param": (ctypes.c_int, [vp, ctypes.c_char_p, ctypes.c_size_t]),
        "lvc_shape_candidates": (ctypes.c_int, [vp, i32, i32, i32, ctypes.POINTER(Shape), i32, ctypes.POINTER(i32)]),
        "lvc_tuning_set": (ctypes.c_int, [vp, i32, i32, i32, ctypes.POINTER(Shape)]),
        "lvc_tuning_get": (ctypes.c_int, [vp, i32, i32, i32, ctypes.POINTER(TuningEntry)]),
        "lvc_plan_shape": (ctypes.c_int, [vp, i32, ctypes.POINTER(Shape)]),
        "lvc_tuning_entries": (i32, [vp, ctypes.POINTER(TuningEntry), i32]),
        "lvc_autotune": (ctypes.c_int, [vp, ctypes.POINTER(_Calib), i32, i32, i32]),
        "lvc_autotune_plan": (ctypes.c_int, [vp, ctypes.POINTER(_Calib), i32, i32, i32, ctypes.POINTER(i32),
                                             ctypes.POINTER(i32), ctypes.POINTER(f64)]),
        "lvc_tuning_save": (ctypes.c_int, [vp, ctypes.c_char_p]),
        "lvc_tuning_load": (ctypes.c_int, [vp, ctypes.c_char_p]),
        "futhark_context_new": (vp, [vp]),
        "futhark_context_free": (None, [vp]),
        "futhark_context_sync": (ctypes.c_int, [vp]),
        "futhark_context_get_error": (ctypes.POINTER(ctypes.c_char), [vp]),
        "futhark_context_clear_caches": (ctypes.c_int, [vp]),
        "futhark_new_f32_1d": (vp, [vp, vp, i64]),
        "futhark_new_f64_1d": (vp, [vp, vp, i64]),
        "futhark_free_f32_1d": (ctypes.c_int, [vp, vp]),
        "futhark_free_f64_1d": (ctypes.c_int, [vp, vp]),
        "futhark_values_f32_1d": (ctypes.c_int, [vp, vp, vp]),
        "futhark_values_f64_1d": (ctypes.c_int, [vp, vp, vp]),
        "futhark_shape_f32_1d": (ctypes.POINTER(i64), [vp, vp]),
        "futhark_shape_f64_1d": (ctypes.POINTER(i64), [vp, vp]),
        "futhark_entry_main": (ctypes.c_int, [vp, ctypes.POINTER(vp), i32, i32, i32, i32, f32, f32, f32, f32, f32]),
        "futhark_entry_main_f64": (ctypes.c_int, [vp, ctypes.POINTER(vp), i32, i32, i32, i32, f64, f64, f64, f64, f64]),
        "lvc_plan_new": (ctypes.c_int, [vp, ctypes.POINTER(_Calib), i32, i32, ctypes.POINTER(vp)]),
        "lvc_plan_free": (ctypes.c_int, [vp, vp]),
        "lvc_plan_num_prices": (i64, [vp]),
        "lvc_plan_set_params": (ctypes.c_int, [vp, vp, ctypes.POINTER(_Calib), i32]),
        "lvc_plan_run": (ctypes.c_int, [vp, vp]),
        "lvc_plan_copy_prices": (ctypes.c_int, [vp, vp, vp]),
        "lvc_plan_device_prices": (vp, [vp]),
        "lvc_plan_time": (ctypes.c_int, [vp, vp, i32, ctypes.POINTER(f64)]),
        "lvc_plan_rollback_ms": (f64, [vp]),
        "lvc_plan_num_launches": (i32, [vp]),
        "lvc_plan_num_classes": (i32, [vp]),
        "lvc_plan_launch_info": (ctypes.c_int, [vp, i32, ctypes.POINTER(LaunchInfo)]),
        "lvc_batch": (ctypes.c_int, [vp, ctypes.POINTER(_Calib), i32, i32, vp]),
        "lvc_context_stream": (vp, [vp]),
        "futhark_new_f32_2d": (vp, [vp, vp, i64, i64]),
        "futhark_free_f32_2d": (ctypes.c_int, [vp, vp]),
        "futhark_values_f32_2d": (ctypes.c_int, [vp, vp, vp]),
        "futhark_shape_f32_2d": (ctypes.POINTER(i64), [vp, vp]),
        "futhark_entry_tridagNested": (ctypes.c_int, [vp, ctypes.POINTER(vp), vp, vp, vp, vp]),
        "futhark_entry_tridagNestedConst": (ctypes.c_int, [vp, ctypes.POINTER(vp), vp, vp, vp, vp]),
        "futhark_entry_tridagNestedSeq": (ctypes.c_int, [vp, ctypes.POINTER(vp), vp, vp, vp, vp]),
        "futhark_entry_tridagNestedSeqConst": (ctypes.c_int, [vp, ctypes.POINTER(vp), vp, vp, vp, vp]),
        "lvc_tridag_f32": (ctypes.c_int, [vp, i32, i64, i64, vp, vp, vp, vp, vp]),
        "lvc_tridag_check": (ctypes.c_int, [vp]),
        "lvc_wait_selftest": (ctypes.c_int, [vp, i32, i32]),
        "lvc_entry_main_f64_noalloc_bytes": (i64, [vp, i32, i32, i32, i32]),
        "lvc_probe_peaks": (ctypes.c_int, [vp, ctypes.POINTER(f64), ctypes.POINTER(f64)]),
        "lvc_server_new": (ctypes.c_int, [vp, ctypes.POINTER(_ServerConfig), ctypes.POINTER(vp)]),
        "lvc_server_submit": (ctypes.c_int, [vp, ctypes.POINTER(_Calib), ctypes.POINTER(ctypes.c_uint64)]),
        "lvc_server_poll": (ctypes.c_int, [vp, ctypes.c_uint64, ctypes.POINTER(i32)]),
        "lvc_server_wait": (ctypes.c_int, [vp, ctypes.c_uint64, vp, f64]),
        "lvc_server_stats": (ctypes.c_int, [vp, ctypes.POINTER(_ServerStats)]),
        "lvc_server_reset_stats": (ctypes.c_int, [vp]),
        "lvc_server_free": (ctypes.c_int, [vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    libc = ctypes.CDLL(None)
    libc.free.argtypes = [vp]
    L._libc_free = libc.free
    _lib = L
    return L


def _calib_array(calibs: Sequence[Calibration]):
    arr = (_Calib * max(1, len(calibs)))()
    for i, c in enumerate(calibs):
        arr[i] = _Calib(*astuple(c))
    return arr


class Context:
    """A futhark_context on one CUDA device ("#N" or a device-name substring)."""

    def __init__(self, device: str | None = None, tuning: dict | None = None):
        self.lib = load_library()
        self._cfg = self.lib.futhark_context_config_new()
        if device is not None:
            self.lib.futhark_context_config_set_device(self._cfg, device.encode())
        for name, value in (tuning or {}).items():
            if self.lib.futhark_context_config_set_tuning_param(self._cfg, name.encode(), int(value)):
                self.lib.futhark_context_config_free(self._cfg)
                self._cfg = None
                raise FutharkError(FUTHARK_PROGRAM_ERROR, f"unknown tuning parameter or value: {name}={value}")
        self._ctx = self.lib.futhark_context_new(self._cfg)
        if not self._ctx:
            raise FutharkError(FUTHARK_OUT_OF_MEMORY, "futhark_context_new failed")
        err = self._take_error()
        if err:
            self.close()
            raise FutharkError(FUTHARK_PROGRAM_ERROR, err)

    # -- plumbing -----------------------------------------------------------
    def _take_error(self) -> str:
        p = self.lib.futhark_context_get_error(self._ctx)
        if not p:
            return ""
        msg = ctypes.cast(p, ctypes.c_char_p).value.decode(errors="replace")
        self.lib._libc_free(ctypes.cast(p, ctypes.c_void_p))
        return msg

    def _check(self, rc: int):
        if rc != 0:
            raise FutharkError(rc, self._take_error() or "unknown error")

    def close(self):
        if getattr(self, "_ctx", None):
            self.lib.futhark_context_free(self._ctx)
            self._ctx = None
        if getattr(self, "_cfg", None):
            self.lib.futhark_context_config_free(self._cfg)
            self._cfg = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def sync(self):
        self._check(self.lib.futhark_context_sync(self._ctx))

    def set_tuning_param(self, name: str, value: int):
        """Tuning parameter for plans created from now on ("lvc.streams", "lvc.grid")."""
        self._check(self.lib.lvc_context_set_tuning_param(self._ctx, name.encode(), int(value)))

    # -- shape autotuner ------------------------------------------------------
    def shape_candidates(self, numX: int, numY: int, precision: int = F64) -> list:
        """Every Shape that can run an numX x numY grid on this device."""
        n = ctypes.c_int32()
        self._check(self.lib.lvc_shape_candidates(self._ctx, numX, numY, precision, None, 0, ctypes.byref(n)))
        arr = (Shape * max(1, n.value))()
        self._check(self.lib.lvc_shape_candidates(self._ctx, numX, numY, precision, arr, n.value, ctypes.byref(n)))
        return list(arr[:n.value])

    def tuning_set(self, numX: int, numY: int, precision: int = F64, shape: Shape | None = None):
        """Pin a shape for a grid class (None: back to the built-in choice)."""
        self._check(self.lib.lvc_tuning_set(self._ctx, numX, numY, precision,
                                            ctypes.byref(shape) if shape is not None else None))

    def tuning_get(self, numX: int, numY: int, precision: int = F64) -> TuningEntry:
        e = TuningEntry()
        self._check(self.lib.lvc_tuning_get(self._ctx, numX, numY, precision, ctypes.byref(e)))
        return e

    def tuning_entries(self) -> list:
        n = self.lib.lvc_tuning_entries(self._ctx, None, 0)
        arr = (TuningEntry * max(1, n))()
        n = self.lib.lvc_tuning_entries(self._ctx, arr, n)
        return list(arr[:n])

    def autotune(self, calibs: Sequence[Calibration], precision: int = F64, probe_steps: int = 8) -> list:
        """Time every candidate shape of every grid class of `calibs`; keep the fastest."""
        arr = _calib_array(calibs)
        self._check(self.lib.lvc_autotune(self._ctx, arr, len(calibs), precision, probe_steps))
        return self.tuning_entries()

    def autotune_plan(self, calibs: Sequence[Calibration], precision: int = F64, max_steps: int = 32) -> dict:
        """Time the whole plan (time lines capped at max_steps) under lvc.grid 0/1 x
        lvc.streams 2/4 and keep the fastest; then keep each class shape the
        per-class autotuner changed only if the plan is faster with it."""
        arr = _calib_array(calibs)
        g, st, ms = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_double()
        self._check(self.lib.lvc_autotune_plan(self._ctx, arr, len(calibs), precision, max_steps,
                                               ctypes.byref(g), ctypes.byref(st), ctypes.byref(ms)))
        return {"lvc.grid": g.value, "lvc.streams": st.value, "capped_plan_ms": ms.value}

    def tuning_save(self, path: str):
        self._check(self.lib.lvc_tuning_save(self._ctx, str(path).encode()))

    def tuning_load(self, path: str):
        self._check(self.lib.lvc_tuning_load(self._ctx, str(path).encode()))

    # -- batched tridiagonal solvers (misc/ocean-sim/tridiag-test.fut) ---------
    TRIDAG_ENTRIES = {("par", False): "tridagNested", ("par", True): "tridagNestedConst",
                      ("seq", False): "tridagNestedSeq", ("seq", True): "tridagNestedSeqConst"}

    def tridag(self, a, b, c, y, form: str = "par", const: bool = False) -> np.ndarray:
        """One of the four tridagNested* entry points on host [n][m] f32 arrays:
        form "par" (tridagPar) or "seq" (tridagSeq); const requires m == 115."""
        arrs = [np.ascontiguousarray(v, dtype=np.float32) for v in (a, b, c, y)]
        if arrs[0].ndim != 2:
            raise ValueError("tridag: 2-D arrays expected")
        ins = []
        try:
            for v in arrs:
                h = self.lib.futhark_new_f32_2d(self._ctx, v.ctypes.data, v.shape[0], v.shape[1])
                if not h:
                    raise FutharkError(FUTHARK_OUT_OF_MEMORY, self._take_error() or "futhark_new_f32_2d failed")
                ins.append(h)
            out = ctypes.c_void_p()
            entry = getattr(self.lib, "futhark_entry_" + self.TRIDAG_ENTRIES[(form, bool(const))])
            self._check(entry(self._ctx, ctypes.byref(out), *ins))
            try:
                shape = self.lib.futhark_shape_f32_2d(self._ctx, out)
                res = np.empty((shape[0], shape[1]), dtype=np.float32)
                self._check(self.lib.futhark_values_f32_2d(self._ctx, out, res.ctypes.data))
            finally:
                self.lib.futhark_free_f32_2d(self._ctx, out)
            return res
        finally:
            for h in ins:
                self.lib.futhark_free_f32_2d(self._ctx, h)

    def tridag_device(self, form: str, rows: int, m: int, a: int, b: int, c: int, y: int, out: int):
        """lvc_tridag_f32 on device pointers, asynchronous on this context's stream."""
        self._check(self.lib.lvc_tridag_f32(self._ctx, 0 if form == "seq" else 1, rows, m, a, b, c, y, out))

    def tridag_check(self):
        """Raises if a device-pointer solve since the last check had a copy time out."""
        self._check(self.lib.lvc_tridag_check(self._ctx))

    def wait_selftest(self, polls: int, arrive: bool):
        """lvc_wait_selftest: a bounded device wait that runs out (arrive=False)
        raises FutharkError; one that completes returns quietly."""
        self._check(self.lib.lvc_wait_selftest(self._ctx, polls, int(bool(arrive))))

    @property
    def stream(self) -> int:
        return self.lib.lvc_context_stream(self._ctx) or 0

    def probe_peaks(self):
        """(FP64 TFLOP/s, shared-memory GB/s) measured on this context's device."""
        f, s = ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.lvc_probe_peaks(self._ctx, ctypes.byref(f), ctypes.byref(s)))
        return f.value, s.value

    # -- the entry points ---------------------------------------------------
    def _array_values(self, arr, kind: str) -> np.ndarray:
        shape = getattr(self.lib, f"futhark_shape_{kind}_1d")(self._ctx, arr)
        n = int(shape[0])
        out = np.empty(n, dtype=np.float32 if kind == "f32" else np.float64)
        self._check(getattr(self.lib, f"futhark_values_{kind}_1d")(self._ctx, arr, out.ctypes.data))
        return out

    def main(self, outer, numX, numY, numT, s0, t, alpha, nu, beta) -> np.ndarray:
        """futhark_entry_main: f32 inputs, f32 prices (computed in f64)."""
        arr = ctypes.c_void_p()
        self._check(self.lib.futhark_entry_main(self._ctx, ctypes.byref(arr), outer, numX, numY, numT,
                                                s0, t, alpha, nu, beta))
        try:
            return self._array_values(arr, "f32")
        finally:
            self.lib.futhark_free_f32_1d(self._ctx, arr)

    def main_f64(self, outer, numX, numY, numT, s0, t, alpha, nu, beta) -> np.ndarray:
        """futhark_entry_main_f64: the f64 instantiation of `main`."""
        arr = ctypes.c_void_p()
        self._check(self.lib.futhark_entry_main_f64(self._ctx, ctypes.byref(arr), outer, numX, numY,
                                                    numT, s0, t, alpha, nu, beta))
        try:
            return self._array_values(arr, "f64")
        finally:
            self.lib.futhark_free_f64_1d(self._ctx, arr)

    # -- batched form -------------------------------------------------------
    def plan(self, calibs: Sequence[Calibration], precision: int = F64) -> "Plan":
        return Plan(self, calibs, precision)

    def batch(self, calibs: Sequence[Calibration], precision: int = F64) -> np.ndarray:
        """lvc_batch: one-shot batched call from host memory; prices concatenated."""
        arr = _calib_array(calibs)
        n = sum(c.outer for c in calibs)
        out = np.empty(max(n, 1), dtype=np.float64)
        self._check(self.lib.lvc_batch(self._ctx, arr, len(calibs), precision, out.ctypes.data))
        return out[:n]


class Plan:
    """lvc_plan: device tables, work lists and the captured graph of a batch."""

    def __init__(self, ctx: Context, calibs: Sequence[Calibration], precision: int = F64):
        self.ctx = ctx
        self.calibs = list(calibs)
        self.precision = precision
        self._p = ctypes.c_void_p()
        ctx._check(ctx.lib.lvc_plan_new(ctx._ctx, _calib_array(self.calibs), len(self.calibs),
                                        precision, ctypes.byref(self._p)))
        self.num_prices = int(ctx.lib.lvc_plan_num_prices(self._p))
        self.offsets = np.concatenate([[0], np.cumsum([c.outer for c in self.calibs])]).astype(np.int64)

    def run(self):
        self.ctx._check(self.ctx.lib.lvc_plan_run(self.ctx._ctx, self._p))

    def set_params(self, calibs: Sequence[Calibration]):
        self.ctx._check(self.ctx.lib.lvc_plan_set_params(self.ctx._ctx, self._p, _calib_array(calibs),
                                                         len(calibs)))
        self.calibs = list(calibs)

    def prices(self) -> np.ndarray:
        out = np.empty(max(self.num_prices, 1), dtype=np.float64)
        self.ctx._check(self.ctx.lib.lvc_plan_copy_prices(self.ctx._ctx, self._p, out.ctypes.data))
        return out[: self.num_prices]

    def split(self, prices: np.ndarray) -> List[np.ndarray]:
        return [prices[self.offsets[i]:self.offsets[i + 1]] for i in range(len(self.calibs))]

    def time(self, iters: int = 3) -> float:
        """Mean milliseconds per run over `iters` graph launches (CUDA events)."""
        ms = ctypes.c_double()
        self.ctx._check(self.ctx.lib.lvc_plan_time(self.ctx._ctx, self._p, iters, ctypes.byref(ms)))
        return ms.value

    @property
    def rollback_ms(self) -> float:
        return float(self.ctx.lib.lvc_plan_rollback_ms(self._p))

    @property
    def num_launches(self) -> int:
        return int(self.ctx.lib.lvc_plan_num_launches(self._p))

    def classes(self) -> list:
        """The plan's rollback launch classes (largest work first), with their
        device times from the last time() call."""
        out = []
        for i in range(int(self.ctx.lib.lvc_plan_num_classes(self._p))):
            li = LaunchInfo()
            if self.ctx.lib.lvc_plan_launch_info(self._p, i, ctypes.byref(li)) == 0:
                out.append(li.as_dict())
        return out

    @property
    def device_prices(self) -> int:
        return int(self.ctx.lib.lvc_plan_device_prices(self._p) or 0)

    def shape(self, calib: int = 0) -> "Shape":
        """The shape (kernel family, cluster size, ...) calibration `calib` runs under."""
        sh = Shape()
        if self.ctx.lib.lvc_plan_shape(self._p, calib, ctypes.byref(sh)):
            raise FutharkError(FUTHARK_PROGRAM_ERROR, f"no calibration {calib} in this plan")
        return sh

    def free(self):
        if self._p:
            self.ctx.lib.lvc_plan_free(self.ctx._ctx, self._p)
            self._p = ctypes.c_void_p()

    def __del__(self):
        try:
            if self._p and self.ctx._ctx:
                self.free()
        except Exception:
            pass


def run_dataset(ctx: Context, path: str, f64: bool = False) -> np.ndarray:
    """Run `main` on a reference dataset file (finpar/LocVolCalib-data/*.in)."""
    from . import futhark_data
    vals = futhark_data.read_file(path)
    if len(vals) != 9:
        raise ValueError(f"{path}: expected the 9 inputs of main, got {len(vals)} values")
    args = [int(v) for v in vals[:4]] + [float(v) for v in vals[4:]]
    return ctx.main_f64(*args) if f64 else ctx.main(*args)


class Server:
    """lvc_server: continuous batching of calibration requests on one device.

    submit() returns a ticket at once; result(ticket) blocks until that
    request's prices are ready.  Requests that arrive while others run are
    admitted as streams, the HBM budget and SMs free up, and run concurrently.
    """

    def __init__(self, ctx: Context, precision: int = F64, max_inflight_requests: int = 0,
                 max_batch_requests: int = 0, num_streams: int = 0, hbm_budget_bytes: int = 0):
        self.ctx = ctx
        cfg = _ServerConfig(precision, max_inflight_requests, max_batch_requests, num_streams, hbm_budget_bytes)
        self._s = ctypes.c_void_p()
        ctx._check(ctx.lib.lvc_server_new(ctx._ctx, ctypes.byref(cfg), ctypes.byref(self._s)))
        self._outer = {}

    def submit(self, c: Calibration) -> int:
        t = ctypes.c_uint64()
        self.ctx._check(self.ctx.lib.lvc_server_submit(self._s, ctypes.byref(_Calib(*astuple(c))), ctypes.byref(t)))
        self._outer[t.value] = c.outer
        return t.value

    def done(self, ticket: int) -> bool:
        d = ctypes.c_int32()
        self.ctx._check(self.ctx.lib.lvc_server_poll(self._s, ticket, ctypes.byref(d)))
        return bool(d.value)

    def result(self, ticket: int, timeout_s: float = 0.0) -> np.ndarray:
        n = self._outer.pop(ticket)
        out = np.empty(max(n, 1), dtype=np.float64)
        self.ctx._check(self.ctx.lib.lvc_server_wait(self._s, ticket, out.ctypes.data, timeout_s))
        return out[:n]

    def stats(self) -> dict:
        st = _ServerStats()
        self.ctx._check(self.ctx.lib.lvc_server_stats(self._s, ctypes.byref(st)))
        return {k: getattr(st, k) for k, _ in _ServerStats._fields_}

    def reset_stats(self):
        self.ctx.lib.lvc_server_reset_stats(self._s)

    def close(self):
        if self._s:
            self.ctx.lib.lvc_server_free(self._s)
            self._s = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
