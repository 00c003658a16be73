"""ctypes plumbing shared by the mirrors of the engine's one-program libraries
(libtke.so, libop.so): each exports the generated API's configuration,
context and array functions (csrc/fut_api.cuh) plus its own entry point.
"""
from __future__ import annotations

import ctypes
import os
from typing import Dict, Iterable, Tuple

import numpy as np

from . import FUTHARK_OUT_OF_MEMORY, FUTHARK_PROGRAM_ERROR, FutharkError

# element type name -> numpy dtype
ELEM = {"f32": np.float32, "i32": np.int32}


def load_program_library(path: str, array_kinds: Iterable[str], extra: Dict[str, tuple]):
    """Load a one-program library and declare the generated API's C
    signatures: the context functions, the array functions of array_kinds
    ("f32_3d", ...), and `extra` (name -> (restype, argtypes))."""
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
    }
    for kind in array_kinds:
        rank = int(kind[4])
        sig[f"futhark_new_{kind}"] = (vp, [vp, vp] + [i64] * rank)
        sig[f"futhark_free_{kind}"] = (c_int, [vp, vp])
        sig[f"futhark_values_{kind}"] = (c_int, [vp, vp, vp])
        sig[f"futhark_shape_{kind}"] = (ctypes.POINTER(i64), [vp, vp])
    sig.update(extra)
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    libc = ctypes.CDLL(None)
    libc.free.argtypes = [vp]
    libc.free.restype = None
    L.free_str = libc.free
    return L


class ProgramContext:
    """A context of a one-program library on one CUDA device ("#k" selects
    device k); subclasses set `lib` through their loader."""

    def __init__(self, lib, device: str | None = None):
        self.lib = lib
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

    def new_array(self, kind: str, v) -> Tuple[int, str]:
        """A device array of `kind` ("f32_3d", ...) from host data."""
        etype, rank = kind[:3], int(kind[4])
        v = np.ascontiguousarray(v, dtype=ELEM[etype])
        if v.ndim != rank:
            raise ValueError(f"expected a rank-{rank} array, got shape {v.shape}")
        h = getattr(self.lib, f"futhark_new_{kind}")(self._ctx, v.ctypes.data, *v.shape)
        if not h:
            raise FutharkError(FUTHARK_OUT_OF_MEMORY, self._take_error() or "array allocation failed")
        return h, kind

    def fetch(self, kind: str, h) -> np.ndarray:
        shape = getattr(self.lib, f"futhark_shape_{kind}")(self._ctx, h)
        rank = int(kind[4])
        res = np.empty(tuple(shape[r] for r in range(rank)), dtype=ELEM[kind[:3]])
        self._check(getattr(self.lib, f"futhark_values_{kind}")(self._ctx, h, res.ctypes.data))
        return res

    def free(self, kind: str, h):
        if h:
            getattr(self.lib, f"futhark_free_{kind}")(self._ctx, h)

    def sync(self):
        self._check(self.lib.futhark_context_sync(self._ctx))
