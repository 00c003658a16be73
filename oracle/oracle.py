"""ctypes binding of the CPU oracle (liblvc_oracle.so) -- TEST INFRASTRUCTURE ONLY.

Importers: tests/, __graft_entry__.smoke() and bench.py's CPU-baseline and
reference legs.  The engine never imports this module.

The oracle restates finpar/LocVolCalib.fut line by line (see lvc_oracle.cpp);
`main_f32`/`main_f64` are the reference `main` at f32 (the reference's own
precision) and at f64.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liblvc_oracle.so")
_lib = None


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB):
        subprocess.run(["make", "-C", HERE, "--no-print-directory"], check=True)
    L = ctypes.CDLL(LIB)
    i32, i64, f32, f64, vp = ctypes.c_int32, ctypes.c_int64, ctypes.c_float, ctypes.c_double, ctypes.c_void_p
    L.lvc_oracle_main_f32.argtypes = [i32] * 4 + [f32] * 5 + [vp, ctypes.c_int, ctypes.c_int]
    L.lvc_oracle_main_f32.restype = ctypes.c_int
    L.lvc_oracle_main_f64.argtypes = [i32] * 4 + [f64] * 5 + [vp, ctypes.c_int, ctypes.c_int]
    L.lvc_oracle_main_f64.restype = ctypes.c_int
    L.lvc_oracle_value_f64.argtypes = [i32] * 3 + [f64] * 6 + [ctypes.c_int]
    L.lvc_oracle_value_f64.restype = f64
    L.lvc_oracle_value_f32.argtypes = [i32] * 3 + [f32] * 6 + [ctypes.c_int]
    L.lvc_oracle_value_f32.restype = f32
    L.lvc_oracle_xindex_f64.argtypes = [i32, f64, f64, f64]
    L.lvc_oracle_xindex_f64.restype = ctypes.c_int
    L.lvc_oracle_batch_f64.argtypes = [i32] + [vp] * 9 + [vp, vp, ctypes.c_int]
    L.lvc_oracle_batch_f64.restype = ctypes.c_int
    for name in ("lvc_oracle_tridag_par_f32", "lvc_oracle_tridag_par_f64",
                 "lvc_oracle_tridag_seq_f32", "lvc_oracle_tridag_seq_f64",
                 "lvc_oracle_tridag_par4_f32", "lvc_oracle_tridag_par4_f64"):
        fn = getattr(L, name)
        fn.argtypes = [i64, i64] + [vp] * 5
        fn.restype = None
    L.lvc_oracle_max_threads.restype = ctypes.c_int
    _lib = L
    return L


def max_threads() -> int:
    return int(load().lvc_oracle_max_threads())


def main_f32(outer, numX, numY, numT, s0, t, alpha, nu, beta, threads=0, seq=False) -> np.ndarray:
    out = np.zeros(max(outer, 1), dtype=np.float32)
    rc = load().lvc_oracle_main_f32(outer, numX, numY, numT, s0, t, alpha, nu, beta,
                                    out.ctypes.data, threads, int(seq))
    if rc:
        raise ValueError("oracle: invalid inputs")
    return out[:outer]


def main_f64(outer, numX, numY, numT, s0, t, alpha, nu, beta, threads=0, seq=False) -> np.ndarray:
    out = np.zeros(max(outer, 1), dtype=np.float64)
    rc = load().lvc_oracle_main_f64(outer, numX, numY, numT, s0, t, alpha, nu, beta,
                                    out.ctypes.data, threads, int(seq))
    if rc:
        raise ValueError("oracle: invalid inputs")
    return out[:outer]


def value_f64(numX, numY, numT, s0, strike, t, alpha, nu, beta, seq=False) -> float:
    return float(load().lvc_oracle_value_f64(numX, numY, numT, s0, strike, t, alpha, nu, beta, int(seq)))


def batch_f64(calibs: Sequence, threads=0) -> np.ndarray:
    """Prices of many calibrations (objects with the nine fields of `main`), concatenated."""
    n = len(calibs)
    cols = {k: np.array([getattr(c, k) for c in calibs], dtype=np.int32 if k in ("outer", "numX", "numY", "numT") else np.float64)
            for k in ("outer", "numX", "numY", "numT", "s0", "t", "alpha", "nu", "beta")}
    offsets = np.concatenate([[0], np.cumsum(cols["outer"])]).astype(np.int64)
    out = np.zeros(max(int(offsets[-1]), 1), dtype=np.float64)
    rc = load().lvc_oracle_batch_f64(n, *[cols[k].ctypes.data for k in
                                          ("outer", "numX", "numY", "numT", "s0", "t", "alpha", "nu", "beta")],
                                     offsets.ctypes.data, out.ctypes.data, threads)
    if rc:
        raise ValueError("oracle: invalid inputs")
    return out[:offsets[-1]]


def tridag(a, b, c, y, form="par") -> np.ndarray:
    a = np.ascontiguousarray(a)
    dt = a.dtype
    b, c, y = (np.ascontiguousarray(v, dtype=dt) for v in (b, c, y))
    rows, n = a.shape
    out = np.zeros_like(a)
    name = f"lvc_oracle_tridag_{form}_{'f32' if dt == np.float32 else 'f64'}"
    getattr(load(), name)(rows, n, a.ctypes.data, b.ctypes.data, c.ctypes.data, y.ctypes.data,
                          out.ctypes.data)
    return out


TKE_INPUTS = ["tketau", "tketaup1", "tketaum1", "dtketau", "dtketaup1", "dtketaum1", "utau", "vtau", "wtau",
              "maskU", "maskV", "maskW", "dxt", "dxu", "dyt", "dyu", "dzt", "dzw", "cost", "cosu", "kbot",
              "kappaM", "mxl", "forc", "forc_tke_surface"]


def tke(*inputs):
    """misc/ocean-sim/tke.fut's entry main (f32) on the 25 inputs in the
    reference's order; returns its 7 outputs (tketau, tketaup1, tketaum1,
    dtketau, dtketaup1, dtketaum1, tke_surf_corr)."""
    v = dict(zip(TKE_INPUTS, inputs))
    f32 = {k: np.ascontiguousarray(x, dtype=np.float32) for k, x in v.items() if k != "kbot"}
    kbot = np.ascontiguousarray(v["kbot"], dtype=np.int32)
    X, Y, Z = f32["tketau"].shape
    tp1 = np.empty((X, Y, Z), np.float32)
    dtk = np.empty((X, Y, Z), np.float32)
    corr = np.empty((X, Y), np.float32)
    L = load()
    fn = L.lvc_oracle_tke_f32
    fn.restype = None
    fn.argtypes = [ctypes.c_int] * 3 + [ctypes.c_void_p] * 26
    order = ["tketau", "tketaup1", "dtketau", "dtketaum1", "utau", "vtau", "wtau", "maskU", "maskV", "maskW",
             "dxt", "dxu", "dyt", "dyu", "dzt", "dzw", "cost", "cosu"]
    args = [f32[k].ctypes.data for k in order] + [kbot.ctypes.data] + \
           [f32[k].ctypes.data for k in ("kappaM", "mxl", "forc", "forc_tke_surface")] + \
           [tp1.ctypes.data, dtk.ctypes.data, corr.ctypes.data]
    fn(X, Y, Z, *args)
    return (f32["tketau"].copy(), tp1, f32["tketaum1"].copy(), dtk, f32["dtketaup1"].copy(),
            f32["dtketaum1"].copy(), corr)


# finpar/OptionPricing.fut's entry main (op_oracle.cpp): the inputs in the
# entry point's order.
OP_INPUTS = ["contract_number", "num_mc_it", "dir_vs", "md_cs", "md_vols", "md_drifts", "md_sts", "md_detvals",
             "md_discts", "bb_inds", "bb_data"]


def _op_arrays(inputs):
    v = dict(zip(OP_INPUTS, inputs))
    a = {k: np.ascontiguousarray(v[k], dtype=np.int32 if k in ("dir_vs", "bb_inds") else np.float32)
         for k in OP_INPUTS[2:]}
    num_models, num_dates, num_und = a["md_vols"].shape
    dims = (int(v["contract_number"]), int(a["dir_vs"].shape[1]), num_models, num_und, num_dates,
            int(a["md_discts"].shape[1]))
    return int(v["num_mc_it"]), a, dims


def option_pricing_sums(*inputs, first: int = 0, count: int | None = None, threads: int | None = None):
    """Per-model f64 sums of the payoffs of paths [first, first + count)."""
    num_mc_it, a, dims = _op_arrays(inputs)
    L = load()
    fn = L.lvc_oracle_op_sums
    fn.restype = None
    fn.argtypes = [ctypes.c_int] * 6 + [ctypes.c_void_p] * 9 + [ctypes.c_int64, ctypes.c_int64, ctypes.c_int,
                                                                  ctypes.c_void_p]
    count = num_mc_it - first if count is None else count
    threads = threads or max(1, min(os.cpu_count() or 1, 64))
    sums = np.zeros(dims[2], np.float64)
    fn(*dims, *[a[k].ctypes.data for k in OP_INPUTS[2:]], first, count, threads, sums.ctypes.data)
    return sums


def option_pricing(*inputs, threads: int | None = None, order: str = "f64") -> np.ndarray:
    """finpar/OptionPricing.fut's main (f32): [num_models] mean payoffs.

    order="f64": the sum over paths (a reduce whose order the program leaves
    open, finpar/OptionPricing.fut:321) accumulated in f64 and rounded once --
    the order the GPU kernels use.  order="sequential_f32": an f32 running sum
    in path order, the order that reproduces the reference's own golden
    outputs (finpar/OptionPricing-data/{small,medium}.out bit for bit)."""
    num_mc_it = int(inputs[1])
    if order == "sequential_f32":
        p = option_pricing_payoffs(*inputs, threads=threads)
        tot = np.cumsum(p, axis=0, dtype=np.float32)[-1] if len(p) else np.zeros(p.shape[1], np.float32)
        return (tot / np.float32(num_mc_it)).astype(np.float32)
    if order != "f64":
        raise ValueError(f"unknown order {order!r}")
    sums = option_pricing_sums(*inputs, threads=threads)
    return (sums.astype(np.float32) / np.float32(num_mc_it)).astype(np.float32)


def option_pricing_payoffs(*inputs, first: int = 0, count: int | None = None,
                           threads: int | None = None) -> np.ndarray:
    """The f32 payoffs of paths [first, first + count), [path][model]."""
    num_mc_it, a, dims = _op_arrays(inputs)
    L = load()
    fn = L.lvc_oracle_op_payoffs
    fn.restype = None
    fn.argtypes = [ctypes.c_int] * 6 + [ctypes.c_void_p] * 9 + [ctypes.c_int64, ctypes.c_int64, ctypes.c_int,
                                                                  ctypes.c_void_p]
    count = num_mc_it - first if count is None else count
    threads = threads or max(1, min(os.cpu_count() or 1, 64))
    out = np.zeros((count, dims[2]), np.float32)
    fn(*dims, *[a[k].ctypes.data for k in OP_INPUTS[2:]], first, count, threads, out.ctypes.data)
    return out


def option_pricing_path(*inputs, n: int) -> np.ndarray:
    """One path's (Sobol index n, 1-based) f32 payoffs per model."""
    _, a, dims = _op_arrays(inputs)
    L = load()
    fn = L.lvc_oracle_op_path
    fn.restype = None
    fn.argtypes = [ctypes.c_int] * 6 + [ctypes.c_void_p] * 9 + [ctypes.c_int32, ctypes.c_void_p]
    out = np.zeros(dims[2], np.float64)
    fn(*dims, *[a[k].ctypes.data for k in OP_INPUTS[2:]], n, out.ctypes.data)
    return out.astype(np.float32)
