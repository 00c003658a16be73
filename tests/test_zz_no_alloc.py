"""The entry point that allocates no device memory (lvc_entry_main_f64_noalloc).

It serves callers that cannot call cudaMalloc when they need prices (for
example a serving loop that must not pay cudaMalloc's device-wide
synchronisation, or a host whose allocator already owns all of HBM): the
caller passes the output buffer, and all scratch comes from one static device
array.  This file is collected last so that a failure here stops a `-x` run
only after every other test has run.

Checked through the C ABI against the allocating entry point
futhark_entry_main_f64, at the suite's f64 tolerance (1e-9 relative), on two
calls in a row with different calibrations (the static scratch keeps the
previous call's contents), plus the size check.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ["outer", "numX", "numY", "numT", "s0", "t", "alpha", "nu", "beta"]
F64_RTOL = 1e-9


def _bind(lib):
    fn = lib.lvc_entry_main_f64_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p] + [ctypes.c_int32] * 4 + [ctypes.c_double] * 5
    return fn


def test_noalloc_matches_allocating_entry_twice(pkg):
    import torch

    calls = [
        (16, 32, 256, 40, 0.03, 5.0, 0.2, 0.6, 0.5),     # small dataset's grid, shorter time line
        (128, 256, 32, 64, 0.03, 5.0, 0.2, 0.6, 0.5),    # the medium dataset
    ]
    with pkg.Context("#0") as ctx:
        fn = _bind(pkg.load_library())
        for args in calls:
            expected = ctx.main_f64(*args)
            out = torch.full((args[0],), float("nan"), dtype=torch.float64, device="cuda:0")
            torch.cuda.synchronize()
            rc = fn(ctx._ctx, ctypes.c_void_p(out.data_ptr()), *args)
            assert rc == 0, ctx._take_error()
            ctx.sync()
            got = out.cpu().numpy()
            assert np.all(np.isfinite(got))
            rel = np.max(np.abs(got - expected) / np.abs(expected))
            assert rel <= F64_RTOL, rel


def test_noalloc_rejects_oversized_calibration(pkg):
    import torch

    with pkg.Context("#0") as ctx:
        fn = _bind(pkg.load_library())
        out = torch.empty((4,), dtype=torch.float64, device="cuda:0")
        # 256 x 256 grid with 255 steps: ~135 MB of pivot rows > the 64 MiB array
        rc = fn(ctx._ctx, ctypes.c_void_p(out.data_ptr()), 4, 256, 256, 256, 0.03, 5.0, 0.2, 0.6, 0.5)
        assert rc == pkg.FUTHARK_PROGRAM_ERROR
        assert "scratch" in ctx._take_error()
        # the context is still usable
        rc = fn(ctx._ctx, ctypes.c_void_p(out.data_ptr()), 4, 32, 32, 8, 0.03, 5.0, 0.2, 0.6, 0.5)
        assert rc == 0


def test_noalloc_size_query(pkg):
    # the size query gives the figure the entry point checks: the medium
    # dataset fits, the oversized calibration above does not, bad sizes are -1
    with pkg.Context("#0") as ctx:
        q = pkg.load_library().lvc_entry_main_f64_noalloc_bytes
        limit = 64 << 20
        assert 0 < q(ctx._ctx, 128, 256, 32, 64) <= limit
        assert q(ctx._ctx, 4, 256, 256, 256) > limit
        assert q(ctx._ctx, 4, 2, 16, 8) == -1
