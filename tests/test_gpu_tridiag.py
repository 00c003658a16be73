"""Batched tridiagonal solvers (GPU): the tridagNested* entry points of
misc/ocean-sim/tridiag-test.fut through the C ABI.

Parity bar: bit-exact.  The GPU folds each system's recurrences in the same
order, with the same IEEE-rounded f32 operations, as the CPU oracle:
tridagSeq against oracle form "seq" (which reproduces the reference's golden
file bit for bit) and tridagPar against oracle form "par4" (the 4-tuple scan
of misc/ocean-sim/tridiag.fut:4-79, pinned at f64 against Thomas in
test_oracle.py)."""
import ctypes
import importlib
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden_npz

pytestmark = pytest.mark.gpu

wl = importlib.import_module("futhark-benchmarks_b200.workloads")


@pytest.fixture(scope="module")
def golden_tridiag():
    return golden_npz("tridiag32_small")


@pytest.mark.parametrize("const", [False, True])
def test_seq_reproduces_reference_golden_bit_exact(ctx, golden_tridiag, const):
    z = golden_tridiag
    got = ctx.tridag(z["a"], z["b"], z["c"], z["y"], form="seq", const=const)
    assert got.dtype == np.float32 and got.shape == z["x"].shape
    assert np.array_equal(got, z["x"])


@pytest.mark.parametrize("const", [False, True])
def test_par_matches_oracle_bit_exact_on_golden_inputs(ctx, oracle, golden_tridiag, const):
    z = golden_tridiag
    got = ctx.tridag(z["a"], z["b"], z["c"], z["y"], form="par", const=const)
    assert np.array_equal(got, oracle.tridag(z["a"], z["b"], z["c"], z["y"], form="par4"))


# (rows, m): empty, single-element systems, partial warps and CTAs, the
# stanza's inner size, the tensor-memory kernel's two allocation sizes and
# their limits (128, 256) and just above them, odd and even m, the
# shared-memory kernels' limit (400) and the kernel with global scratch
# above it; rows % 4 == 0 with odd m (the tensor-copy staging of 4-system
# groups: m = 1 and 3 with boxes wider than the group, partial and whole
# CTAs, both allocation sizes) beside odd m with rows % 4 != 0 (the
# per-lane window copies)
@pytest.mark.parametrize("shape", [(0, 5), (3, 1), (7, 2), (33, 3), (129, 64), (1000, 115), (257, 128),
                                   (65, 129), (70, 200), (40, 256), (9, 257), (70, 399), (130, 400), (40, 401),
                                   (5, 1000), (4, 1), (8, 3), (132, 7), (260, 63), (4096, 115), (512, 129),
                                   (36, 255), (1001, 115)])
@pytest.mark.parametrize("form,oform", [("seq", "seq"), ("par", "par4")])
def test_random_batches_match_oracle_bit_exact(ctx, oracle, shape, form, oform):
    rows, m = shape
    a, b, c, y = wl.tridiag_inputs(rows, m, seed=rows * 7 + m)
    got = ctx.tridag(a, b, c, y, form=form)
    assert got.shape == (rows, m)
    if rows:
        assert np.array_equal(got, oracle.tridag(a, b, c, y, form=oform))


def test_const_entries_require_inner_dim_115(ctx, pkg):
    a, b, c, y = wl.tridiag_inputs(4, 100, seed=3)
    for form in ("seq", "par"):
        with pytest.raises(pkg.FutharkError) as ei:
            ctx.tridag(a, b, c, y, form=form, const=True)
        assert ei.value.code == pkg.FUTHARK_PROGRAM_ERROR
    assert ctx.tridag(a, b, c, y, form="seq").shape == (4, 100)  # context still usable


def test_mismatched_shapes_are_errors(ctx, pkg):
    a, b, c, y = wl.tridiag_inputs(4, 16, seed=4)
    with pytest.raises(pkg.FutharkError):
        ctx.tridag(a, b[:, :8], c, y)


def test_device_pointer_form_matches_entry_point(ctx, oracle):
    import torch
    rows, m = 2000, 115
    host = wl.tridiag_inputs(rows, m, seed=11)
    dev = [torch.from_numpy(v).to("cuda:0") for v in host]
    out = torch.empty_like(dev[0])
    for form, oform in (("seq", "seq"), ("par", "par4")):
        torch.cuda.synchronize()
        ctx.tridag_device(form, rows, m, *[t.data_ptr() for t in dev], out.data_ptr())
        ctx.tridag_check()
        assert np.array_equal(out.cpu().numpy(), oracle.tridag(*host, form=oform))


def test_device_pointer_form_reuses_arrays(ctx, oracle):
    # the tensor maps of a batch are kept while its arrays and shape repeat:
    # new contents in the same arrays, then a shorter batch and another inner
    # size over the same memory, must all give the oracle's solutions
    import torch
    rows, m = 1024, 115
    dev = [torch.empty(rows * m, dtype=torch.float32, device="cuda:0") for _ in range(4)]
    out = torch.empty(rows * m, dtype=torch.float32, device="cuda:0")
    for seed, r, mm in ((21, rows, m), (22, rows, m), (23, rows // 2, m), (24, 256, 111)):
        host = wl.tridiag_inputs(r, mm, seed=seed)
        for t, v in zip(dev, host):
            t[:r * mm] = torch.from_numpy(v.ravel()).to("cuda:0")
        for form, oform in (("seq", "seq"), ("par", "par4")):
            torch.cuda.synchronize()
            ctx.tridag_device(form, r, mm, *[t.data_ptr() for t in dev], out.data_ptr())
            ctx.tridag_check()
            got = out[:r * mm].cpu().numpy().reshape(r, mm)
            assert np.array_equal(got, oracle.tridag(*host, form=oform)), (seed, form)


@pytest.mark.parametrize("m", [115, 200, 300])
def test_device_pointer_form_with_unaligned_arrays(ctx, oracle, m):
    # device arrays that start 4 bytes past a 16-byte boundary (the kernels'
    # window copies are 4-byte copies: no alignment beyond the element's);
    # the tensor-memory kernel (m <= 256) and the streaming kernel above it
    import torch
    rows = 100
    host = wl.tridiag_inputs(rows, m, seed=12)
    dev = []
    for v in host:
        t = torch.zeros(rows * m + 1, dtype=torch.float32, device="cuda:0")
        t[1:] = torch.from_numpy(v.ravel()).to("cuda:0")
        dev.append(t)
    out = torch.zeros(rows * m + 1, dtype=torch.float32, device="cuda:0")
    for form, oform in (("seq", "seq"), ("par", "par4")):
        torch.cuda.synchronize()
        ctx.tridag_device(form, rows, m, *[t[1:].data_ptr() for t in dev], out[1:].data_ptr())
        ctx.tridag_check()
        got = out[1:].cpu().numpy().reshape(rows, m)
        assert np.array_equal(got, oracle.tridag(*host, form=oform))


def test_bounded_wait_runs_out_safely(ctx, pkg):
    # a device wait on a barrier nothing completes gives up after its poll
    # limit and reports the timeout through the error flag the solvers use;
    # the context stays usable
    with pytest.raises(pkg.FutharkError) as ei:
        ctx.wait_selftest(64, arrive=False)
    assert ei.value.code == pkg.FUTHARK_PROGRAM_ERROR and "timed out" in str(ei.value)
    ctx.wait_selftest(1 << 20, arrive=True)  # completes: no error, and the flag was cleared
    ctx.tridag_check()
    z = golden_npz("tridiag32_small")
    assert np.array_equal(ctx.tridag(z["a"], z["b"], z["c"], z["y"], form="seq"), z["x"])
    with pytest.raises(pkg.FutharkError):
        ctx.wait_selftest(0, arrive=True)  # poll limit out of range
