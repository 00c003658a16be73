"""finpar/OptionPricing.fut (entry main, f32) on the GPU through libop.so,
against the reference's golden outputs (at the reference test runner's
relative 2e-3) and against the CPU oracle, which computes every path with the
same f32 operations in the same order: the GPU agrees with it to within a few
f32 ulps (only the f64 sum over paths runs in another order)."""
import importlib
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden_npz

pytestmark = pytest.mark.gpu

OP_GOLDEN_REL_TOL = 2e-3
ORACLE_REL_TOL = 1e-6


def load_op(name):
    z = golden_npz(f"optionpricing_{name}")
    return [z[f"in{i:02d}"] for i in range(11)], z["out0"]


@pytest.fixture(scope="module")
def op():
    return importlib.import_module("futhark-benchmarks_b200.op")


@pytest.fixture(scope="module")
def octx(op):
    c = op.OpContext()
    yield c
    c.close()


def close_to(got, want, rel):
    got = np.asarray(got, np.float64)
    want = np.asarray(want, np.float64)
    return got.shape == want.shape and np.all(np.abs(got - want) <= rel * np.maximum(np.abs(want), 1e-30))


@pytest.mark.parametrize("name", ["small", "medium", "large"])
def test_golden_datasets(octx, oracle, name):
    ins, want = load_op(name)
    got = octx.main(*ins)
    assert close_to(got, want, OP_GOLDEN_REL_TOL), (got, want)
    assert close_to(got, oracle.option_pricing(*ins), ORACLE_REL_TOL), (got, oracle.option_pricing(*ins))


@pytest.mark.parametrize("name,paths", [("small", 1), ("small", 7), ("medium", 1), ("medium", 12345),
                                        ("large", 1), ("large", 300), ("large", 4097)])
def test_path_counts_vs_oracle(octx, oracle, name, paths):
    # one path is a single payoff: the f32 value must match the oracle's exactly
    ins, _ = load_op(name)
    ins[1] = np.int32(paths)
    got = octx.main(*ins)
    want = oracle.option_pricing(*ins)
    if paths == 1:
        assert np.array_equal(got, want), (got, want)
    else:
        assert close_to(got, want, ORACLE_REL_TOL), (got, want)


def many_models(ins, m):
    """The dataset's single model repeated m times with perturbed drifts,
    volatilities and starts."""
    v = list(ins)
    k = np.arange(m, dtype=np.float32)[:, None, None]
    v[3] = np.repeat(ins[3], m, axis=0)
    v[4] = (np.repeat(ins[4], m, axis=0) * (1 + 0.02 * k)).astype(np.float32)
    v[5] = (np.repeat(ins[5], m, axis=0) + 0.001 * k).astype(np.float32)
    v[6] = (np.repeat(ins[6], m, axis=0) * (1 + 0.01 * k[:, :, 0])).astype(np.float32)
    v[7] = np.repeat(ins[7], m, axis=0)
    v[8] = np.repeat(ins[8], m, axis=0)
    return v


@pytest.mark.parametrize("name", ["small", "medium", "large"])
def test_several_models(octx, oracle, name):
    # six models: two launch windows of the per-model accumulators
    ins, _ = load_op(name)
    ins = many_models(ins, 6)
    ins[1] = np.int32(5000)
    got = octx.main(*ins)
    assert got.shape == (6,)
    assert close_to(got, oracle.option_pricing(*ins), ORACLE_REL_TOL)


def test_other_contracts_price_zero(octx, oracle):
    ins, _ = load_op("medium")
    for contract in (0, 4, -1):
        v = list(ins)
        v[0] = np.int32(contract)
        assert np.array_equal(octx.main(*v), np.zeros(1, np.float32))
        assert np.array_equal(oracle.option_pricing(*v), np.zeros(1, np.float32))


def test_no_paths_is_nan(octx):
    ins, _ = load_op("small")
    ins[1] = np.int32(0)
    assert np.isnan(octx.main(*ins)).all()  # 0 / 0, as the reference divides


def test_errors_leave_context_usable(octx, pkg):
    ins, want = load_op("small")
    bad = list(ins)
    bad[0] = np.int32(2)  # contract 2 needs [5][3] paths
    with pytest.raises(pkg.FutharkError) as ei:
        octx.main(*bad)
    assert ei.value.code == pkg.FUTHARK_PROGRAM_ERROR and "size coercion" in ei.value.msg
    bad = list(ins)
    bad[9] = np.array([[2], [0], [0]], np.int32)  # bridge index outside one date
    with pytest.raises(pkg.FutharkError) as ei:
        octx.main(*bad)
    assert "bb_inds" in ei.value.msg
    bad = list(ins)
    bad[1] = np.int32(-5)
    with pytest.raises(pkg.FutharkError):
        octx.main(*bad)
    bad = list(ins)
    bad[2] = np.zeros((2, 30), np.int32)  # dir_vs rows != num_dates * num_und
    with pytest.raises(pkg.FutharkError) as ei:
        octx.main(*bad)
    assert "sizes" in ei.value.msg
    small = list(ins)
    small[1] = np.int32(1000)
    assert np.isfinite(octx.main(*small)).all()


def test_device_pointer_form_matches_entry(octx, op, oracle):
    import torch
    ins, _ = load_op("medium")
    ins[1] = np.int32(100000)
    dims = op.dims_of(ins)
    dev = {n: torch.from_numpy(np.ascontiguousarray(v)).cuda() for n, v in zip(op.ARRAY_NAMES, ins[2:])}
    out = torch.empty(dims["num_models"], dtype=torch.float32, device="cuda")
    scratch = torch.empty(octx.scratch_bytes(int(ins[0]), int(ins[1]), dims), dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    octx.price(int(ins[0]), int(ins[1]), dims, {n: t.data_ptr() for n, t in dev.items()}, out.data_ptr(),
               scratch.data_ptr())
    octx.check()
    assert np.array_equal(out.cpu().numpy(), octx.main(*ins))
    assert close_to(out.cpu().numpy(), oracle.option_pricing(*ins), ORACLE_REL_TOL)


@pytest.mark.parametrize("name", ["small", "medium", "large"])
def test_device_form_guards_bridge_indices(octx, op, name):
    # op_price_f32 leaves bb_inds' values to the caller; the kernels check
    # them themselves and price NaN rather than read outside a path
    import torch
    ins, _ = load_op(name)
    ins[1] = np.int32(1000)
    bad = np.array(ins[9], copy=True)
    bad[0, -1] = bad.shape[1] + 1  # a date past the path's end
    ins[9] = bad
    dims = op.dims_of(ins)
    dev = {n: torch.from_numpy(np.ascontiguousarray(v)).cuda() for n, v in zip(op.ARRAY_NAMES, ins[2:])}
    out = torch.zeros(dims["num_models"], dtype=torch.float32, device="cuda")
    scratch = torch.empty(octx.scratch_bytes(int(ins[0]), int(ins[1]), dims), dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    octx.price(int(ins[0]), int(ins[1]), dims, {n: t.data_ptr() for n, t in dev.items()}, out.data_ptr(),
               scratch.data_ptr())
    octx.check()
    assert np.isnan(out.cpu().numpy()).all()
    good, _ = load_op(name)
    good[1] = np.int32(1000)
    assert np.isfinite(octx.main(*good)).all()


@pytest.mark.parametrize("name", ["small", "medium", "large"])
def test_reference_order_reproduces_golden_outputs(op, oracle, name):
    """OP_ORDER_SEQUENTIAL_F32 (an f32 running sum over paths in path order):
    the GPU equals the oracle in that order bit for bit, which reproduces the
    reference's golden small.out and medium.out bit for bit and large.out to
    3.7e-6."""
    ins, want = load_op(name)
    with op.OpContext() as c:
        c.set_reduction_order(c.ORDER_SEQUENTIAL_F32)
        got = c.main(*ins)
    assert np.array_equal(got, oracle.option_pricing(*ins, order="sequential_f32"))
    tol = 0.0 if name in ("small", "medium") else 4e-6
    assert close_to(got, want, tol), (got, want)


@pytest.mark.parametrize("name,paths", [("small", 1), ("small", 100003), ("medium", 77777), ("large", 4097)])
def test_reference_order_path_counts(op, oracle, name, paths):
    ins, _ = load_op(name)
    ins[1] = np.int32(paths)
    with op.OpContext() as c:
        c.set_reduction_order(c.ORDER_SEQUENTIAL_F32)
        got = c.main(*ins)
        c.set_reduction_order(c.ORDER_F64)  # back to the default
        f64 = c.main(*ins)
    assert np.array_equal(got, oracle.option_pricing(*ins, order="sequential_f32"))
    assert close_to(f64, oracle.option_pricing(*ins), ORACLE_REL_TOL)
