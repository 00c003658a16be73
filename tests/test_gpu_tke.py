"""The ocean model's tke step (misc/ocean-sim/tke.fut, entry main, f32) on the
GPU through libtke.so, against the reference's golden outputs and the CPU
oracle: bit for bit, as every operation is rounded in the reference's order."""
import ctypes
import importlib
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden_npz

pytestmark = pytest.mark.gpu

W = importlib.import_module("futhark-benchmarks_b200.workloads")


def same_bits(got, want):
    got = np.asarray(got)
    want = np.asarray(want)
    assert got.shape == want.shape and got.dtype == want.dtype
    return np.array_equal(got.view(np.uint32), want.view(np.uint32))


@pytest.fixture(scope="module")
def tctx(tke):
    c = tke.TkeContext()
    yield c
    c.close()


def test_golden_bit_exact(tctx, tke):
    # misc/ocean-sim/data/tke32-small.{in,out}: [20][20][10]
    z = golden_npz("tke32_small")
    outs = tctx.main(*[z[f"in{i:02d}"] for i in range(25)])
    for k, name in enumerate(tke.OUTPUT_NAMES):
        assert same_bits(outs[k], z[f"out{k}"]), name


@pytest.mark.parametrize("shape,wet,seed", [
    ((20, 20, 10), True, 1), ((8, 9, 5), True, 2), ((33, 17, 12), True, 3), ((6, 6, 2), True, 4),
    ((5, 7, 3), False, 5), ((40, 37, 100), True, 6), ((4, 4, 7), True, 7), ((9, 6, 401), True, 8),
    ((64, 48, 33), False, 9),
], ids=lambda v: "x".join(map(str, v)) if isinstance(v, tuple) else str(v))
def test_random_bit_exact_vs_oracle(tctx, tke, oracle, shape, wet, seed):
    ins = W.tke_inputs(*shape, seed=seed, wet=wet)
    want = oracle.tke(*ins)
    got = tctx.main(*ins)
    for k, name in enumerate(tke.OUTPUT_NAMES):
        assert same_bits(got[k], want[k]), (name, shape)


def test_pass_through_outputs_share_storage(tctx, tke):
    # tketau, tketaum1, dtketaup1 and dtketaum1 come back unchanged
    ins = W.tke_inputs(10, 11, 6, seed=11, wet=True)
    got = tctx.main(*ins)
    for out_k, in_k in ((0, 0), (2, 2), (4, 4), (5, 5)):
        assert same_bits(got[out_k], ins[in_k])


def test_shape_errors(tctx, tke, pkg):
    ins = list(W.tke_inputs(8, 8, 4, seed=12))
    bad = list(ins)
    bad[16] = ins[16][:3]  # dzt of the wrong length
    with pytest.raises(pkg.FutharkError) as ei:
        tctx.main(*bad)
    assert ei.value.code == pkg.FUTHARK_PROGRAM_ERROR and "size" in ei.value.msg
    bad = list(ins)
    bad[7] = ins[7][:, :, :3]  # vtau of another shape
    with pytest.raises(pkg.FutharkError) as ei:
        tctx.main(*bad)
    assert "shape" in ei.value.msg
    # zdim 1: the reference's dtketau indexes flux_top at z - 1 = -1
    with pytest.raises(pkg.FutharkError) as ei:
        tctx.main(*W.tke_inputs(6, 6, 1, seed=13))
    assert "out of bounds" in ei.value.msg
    # the context is still usable
    ok = tctx.main(*ins)
    assert ok[1].shape == (8, 8, 4)


def test_empty_dimensions(tctx, tke):
    outs = tctx.main(*W.tke_inputs(0, 5, 4, seed=14))
    assert outs[1].shape == (0, 5, 4) and outs[6].shape == (0, 5)
    outs = tctx.main(*W.tke_inputs(5, 5, 0, seed=15))
    assert outs[1].shape == (5, 5, 0)


def test_device_step_matches_entry(tctx, tke, oracle):
    import torch
    X, Y, Z = 24, 20, 16
    ins = dict(zip(tke.INPUT_NAMES, W.tke_inputs(X, Y, Z, seed=16, wet=True)))
    dev = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in ins.items()}
    out = {"tketaup1_out": torch.empty((X, Y, Z), dtype=torch.float32, device="cuda"),
           "dtketau_out": torch.empty((X, Y, Z), dtype=torch.float32, device="cuda"),
           "tke_surf_corr_out": torch.empty((X, Y), dtype=torch.float32, device="cuda")}
    scratch = torch.empty(tctx.scratch_bytes(X, Y, Z), dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    ptrs = {k: dev[k].data_ptr() for k in tke.STEP_INPUTS}
    ptrs.update({k: v.data_ptr() for k, v in out.items()})
    ptrs["scratch"] = scratch.data_ptr()
    tctx.step((X, Y, Z), ptrs)
    tctx.check()
    want = oracle.tke(*[ins[k] for k in tke.INPUT_NAMES])
    assert same_bits(out["tketaup1_out"].cpu().numpy(), want[1])
    assert same_bits(out["dtketau_out"].cpu().numpy(), want[3])
    assert same_bits(out["tke_surf_corr_out"].cpu().numpy(), want[6])


@pytest.mark.parametrize("off", [0, 1])
def test_device_step_any_alignment_and_ragged_size(tctx, tke, oracle, off):
    # the Adams-Bashforth update moves four cells per 16-byte access where the
    # arrays allow it and one at a time otherwise: arrays 4 bytes past the
    # 16-byte grid (off = 1) and a cell count that is not a multiple of 4 take
    # the one-at-a-time path and its tail
    import torch
    X, Y, Z = 7, 6, 5
    ins = dict(zip(tke.INPUT_NAMES, W.tke_inputs(X, Y, Z, seed=18, wet=True)))

    def place(a):
        a = np.ascontiguousarray(a, dtype=np.float32 if a.dtype.kind == "f" else a.dtype)
        t = torch.zeros(a.size + off, dtype=torch.from_numpy(a).dtype, device="cuda")
        t[off:] = torch.from_numpy(a.ravel()).cuda()
        return t

    dev = {k: place(v) for k, v in ins.items()}
    out = {k: torch.zeros(n + off, dtype=torch.float32, device="cuda")
           for k, n in (("tketaup1_out", X * Y * Z), ("dtketau_out", X * Y * Z), ("tke_surf_corr_out", X * Y))}
    scratch = torch.empty(tctx.scratch_bytes(X, Y, Z), dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    ptrs = {k: dev[k][off:].data_ptr() for k in tke.STEP_INPUTS}
    ptrs.update({k: v[off:].data_ptr() for k, v in out.items()})
    ptrs["scratch"] = scratch.data_ptr()
    tctx.step((X, Y, Z), ptrs)
    tctx.check()
    want = oracle.tke(*[ins[k] for k in tke.INPUT_NAMES])
    assert same_bits(out["tketaup1_out"][off:].cpu().numpy().reshape(X, Y, Z), want[1])
    assert same_bits(out["dtketau_out"][off:].cpu().numpy().reshape(X, Y, Z), want[3])
    assert same_bits(out["tke_surf_corr_out"][off:].cpu().numpy().reshape(X, Y), want[6])


def test_device_step_rejects_unaligned_scratch(tctx, tke, pkg):
    import torch
    X, Y, Z = 6, 6, 4
    scratch = torch.empty(tctx.scratch_bytes(X, Y, Z) + 256, dtype=torch.uint8, device="cuda")
    ptrs = {k: scratch.data_ptr() for k in tke.STEP_INPUTS + tke.STEP_OUTPUTS}
    ptrs["scratch"] = scratch.data_ptr() + 4
    with pytest.raises(pkg.FutharkError) as ei:
        tctx.step((X, Y, Z), ptrs)
    assert "128-byte" in ei.value.msg


def test_many_steps_in_sequence(tctx, tke, oracle):
    # a time loop through the generated API: each step's outputs are the next
    # step's state inputs (tketaup1 -> tketau and so on as the model rotates them)
    ins = list(W.tke_inputs(16, 14, 9, seed=17, wet=True))
    cpu = list(ins)
    for _ in range(3):
        g = tctx.main(*ins)
        c = oracle.tke(*cpu)
        for k in range(7):
            assert same_bits(g[k], c[k])
        # rotate: tau <- taup1, taum1 <- tau; dtau <- new, dtaum1 <- old dtau
        ins = [g[1], g[1].copy(), g[0], g[3], g[4], g[3].copy()] + ins[6:]
        cpu = [c[1], c[1].copy(), c[0], c[3], c[4], c[3].copy()] + cpu[6:]
