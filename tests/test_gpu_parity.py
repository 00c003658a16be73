"""Parity of the CUDA engine with the CPU oracle, through the C ABI (GPU).

Tolerances (relative, against the f64 oracle, which restates
finpar/LocVolCalib.fut line by line):
  * f64 engine: 1e-9 on every price;
  * f32-state engine: 1e-4 on every price above 1e-3 of the largest price of
    its calibration, 1e-7 absolute below that;
  * f32 entry point vs the reference's golden .out files: 5e-6 absolute (the
    golden files are f32 results carrying up to 2.8e-6 of their own error).
"""
import importlib
import os

import numpy as np
import pytest

from conftest import FIELDS, dataset_args

pytestmark = pytest.mark.gpu

wl = importlib.import_module("futhark-benchmarks_b200.workloads")

F64_RTOL = 1e-9
F32S_RTOL = 1e-4


def rel_err(got, exp):
    got = np.asarray(got, dtype=np.float64)
    exp = np.asarray(exp, dtype=np.float64)
    return np.max(np.abs(got - exp) / np.maximum(np.abs(exp), 1e-300)) if exp.size else 0.0


def oracle_for(oracle, c, strikes=None):
    """f64 oracle prices of calibration c (optionally only some strike indices,
    priced on all host threads)."""
    if strikes is None:
        return oracle.main_f64(*[getattr(c, k) for k in FIELDS])
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, os.cpu_count() or 1)) as ex:
        return np.array(list(ex.map(
            lambda i: oracle.value_f64(c.numX, c.numY, c.numT, c.s0, 0.001 * i, c.t, c.alpha, c.nu, c.beta),
            strikes)))


def check_f32_state(got, exp):
    """The FP32-state contract: 1e-4 relative on every price above 1e-3 of the
    calibration's largest, 1e-7 absolute below; returns the max relative error
    over the significant prices."""
    big = np.abs(exp) > 1e-3 * np.max(np.abs(exp))
    err = rel_err(got[big], exp[big])
    assert err <= F32S_RTOL
    assert np.max(np.abs(got[~big] - exp[~big]), initial=0.0) <= 1e-7
    return err


@pytest.mark.parametrize("name", ["small", "medium"])
def test_entry_f64_matches_oracle(ctx, oracle, name):
    c = wl.DATASETS[name]
    got = ctx.main_f64(*[getattr(c, k) for k in FIELDS])
    exp = oracle_for(oracle, c)
    assert got.shape == (c.outer,)
    assert rel_err(got, exp) <= F64_RTOL


def test_entry_f64_large_matches_oracle(ctx, oracle):
    # 256 x 256 grid: split over a thread-block cluster; oracle on 32 of the 256 strikes
    c = wl.LARGE
    got = ctx.main_f64(*[getattr(c, k) for k in FIELDS])
    idx = list(range(0, 256, 8))
    assert rel_err(got[idx], oracle_for(oracle, c, idx)) <= F64_RTOL


@pytest.mark.parametrize("name", ["small", "medium", "large"])
def test_entry_f32_matches_reference_golden(ctx, golden, name):
    e = golden[name]
    got = ctx.main(*dataset_args(e))
    assert got.dtype == np.float32
    exp = np.asarray(e["expected_f32"], dtype=np.float64)
    assert np.max(np.abs(got.astype(np.float64) - exp)) <= 5e-6


def test_batched_uneven_matches_oracle(ctx, oracle):
    calibs = wl.uneven_mix(12, seed=11, sizes=(32, 64), numT=(8, 24), outer=(2, 6))
    got = ctx.batch(calibs)
    exp = oracle.batch_f64(calibs)
    assert got.shape == exp.shape
    assert rel_err(got, exp) <= F64_RTOL


def test_batched_all_grid_classes(ctx, oracle):
    # every (numX, numY) pair of the uneven workload, short time lines
    calibs = []
    for X in (32, 64, 128, 256):
        for Y in (32, 64, 128, 256):
            calibs.append(wl.Calibration(2, X, Y, 5, 0.031, 3.0, 0.25, 0.5, 0.6))
    got = ctx.batch(calibs)
    exp = oracle.batch_f64(calibs)
    assert rel_err(got, exp) <= F64_RTOL


def test_f32_state_error_vs_oracle(ctx, oracle):
    calibs = wl.uneven_mix(8, seed=5, sizes=(32, 64, 128), numT=(16, 48), outer=(3, 8))
    got = ctx.batch(calibs, precision=1)
    exp = oracle.batch_f64(calibs)
    offs = np.concatenate([[0], np.cumsum([c.outer for c in calibs])])
    for i in range(len(calibs)):
        g, e = got[offs[i]:offs[i + 1]], exp[offs[i]:offs[i + 1]]
        big = np.abs(e) > 1e-3 * np.max(np.abs(e))
        assert rel_err(g[big], e[big]) <= F32S_RTOL
        assert np.max(np.abs(g[~big] - e[~big]), initial=0.0) <= 1e-7


def test_f32_state_large_config(ctx, oracle):
    # the large dataset's shape (256 x 256 x 64, a cluster per strike) in FP32
    # state; the oracle prices every eighth strike
    c = wl.LARGE
    got = ctx.batch([c], precision=1)
    idx = np.arange(0, 256, 8)
    check_f32_state(got[idx], oracle_for(oracle, c, idx))


def test_f32_state_long_time_line(ctx, oracle):
    # 255 steps on 256-sized grids, where the f32 drift is largest
    for X, Y in ((256, 256), (256, 64), (64, 256)):
        c = wl.Calibration(12, X, Y, 256, 0.041, 9.5, 0.27, 0.75, 0.65)
        got = ctx.batch([c], precision=1)
        check_f32_state(got, oracle.main_f64(*[getattr(c, k) for k in FIELDS]))


def mix_slice(n_big=3, n_rand=8):
    """Calibrations of the benchmark's own mix (512 from seed 0): its n_big
    largest by work and n_rand more at random."""
    mix = wl.uneven_mix(512, seed=0)
    order = sorted(range(len(mix)), key=lambda i: -mix[i].work())
    rng = np.random.default_rng(1)
    pick = order[:n_big] + list(rng.choice(order[n_big:], size=n_rand, replace=False))
    return [mix[i] for i in sorted(pick)]


def test_benchmark_mix_slice_f64(ctx, oracle):
    calibs = mix_slice()
    assert max(c.numT for c in calibs) > 200 and max(c.numX * c.numY for c in calibs) == 65536
    got = ctx.batch(calibs)
    exp = oracle.batch_f64(calibs)
    assert rel_err(got, exp) <= F64_RTOL


def test_benchmark_mix_slice_f32_state(ctx, oracle):
    calibs = mix_slice(2, 5)
    got = ctx.batch(calibs, precision=1)
    exp = oracle.batch_f64(calibs)
    offs = np.concatenate([[0], np.cumsum([c.outer for c in calibs])])
    for i in range(len(calibs)):
        check_f32_state(got[offs[i]:offs[i + 1]], exp[offs[i]:offs[i + 1]])


def test_alone_equals_in_mix(ctx):
    # the arithmetic of an instance does not depend on what runs beside it
    a = wl.Calibration(5, 64, 32, 20, 0.033, 4.0, 0.22, 0.55, 0.45)
    others = wl.uneven_mix(6, seed=2, sizes=(32, 64, 128), numT=(8, 30), outer=(2, 9))
    alone = ctx.batch([a])
    mixed = ctx.batch(others[:3] + [a] + others[3:])
    off = sum(c.outer for c in others[:3])
    assert np.array_equal(alone, mixed[off:off + a.outer])


@pytest.mark.parametrize("shape", [(3, 3, 2), (37, 45, 17), (9, 130, 6), (200, 7, 5), (130, 33, 4)])
def test_ragged_sizes_match_oracle(ctx, oracle, shape):
    X, Y, T = shape
    c = wl.Calibration(4, X, Y, T, 0.03, 5.0, 0.2, 0.6, 0.5)
    got = ctx.main_f64(*[getattr(c, k) for k in FIELDS])
    assert rel_err(got, oracle_for(oracle, c)) <= F64_RTOL


@pytest.mark.parametrize("shape", [(128, 128), (256, 64), (64, 256)])
def test_cluster_runs_many_instances_per_cluster(ctx, oracle, shape):
    # more strikes than resident clusters: every cluster prices several
    # instances in a row, which exercises the hand-over of halo rows between them
    X, Y = shape
    c = wl.Calibration(300, X, Y, 5, 0.03, 5.0, 0.2, 0.6, 0.5)
    got = ctx.main_f64(*[getattr(c, k) for k in FIELDS])
    idx = list(range(0, 300, 23)) + [299]
    assert rel_err(got[idx], oracle_for(oracle, c, idx)) <= F64_RTOL


def test_hbm_state_fallback_matches_oracle(ctx, oracle):
    # 512 x 512 f64 does not fit on chip even over a 16-CTA cluster
    c = wl.Calibration(2, 512, 512, 3, 0.03, 5.0, 0.2, 0.6, 0.5)
    got = ctx.main_f64(*[getattr(c, k) for k in FIELDS])
    assert rel_err(got, oracle_for(oracle, c)) <= F64_RTOL


def test_numT_one_and_empty(ctx):
    got = ctx.main_f64(5, 16, 16, 1, 0.03, 5.0, 0.2, 0.6, 0.5)
    assert np.allclose(got, np.maximum(0.03 - 0.001 * np.arange(5), 0.0), rtol=0, atol=1e-17)
    assert ctx.main_f64(0, 32, 32, 8, 0.03, 5.0, 0.2, 0.6, 0.5).shape == (0,)


def test_invalid_inputs_are_errors(ctx, pkg):
    for args in [(4, 2, 16, 8), (4, 16, 2, 8), (4, 16, 16, 0), (-1, 16, 16, 8), (4, 1024, 16, 8)]:
        with pytest.raises(pkg.FutharkError) as ei:
            ctx.main_f64(*args, 0.03, 5.0, 0.2, 0.6, 0.5)
        assert ei.value.code == pkg.FUTHARK_PROGRAM_ERROR
    # spot index outside the grid (alpha * sqrt(t) tiny)
    with pytest.raises(pkg.FutharkError):
        ctx.main_f64(4, 32, 32, 8, 0.03, 1e-4, 0.001, 0.6, 0.5)
    # the context stays usable after an error
    assert ctx.main_f64(2, 32, 32, 4, 0.03, 5.0, 0.2, 0.6, 0.5).shape == (2,)


def test_plan_reuse_and_set_params(ctx, oracle):
    calibs = wl.uneven_mix(3, seed=9, sizes=(32, 64), numT=(6, 12), outer=(2, 4))
    plan = ctx.plan(calibs)
    plan.run()
    p1 = plan.prices()
    plan.run()
    assert np.array_equal(plan.prices(), p1)
    moved = [wl.Calibration(c.outer, c.numX, c.numY, c.numT, c.s0 * 1.1, c.t, c.alpha, c.nu, c.beta)
             for c in calibs]
    plan.set_params(moved)
    plan.run()
    assert rel_err(plan.prices(), oracle.batch_f64(moved)) <= F64_RTOL
    plan.free()
