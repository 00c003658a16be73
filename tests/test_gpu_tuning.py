"""Shape autotuner (GPU): every candidate shape of a grid class prices the
same options as the FP64 oracle, the autotuner keeps a shape no slower than
the built-in one, and the tuning file round-trips.

Tolerances as in test_gpu_parity: 1e-9 relative (f64), 1e-4 relative on
prices above 1e-3 of the largest (FP32 state)."""
import importlib

import numpy as np
import pytest

from conftest import FIELDS

pytestmark = pytest.mark.gpu

wl = importlib.import_module("futhark-benchmarks_b200.workloads")


def rel_err(got, exp):
    got = np.asarray(got, dtype=np.float64)
    exp = np.asarray(exp, dtype=np.float64)
    return np.max(np.abs(got - exp) / np.maximum(np.abs(exp), 1e-300)) if exp.size else 0.0


SHAPES = [(32, 32), (64, 128), (128, 64), (256, 256), (256, 32), (96, 64), (37, 45), (200, 7), (512, 64)]


@pytest.mark.parametrize("grid", SHAPES, ids=[f"{x}x{y}" for x, y in SHAPES])
def test_every_candidate_shape_matches_oracle(ctx, oracle, grid):
    X, Y = grid
    c = wl.Calibration(5, X, Y, 6, 0.03, 5.0, 0.2, 0.6, 0.5)
    exp = oracle.main_f64(*[getattr(c, k) for k in FIELDS])
    cands = ctx.shape_candidates(X, Y)
    assert cands
    try:
        for sh in cands:
            ctx.tuning_set(X, Y, 0, sh)
            assert ctx.tuning_get(X, Y, 0).shape.key() == sh.key()
            # a fresh plan takes the pinned shape ...
            plan = ctx.plan([c])
            assert plan.shape(0).key() == sh.key()
            plan.run()
            assert rel_err(plan.prices(), exp) <= 1e-9, sh
            plan.free()
            # ... and so does the entry point, whose cached plan (same sizes on
            # every pass of this loop) is rebuilt when the tuning table changes
            got = ctx.main_f64(*[getattr(c, k) for k in FIELDS])
            assert rel_err(got, exp) <= 1e-9, sh
    finally:
        ctx.tuning_set(X, Y, 0, None)


@pytest.mark.parametrize("grid", [(64, 128), (256, 256), (37, 45)], ids=["64x128", "256x256", "37x45"])
def test_every_candidate_shape_f32_state(ctx, oracle, grid):
    X, Y = grid
    c = wl.Calibration(5, X, Y, 6, 0.03, 5.0, 0.2, 0.6, 0.5)
    exp = oracle.main_f64(*[getattr(c, k) for k in FIELDS])
    big = np.abs(exp) > 1e-3 * np.max(np.abs(exp))
    try:
        for sh in ctx.shape_candidates(X, Y, 1):
            ctx.tuning_set(X, Y, 1, sh)
            plan = ctx.plan([c], precision=1)
            assert plan.shape(0).key() == sh.key()
            plan.free()
            got = ctx.batch([c], precision=1)
            assert rel_err(got[big], exp[big]) <= 1e-4, sh
            assert np.max(np.abs(got[~big] - exp[~big]), initial=0.0) <= 1e-7, sh
    finally:
        ctx.tuning_set(X, Y, 1, None)


def test_autotune_then_batch_matches_oracle(pkg, oracle, tmp_path):
    calibs = wl.uneven_mix(10, seed=21, sizes=(32, 64, 128, 256), numT=(6, 12), outer=(2, 6))
    with pkg.Context() as c:
        entries = c.autotune(calibs, probe_steps=4)
        classes = {(x.numX, x.numY) for x in calibs}
        assert {(e.numX, e.numY) for e in entries} == classes
        for e in entries:
            assert e.tuned == 1
            if e.us_per_step_default > 0:
                assert e.us_per_step_best <= e.us_per_step_default * 1.0001
        got = c.batch(calibs)
        assert rel_err(got, oracle.batch_f64(calibs)) <= 1e-9
        path = tmp_path / "lvc.tuning"
        c.tuning_save(path)
        text = path.read_text()
        assert "lvc.streams=" in text and "lvc.shape.f64." in text
    with pkg.Context() as d:
        d.tuning_load(path)
        again = {(e.numX, e.numY, e.shape.key()) for e in d.tuning_entries()}
        assert again == {(e.numX, e.numY, e.shape.key()) for e in entries}
        assert np.array_equal(d.batch(calibs), got)


def test_tuning_errors(ctx, pkg, tmp_path):
    with pytest.raises(pkg.FutharkError):
        ctx.shape_candidates(2, 32)
    bad = pkg.Shape(family=2, cluster=3)
    with pytest.raises(pkg.FutharkError):
        ctx.tuning_set(64, 64, 0, bad)
    p = tmp_path / "bad.tuning"
    p.write_text("lvc.shape.f64.64x64=line_full,3\n")
    with pytest.raises(pkg.FutharkError):
        ctx.tuning_load(p)
    with pytest.raises(pkg.FutharkError):
        ctx.set_tuning_param("lvc.streams", 0)
    assert ctx.main_f64(2, 32, 32, 4, 0.03, 5.0, 0.2, 0.6, 0.5).shape == (2,)


def test_plan_autotuner_keeps_valid_parameters(pkg, oracle):
    calibs = wl.uneven_mix(8, seed=23, sizes=(32, 64, 128), numT=(6, 12), outer=(2, 5))
    with pkg.Context() as c:
        for prec in (0, 1):
            res = c.autotune_plan(calibs, precision=prec, max_steps=4)
            assert res["lvc.grid"] in (0, 1) and res["lvc.streams"] in (2, 4) and res["capped_plan_ms"] > 0
        got = c.batch(calibs)  # plans built afterwards run under the chosen parameters
        assert rel_err(got, oracle.batch_f64(calibs)) <= 1e-9


def test_plan_autotuner_checks_changed_shapes(pkg, oracle):
    # a class pinned to a non-built-in shape is checked against the whole
    # plan: afterwards it holds either that shape or the built-in one, and
    # plans built afterwards are still right
    calibs = wl.uneven_mix(8, seed=29, sizes=(64, 128), numT=(6, 12), outer=(2, 5))
    X, Y = calibs[0].numX, calibs[0].numY
    with pkg.Context() as c:
        builtin = c.tuning_get(X, Y).shape.key()
        other = [s for s in c.shape_candidates(X, Y) if s.key() != builtin]
        assert other
        c.tuning_set(X, Y, 0, other[0])
        c.autotune_plan(calibs, precision=0, max_steps=4)
        assert c.tuning_get(X, Y).shape.key() in (builtin, other[0].key())
        got = c.batch(calibs)
        assert rel_err(got, oracle.batch_f64(calibs)) <= 1e-9
