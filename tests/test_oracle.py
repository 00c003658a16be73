"""The CPU oracle pinned against the reference's own golden data (no GPU).

* finpar/LocVolCalib-data/{small,medium,large}.out: prices of the reference's
  f32 program.  Those files are f32 results printed to 6 significant digits
  (large: 6 decimals), and they differ from the f64 solution by up to
  2.8e-6 absolute; the restated f32 and f64 oracles must both land within
  5e-6 absolute of every golden price.
* misc/ocean-sim/data/tridiag32-small.{in,out}: the sequential Thomas solver
  restated from misc/ocean-sim/tridiag.fut:81-95 reproduces the golden file
  bit for bit.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN, dataset_args, golden_npz

GOLDEN_ABS_TOL = 5e-6


@pytest.mark.parametrize("name", ["small", "medium"])
def test_oracle_f32_matches_reference_outputs(oracle, golden, name):
    e = golden[name]
    got = oracle.main_f32(*dataset_args(e)).astype(np.float64)
    exp = np.asarray(e["expected_f32"], dtype=np.float64)
    assert got.shape == exp.shape
    assert np.max(np.abs(got - exp)) <= GOLDEN_ABS_TOL


@pytest.mark.parametrize("name", ["small", "medium"])
def test_oracle_f64_matches_reference_outputs(oracle, golden, name):
    e = golden[name]
    got = oracle.main_f64(*dataset_args(e))
    exp = np.asarray(e["expected_f32"], dtype=np.float64)
    assert np.max(np.abs(got - exp)) <= GOLDEN_ABS_TOL


@pytest.mark.slow
def test_oracle_large_matches_reference_outputs(oracle, golden):
    e = golden["large"]
    exp = np.asarray(e["expected_f32"], dtype=np.float64)
    got32 = oracle.main_f32(*dataset_args(e)).astype(np.float64)
    assert np.max(np.abs(got32 - exp)) <= GOLDEN_ABS_TOL
    got64 = oracle.main_f64(*dataset_args(e))
    assert np.max(np.abs(got64 - exp)) <= GOLDEN_ABS_TOL


def test_tridag_seq_reproduces_golden_bit_exact(oracle):
    z = golden_npz("tridiag32_small")
    x = oracle.tridag(z["a"], z["b"], z["c"], z["y"], form="seq")
    assert x.dtype == np.float32
    assert np.array_equal(x, z["x"])


def test_tridag_scan_form_agrees_with_thomas_f64(oracle):
    z = golden_npz("tridiag32_small")
    a, b, c, y = (z[k].astype(np.float64) for k in "abcy")
    xp = oracle.tridag(a, b, c, y, form="par")
    xs = oracle.tridag(a, b, c, y, form="seq")
    # the fixture's systems are not diagonally dominant; the two f64 forms
    # still agree to ~1e-9 of the solution's scale, row by row
    scale = np.max(np.abs(xs), axis=1, keepdims=True)
    assert np.max(np.abs(xp - xs) / scale) < 1e-8


def test_tridag_diagonally_dominant_forms_agree(oracle):
    rng = np.random.default_rng(7)
    rows, n = 64, 200
    a = rng.uniform(-1, 1, (rows, n))
    c = rng.uniform(-1, 1, (rows, n))
    b = np.abs(a) + np.abs(c) + rng.uniform(0.5, 2, (rows, n))
    y = rng.uniform(-1, 1, (rows, n))
    xp = oracle.tridag(a, b, c, y, form="par")
    xs = oracle.tridag(a, b, c, y, form="seq")
    assert np.max(np.abs(xp - xs)) < 1e-13
    # and both solve the system
    r = b * xs + np.pad(a[:, 1:] * xs[:, :-1], ((0, 0), (1, 0))) + np.pad(c[:, :-1] * xs[:, 1:], ((0, 0), (0, 1)))
    assert np.max(np.abs(r - y)) < 1e-12


def test_value_scan_vs_thomas_f64(oracle):
    # the whole rollback with the two tridiagonal formulations
    args = (24, 20, 30, 0.03, 0.004, 5.0, 0.2, 0.6, 0.5)
    v_par = oracle.value_f64(*args, seq=False)
    v_seq = oracle.value_f64(*args, seq=True)
    assert abs(v_par - v_seq) <= 1e-13 * abs(v_seq)


def test_numT_one_is_the_payoff(oracle):
    # no time step: res[myYindex, myXindex] of setPayoff, i.e. max(s0 - strike, 0)
    out = oracle.main_f64(5, 16, 16, 1, 0.03, 5.0, 0.2, 0.6, 0.5)
    strikes = 0.001 * np.arange(5)
    assert np.allclose(out, np.maximum(0.03 - strikes, 0.0), rtol=0, atol=1e-16)


def test_invalid_sizes_rejected(oracle):
    with pytest.raises(ValueError):
        oracle.main_f64(4, 2, 16, 8, 0.03, 5.0, 0.2, 0.6, 0.5)
    with pytest.raises(ValueError):
        oracle.main_f64(4, 16, 16, 0, 0.03, 5.0, 0.2, 0.6, 0.5)


def test_batch_equals_per_calibration(oracle, pkg):
    from importlib import import_module
    wl = import_module("futhark-benchmarks_b200.workloads")
    calibs = wl.uneven_mix(4, seed=3, sizes=(16, 24), numT=(4, 9), outer=(1, 4))
    got = oracle.batch_f64(calibs)
    exp = np.concatenate([oracle.main_f64(*[getattr(c, k) for k in
                                           ("outer", "numX", "numY", "numT", "s0", "t", "alpha", "nu", "beta")])
                          for c in calibs])
    assert np.array_equal(got, exp)


def test_tridag_par4_agrees_with_thomas_f64(oracle):
    # misc/ocean-sim/tridiag.fut's tridagPar (4-tuple matrix scan) is the same
    # solution as tridagSeq in exact arithmetic: at f64 on the reference's own
    # test inputs the two agree to ~4e-11 (the f32 runs differ by up to 6e-2
    # on the worst element of these ill-conditioned random systems, median 2e-6)
    z = golden_npz("tridiag32_small")
    a, b, c, y = (z[k].astype(np.float64) for k in "abcy")
    xs = oracle.tridag(a, b, c, y, form="seq")
    for form in ("par", "par4"):
        xp = oracle.tridag(a, b, c, y, form=form)
        assert np.max(np.abs(xp - xs) / np.abs(xs)) <= 1e-9


def test_tke_reproduces_golden_bit_exact(oracle):
    # misc/ocean-sim/tke.fut's entry main restated in f32 with the reference's
    # operand order: all seven outputs equal tke32-small.out bit for bit
    z = golden_npz("tke32_small")
    got = oracle.tke(*[z[f"in{i:02d}"] for i in range(25)])
    for i, g in enumerate(got):
        assert np.array_equal(g, z[f"out{i}"]), i


def load_op(name):
    z = golden_npz(f"optionpricing_{name}")
    return [z[f"in{i:02d}"] for i in range(11)], z["out0"]


# finpar/OptionPricing-data/*.out hold the reference's f32 results.  They are
# the sum over paths taken as an f32 running sum in path order (a sequential
# left fold of the program's reduce, finpar/OptionPricing.fut:321): the
# oracle in that order reproduces small.out and medium.out bit for bit and
# large.out to 3.7e-6 (32 ulps of the running sum; contract 3's per-path
# payoffs are the only other input).  The f64 accumulation the GPU kernels
# use is the more accurate mean: it sits 4e-4 .. 1.1e-3 (relative) from
# those files, the error of the f32 running sum over 1e5 .. 8e6 paths.
OP_GOLDEN_REL_TOL = 2e-3


@pytest.mark.parametrize("name,tol", [("small", 0.0), ("medium", 0.0), ("large", 4e-6)])
def test_option_pricing_reference_order_reproduces_golden(oracle, name, tol):
    ins, want = load_op(name)
    got = oracle.option_pricing(*ins, order="sequential_f32")
    assert got.dtype == np.float32 and got.shape == want.shape
    assert np.all(np.abs(got.astype(np.float64) - want) <= tol * np.abs(want))
    # the f64 order's distance from the file is that f32 running sum's error
    f64 = oracle.option_pricing(*ins)
    d = np.abs(f64.astype(np.float64) - want) / np.abs(want)
    assert np.all((d > 3e-4) & (d < 2e-3))


@pytest.mark.parametrize("name", ["small", "medium", "large"])
def test_option_pricing_within_golden_tolerance(oracle, name):
    ins, want = load_op(name)
    got = oracle.option_pricing(*ins)
    assert got.shape == want.shape
    assert np.all(np.abs(got - want) <= OP_GOLDEN_REL_TOL * np.abs(want))


def test_option_pricing_small_matches_black_scholes_closed_form(oracle):
    # the small dataset is a European call on one underlying with one date:
    # the Sobol mean over 2^23 paths must reproduce the closed-form
    # Black-Scholes value of the same model (exact to ~1e-6 relative)
    from math import erf, exp, log, sqrt
    ins, _ = load_op("small")
    v = dict(zip(oracle.OP_INPUTS, ins))
    S = float(v["md_sts"][0, 0])
    mu = float(v["md_drifts"][0, 0, 0])
    s = float(v["md_vols"][0, 0, 0]) * float(v["bb_data"][0, 0]) * float(v["md_cs"][0, 0, 0])
    K, det, disc = 4000.0, float(v["md_detvals"][0, 0]), float(v["md_discts"][0, 0])
    N = lambda x: 0.5 * (1.0 + erf(x / sqrt(2.0)))
    d2 = (log(S / K) + mu) / s
    exact = (S * exp(mu + s * s / 2) * N(d2 + s) - K * N(d2)) * det * disc
    got = float(oracle.option_pricing(*ins)[0])
    assert abs(got - exact) <= 1e-5 * exact


def test_option_pricing_path_sum_consistency(oracle):
    # the per-path payoffs add up to the sums the pricer averages
    ins, _ = load_op("medium")
    ins = list(ins)
    ins[1] = np.int32(64)
    sums = oracle.option_pricing_sums(*ins, threads=3)
    paths = sum(oracle.option_pricing_path(*ins, n=n).astype(np.float64) for n in range(1, 65))
    assert np.allclose(sums, paths, rtol=0, atol=1e-9 * np.abs(sums).max())
