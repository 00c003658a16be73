"""The serving runtime (continuous batching), through the C ABI (GPU).

Every result is the same alone and in the mix (the per-instance arithmetic
does not depend on what runs beside it: bit-identical), results match the
FP64 oracle at the suite's f64 tolerance, overlapping requests complete,
the HBM budget and in-flight caps hold, and invalid requests are rejected
at submission without disturbing the server.
"""
import importlib
import threading
import time

import numpy as np
import pytest

from conftest import FIELDS

pytestmark = pytest.mark.gpu

wl = importlib.import_module("futhark-benchmarks_b200.workloads")


def test_server_results_alone_equal_in_mix(ctx, pkg, oracle):
    a = wl.Calibration(6, 64, 128, 20, 0.032, 4.0, 0.21, 0.55, 0.45)
    mix = wl.uneven_mix(24, seed=21, sizes=(32, 64, 128), numT=(8, 40), outer=(2, 12))
    with pkg.Server(ctx) as srv:
        alone = srv.result(srv.submit(a))
        tickets = [srv.submit(c) for c in mix[:10]]
        ta = srv.submit(a)
        tickets += [srv.submit(c) for c in mix[10:]]
        in_mix = srv.result(ta)
        others = [srv.result(t) for t in tickets]
        st = srv.stats()
    assert np.array_equal(alone, in_mix)
    exp = oracle.main_f64(*[getattr(a, k) for k in FIELDS])
    assert np.max(np.abs(alone - exp) / np.abs(exp)) <= 1e-9
    got = np.concatenate(others)
    ref = oracle.batch_f64(mix)
    assert np.max(np.abs(got - ref) / np.abs(ref)) <= 1e-9
    assert st["completed"] == 26 and st["failed"] == 0
    assert st["p50_ms"] > 0 and st["p99_ms"] >= st["p50_ms"]


def test_server_concurrent_submitters(ctx, pkg):
    calibs = wl.uneven_mix(32, seed=4, sizes=(32, 64), numT=(8, 20), outer=(2, 8))
    expected = ctx.batch(calibs)
    offs = np.concatenate([[0], np.cumsum([c.outer for c in calibs])])
    results = {}
    with pkg.Server(ctx, num_streams=3, max_batch_requests=4) as srv:
        def worker(ids):
            for i in ids:
                results[i] = srv.result(srv.submit(calibs[i]))
        th = [threading.Thread(target=worker, args=(range(k, 32, 4),)) for k in range(4)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        st = srv.stats()
    for i in range(32):
        assert np.array_equal(results[i], expected[offs[i]:offs[i + 1]])
    assert st["batches"] >= 8  # batches of at most 4 requests


def test_server_hbm_budget_admits_within_budget(ctx, pkg):
    # a budget that holds about two of these calibrations at a time
    c = wl.Calibration(4, 128, 128, 40, 0.03, 5.0, 0.2, 0.6, 0.5)
    per = 8 * 129 * 128 * 39 + 64 * 128 * 39 * 2 + (1 << 20)
    with pkg.Server(ctx, hbm_budget_bytes=2 * per + (4 << 20)) as srv:
        ts = [srv.submit(c) for _ in range(6)]
        res = [srv.result(t) for t in ts]
        st = srv.stats()
    assert st["completed"] == 6 and st["hbm_reserved_bytes"] <= 2 * per + (4 << 20)
    for r in res[1:]:
        assert np.array_equal(r, res[0])


def test_server_rejects_invalid_request(ctx, pkg):
    with pkg.Server(ctx) as srv:
        with pytest.raises(pkg.FutharkError):
            srv.submit(wl.Calibration(4, 2, 16, 8, 0.03, 5.0, 0.2, 0.6, 0.5))
        ok = srv.result(srv.submit(wl.Calibration(2, 32, 32, 6, 0.03, 5.0, 0.2, 0.6, 0.5)))
        assert ok.shape == (2,)


def test_server_poisson_stream_every_request_vs_oracle(ctx, pkg, oracle):
    # a Poisson stream drawn as the uneven mix (short time lines so that the
    # oracle stays cheap), submitted at its arrival times: every request's
    # prices within 1e-9 of the FP64 oracle and bit-identical to a batched run
    reqs = wl.uneven_mix(60, seed=77, numT=(8, 40))
    arrivals = wl.poisson_arrivals(2000.0, len(reqs), seed=78)
    with pkg.Server(ctx) as srv:
        t0 = time.perf_counter()
        tickets = []
        for c, ta in zip(reqs, arrivals):
            dt = t0 + ta - time.perf_counter()
            if dt > 0:
                time.sleep(dt)
            tickets.append(srv.submit(c))
        got = [srv.result(t) for t in tickets]
        st = srv.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    ref = oracle.batch_f64(reqs)
    batched = ctx.batch(reqs)
    flat = np.concatenate(got)
    assert np.array_equal(flat, batched)
    assert np.max(np.abs(flat - ref) / np.abs(ref)) <= 1e-9
