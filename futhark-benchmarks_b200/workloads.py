"""The workloads of the LocVolCalib path: the reference's three datasets and
seeded synthetic calibration mixes.

* `SMALL`, `MEDIUM`, `LARGE`: the inputs of finpar/LocVolCalib-data/{small,
  medium,large}.in (16x32x256x256, 128x256x32x64, 256x256x256x64; s0=0.03,
  t=5, alpha=0.2, nu=0.6, beta=0.5).
* `uneven_mix(n, seed)`: n calibrations with numX, numY uniform on
  {32, 64, 128, 256}, numT uniform on [32, 256], s0 ~ U[0.02, 0.05],
  alpha ~ U[0.1, 0.3], nu ~ U[0.4, 0.8], beta ~ U[0.3, 0.7], t ~ U[1, 10],
  outer uniform on [8, 64] (strikes 0.001*i as in `main`).  The reference
  suite has no such dataset; this seeded generator stands in for it with the
  value ranges of the reference's own inputs around them.
* `poisson_arrivals(rate, n, seed)`: arrival times of a Poisson request stream.
"""
from __future__ import annotations

from typing import List

import numpy as np

from . import Calibration

REF = dict(s0=0.03, t=5.0, alpha=0.2, nu=0.6, beta=0.5)
SMALL = Calibration(16, 32, 256, 256, **REF)
MEDIUM = Calibration(128, 256, 32, 64, **REF)
LARGE = Calibration(256, 256, 256, 64, **REF)
DATASETS = {"small": SMALL, "medium": MEDIUM, "large": LARGE}

GRID_SIZES = (32, 64, 128, 256)


def uneven_mix(n: int = 512, seed: int = 0, sizes=GRID_SIZES, numT=(32, 256),
               outer=(8, 64)) -> List[Calibration]:
    rng = np.random.default_rng(seed)
    X = rng.choice(np.asarray(sizes), size=n)
    Y = rng.choice(np.asarray(sizes), size=n)
    T = rng.integers(numT[0], numT[1] + 1, size=n)
    s0 = rng.uniform(0.02, 0.05, size=n)
    alpha = rng.uniform(0.1, 0.3, size=n)
    nu = rng.uniform(0.4, 0.8, size=n)
    beta = rng.uniform(0.3, 0.7, size=n)
    t = rng.uniform(1.0, 10.0, size=n)
    O = rng.integers(outer[0], outer[1] + 1, size=n)
    return [Calibration(int(O[i]), int(X[i]), int(Y[i]), int(T[i]), float(s0[i]), float(t[i]),
                        float(alpha[i]), float(nu[i]), float(beta[i])) for i in range(n)]


def total_options(calibs) -> int:
    return int(sum(c.outer for c in calibs))


def total_work(calibs) -> int:
    """Option-cell-steps: sum of outer * numX * numY * (numT - 1)."""
    return int(sum(c.work() for c in calibs))


def poisson_arrivals(rate: float, n: int, seed: int = 0) -> np.ndarray:
    """Arrival times (seconds) of n requests of a Poisson process of `rate` per second."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, size=n))


# Batched tridiagonal systems of misc/ocean-sim/tridiag-test.fut: [rows][m] f32
# arrays a, b, c, y drawn uniformly from the bounds the reference's dataset
# script gives futhark dataset (misc/ocean-sim/data/rand-dataset-tridiag.sh:
# a 0.3:1.3, b 0.4:1.4, c 0.5:1.5, y 0.2:1.2), here from a seeded numpy
# generator.  The benchmark stanza's size is [57600][115] (tridiag-test.fut:12).
TRIDIAG_BOUNDS = ((0.3, 1.3), (0.4, 1.4), (0.5, 1.5), (0.2, 1.2))
TRIDIAG_BENCH = (57600, 115)


def tridiag_inputs(rows: int, m: int, seed: int = 0):
    rng = np.random.default_rng(seed)
    return tuple(rng.uniform(lo, hi, size=(rows, m)).astype(np.float32) for lo, hi in TRIDIAG_BOUNDS)


# misc/ocean-sim/tke.fut: the benchmark's "200x200x100" dataset shape, and the
# value ranges of the reference's random-dataset recipe
# (misc/ocean-sim/data/rand-dataset-tke.sh): f32 fields uniform on [0.5, 1.5],
# kbot uniform on [-100, 10000].
TKE_BENCH = (200, 200, 100)
TKE_F32_BOUNDS = (0.5, 1.5)
TKE_KBOT_BOUNDS = (-100, 10000)


def tke_inputs(xdim: int, ydim: int, zdim: int, seed: int = 0, wet: bool = False):
    """The 25 inputs of tke.fut's main, in the entry's order.  wet=False draws
    them as the reference's recipe does; wet=True puts most columns' bottom
    inside [0, zdim] and gives the state and velocity fields both signs, so that
    every branch (land, edge and water cells, both upwind directions, the clip
    of a negative surface value) is taken."""
    rng = np.random.default_rng(seed)
    lo, hi = TKE_F32_BOUNDS
    f3 = lambda: rng.uniform(lo, hi, size=(xdim, ydim, zdim)).astype(np.float32)
    f1 = lambda n: rng.uniform(lo, hi, size=n).astype(np.float32)
    state = [f3() for _ in range(6)]
    vel = [f3() for _ in range(3)]
    masks = [f3() for _ in range(3)]
    if wet:
        state = [(s - np.float32(1.1)).astype(np.float32) for s in state]
        vel = [(v - np.float32(1.0)).astype(np.float32) for v in vel]
        masks = [(rng.uniform(size=(xdim, ydim, zdim)) < 0.85).astype(np.float32) for _ in range(3)]
        kbot = rng.integers(-1, zdim + 1, size=(xdim, ydim), endpoint=True).astype(np.int32)
    else:
        kbot = rng.integers(TKE_KBOT_BOUNDS[0], TKE_KBOT_BOUNDS[1], size=(xdim, ydim), endpoint=True).astype(np.int32)
    grid = [f1(xdim), f1(xdim), f1(ydim), f1(ydim), f1(zdim), f1(zdim), f1(ydim), f1(ydim)]
    forcing = [f3() for _ in range(3)]
    surf = rng.uniform(lo, hi, size=(xdim, ydim)).astype(np.float32)
    if wet:
        surf = (surf - np.float32(1.2)).astype(np.float32)
    return (*state, *vel, *masks, *grid, kbot, *forcing, surf)
