"""Futhark value-file reader/writer (text and binary), no GPU."""
import importlib
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden_npz

fd = importlib.import_module("futhark-benchmarks_b200.futhark_data")

SMALL_IN = """16 --128  -- OUTER -- no restrictions
32 --32   -- NUM_X -- 2^x, where x \\in {5, ..., 9}
256 --32   -- NUM_Y
256  -- NUM_T -- no restrictions
0.03f32 --s0
5.0f32 -- t
0.2f32 -- alpha
0.6f32 -- nu
0.5f32 -- beta
"""


def test_text_scalars_with_comments():
    vals = fd.read_values(SMALL_IN)
    assert len(vals) == 9
    assert [int(v) for v in vals[:4]] == [16, 32, 256, 256]
    assert vals[0].dtype == np.int32
    assert vals[4].dtype == np.float32 and vals[4] == np.float32(0.03)


def test_text_array():
    (a,) = fd.read_values("[ 0.0300001f32,  0.0290001f32,\n 0.026f32 ] -- trailing")
    assert a.dtype == np.float32 and a.shape == (3,)
    assert a[2] == np.float32(0.026)


def test_text_nested_and_empty_and_bool():
    vals = fd.read_values("[[1i64, 2i64], [3i64, 4i64]] empty([0]f64) true [false, true]")
    assert vals[0].shape == (2, 2) and vals[0].dtype == np.int64
    assert vals[1].shape == (0,) and vals[1].dtype == np.float64
    assert bool(vals[2]) is True
    assert vals[3].tolist() == [False, True]


def test_binary_roundtrip_and_mixed():
    a = np.arange(12, dtype=np.float32).reshape(3, 4)
    b = np.array([1, -2, 3], dtype=np.int64)
    blob = fd.write_binary([a, b, np.float64(2.5)])
    vals = fd.read_values(b"16 " + blob)
    assert int(vals[0]) == 16
    assert np.array_equal(vals[1], a) and vals[1].dtype == np.float32
    assert np.array_equal(vals[2], b)
    assert float(vals[3]) == 2.5


def test_text_roundtrip():
    vals = [np.float32(0.5), np.array([1.5, 2.5], dtype=np.float64), np.int32(7)]
    back = fd.read_values(fd.write_text(vals))
    assert back[0] == vals[0] and back[0].dtype == np.float32
    assert np.array_equal(back[1], vals[1]) and back[1].dtype == np.float64
    assert back[2] == 7


def test_tridiag_fixture_shapes():
    z = golden_npz("tridiag32_small")
    for k in "abcyx":
        assert z[k].shape == (100, 115) and z[k].dtype == np.float32


def test_malformed_rejected():
    with pytest.raises(fd.FutharkDataError):
        fd.read_values("[1.0f32, 2.0f32")
    with pytest.raises(fd.FutharkDataError):
        fd.read_values(b"b\x02\x01 f32" + b"\x05\x00\x00\x00\x00\x00\x00\x00" + b"\x00" * 8)
