"""Reader and writer for Futhark's value files (`.in` / `.out` datasets).

Futhark benchmark datasets come in two encodings, both accepted by the
reference's `futhark test` / `futhark bench` harness (finpar/LocVolCalib.fut:1-10
points at text files; misc/ocean-sim/tridiag-test.fut:9-10 at binary ones):

* text: whitespace-separated values with `--` line comments, scalars carrying a
  type suffix (``0.03f32``, ``16``, ``5i64``), arrays in brackets
  (``[1.0f32, 2.0f32]``), ``true``/``false`` and ``empty([0]f32)``;
* binary: per value ``b'b'``, version byte 2, rank byte, a 4-byte type name
  (``" f32"``, ``" i32"``, ``"bool"`` ...), ``rank`` little-endian int64 shape
  entries, then the little-endian elements.

`read_values` sniffs the encoding per value, so a file may mix them.  Scalars
come back as numpy scalars (an un-suffixed integer literal is i32, an
un-suffixed decimal literal f64, as in Futhark), arrays as numpy arrays.
"""
from __future__ import annotations

import re
import struct
from typing import Iterable, List

import numpy as np

_BIN_TYPES = {
    b"  i8": np.int8, b" i16": np.int16, b" i32": np.int32, b" i64": np.int64,
    b"  u8": np.uint8, b" u16": np.uint16, b" u32": np.uint32, b" u64": np.uint64,
    b" f16": np.float16, b" f32": np.float32, b" f64": np.float64, b"bool": np.bool_,
}
_SUFFIX_TYPES = {
    "i8": np.int8, "i16": np.int16, "i32": np.int32, "i64": np.int64,
    "u8": np.uint8, "u16": np.uint16, "u32": np.uint32, "u64": np.uint64,
    "f16": np.float16, "f32": np.float32, "f64": np.float64,
}
_TYPE_NAMES = {np.dtype(v): k for k, v in _BIN_TYPES.items()}

_TOKEN = re.compile(
    r"""\s*(?:
        (?P<comment>--[^\n]*) |
        (?P<open>\[) | (?P<close>\]) | (?P<comma>,) |
        (?P<empty>empty\s*\(\s*(?P<edims>(?:\[\d+\])+)\s*(?P<etype>[a-z]+\d*)\s*\)) |
        (?P<bool>true|false) |
        (?P<num>[-+]?(?:inf|nan|(?:\d[\d_]*(?:\.\d[\d_]*)?(?:[eE][-+]?\d+)?))
                (?:(?P<suffix>[iuf]\d+))?)
    )""",
    re.VERBOSE,
)


class FutharkDataError(ValueError):
    """Raised for malformed value files."""


def _parse_number(text: str, suffix: str | None):
    body = text[: len(text) - len(suffix)] if suffix else text
    body = body.replace("_", "")
    if suffix:
        dt = _SUFFIX_TYPES.get(suffix)
        if dt is None:
            raise FutharkDataError(f"unknown type suffix {suffix!r}")
        if np.dtype(dt).kind == "f":
            return dt(float(body))
        return dt(int(body))
    if any(ch in body for ch in ".eE") or body.lstrip("+-") in ("inf", "nan"):
        return np.float64(float(body))
    return np.int32(int(body))


class _TextParser:
    def __init__(self, text: str):
        self.text = text
        self.pos = 0

    def _next(self):
        while True:
            if self.pos >= len(self.text) or not self.text[self.pos:].strip():
                self.pos = len(self.text)
                return None
            m = _TOKEN.match(self.text, self.pos)
            if not m or m.end() == self.pos:
                raise FutharkDataError(f"cannot parse near {self.text[self.pos:self.pos + 30]!r}")
            self.pos = m.end()
            if m.group("comment") is None:
                return m

    def _peek(self):
        save = self.pos
        tok = self._next()
        self.pos = save
        return tok

    def value(self):
        tok = self._next()
        if tok is None:
            return None
        return self._value_from(tok)

    def _value_from(self, tok):
        if tok.group("num") is not None:
            return _parse_number(tok.group("num"), tok.group("suffix"))
        if tok.group("bool") is not None:
            return np.bool_(tok.group("bool") == "true")
        if tok.group("empty") is not None:
            dims = [int(d) for d in re.findall(r"\[(\d+)\]", tok.group("edims"))]
            dt = _SUFFIX_TYPES.get(tok.group("etype"), np.bool_ if tok.group("etype") == "bool" else None)
            if dt is None:
                raise FutharkDataError(f"unknown element type {tok.group('etype')!r}")
            return np.zeros(dims, dtype=dt)
        if tok.group("open") is not None:
            elems = []
            while True:
                nxt = self._next()
                if nxt is None:
                    raise FutharkDataError("unterminated array")
                if nxt.group("close") is not None:
                    break
                if nxt.group("comma") is not None:
                    continue
                elems.append(self._value_from(nxt))
            if not elems:
                raise FutharkDataError("use empty(...) for empty arrays")
            kinds = {np.asarray(e).dtype for e in elems}
            if len(kinds) > 1:
                # un-suffixed literals adopt the suffixed element type
                typed = [k for k in kinds if k not in (np.dtype(np.int32), np.dtype(np.float64))]
                target = typed[0] if typed else np.result_type(*kinds)
                elems = [np.asarray(e).astype(target) for e in elems]
            return np.stack([np.asarray(e) for e in elems])
        raise FutharkDataError(f"unexpected token {tok.group(0)!r}")


def _read_binary(buf: bytes, pos: int):
    if len(buf) < pos + 7 or buf[pos:pos + 1] != b"b":
        raise FutharkDataError("not a binary value")
    version, rank = buf[pos + 1], buf[pos + 2]
    if version != 2:
        raise FutharkDataError(f"unsupported binary version {version}")
    tname = buf[pos + 3:pos + 7]
    dt = _BIN_TYPES.get(tname)
    if dt is None:
        raise FutharkDataError(f"unknown binary type {tname!r}")
    pos += 7
    shape = struct.unpack_from("<" + "q" * rank, buf, pos) if rank else ()
    pos += 8 * rank
    count = int(np.prod(shape)) if rank else 1
    itemsize = np.dtype(dt).itemsize
    end = pos + count * itemsize
    if end > len(buf):
        raise FutharkDataError("truncated binary value")
    arr = np.frombuffer(buf, dtype=np.dtype(dt).newbyteorder("<"), count=count, offset=pos)
    arr = arr.astype(dt)
    value = arr.reshape(shape) if rank else arr[0]
    return value, end


def read_values(data: bytes | str) -> List[np.ndarray]:
    """Parse every value in a Futhark value file (text, binary, or mixed)."""
    if isinstance(data, str):
        data = data.encode()
    out = []
    pos = 0
    n = len(data)
    while pos < n:
        while pos < n and data[pos:pos + 1].isspace():
            pos += 1
        if pos >= n:
            break
        if data[pos:pos + 1] == b"b" and pos + 1 < n and data[pos + 1] == 2:
            v, pos = _read_binary(data, pos)
            out.append(v)
            continue
        # a text value runs until the next binary marker (or the end)
        nxt = data.find(b"b\x02", pos)
        chunk_end = n if nxt < 0 else nxt
        parser = _TextParser(data[pos:chunk_end].decode("utf-8"))
        while True:
            v = parser.value()
            if v is None:
                break
            out.append(v)
        pos = chunk_end
    return out


def read_file(path: str) -> List[np.ndarray]:
    """Values of a dataset file; a name ending in ``.gz`` is gunzipped first."""
    if path.endswith(".gz"):
        import gzip
        with gzip.open(path, "rb") as f:
            return read_values(f.read())
    with open(path, "rb") as f:
        return read_values(f.read())


def write_binary(values: Iterable) -> bytes:
    """Encode values in Futhark's binary format (version 2)."""
    parts = []
    for v in values:
        a = np.asarray(v)
        name = _TYPE_NAMES.get(a.dtype)
        if name is None:
            raise FutharkDataError(f"no Futhark binary type for {a.dtype}")
        parts.append(b"b" + bytes([2, a.ndim]) + name)
        parts.append(struct.pack("<" + "q" * a.ndim, *a.shape))
        parts.append(np.ascontiguousarray(a, dtype=a.dtype.newbyteorder("<")).tobytes())
    return b"".join(parts)


def _fmt_scalar(x) -> str:
    a = np.asarray(x)
    if a.dtype == np.bool_:
        return "true" if bool(a) else "false"
    suffix = {v: k for k, v in _SUFFIX_TYPES.items()}[a.dtype.type]
    if a.dtype.kind == "f":
        return f"{float(a)!r}{suffix}"
    return f"{int(a)}{suffix}"


def write_text(values: Iterable) -> str:
    """Encode values in Futhark's text format."""
    def enc(a):
        a = np.asarray(a)
        if a.ndim == 0:
            return _fmt_scalar(a)
        if a.size == 0:
            suffix = "bool" if a.dtype == np.bool_ else {v: k for k, v in _SUFFIX_TYPES.items()}[a.dtype.type]
            return "empty(" + "".join(f"[{d}]" for d in a.shape) + suffix + ")"
        return "[" + ", ".join(enc(e) for e in a) + "]"
    return "\n".join(enc(v) for v in values) + "\n"
