"""Test-stanza runner: the ``-- ==`` blocks of a Futhark program, run against
this repository's libraries.

A benchmark program of the reference declares its test and benchmark runs in a
comment block (finpar/LocVolCalib.fut:1-10, misc/ocean-sim/tridiag-test.fut:6-12,
misc/ocean-sim/tke.fut:55-62, finpar/OptionPricing.fut:1-10)::

    -- ==
    -- entry: tridagNested tridagNestedSeq            (optional; default: main)
    -- compiled input @ data/tridiag32-small.in       (input from a dataset file)
    -- output @ data/tridiag32-small.out              (expected output file)
    --
    -- "200x200x100" compiled random input { [200][200][100]f32 ... }

`parse` turns such a block into `Run` records (entries, tags, name, input
file / inline values / random type list, output file / inline values).
`run_stanzas` executes each run through a caller-supplied table of entry
points: dataset files are read with `futhark_data` (text or binary, gzipped
or not) relative to a dataset root, random inputs come from a caller-supplied
generator keyed by the run's type list, and outputs are compared with
`compare_values`.

Comparison rule (this runner's; the reference's `futhark test` tool is part of
the Futhark compiler, which the reference tree does not contain): integers and
booleans must be equal; floats of one output array must satisfy
``|got - expected| <= FLOAT_TOL * max(1, max|expected|)`` elementwise, i.e. a
relative tolerance of 0.002 scaled by the largest magnitude of the expected
array, so that elements close to zero in a well-scaled result are not held to a
relative bound they cannot carry after a change of summation order.  NaNs must
match NaNs.  Every comparison also reports the elementwise maximum relative
and absolute errors, so a caller can assert a tighter bound.
"""
from __future__ import annotations

import os
import re
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional, Sequence

import numpy as np

from . import futhark_data

FLOAT_TOL = 0.002
RUN_TAGS = ("compiled", "nobench", "notest", "random", "script", "interpreted")


class StanzaError(ValueError):
    """A malformed test block."""


@dataclass
class Run:
    entries: List[str]
    tags: List[str] = field(default_factory=list)
    name: Optional[str] = None
    input_file: Optional[str] = None      # path relative to the program's directory
    input_values: Optional[str] = None    # inline value text
    random_types: Optional[List[str]] = None  # e.g. ["[57600][115]f32", ...]
    output_file: Optional[str] = None
    output_values: Optional[str] = None
    error: Optional[str] = None

    @property
    def label(self) -> str:
        src = self.name or self.input_file or ("random " + " ".join(self.random_types or []))
        return f"{'/'.join(self.entries)}: {src}"


def _strip(block: str) -> str:
    lines = []
    for ln in block.splitlines():
        s = ln.strip()
        if not s.startswith("--"):
            continue
        lines.append(s[2:])
    return "\n".join(lines)


def _braced(text: str, pos: int):
    """The text between the brace at `pos` and its match; returns (inner, end)."""
    if text[pos] != "{":
        raise StanzaError(f"expected '{{' at {text[pos:pos + 20]!r}")
    depth, i = 0, pos
    while i < len(text):
        if text[i] == "{":
            depth += 1
        elif text[i] == "}":
            depth -= 1
            if depth == 0:
                return text[pos + 1:i], i + 1
        i += 1
    raise StanzaError("unterminated '{'")


_WORD = re.compile(r"\s*(\"[^\"]*\"|[A-Za-z_][\w]*:?|@|\{|==)")


def block_of(program: str) -> str:
    """The test block of a whole program text: its ``-- ==`` line and the rest
    of that comment block."""
    lines = program.splitlines()
    for start, ln in enumerate(lines):
        if ln.strip() == "-- ==":
            break
    else:
        raise StanzaError("no '-- ==' line")
    end = start
    while end < len(lines) and lines[end].lstrip().startswith("--"):
        end += 1
    return "\n".join(lines[start:end]) + "\n"


def parse(block: str) -> List[Run]:
    """Parse a program's test block; given a whole program text, its block."""
    if any(ln.strip() and not ln.lstrip().startswith("--") for ln in block.splitlines()):
        block = block_of(block)
    text = _strip(block)
    pos = 0
    entries = ["main"]
    runs: List[Run] = []
    pending_tags: List[str] = []
    pending_name: Optional[str] = None
    seen_marker = False
    while True:
        m = _WORD.match(text, pos)
        if not m:
            rest = text[pos:].strip()
            if rest:
                raise StanzaError(f"cannot parse {rest[:40]!r}")
            break
        tok = m.group(1)
        pos = m.end()
        if tok == "==":
            seen_marker = True
        elif tok == "entry:":
            eol = text.find("\n", pos)
            eol = len(text) if eol < 0 else eol
            entries = text[pos:eol].split()
            if not entries:
                raise StanzaError("entry: without names")
            pos = eol
        elif tok == "tags":
            _, pos = _braced(text, text.index("{", pos))
        elif tok in RUN_TAGS:
            pending_tags.append(tok)
        elif tok.startswith('"'):
            pending_name = tok.strip('"')
        elif tok == "input":
            run = Run(entries=list(entries), tags=pending_tags, name=pending_name)
            pending_tags, pending_name = [], None
            m2 = re.compile(r"\s*(@|\{)").match(text, pos)
            if not m2:
                raise StanzaError("input without '@ file' or '{ values }'")
            if m2.group(1) == "@":
                m3 = re.compile(r"\s*(\S+)").match(text, m2.end())
                run.input_file = m3.group(1)
                pos = m3.end()
            else:
                inner, pos = _braced(text, m2.end() - 1)
                if "random" in run.tags:
                    run.random_types = inner.split()
                else:
                    run.input_values = inner
            runs.append(run)
        elif tok == "output":
            if not runs:
                raise StanzaError("output before any input")
            m2 = re.compile(r"\s*(@|\{)").match(text, pos)
            if not m2:
                raise StanzaError("output without '@ file' or '{ values }'")
            if m2.group(1) == "@":
                m3 = re.compile(r"\s*(\S+)").match(text, m2.end())
                runs[-1].output_file = m3.group(1)
                pos = m3.end()
            else:
                runs[-1].output_values, pos = _braced(text, m2.end() - 1)
        elif tok == "error:":
            eol = text.find("\n", pos)
            eol = len(text) if eol < 0 else eol
            if not runs:
                raise StanzaError("error: before any input")
            runs[-1].error = text[pos:eol].strip()
            pos = eol
        else:
            raise StanzaError(f"unexpected word {tok!r}")
    if not seen_marker:
        raise StanzaError("no '==' marker")
    return runs


@dataclass
class Comparison:
    ok: bool
    max_rel: float
    max_abs: float
    detail: str = ""


def compare_values(got: Sequence, expected: Sequence, tol: float = FLOAT_TOL) -> Comparison:
    """Compare the outputs of one run with the expected values (rule in the
    module docstring)."""
    if len(got) != len(expected):
        return Comparison(False, np.inf, np.inf, f"{len(got)} outputs, expected {len(expected)}")
    max_rel = max_abs = 0.0
    for k, (g, e) in enumerate(zip(got, expected)):
        g = np.asarray(g)
        e = np.asarray(e)
        if g.shape != e.shape:
            return Comparison(False, np.inf, np.inf, f"output {k}: shape {g.shape}, expected {e.shape}")
        if e.dtype.kind != "f":
            if not np.array_equal(g, e):
                return Comparison(False, np.inf, np.inf, f"output {k}: values differ")
            continue
        g64 = g.astype(np.float64)
        e64 = e.astype(np.float64)
        nan_g, nan_e = np.isnan(g64), np.isnan(e64)
        if not np.array_equal(nan_g, nan_e):
            return Comparison(False, np.inf, np.inf, f"output {k}: NaNs differ")
        fin = ~nan_e
        d = np.abs(g64[fin] - e64[fin])
        if d.size:
            scale = max(1.0, float(np.max(np.abs(e64[fin]))))
            rel = d / np.maximum(np.abs(e64[fin]), 1e-300)
            max_rel = max(max_rel, float(np.max(rel)))
            max_abs = max(max_abs, float(np.max(d)))
            if float(np.max(d)) > tol * scale:
                i = int(np.argmax(d))
                return Comparison(False, max_rel, max_abs,
                                  f"output {k}: |diff| {float(d[i]):.3e} > {tol} x {scale:.3e}")
    return Comparison(True, max_rel, max_abs)


@dataclass
class RunResult:
    run: Run
    entry: str
    status: str              # "passed", "failed", "ran" (no expected output), "skipped"
    comparison: Optional[Comparison] = None
    detail: str = ""


def run_stanzas(runs: Sequence[Run], program_dir: str, dataset_root: str,
                entries: Dict[str, Callable[..., Sequence]],
                random_inputs: Optional[Callable[[Run], Sequence]] = None,
                tol: float = FLOAT_TOL) -> List[RunResult]:
    """Execute every run of a program's test block.

    program_dir   the program's directory in the reference tree (for example
                  "finpar"); dataset paths of the block are relative to it
    dataset_root  where the dataset files live; a file named NAME is read from
                  dataset_root/program_dir/NAME, or NAME.gz if only that exists
    entries       entry name -> callable taking the input values and returning
                  the tuple of outputs
    random_inputs callable producing the input values of a random run (given
                  the run); None skips random runs
    """
    def path_of(rel):
        p = os.path.join(dataset_root, program_dir, rel)
        return p if os.path.exists(p) else p + ".gz"

    results = []
    for run in runs:
        for entry in run.entries:
            fn = entries.get(entry)
            if fn is None:
                results.append(RunResult(run, entry, "skipped", detail="no such entry point"))
                continue
            if run.input_file is not None:
                ins = futhark_data.read_file(path_of(run.input_file))
            elif run.input_values is not None:
                ins = futhark_data.read_values(run.input_values)
            elif run.random_types is not None:
                if random_inputs is None:
                    results.append(RunResult(run, entry, "skipped", detail="random input"))
                    continue
                ins = random_inputs(run)
            else:
                raise StanzaError(f"{run.label}: no input")
            if run.error is not None:
                try:
                    fn(*ins)
                except Exception as ex:  # the run is expected to fail
                    ok = re.search(run.error, str(ex)) is not None
                    results.append(RunResult(run, entry, "passed" if ok else "failed", detail=str(ex)))
                    continue
                results.append(RunResult(run, entry, "failed", detail="expected an error"))
                continue
            outs = fn(*ins)
            if run.output_file is not None:
                want = futhark_data.read_file(path_of(run.output_file))
            elif run.output_values is not None:
                want = futhark_data.read_values(run.output_values)
            else:
                results.append(RunResult(run, entry, "ran"))
                continue
            cmp = compare_values(outs, want, tol)
            results.append(RunResult(run, entry, "passed" if cmp.ok else "failed", cmp, cmp.detail))
    return results
