"""The test-stanza runner over the reference programs' own test blocks.

The ``-- ==`` blocks of finpar/LocVolCalib.fut, misc/ocean-sim/tridiag-test.fut,
misc/ocean-sim/tke.fut and finpar/OptionPricing.fut (tests/golden/stanzas.json)
name the reference's datasets (tests/golden/datasets, byte for byte).  The CPU
tests parse every block, check the comparison rule, and drive the runner with
the oracle; the GPU test runs every run of every block through this
repository's libraries: dataset runs against their expected outputs at the
runner's tolerance, random runs (seeded inputs of the stated types) against the
oracle, bit for bit where the kernels are bit-exact.
"""
import importlib
import json
import os
import re

import numpy as np
import pytest

from conftest import DATASETS, GOLDEN

st = importlib.import_module("futhark-benchmarks_b200.stanza")
wl = importlib.import_module("futhark-benchmarks_b200.workloads")

with open(os.path.join(GOLDEN, "stanzas.json")) as _f:
    STANZAS = json.load(_f)["stanzas"]


def runs_of(prog):
    return st.parse(STANZAS[prog])


def test_every_block_parses():
    counts = {p: len(runs_of(p)) for p in STANZAS}
    assert counts == {"finpar/LocVolCalib.fut": 3, "misc/ocean-sim/tridiag-test.fut": 2,
                      "misc/ocean-sim/tke.fut": 2, "finpar/OptionPricing.fut": 3}
    tri = runs_of("misc/ocean-sim/tridiag-test.fut")
    assert tri[0].entries == ["tridagNested", "tridagNestedConst", "tridagNestedSeq", "tridagNestedSeqConst"]
    assert tri[1].random_types == ["[57600][115]f32"] * 4 and "random" in tri[1].tags
    tke = runs_of("misc/ocean-sim/tke.fut")
    assert tke[0].name == "200x200x100" and len(tke[0].random_types) == 25
    assert tke[1].input_file == "data/tke32-small.in" and tke[1].output_file == "data/tke32-small.out"
    # every dataset a block names is a committed fixture
    for prog in STANZAS:
        for r in runs_of(prog):
            for rel in (r.input_file, r.output_file):
                if rel:
                    assert os.path.exists(os.path.join(DATASETS, os.path.dirname(prog), rel + ".gz")), rel


def test_parse_whole_program_text():
    # a program's code and its other comments around the block are skipped
    prog = "-- A program\n-- ==\n-- input { 1i32 }\n-- output { 2i32 }\n\n-- a comment\ndef main (x: i32) = x + 1\n"
    runs = st.parse(prog)
    assert len(runs) == 1 and runs[0].output_values.strip() == "2i32"


def test_parser_inline_values_and_errors():
    block = """-- ==
-- entry: f g
-- input { 1i32 [2.0f32, 3.0f32] }
-- output { [2.0f32] }
-- nobench input { 0i32 empty([0]f32) }
-- error: too small
"""
    runs = st.parse(block)
    assert [r.entries for r in runs] == [["f", "g"], ["f", "g"]]
    assert runs[0].output_values.strip() == "[2.0f32]"
    assert runs[1].tags == ["nobench"] and runs[1].error == "too small"
    with pytest.raises(st.StanzaError):
        st.parse("-- input { 1 }\n")  # no == marker
    with pytest.raises(st.StanzaError):
        st.parse("-- ==\n-- output { 1 }\n")


def test_compare_values_rule():
    e = [np.array([1.0, 2.0, 1e-8], dtype=np.float32)]
    assert st.compare_values([e[0] * np.float32(1.001)], e).ok
    assert not st.compare_values([e[0] * np.float32(1.01)], e).ok
    # an element near zero is held to the array's scale, not to its own magnitude
    near0 = [np.array([1.0, 2.0, 3e-8], dtype=np.float32)]
    c = st.compare_values(near0, e)
    assert c.ok and c.max_rel > 0.4
    assert not st.compare_values([np.array([1, 2], dtype=np.int32)], [np.array([1, 3], dtype=np.int32)]).ok
    assert not st.compare_values([np.array([np.nan])], [np.array([1.0])]).ok
    assert st.compare_values([np.array([np.nan])], [np.array([np.nan])]).ok
    assert not st.compare_values([np.zeros(2)], [np.zeros(3)]).ok


def test_oracle_through_the_runner(oracle):
    """The runner with the oracle as the entry points: LocVolCalib small,
    tridiagonal solvers, tke, OptionPricing small (a fast subset)."""
    res = st.run_stanzas(runs_of("finpar/LocVolCalib.fut")[:1], "finpar", DATASETS,
                         {"main": lambda *v: (oracle.main_f32(*[x.item() for x in v]),)})
    assert [r.status for r in res] == ["passed"] and res[0].comparison.max_abs <= 5e-6
    ents = {"tridagNestedSeq": lambda a, b, c, y: (oracle.tridag(a, b, c, y, form="seq"),),
            "tridagNestedSeqConst": lambda a, b, c, y: (oracle.tridag(a, b, c, y, form="seq"),),
            "tridagNested": lambda a, b, c, y: (oracle.tridag(a, b, c, y, form="par4"),),
            "tridagNestedConst": lambda a, b, c, y: (oracle.tridag(a, b, c, y, form="par4"),)}
    res = st.run_stanzas(runs_of("misc/ocean-sim/tridiag-test.fut")[:1], "misc/ocean-sim", DATASETS, ents)
    assert [r.status for r in res] == ["passed"] * 4
    seq = [r for r in res if r.entry == "tridagNestedSeq"][0]
    assert seq.comparison.max_abs == 0.0  # tridagSeq reproduces the golden file bit for bit
    res = st.run_stanzas(runs_of("misc/ocean-sim/tke.fut"), "misc/ocean-sim", DATASETS,
                         {"main": lambda *v: oracle.tke(*v)})
    assert [r.status for r in res] == ["skipped", "passed"] and res[1].comparison.max_abs == 0.0
    res = st.run_stanzas(runs_of("finpar/OptionPricing.fut")[:1], "finpar", DATASETS,
                         {"main": lambda *v: (oracle.option_pricing(*v),)})
    assert [r.status for r in res] == ["passed"]


@pytest.mark.gpu
def test_every_stanza_through_the_libraries(ctx, pkg, oracle):
    tke = importlib.import_module("futhark-benchmarks_b200.tke")
    op = importlib.import_module("futhark-benchmarks_b200.op")
    seen = {}

    def remember(key, fn):
        def call(*v):
            out = fn(*v)
            seen.setdefault(key, []).append((v, out))
            return out
        return call

    def random_inputs(run):
        if run.name == "200x200x100":
            return wl.tke_inputs(200, 200, 100, seed=3)
        rows, m = (int(d) for d in re.findall(r"\[(\d+)\]", run.random_types[0]))
        return wl.tridiag_inputs(rows, m, seed=3)

    results = []
    results += st.run_stanzas(runs_of("finpar/LocVolCalib.fut"), "finpar", DATASETS,
                              {"main": lambda *v: (ctx.main(*[x.item() for x in v]),)})
    ents = {name: remember(name, (lambda f, c: lambda a, b, cc, y: (ctx.tridag(a, b, cc, y, form=f, const=c),))(f, c))
            for name, f, c in (("tridagNested", "par", False), ("tridagNestedConst", "par", True),
                               ("tridagNestedSeq", "seq", False), ("tridagNestedSeqConst", "seq", True))}
    results += st.run_stanzas(runs_of("misc/ocean-sim/tridiag-test.fut"), "misc/ocean-sim", DATASETS, ents,
                              random_inputs)
    with tke.TkeContext() as tctx:
        results += st.run_stanzas(runs_of("misc/ocean-sim/tke.fut"), "misc/ocean-sim", DATASETS,
                                  {"main": remember("tke", tctx.main)}, random_inputs)
    with op.OpContext() as octx:
        results += st.run_stanzas(runs_of("finpar/OptionPricing.fut"), "finpar", DATASETS,
                                  {"main": lambda *v: (octx.main(*v),)})
    bad = [(r.run.label, r.entry, r.detail) for r in results if r.status not in ("passed", "ran")]
    assert not bad, bad
    assert len(results) == 3 + 4 * 2 + 2 + 3
    # dataset runs: the LocVolCalib f32 prices within 5e-6 of the golden files,
    # tke and tridagSeq bit for bit
    for r in results:
        if r.run.input_file and "LocVolCalib" in r.run.input_file:
            assert r.comparison.max_abs <= 5e-6
        if r.run.input_file and ("tke32" in r.run.input_file or r.entry.startswith("tridagNestedSeq")):
            assert r.comparison.max_abs == 0.0, r.run.label
    # random runs against the oracle, bit for bit
    (tv, tout), = [x for x in seen["tke"] if x[0][0].shape == (200, 200, 100)]
    want = oracle.tke(*tv)
    for k in (1, 3, 6):  # tketaup1, dtketau, tke_surf_corr: the step's results
        assert np.array_equal(tout[k].view(np.uint32), want[k].view(np.uint32)), k
    for name, form in (("tridagNested", "par4"), ("tridagNestedSeq", "seq")):
        (v, out), = [x for x in seen[name] if x[0][0].shape == (57600, 115)]
        sub = slice(0, 4096)
        assert np.array_equal(out[0][sub], oracle.tridag(*[a[sub] for a in v], form=form)), name


@pytest.mark.gpu
def test_run_dataset_reads_reference_files(ctx, pkg, golden):
    # run_dataset: a dataset file of finpar/LocVolCalib-data straight through main
    for name in ("small", "medium"):
        got = pkg.run_dataset(ctx, os.path.join(DATASETS, "finpar", "LocVolCalib-data", name + ".in.gz"))
        exp = np.asarray(golden[name]["expected_f32"], dtype=np.float64)
        assert got.dtype == np.float32 and np.max(np.abs(got - exp)) <= 5e-6
