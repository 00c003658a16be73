"""Regenerate the golden fixtures in this directory from a reference checkout.

The reference's own test data for the programs this repository builds are the
datasets named in the test stanzas (the ``-- ==`` comment blocks) of

  finpar/LocVolCalib.fut:1-10           LocVolCalib-data/{small,medium,large}.{in,out}
  misc/ocean-sim/tridiag-test.fut:6-12  data/tridiag32-small.{in,out}
  misc/ocean-sim/tke.fut:55-62          data/tke32-small.{in,out}
  finpar/OptionPricing.fut:1-10         OptionPricing-data/{small,medium,large}.{in,out}

This script copies them into self-contained fixtures, so that the tests run
where the reference tree is not present:

  datasets/<program dir>/<dataset path>.gz
                            every dataset file a stanza names, byte for byte,
                            gzip-compressed (futhark_data.read_file reads .gz)
  stanzas.json              the four programs' stanza blocks, verbatim, keyed
                            by the program's path in the reference tree
  locvolcalib_golden.json   LocVolCalib's inputs and expected f32 prices (with
                            the printed text of each, to know its precision)

Usage:  python tests/golden/make_golden.py REFERENCE_ROOT
        (or set FUTHARK_BENCHMARKS_ROOT and give no argument)
"""
import gzip
import importlib
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
fd = importlib.import_module("futhark-benchmarks_b200.futhark_data")
stanza = importlib.import_module("futhark-benchmarks_b200.stanza")

NAMES = ["outer", "numX", "numY", "numT", "s0", "t", "alpha", "nu", "beta"]
PROGRAMS = ["finpar/LocVolCalib.fut", "misc/ocean-sim/tridiag-test.fut", "misc/ocean-sim/tke.fut",
            "finpar/OptionPricing.fut"]


def main(ref_root: str) -> None:
    stanzas = {}
    for prog in PROGRAMS:
        with open(os.path.join(ref_root, prog)) as f:
            block = stanza.block_of(f.read())
        stanzas[prog] = block
        for run in stanza.parse(block):
            for rel in (run.input_file, run.output_file):
                if rel is None:
                    continue
                src = os.path.join(ref_root, os.path.dirname(prog), rel)
                dst = os.path.join(HERE, "datasets", os.path.dirname(prog), rel + ".gz")
                os.makedirs(os.path.dirname(dst), exist_ok=True)
                with open(src, "rb") as f:
                    raw = f.read()
                # mtime=0: the same bytes on every regeneration
                with open(dst, "wb") as f:
                    f.write(gzip.compress(raw, compresslevel=9, mtime=0))
    with open(os.path.join(HERE, "stanzas.json"), "w") as f:
        json.dump({"source": "the -- == blocks of these programs in the reference tree", "stanzas": stanzas},
                  f, indent=1)

    data_dir = os.path.join(ref_root, "finpar", "LocVolCalib-data")
    golden = {"source": "finpar/LocVolCalib-data/{small,medium,large}.{in,out}", "datasets": {}}
    for name in ("small", "medium", "large"):
        ins = fd.read_file(os.path.join(data_dir, f"{name}.in"))
        outs = fd.read_file(os.path.join(data_dir, f"{name}.out"))
        assert len(ins) == 9 and len(outs) == 1, (name, len(ins), len(outs))
        entry = {}
        for key, v in zip(NAMES, ins):
            entry[key] = int(v) if np.asarray(v).dtype.kind == "i" else float(np.float32(v))
        entry["expected_f32"] = [float(x) for x in np.asarray(outs[0], dtype=np.float32)]
        with open(os.path.join(data_dir, f"{name}.out")) as f:
            text = f.read()
        entry["expected_text"] = re.findall(r"[-+]?\d+\.\d+(?:e[-+]?\d+)?(?=f32)", text)
        assert len(entry["expected_text"]) == len(entry["expected_f32"]), name
        golden["datasets"][name] = entry
    with open(os.path.join(HERE, "locvolcalib_golden.json"), "w") as f:
        json.dump(golden, f, indent=1)
    print("wrote", sorted(os.listdir(HERE)))


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("FUTHARK_BENCHMARKS_ROOT")
    if not root:
        sys.exit("usage: make_golden.py REFERENCE_ROOT  (or set FUTHARK_BENCHMARKS_ROOT)")
    main(root)
