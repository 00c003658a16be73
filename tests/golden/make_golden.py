"""Regenerate the golden fixtures in this directory from the reference checkout.

The reference's own test data for the LocVolCalib path are the three dataset
pairs named in the test stanza of finpar/LocVolCalib.fut:1-10, and its
tridiagonal-solver fixture is misc/ocean-sim/data/tridiag32-small.{in,out}
(misc/ocean-sim/tridiag-test.fut:6-12).  This script copies their values into
self-contained fixtures so the tests can run where the reference tree is not
present:

  locvolcalib_golden.json   inputs + expected f32 prices for small/medium/large
  tridiag32_small.npz       a, b, c, y [100][115] f32 and the expected x
  tke32_small.npz           misc/ocean-sim/data/tke32-small.{in,out}: in00..in24
                            (the 25 inputs of tke.fut's main) and out0..out6
  optionpricing_{small,medium,large}.npz
                            finpar/OptionPricing-data/*.{in,out} (the test stanza of
                            finpar/OptionPricing.fut:1-11): in00..in10 (the 11 inputs
                            of main) and out0

Usage:  python tests/golden/make_golden.py [REFERENCE_ROOT]
(REFERENCE_ROOT defaults to /root/reference.)
"""
import importlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
fd = importlib.import_module("futhark-benchmarks_b200.futhark_data")

NAMES = ["outer", "numX", "numY", "numT", "s0", "t", "alpha", "nu", "beta"]


def main(ref_root: str) -> None:
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
        # the text of each printed value, to know its printed precision
        with open(os.path.join(data_dir, f"{name}.out")) as f:
            text = f.read()
        import re
        entry["expected_text"] = re.findall(r"[-+]?\d+\.\d+(?:e[-+]?\d+)?(?=f32)", text)
        assert len(entry["expected_text"]) == len(entry["expected_f32"]), name
        golden["datasets"][name] = entry
    with open(os.path.join(HERE, "locvolcalib_golden.json"), "w") as f:
        json.dump(golden, f, indent=1)

    tdir = os.path.join(ref_root, "misc", "ocean-sim", "data")
    a, b, c, y = fd.read_file(os.path.join(tdir, "tridiag32-small.in"))
    (x,) = fd.read_file(os.path.join(tdir, "tridiag32-small.out"))
    np.savez_compressed(os.path.join(HERE, "tridiag32_small.npz"), a=a, b=b, c=c, y=y, x=x)

    # misc/ocean-sim/tke.fut's test stanza: 25 inputs, 7 outputs ([20][20][10])
    ins = fd.read_file(os.path.join(tdir, "tke32-small.in"))
    outs = fd.read_file(os.path.join(tdir, "tke32-small.out"))
    np.savez_compressed(os.path.join(HERE, "tke32_small.npz"),
                        **{f"in{i:02d}": v for i, v in enumerate(ins)},
                        **{f"out{i}": v for i, v in enumerate(outs)})
    # finpar/OptionPricing.fut's test stanza: 11 inputs, 1 output
    odir = os.path.join(ref_root, "finpar", "OptionPricing-data")
    for name in ("small", "medium", "large"):
        ins = fd.read_file(os.path.join(odir, f"{name}.in"))
        outs = fd.read_file(os.path.join(odir, f"{name}.out"))
        np.savez_compressed(os.path.join(HERE, f"optionpricing_{name}.npz"),
                            **{f"in{i:02d}": np.asarray(v) for i, v in enumerate(ins)},
                            **{f"out{i}": np.asarray(v) for i, v in enumerate(outs)})
    print("wrote", os.listdir(HERE))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
