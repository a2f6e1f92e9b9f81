"""Copies small input files of the reference's toy examples into
tests/golden/reference_files/ and records the structure of two binary
files (a model file and a SAC trace) in reference_files/summary.json, for
the file-format tests.  Usage: python make_reference_fixtures.py
<SpecFWAT source tree> (or SPECFWAT_REFERENCE_ROOT set); the tests use only
what this writes."""
import json
import os
import shutil
import struct
import sys

import numpy as np

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SPECFWAT_REFERENCE_ROOT", "")
if not REF or not os.path.isdir(REF):
    sys.exit("usage: make_reference_fixtures.py <SpecFWAT source tree>")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_files")
os.makedirs(OUT, exist_ok=True)

shutil.copy(os.path.join(REF, "tests/toy_example_HTI/DATA/CMTSOLUTION"),
            os.path.join(OUT, "CMTSOLUTION"))
with open(os.path.join(REF, "tests/toy_example_HTI/DATA/STATIONS")) as f:
    lines = f.readlines()[:5]
with open(os.path.join(OUT, "STATIONS"), "w") as f:
    f.writelines(lines)

summary = {}
p = os.path.join(REF, "tests/toy_example_rf/model_target/proc000000_vs.bin")
raw = open(p, "rb").read()
n = struct.unpack("<i", raw[:4])[0]
a = np.frombuffer(raw[4:4 + n], "<f4")
summary["model_bin"] = {"file": "tests/toy_example_rf/model_target/proc000000_vs.bin",
                        "bytes": len(raw), "record_bytes": n,
                        "nspec": n // 500, "first": [float(v) for v in a[:5]],
                        "min": float(a.min()), "max": float(a.max()),
                        "sum": float(a.astype(np.float64).sum())}
p = os.path.join(REF, "tests/toy_example_tele/src_rec/STF_0.sac")
raw = open(p, "rb").read()
fl = np.frombuffer(raw[:280], "<f4")
it = np.frombuffer(raw[280:440], "<i4")
d = np.frombuffer(raw[632:], "<f4")
summary["sac"] = {"file": "tests/toy_example_tele/src_rec/STF_0.sac", "bytes": len(raw),
                  "delta": float(fl[0]), "b": float(fl[5]), "npts": int(it[9]),
                  "nvhdr": int(it[6]), "first": [float(v) for v in d[:5]],
                  "sum": float(d.astype(np.float64).sum())}
with open(os.path.join(OUT, "summary.json"), "w") as f:
    json.dump(summary, f, indent=1)
print(json.dumps(summary, indent=1))
