"""Regenerate the golden fixtures in this directory from the reference tree.

Copies (verbatim) the reference's regression goldens `regress/*.ok` and
`regress/MPI/*.ok` -- the ∞-norm errors `compare -n` printed after `dns -chk`
(test/testregress:14-30) -- into regress_ok.json, and copies the session
files those tests and the elliptic suite run (mesh/<name>) into sessions/.

Usage:  python tests/golden/make_golden.py /path/to/reference
"""

from __future__ import annotations

import glob
import json
import os
import re
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SESSIONS = ["taylor2", "taylor3", "taylor4", "taylor5", "kovas1", "kovas2", "kovas3", "kovas4", "kovas5",
            "helmholtz1", "laplace1",
            "laplace3", "laplace4", "poisson1", "tgreen", "mixed1", "tgreen100", "sbr", "tc1", "tube1", "tube2", "tube3", "cylkov2", "laplace8", "laplace9"]


def main(ref):
    out = {}
    for sub in ("", "MPI"):
        for f in sorted(glob.glob(os.path.join(ref, "regress", sub, "*.ok"))):
            name = ("MPI/" if sub else "") + os.path.basename(f)[:-3]
            vals = {}
            for ln in open(f):
                m = re.match(r"Field '(\w)': norm_inf: (\S+)", ln.strip())
                if m:
                    vals[m.group(1)] = m.group(2)
            out[name] = vals
    with open(os.path.join(HERE, "regress_ok.json"), "w") as fp:
        json.dump({"source": "reference regress/*.ok (utility/compare.cpp:226-232 format)",
                   "goldens": out}, fp, indent=1, sort_keys=True)
    os.makedirs(os.path.join(HERE, "sessions"), exist_ok=True)
    for s in SESSIONS:
        shutil.copy(os.path.join(ref, "mesh", s), os.path.join(HERE, "sessions", s))
    print(f"{len(out)} goldens, {len(SESSIONS)} sessions written")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py /path/to/reference")
    main(sys.argv[1])
