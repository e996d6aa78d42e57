"""Make tests/golden/globind_n30_p3.json from the reference's GlobInd fixture.

The reference ships TestKernels/GlobInd (identical to TestAMD/GlobInd): the
Glob map of the cubed sphere at nPanel=30, OrdPoly=3 as raw little-endian
Int64, shape (16, 5400), column-major, 1-based.  This script records its
SHA-256, shape, extrema and a few full columns, so the tests can pin the grid
chain bit-exactly without the 691 KB file (and without the reference tree).

    python tests/golden/make_globind_digest.py [path/to/CGDycore.jl]

The checkout is the argument, else the CGD_REFERENCE_DIR environment
variable.
"""
import hashlib
import json
import os
import sys

import numpy as np

ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CGD_REFERENCE_DIR", "")
if not ref:
    sys.exit("usage: make_globind_digest.py path/to/CGDycore.jl (or set CGD_REFERENCE_DIR)")
raw = open(os.path.join(ref, "TestKernels", "GlobInd"), "rb").read()
g = np.frombuffer(raw, dtype="<i8").reshape((16, 5400), order="F")
cols = [0, 1, 29, 30, 899, 900, 1799, 2700, 3599, 4500, 5399]
out = {
    "source": "TestKernels/GlobInd (CGDycore.jl), nPanel=30, OrdPoly=3",
    "dtype": "int64 little-endian, column-major (16, 5400), 1-based",
    "sha256": hashlib.sha256(raw).hexdigest(),
    "shape": [16, 5400],
    "min": int(g.min()), "max": int(g.max()), "n_unique": int(np.unique(g).size),
    "columns": {str(c): [int(x) for x in g[:, c]] for c in cols},
}
here = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(here, "globind_n30_p3.json"), "w") as f:
    json.dump(out, f, indent=1)
print(out["sha256"])
