"""Every reference citation of the form `src/.../File.jl:L` or `:L0-L1` in
the library, the host package and the oracle names a file of the CGDycore.jl
checkout whose length covers the cited lines.  Runs only where a checkout is
given (CGD_REFERENCE_DIR); skipped otherwise.
"""
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_DIR = os.environ.get("CGD_REFERENCE_DIR", "")
SOURCES = (glob.glob(os.path.join(ROOT, "include", "*.h")) +
           glob.glob(os.path.join(ROOT, "cgdycore.jl_b200", "csrc", "*")) +
           glob.glob(os.path.join(ROOT, "cgdycore.jl_b200", "cgd_b200", "*.py")) +
           glob.glob(os.path.join(ROOT, "cgdycore.jl_b200", "julia", "*.jl")) +
           glob.glob(os.path.join(ROOT, "oracle", "*.cpp")) + glob.glob(os.path.join(ROOT, "oracle", "*.py")))
CITE = re.compile(r"\b((?:src|TestKernels|Examples|Jobs)/[A-Za-z0-9_/]+\.jl)(?::([0-9]+)(?:-([0-9]+))?)?")


def _citations():
    out = []
    for f in sorted(SOURCES):
        for m in CITE.finditer(open(f, errors="ignore").read()):
            out.append((os.path.relpath(f, ROOT), m.group(1), int(m.group(3) or m.group(2) or 0)))
    return out


def test_sources_cite_the_reference():
    assert len(_citations()) >= 100


@pytest.mark.skipif(not REF_DIR or not os.path.isdir(REF_DIR), reason="no CGDycore.jl checkout (CGD_REFERENCE_DIR)")
def test_citations_point_into_the_reference():
    bad = []
    nlines = {}
    for src, path, last in _citations():
        p = os.path.join(REF_DIR, path)
        if not os.path.isfile(p):
            bad.append(f"{src}: {path} does not exist")
            continue
        if path not in nlines:
            with open(p, errors="ignore") as fh:
                nlines[path] = sum(1 for _ in fh)
        if last > nlines[path]:
            bad.append(f"{src}: {path}:{last} beyond its {nlines[path]} lines")
    assert bad == []
