"""Pin the grid chain: the oracle's and the product's Glob at nPanel=30, p=3
against the reference's GlobInd fixture (tests/golden/globind_n30_p3.json,
made by tests/golden/make_globind_digest.py), plus structural invariants."""
import hashlib
import json
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "globind_n30_p3.json")))
# the reference checkout, when present (CGD_REFERENCE_DIR); the digest above
# stands in for it everywhere else
REF_DIR = os.environ.get("CGD_REFERENCE_DIR", "")
REF_FILE = os.path.join(REF_DIR, "TestKernels", "GlobInd") if REF_DIR else ""


def _check_against_digest(glob):
    assert list(glob.shape) == GOLD["shape"]
    raw = np.ascontiguousarray(glob.T).astype("<i8").tobytes()   # column-major bytes
    assert hashlib.sha256(raw).hexdigest() == GOLD["sha256"]
    for c, col in GOLD["columns"].items():
        assert list(glob[:, int(c)]) == col


def test_oracle_glob_matches_globind(oracle_mod):
    o = oracle_mod.Oracle(30, 3, 2, 0, np.array([0.0, 15000.0, 30000.0]))
    g = o.glob()
    assert o.NumG == GOLD["max"] == 6 * 30 * 30 * 9 + 2
    _check_against_digest(g)


def test_product_glob_matches_globind():
    from cgd_b200 import grid as G
    FN, FE, EN, FP, nn, ne = G.build_topology(30, 6.371e6)
    glob, numg = G.numbering_cg_quad(FN, FE, EN, nn, ne, 3)
    assert numg == GOLD["max"]
    _check_against_digest(glob)


@pytest.mark.skipif(not os.path.exists(REF_FILE), reason="reference tree not present")
def test_digest_matches_reference_file():
    raw = open(REF_FILE, "rb").read()
    assert hashlib.sha256(raw).hexdigest() == GOLD["sha256"]


@pytest.mark.parametrize("n,p", [(2, 4), (6, 4), (5, 2), (4, 1), (7, 3)])
def test_glob_structure(oracle_mod, n, p):
    """NumG = 6 n^2 p^2 + 2; corner ids shared by 3 or 4 elements, edge ids by
    2, interior ids by 1; product and oracle agree bit-exactly."""
    from cgd_b200 import grid as G
    o = oracle_mod.Oracle(n, p, 2, 0, np.array([0.0, 1.0, 2.0]), H=2.0)
    g = o.glob()
    assert o.NumG == 6 * n * n * p * p + 2
    counts = np.bincount(g.ravel(), minlength=o.NumG + 1)[1:]
    assert counts.min() >= 1
    N = p + 1
    loc = np.zeros((N, N), int)
    loc[[0, 0, -1, -1], [0, -1, 0, -1]] = 1            # corners
    for ID in range(N * N):
        I, J = ID % N, ID // N
        c = counts[g[ID] - 1]
        if (I in (0, p)) and (J in (0, p)):
            assert set(np.unique(c)) <= {3, 4}
        elif I in (0, p) or J in (0, p):
            assert np.all(c == 2)
        else:
            assert np.all(c == 1)
    FN, FE, EN, FP, nn, ne = G.build_topology(n, 6.371e6)
    glob, numg = G.numbering_cg_quad(FN, FE, EN, nn, ne, p)
    assert numg == o.NumG
    assert np.array_equal(glob, g)


def test_product_grid_matches_oracle(oracle_mod):
    """Product host grid (metric, mass, dz, D matrices) vs the oracle."""
    from cgd_b200 import grid as G
    nz = 10
    z = G.vertical_uniform(nz, 30000.0)
    g = G.init_grid_sphere(6, 4, z, 30000.0, 6.371e6)
    o = oracle_mod.Oracle(6, 4, nz, 0, z)
    assert np.array_equal(g.glob, o.glob())
    xw, w, DS, DW = o.gll()
    assert np.array_equal(g.DS, DS) and np.array_equal(g.DW, DW)
    assert np.array_equal(np.transpose(o.faces(), (2, 0, 1)), g.faces)
    X, dX, J = o.metric()
    assert np.array_equal(g.X, X)
    # sin/cos/asin/atan2 of numpy and of the C library differ by ulps
    assert np.abs(g.dXdxI - dX).max() <= 1e-14 * np.abs(dX).max()
    assert np.abs(g.J - J).max() <= 1e-14 * np.abs(J).max()
    M, MM = o.mass()
    assert np.abs(g.M - M).max() <= 1e-14 * np.abs(M).max()
    assert np.abs(g.MMass - MM).max() <= 1e-14 * np.abs(MM).max()
    assert np.array_equal(g.dz, o.dz())
