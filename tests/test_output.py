"""Output interpolation, host side (no GPU): the sub-cell weights of the
library (cgd_vtk_inter) against the oracle's restatement of vtkStruct, the
cell corner points against pure-Python loops over TransSphereX!, and the VTK
file round trip."""
import numpy as np
import pytest


@pytest.mark.parametrize("p", [1, 2, 3, 4])
@pytest.mark.parametrize("OP", [1, 2, 3, 8])
def test_vtk_inter_matches_oracle(oracle_mod, built_lib, p, OP):
    from cgd_b200 import grid as G
    from cgd_b200 import output
    xw = G.gauss_lobatto(p)[0]
    a = output.vtk_inter(p, OP, xw)
    b = oracle_mod.vtk_inter(p, OP, xw)
    assert a.shape == (OP, OP, p + 1, p + 1)
    assert np.array_equal(a, b)
    # every cell value is a convex-like combination: the weights sum to one
    assert np.allclose(a.sum(axis=(2, 3)), 1.0, rtol=0, atol=1e-13)


def test_vtk_inter_centre_node(built_lib):
    """OrdPrint 1 at p = 4 samples the element centre, a GLL node."""
    from cgd_b200 import grid as G
    from cgd_b200 import output
    a = output.vtk_inter(4, 1, G.gauss_lobatto(4)[0])
    e = np.zeros((1, 1, 5, 5))
    e[0, 0, 2, 2] = 1.0
    assert np.allclose(a, e, rtol=0, atol=1e-15)


def test_vtk_inter_rejects_bad_sizes(built_lib):
    from cgd_b200 import _lib
    from cgd_b200 import output
    for p, OP in [(0, 1), (5, 1), (2, 0), (2, 9)]:
        with pytest.raises(_lib.CgdError):
            output.vtk_inter(p, OP, np.linspace(-1, 1, max(p + 1, 2)))


@pytest.mark.parametrize("OP", [1, 2])
def test_cell_points_match_loops(oracle_mod, OP):
    from _cases import make_case
    from cgd_b200 import output
    o, g, U, nu = make_case(oracle_mod, 2, 2, 3, 0)
    a = output.cell_points(g.X, g.xw, OP, g.Rad)
    b = oracle_mod.cell_points_loops(g.X, list(g.xw), OP, g.Rad)
    assert a.shape == (3, 8 * OP * OP * g.nz * g.NF)
    assert np.array_equal(a, b)
    # every corner lies on a sphere of radius RadPrint + height (heights 0 .. H)
    r = np.sqrt((a * a).sum(axis=0))
    assert r.min() >= 1000.0 - 1e-9 and r.max() <= 1000.0 + g.H + 1e-6
    af = output.cell_points(g.X, g.xw, OP, g.Rad, flat=True, H=g.H)
    bf = oracle_mod.cell_points_loops(g.X, list(g.xw), OP, g.Rad, flat=True, H=g.H)
    assert np.allclose(af, bf, rtol=1e-15, atol=1e-15)


def test_vtu_round_trip(tmp_path):
    from cgd_b200 import output
    rng = np.random.default_rng(3)
    pts = rng.standard_normal((3, 8 * 5))
    data = {"rho": rng.standard_normal(5), "Th": rng.standard_normal(5)}
    path = str(tmp_path / "x0.vtu")
    output.write_vtu(path, pts, data)
    p, conn, offs, types, d = output.read_vtu(path)
    assert np.array_equal(p, pts)
    assert np.array_equal(conn, np.arange(40)) and np.array_equal(offs, 8 * np.arange(1, 6))
    assert np.all(types == output.VTK_HEXAHEDRON)
    assert set(d) == {"rho", "Th"} and all(np.array_equal(d[k], data[k]) for k in data)
    with pytest.raises(ValueError):
        output.write_vtu(path, pts, {"bad": np.zeros(4)})
    output.write_pvtu(str(tmp_path / "x0.pvtu"), ["x0_0.vtu", "x0_1.vtu"], ["rho"])
    import xml.etree.ElementTree as ET
    root = ET.parse(str(tmp_path / "x0.pvtu")).getroot()
    assert [p.get("Source") for p in root.iter("Piece")] == ["x0_0.vtu", "x0_1.vtu"]
