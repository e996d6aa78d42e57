"""Output interpolation on the GPU against the oracle's restatement of the
reference's kernels (src/Outputs/vtkOutputKernel.jl): plain, density-weighted,
layer-mean w, vorticity and the batched cgd_output_fields, bit for bit in
both builds (the potential temperature to rounding: its power function is
CUDA's against the host libm's); host and device pointers agree; the VTK
writer's file holds the same values."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case(oracle_mod):
    from _cases import make_case
    o, g, U, nu = make_case(oracle_mod, 4, 4, 9, 2, "quadratic")
    U = o.ros_step(U, 300.0, 2)   # vertical motion, w != 0
    return o, g, U, nu


@pytest.mark.parametrize("shape", [(3, 2, 7, 0), (4, 3, 8, 1), (2, 1, 5, 0)])
def test_interpolate_lower_orders(built_lib, cuda_ok, oracle_mod, shape):
    """Polynomial orders 1-3 (the vorticity kernel's other node counts),
    OrdPrint 2, exact build, every kernel bit for bit."""
    from _cases import make_case
    from cgd_b200 import Dycore, _lib
    from cgd_b200 import output
    n, p, nz, nt = shape
    o, g, U, nu = make_case(oracle_mod, n, p, nz, nt, "quadratic")
    U = o.ros_step(U, 300.0, 1)
    d = Dycore(g, nt, nu, exact=True)
    inter = output.vtk_inter(p, 2, g.xw)
    f = lambda k: np.asfortranarray(U[..., k])
    assert np.array_equal(d.interpolate(f(1), inter), o.interpolate(f(1), inter))
    assert np.array_equal(d.interpolate(f(4), inter, rhoc=f(0)), o.interpolate(f(4), inter, rhoc=f(0)))
    assert np.array_equal(d.interpolate_wb(f(1), f(2), f(3), inter), o.interpolate_wb(f(1), f(2), f(3), inter))
    assert np.array_equal(d.interpolate_vort(U, inter), o.interpolate_vort(U, inter))
    out = d.output_fields(U, [_lib.OUT_PRES, _lib.OUT_VORT], inter)
    assert np.array_equal(out[0].reshape(-1), o.interpolate(f(4), inter, kind=1).reshape(-1, order="F"))
    assert np.array_equal(out[1].reshape(-1), o.interpolate_vort(U, inter).reshape(-1, order="F"))
    d.close()


def _tensor(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(np.asarray(a).transpose(*reversed(range(a.ndim))))).cuda()


def _host(t, shape):
    return np.asfortranarray(t.cpu().numpy().reshape(-1).reshape(shape, order="F"))


@pytest.mark.parametrize("variant", ["exact", "fast"])
@pytest.mark.parametrize("OP", [1, 2, 3])
def test_interpolate_kernels(built_lib, cuda_ok, oracle_mod, case, variant, OP):
    from cgd_b200 import Dycore
    from cgd_b200 import output
    o, g, U, nu = case
    d = Dycore(g, 2, nu, exact=variant == "exact")
    inter = output.vtk_inter(g.OrdPoly, OP, g.xw)
    cs = (OP, OP, g.nz, g.NF)
    f = lambda k: np.asfortranarray(U[..., k])
    for k in range(d.NV):
        assert np.array_equal(d.interpolate(f(k), inter), o.interpolate(f(k), inter)), k
    for q in range(2):
        assert np.array_equal(d.interpolate(f(5 + q), inter, rhoc=f(0)), o.interpolate(f(5 + q), inter, rhoc=f(0)))
    assert np.array_equal(d.interpolate_wb(f(1), f(2), f(3), inter), o.interpolate_wb(f(1), f(2), f(3), inter))
    assert np.array_equal(d.interpolate_vort(U, inter), o.interpolate_vort(U, inter))
    # device pointers give the host pointers' values
    Ut = _tensor(U)
    fd = lambda k: Ut[k].contiguous()
    assert np.array_equal(_host(d.interpolate(fd(4), inter, rhoc=fd(0)), cs), o.interpolate(f(4), inter, rhoc=f(0)))
    assert np.array_equal(_host(d.interpolate_wb(fd(1), fd(2), fd(3), inter), cs),
                          o.interpolate_wb(f(1), f(2), f(3), inter))
    assert np.array_equal(_host(d.interpolate_vort(Ut, inter), cs), o.interpolate_vort(U, inter))
    d.close()


@pytest.mark.parametrize("variant", ["exact", "fast"])
def test_output_fields(built_lib, cuda_ok, oracle_mod, case, variant):
    from cgd_b200 import Dycore, _lib
    from cgd_b200 import output
    o, g, U, nu = case
    d = Dycore(g, 2, nu, exact=variant == "exact")
    OP = 2
    inter = output.vtk_inter(g.OrdPoly, OP, g.xw)
    f = lambda k: np.asfortranarray(U[..., k])
    codes = [_lib.OUT_RHO, _lib.OUT_U, _lib.OUT_V, _lib.OUT_WB, _lib.OUT_TH, _lib.OUT_PRES, _lib.OUT_VORT,
             _lib.OUT_WB_UV, _lib.OUT_TR, _lib.OUT_TR + 1]
    ref = [o.interpolate(f(0), inter), o.interpolate(f(1), inter), o.interpolate(f(2), inter),
           o.interpolate_wb(f(1), f(1), f(3), inter),           # the reference passes u for v
           o.interpolate(f(4), inter, rhoc=f(0), kind=2), o.interpolate(f(4), inter, kind=1),
           o.interpolate_vort(U, inter), o.interpolate_wb(f(1), f(2), f(3), inter),
           o.interpolate(f(5), inter, rhoc=f(0)), o.interpolate(f(6), inter, rhoc=f(0))]
    out = d.output_fields(U, codes, inter)                       # host result
    outd = d.output_fields(_tensor(U), codes, inter)             # device result
    outd = outd.cpu().numpy().reshape(out.shape)
    assert np.array_equal(out, outd)
    for k, (c, r) in enumerate(zip(codes, ref)):
        a = out[k].reshape(-1)
        b = r.reshape(-1, order="F")
        if c == _lib.OUT_TH:
            assert np.abs(a - b).max() <= 1e-14 * np.abs(b).max(), k
        else:
            assert np.array_equal(a, b), k
    d.close()


def test_output_errors(built_lib, cuda_ok, case):
    from cgd_b200 import Dycore, _lib
    from cgd_b200 import output
    o, g, U, nu = case
    d = Dycore(g, 2, nu)
    inter = output.vtk_inter(g.OrdPoly, 1, g.xw)
    for bad in ([_lib.OUT_TR + 2], [8], [-1]):
        with pytest.raises(_lib.CgdError):
            d.output_fields(U, bad, inter)
    with pytest.raises(ValueError):
        output.VtkOutput(d, names=("Tr3",))
    with pytest.raises(ValueError):
        output.VtkOutput(d, names=("nope",))
    d.close()


def test_vtk_output_file(built_lib, cuda_ok, case, tmp_path):
    """VtkOutput.write from a device state: the file's cell data equal
    cgd_output_fields' values, its points the corner points; a second part
    writes the .pvtu index."""
    from cgd_b200 import Dycore
    from cgd_b200 import output
    o, g, U, nu = case
    d = Dycore(g, 2, nu)
    names = ("Rho", "u", "v", "wB", "Th", "Pres", "Vort", "Tr1", "Tr2")
    w = output.VtkOutput(d, names=names, OrdPrint=2)
    Ut = _tensor(U)
    path = w.write(Ut, str(tmp_path / "out"), step=3, part=0, nparts=2)
    w.wait()
    assert path.endswith("out3_0.vtu") and (tmp_path / "out3.pvtu").exists()
    pts, conn, offs, types, data = output.read_vtu(path)
    assert np.array_equal(pts, w.points)
    vals = d.output_fields(U, w.codes, w.inter)
    for k, n in enumerate(w.vtk_names):
        assert np.array_equal(data[n], vals[k].reshape(-1)), n
    # the host-state path writes the same file contents
    p2 = w.write(U, str(tmp_path / "host"))          # the step counter continues from the last write
    assert p2.endswith("host4.vtu")
    data2 = output.read_vtu(p2)[4]
    assert all(np.array_equal(data2[n], data[n]) for n in data)
    d.close()
