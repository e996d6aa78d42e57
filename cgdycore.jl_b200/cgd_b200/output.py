"""VTK output of the state: the reference's Outputs.vtkStruct and
unstructured_vtkSphere (src/Outputs/vtkSphere.jl:122-220,337-510).

The cell data are the state interpolated on the GPU to OrdPrint x OrdPrint
sub-cells per element and layer (``Dycore.output_fields``, one library call
for all requested quantities); the cell corners are the reference's
TransSphereX! points (src/Grids/Trans.jl:77-99); the file is a VTK XML
unstructured grid of hexahedra (``.vtu``, raw appended binary), with a
``.pvtu`` index when several parts are written.

``VtkOutput.write`` returns once the cell values are computed: their copy to
pinned host memory runs on a stream of its own and the file is written by a
background thread, so the time loop continues meanwhile (``wait()`` joins).
"""
import os
import threading
import xml.etree.ElementTree as ET

import numpy as np

from . import _lib

# cNames of the reference's output (Global.Output.cNames) -> (CGD_OUT_* code, VTK array name)
NAMES = {
    "Rho": (_lib.OUT_RHO, "rho"),
    "u": (_lib.OUT_U, "u"),
    "v": (_lib.OUT_V, "v"),
    "wB": (_lib.OUT_WB, "w"),
    "Th": (_lib.OUT_TH, "Th"),
    "Pres": (_lib.OUT_PRES, "p"),
    "Vort": (_lib.OUT_VORT, "Vort"),
    "Tr1": (_lib.OUT_TR, "Tr1"),
    "Tr2": (_lib.OUT_TR + 1, "Tr2"),
    "Tr3": (_lib.OUT_TR + 2, "Tr3"),
    "Tr4": (_lib.OUT_TR + 3, "Tr4"),
    # not a reference name: the layer-mean w with the surface value from u and v
    "wBuv": (_lib.OUT_WB_UV, "w"),
}

VTK_HEXAHEDRON = 12


def vtk_inter(OrdPoly, OrdPrint, xw):
    """The sub-cell interpolation weights (OrdPrint, OrdPrint, N, N), Fortran
    order: inter[I,J,i,j] = L_i(xi_I) L_j(eta_J) at the sub-cell centres
    (vtkStruct, src/Outputs/vtkSphere.jl:199-219).  Host computation in the
    library (cgd_vtk_inter); needs no GPU."""
    N = OrdPoly + 1
    xw = np.ascontiguousarray(xw, dtype=np.float64)
    out = np.zeros(OrdPrint * OrdPrint * N * N)
    _lib.check(_lib.lib().cgd_vtk_inter(int(OrdPoly), int(OrdPrint), xw.ctypes.data, out.ctypes.data),
               "cgd_vtk_inter")
    return out.reshape((OrdPrint, OrdPrint, N, N), order="F")


def _lagrange(x, xP, iP):
    """DG.Lagrange (src/DG/Lagrange.jl:1-9) of an array of points x."""
    f = np.ones_like(x)
    for i in range(len(xP)):
        if i != iP:
            f = f * (x - xP[i]) / (xP[iP] - xP[i])
    return f


def cell_points(X, xw, OrdPrint, Rad, RadPrint=1000.0, flat=False, H=1.0, dTol=1e-8):
    """The 8 corners of every sub-cell, (3, 8 * OrdPrint^2 * nz * NF), cells
    ordered (iRef, jRef, iz, iF) fastest first, corners bottom then top,
    counter-clockwise (vtkStruct, src/Outputs/vtkSphere.jl:122-178), each
    corner mapped by TransSphereX! (the element's GLL interpolant of the node
    positions X (N*N, 2, 3, nz, NF), projected to radius RadPrint + height).
    flat: longitude, latitude and 3 max(r - Rad, 0) / H instead, as the
    reference's Output.Flat (with r the printed radius)."""
    # a device tensor (NF, nz, 3, 2, N*N) holds the same Fortran-ordered array
    X = X.cpu().numpy().transpose(4, 3, 2, 1, 0) if hasattr(X, "cpu") else np.asarray(X)
    DoF, _, _, nz, NF = X.shape
    N = len(xw)
    # corner coordinates stepped as the reference steps them (ksi1 = ksi0 + dd)
    dd = 2.0 / OrdPrint
    edges = [-1.0]
    for _ in range(OrdPrint):
        edges.append(edges[-1] + dd)
    edges = np.array(edges)
    # per cell (iRef, jRef) and corner c: (ksi, eta, zeta)
    iR, jR = np.meshgrid(np.arange(OrdPrint), np.arange(OrdPrint), indexing="xy")
    iR, jR = iR.ravel(), jR.ravel()                       # iRef fastest
    cks = np.array([0, 1, 1, 0, 0, 1, 1, 0])
    cet = np.array([0, 0, 1, 1, 0, 0, 1, 1])
    czt = np.array([-1.0, -1.0, -1.0, -1.0, 1.0, 1.0, 1.0, 1.0])
    ksi = edges[iR[:, None] + cks[None, :]]               # (OP^2, 8)
    eta = edges[jR[:, None] + cet[None, :]]
    zeta = np.broadcast_to(czt, ksi.shape)
    xwZ = np.array([-1.0, 1.0])
    XP = np.zeros((3, NF, nz, OrdPrint * OrdPrint, 8))
    for j in range(N):
        Lj = _lagrange(eta, xw, j)
        for i in range(N):
            Li = _lagrange(ksi, xw, i) * Lj
            for k in range(2):
                Fac = Li * _lagrange(zeta, xwZ, k)        # (OP^2, 8)
                for l in range(3):
                    Xn = X[i + N * j, k, l].T             # (NF, nz)
                    XP[l] += Fac[None, None] * Xn[:, :, None, None]
    r = np.sqrt(XP[0] * XP[0] + XP[1] * XP[1] + XP[2] * XP[2])
    z = np.maximum(r - Rad, 0.0)
    XP = XP / r * (RadPrint + z)
    if flat:
        # Grids.cart2sphere (src/Grids/Geometry.jl:65-88) and the seam shift
        rr = np.sqrt(XP[0] * XP[0] + XP[1] * XP[1] + XP[2] * XP[2])
        lam = np.arctan2(XP[1], XP[0])
        lam = np.where(XP[1] < 0, lam + 2 * np.pi, lam)
        phi = np.arcsin(XP[2] / rr)
        span = lam.max(axis=-1, keepdims=True) - lam.min(axis=-1, keepdims=True)
        shift = (np.abs(span) > 2 * np.pi - dTol) & (lam > np.pi)
        lam = np.where(shift, lam - 2 * np.pi, lam)
        lam = np.where(shift & (lam > 3 * np.pi), lam - 2 * np.pi, lam)
        XP = np.stack([lam, phi, np.maximum(rr - Rad, 0.0) / H * 3])
    return XP.reshape(3, -1)


# ---------------------------------------------------------------------------
# VTK XML unstructured grid (raw appended binary, UInt64 block headers)
def write_vtu(path, points, cell_data):
    """points (3, 8 * ncells); cell_data: {name: array of ncells values}."""
    pts = np.ascontiguousarray(np.asarray(points, dtype=np.float64).T)
    ncells = pts.shape[0] // 8
    blocks, arrays = [], []

    def add(arr):
        off = sum(8 + b.nbytes for b in blocks)
        blocks.append(np.ascontiguousarray(arr))
        return off

    p_off = add(pts)
    c_off = add(np.arange(8 * ncells, dtype=np.int64))
    o_off = add(8 * np.arange(1, ncells + 1, dtype=np.int64))
    t_off = add(np.full(ncells, VTK_HEXAHEDRON, dtype=np.uint8))
    for name, vals in cell_data.items():
        v = np.asarray(vals, dtype=np.float64).reshape(-1)
        if v.size != ncells:
            raise ValueError(f"{name}: {v.size} values for {ncells} cells")
        arrays.append((name, add(v)))
    cd = "".join(f'        <DataArray type="Float64" Name="{n}" format="appended" offset="{o}"/>\n'
                 for n, o in arrays)
    head = (
        '<?xml version="1.0"?>\n'
        '<VTKFile type="UnstructuredGrid" version="1.0" byte_order="LittleEndian" header_type="UInt64">\n'
        '  <UnstructuredGrid>\n'
        f'    <Piece NumberOfPoints="{pts.shape[0]}" NumberOfCells="{ncells}">\n'
        '      <Points>\n'
        f'        <DataArray type="Float64" NumberOfComponents="3" format="appended" offset="{p_off}"/>\n'
        '      </Points>\n'
        '      <Cells>\n'
        f'        <DataArray type="Int64" Name="connectivity" format="appended" offset="{c_off}"/>\n'
        f'        <DataArray type="Int64" Name="offsets" format="appended" offset="{o_off}"/>\n'
        f'        <DataArray type="UInt8" Name="types" format="appended" offset="{t_off}"/>\n'
        '      </Cells>\n'
        '      <CellData>\n' + cd +
        '      </CellData>\n'
        '    </Piece>\n'
        '  </UnstructuredGrid>\n'
        '  <AppendedData encoding="raw">\n   _')
    with open(path, "wb") as f:
        f.write(head.encode())
        for b in blocks:
            f.write(np.uint64(b.nbytes).tobytes())
            f.write(b.tobytes())
        f.write(b'\n  </AppendedData>\n</VTKFile>\n')


def write_pvtu(path, pieces, names):
    """Index of the parts (`pieces`: their file names, relative to `path`)."""
    cd = "".join(f'      <PDataArray type="Float64" Name="{n}"/>\n' for n in names)
    ps = "".join(f'    <Piece Source="{p}"/>\n' for p in pieces)
    with open(path, "w") as f:
        f.write('<?xml version="1.0"?>\n'
                '<VTKFile type="PUnstructuredGrid" version="1.0" byte_order="LittleEndian" header_type="UInt64">\n'
                '  <PUnstructuredGrid GhostLevel="0">\n'
                '    <PPoints>\n      <PDataArray type="Float64" NumberOfComponents="3"/>\n    </PPoints>\n'
                '    <PCellData>\n' + cd + '    </PCellData>\n' + ps +
                '  </PUnstructuredGrid>\n</VTKFile>\n')


def read_vtu(path):
    """(points (3, npoints), connectivity, offsets, types, {name: cell values})
    of a file written by write_vtu."""
    raw = open(path, "rb").read()
    start = raw.index(b"_", raw.index(b"<AppendedData")) + 1
    root = ET.fromstring(raw[:raw.index(b"<AppendedData")].decode() + "</VTKFile>")
    dt = {"Float64": np.float64, "Int64": np.int64, "UInt8": np.uint8}

    def block(el):
        o = start + int(el.get("offset"))
        n = int(np.frombuffer(raw[o:o + 8], dtype=np.uint64)[0])
        return np.frombuffer(raw[o + 8:o + 8 + n], dtype=dt[el.get("type")])

    piece = root.find("UnstructuredGrid/Piece")
    pts = block(piece.find("Points/DataArray")).reshape(-1, 3).T
    cells = {el.get("Name"): block(el) for el in piece.find("Cells")}
    data = {el.get("Name"): block(el) for el in piece.find("CellData")}
    return pts, cells["connectivity"], cells["offsets"], cells["types"], data


class VtkOutput:
    """The reference's output cache (vtkStruct: weights, cell corners) for one
    Dycore, and unstructured_vtkSphere as ``write``.

    names: the reference's cNames (keys of NAMES); OrdPrint sub-cells per
    element edge; RadPrint, flat as Global.Output.  X: the grid's node
    positions (host or device), from dycore.grid by default."""

    def __init__(self, dycore, names=("Rho", "u", "v", "wB", "Th"), OrdPrint=1, RadPrint=1000.0, flat=False,
                 X=None):
        g = dycore.grid
        unknown = [n for n in names if n not in NAMES]
        if unknown:
            raise ValueError(f"unknown output names {unknown}; known: {sorted(NAMES)}")
        tr = [n for n in names if NAMES[n][0] >= _lib.OUT_TR and NAMES[n][0] - _lib.OUT_TR >= dycore.NumTr]
        if tr:
            raise ValueError(f"{tr}: the model has {dycore.NumTr} tracers")
        self.d, self.names, self.OrdPrint = dycore, list(names), OrdPrint
        self.codes = np.array([NAMES[n][0] for n in names], dtype=np.int32)
        self.vtk_names = [NAMES[n][1] for n in names]
        self.inter = vtk_inter(g.OrdPoly, OrdPrint, g.xw)
        self.points = cell_points(g.X if X is None else X, np.asarray(g.xw), OrdPrint, g.Rad, RadPrint, flat, g.H)
        self.ncells = OrdPrint * OrdPrint * dycore.nz * dycore.NF
        self._thread = None
        self._stream = None
        self.step = 0

    def cells(self, U):
        """All requested quantities of U: {VTK name: cell values (OP, OP, nz,
        NF) flattened in Fortran order}, computed on the GPU and returned in
        host memory."""
        if isinstance(U, np.ndarray):
            out = self.d.output_fields(U, self.codes, self.inter)
            return {n: out[k].reshape(-1) for k, n in enumerate(self.vtk_names)}
        self.wait()   # a background write may still read the pinned buffer
        host = self._device_to_host(U)
        self._event.synchronize()
        return self._split(host)

    def _split(self, flat):
        v = flat.reshape(len(self.codes), self.ncells)
        return {n: v[k] for k, n in enumerate(self.vtk_names)}

    def _device_to_host(self, U):
        import torch
        dev = self.d.output_fields(U, self.codes, self.inter)       # complete on return
        if self._stream is None:
            self._stream = torch.cuda.Stream(device=U.device)
            self._host = torch.empty(dev.numel(), dtype=torch.float64, pin_memory=True)
        self._stream.wait_stream(torch.cuda.current_stream(U.device))
        with torch.cuda.stream(self._stream):
            self._host.copy_(dev, non_blocking=True)
            dev.record_stream(self._stream)
            self._event = torch.cuda.Event()
            self._event.record(self._stream)
        return self._host

    def write(self, U, prefix, step=None, part=None, nparts=1):
        """Writes f"{prefix}{step}.vtu" (or, for part p of nparts,
        f"{prefix}{step}_{p}.vtu" and from part 0 the f"{prefix}{step}.pvtu"
        index) from the state U and returns its path.  For a device state the
        copy to the host and the file write run in the background; call
        wait() before reading the file or changing the pinned buffer's user."""
        self.wait()
        step = self.step if step is None else step
        self.step = step + 1
        base = f"{prefix}{step}"
        path = f"{base}.vtu" if part is None else f"{base}_{part}.vtu"
        if part == 0 and nparts > 1:
            write_pvtu(base + ".pvtu", [os.path.basename(f"{base}_{p}.vtu") for p in range(nparts)], self.vtk_names)
        if isinstance(U, np.ndarray):
            write_vtu(path, self.points, self.cells(U))
            return path
        host = self._device_to_host(U)
        ev = self._event

        def run():
            ev.synchronize()
            write_vtu(path, self.points, self._split(host.numpy()))

        self._thread = threading.Thread(target=run, daemon=True)
        self._thread.start()
        return path

    def wait(self):
        if self._thread is not None:
            self._thread.join()
            self._thread = None
