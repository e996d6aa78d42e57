"""ctypes wrapper of the CPU oracle (TEST INFRASTRUCTURE ONLY).

The oracle is an FP64 CPU restatement of CGDycore.jl's spectral-element hot
path (see cgd_oracle.cpp for the file:line of every restated function).  It is
used by the tests, by ``__graft_entry__.smoke()`` and by the CPU-baseline leg
of ``bench.py`` to check the product; the product never imports it.

Pinning: the Glob numbering is pinned bit for bit to the reference's own
GlobInd golden file; the floating-point restatement is parity unpinned (the
reference records no floating-point vectors for this path and Julia cannot
run here), checked by analytic invariants only.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libcgd_oracle.so")
_lib = None


class OrcCfg(ctypes.Structure):
    _fields_ = [("nPanel", ctypes.c_int), ("OrdPoly", ctypes.c_int), ("nz", ctypes.c_int),
                ("NumTr", ctypes.c_int), ("Rad", ctypes.c_double), ("H", ctypes.c_double),
                ("HyperDCurl", ctypes.c_double), ("HyperDGrad", ctypes.c_double),
                ("HyperDDiv", ctypes.c_double), ("Up", ctypes.c_double)]


def build():
    """Compile the oracle library in place (make)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        vp = ctypes.c_void_p
        L.orc_create.restype = vp
        L.orc_create.argtypes = [ctypes.POINTER(OrcCfg), vp]
        L.orc_destroy.argtypes = [vp]
        L.orc_set_threads.argtypes = [ctypes.c_int]
        L.orc_set_threads.restype = ctypes.c_int
        for f in ["orc_sizes", "orc_get_glob", "orc_get_faces", "orc_get_dz"]:
            getattr(L, f).argtypes = [vp, vp]
        L.orc_get_gll.argtypes = [vp, vp, vp, vp, vp]
        L.orc_get_metric.argtypes = [vp, vp, vp, vp]
        L.orc_get_mass.argtypes = [vp, vp, vp]
        L.orc_set_metric.argtypes = [vp, vp, vp, vp, vp, vp]
        L.orc_init_state.argtypes = [vp, vp, vp]
        for f in ["orc_pressure", "orc_hypervisc1", "orc_rhs", "orc_jac"]:
            getattr(L, f).argtypes = [vp, vp, vp]
        L.orc_contributions.argtypes = [vp, vp, vp, vp]
        L.orc_set_physics.argtypes = [vp, ctypes.c_int, vp, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_double]
        L.orc_schur.argtypes = [vp, vp, vp, ctypes.c_double]
        L.orc_ros_step.argtypes = [vp, vp, ctypes.c_double, ctypes.c_int]
        L.orc_mass_integral.argtypes = [vp, vp]
        L.orc_mass_integral.restype = ctypes.c_double
        L.orc_vtk_inter.argtypes = [ctypes.c_int, ctypes.c_int, vp, vp]
        L.orc_interpolate.argtypes = [vp, vp, vp, ctypes.c_int, vp, ctypes.c_int, vp]
        L.orc_interpolate_wb.argtypes = [vp, vp, vp, vp, vp, ctypes.c_int, vp]
        L.orc_interpolate_vort.argtypes = [vp, vp, vp, ctypes.c_int, vp]
        _lib = L
    return _lib


def set_threads(n):
    return lib().orc_set_threads(int(n))


def _p(a):
    return a.ctypes.data


class Oracle:
    """One oracle model instance (grid, metric, mass, tendencies, steps)."""

    def __init__(self, nPanel, OrdPoly, nz, NumTr, zlev, Rad=6.371e6, H=30000.0,
                 nu=(0.0, 0.0, 0.0), Up=1.0):
        zlev = np.ascontiguousarray(zlev, dtype=np.float64)
        assert zlev.size == nz + 1
        cfg = OrcCfg(nPanel, OrdPoly, nz, NumTr, Rad, H, nu[0], nu[1], nu[2], Up)
        self.h = lib().orc_create(ctypes.byref(cfg), _p(zlev))
        if not self.h:
            raise ValueError("orc_create failed")
        s = np.zeros(6, np.int64)
        lib().orc_sizes(self.h, _p(s))
        self.NF, self.NumG, self.DoF, self.N, self.NumNodes, self.NumEdges = (int(x) for x in s)
        self.nz, self.NumTr, self.NV = nz, NumTr, 5 + NumTr
        self.nPanel, self.OrdPoly = nPanel, OrdPoly

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    # arrays are returned in Fortran order with the reference's shapes
    def glob(self):
        g = np.zeros(self.DoF * self.NF, np.int64)
        lib().orc_get_glob(self.h, _p(g))
        return g.reshape((self.DoF, self.NF), order="F")

    def gll(self):
        N = self.N
        xw, w = np.zeros(N), np.zeros(N)
        DS, DW = np.zeros(N * N), np.zeros(N * N)
        lib().orc_get_gll(self.h, _p(xw), _p(w), _p(DS), _p(DW))
        return xw, w, DS.reshape((N, N), order="F"), DW.reshape((N, N), order="F")

    def faces(self):
        F = np.zeros(12 * self.NF)
        lib().orc_get_faces(self.h, _p(F))
        return F.reshape((4, 3, self.NF), order="F")

    def metric(self):
        DoF, nz, NF = self.DoF, self.nz, self.NF
        X = np.zeros(DoF * 6 * nz * NF)
        dXdxI = np.zeros(18 * DoF * nz * NF)
        J = np.zeros(DoF * 2 * nz * NF)
        lib().orc_get_metric(self.h, _p(X), _p(dXdxI), _p(J))
        return (X.reshape((DoF, 2, 3, nz, NF), order="F"),
                dXdxI.reshape((3, 3, 2, DoF, nz, NF), order="F"),
                J.reshape((DoF, 2, nz, NF), order="F"))

    def mass(self):
        M = np.zeros(self.nz * self.NumG * 2)
        MM = np.zeros(self.nz * self.NumG)
        lib().orc_get_mass(self.h, _p(M), _p(MM))
        return (M.reshape((self.nz, self.NumG, 2), order="F"),
                MM.reshape((self.nz, self.NumG), order="F"))

    def dz(self):
        d = np.zeros(self.nz * self.NumG)
        lib().orc_get_dz(self.h, _p(d))
        return d.reshape((self.nz, self.NumG), order="F")

    def set_metric(self, X=None, dXdxI=None, J=None, M=None, dz=None):
        def q(a):
            return None if a is None else _p(np.asfortranarray(a, dtype=np.float64))
        keep = [np.asfortranarray(a, dtype=np.float64) if a is not None else None
                for a in (X, dXdxI, J, M, dz)]
        lib().orc_set_metric(self.h, *[(_p(a) if a is not None else None) for a in keep])

    def _state(self):
        return np.zeros((self.nz, self.NumG, self.NV), order="F")

    def init_state(self, tracer_lonlat=None):
        U = self._state()
        tl = np.zeros(max(2 * self.NumTr, 2))
        if tracer_lonlat is not None and self.NumTr:
            tl[:2 * self.NumTr] = np.asarray(tracer_lonlat, dtype=np.float64).ravel()
        lib().orc_init_state(self.h, _p(U), _p(tl))
        return U

    def pressure(self, U):
        U = np.asfortranarray(U)
        p = np.zeros((self.nz, self.NumG), order="F")
        lib().orc_pressure(self.h, _p(U), _p(p))
        return p

    def hypervisc1(self, U):
        U = np.asfortranarray(U)
        T = np.zeros((self.nz, self.NumG, 5 + self.NumTr), order="F")
        lib().orc_hypervisc1(self.h, _p(U), _p(T))
        return T

    def set_physics(self, held_suarez=None, damping=None):
        """Column physics in the tendency tail: held_suarez = the 8 parameters
        (k_a, k_f, k_s, DeltaT_y, DeltaTh_z, T_equator, T_min, sigma_b) or
        None; damping = (H, StrideDamp, Relax) or None."""
        hs = np.ascontiguousarray(held_suarez if held_suarez is not None else np.zeros(8), dtype=np.float64)
        dH, dS, dR = damping if damping is not None else (0.0, 1.0, 0.0)
        lib().orc_set_physics(self.h, int(held_suarez is not None), _p(hs), int(damping is not None),
                              float(dH), float(dS), float(dR))

    def contributions(self, U, T1=None):
        """Element-node contributions before the DSS, shape (DoF, nf, nz, NF)
        in Fortran order: phase 1 (T1 None, nf = 5 + NumTr) or phase 2 at the
        DSS'd phase-1 cache T1 (nf = NV)."""
        U = np.asfortranarray(U)
        nf = self.NV if T1 is not None else 5 + self.NumTr
        C = np.zeros(self.DoF * nf * self.nz * self.NF)
        T = np.asfortranarray(T1) if T1 is not None else None
        lib().orc_contributions(self.h, _p(U), _p(T) if T is not None else None, _p(C))
        return C.reshape((self.DoF, nf, self.nz, self.NF), order="F")

    def rhs(self, U):
        U = np.asfortranarray(U)
        F = self._state()
        lib().orc_rhs(self.h, _p(U), _p(F))
        return F

    def jac(self, U):
        U = np.asfortranarray(U)
        b = np.zeros(4 * 2 * (self.nz - 1) * self.NumG)
        lib().orc_jac(self.h, _p(U), _p(b))
        # four bands (JRhoW, JWRho, JWRhoTh, JRhoThW), each (2, nz-1, NumG) column-major
        return b.reshape((4, self.NumG, self.nz - 1, 2)).transpose(0, 3, 2, 1)

    def schur(self, v, fac):
        v = np.array(v, order="F", dtype=np.float64, copy=True)
        k = self._state()
        rc = lib().orc_schur(self.h, _p(k), _p(v), float(fac))
        if rc:
            raise RuntimeError("orc_schur: call jac first")
        return k, v

    def ros_step(self, U, dt, nsteps=1):
        V = np.array(U, order="F", dtype=np.float64, copy=True)
        lib().orc_ros_step(self.h, _p(V), float(dt), int(nsteps))
        return V

    def mass_integral(self, U):
        U = np.asfortranarray(U)
        return lib().orc_mass_integral(self.h, _p(U))

    # ---- output interpolation (src/Outputs/vtkOutputKernel.jl)
    def _cells(self, OP):
        return np.zeros((OP, OP, self.nz, self.NF), order="F")

    def interpolate(self, c, inter, rhoc=None, kind=0):
        """InterpolateKernel! (rhoc None) / InterpolateRhoKernel!; kind 1 the
        dry pressure of c = rho*theta, kind 2 the dry potential temperature
        (c = rho*theta, rhoc = rho).  Cells (OP, OP, nz, NF)."""
        inter = np.asfortranarray(inter, dtype=np.float64)
        OP = inter.shape[0]
        c = np.asfortranarray(c, dtype=np.float64)
        r = np.asfortranarray(rhoc, dtype=np.float64) if rhoc is not None else None
        out = self._cells(OP)
        lib().orc_interpolate(self.h, _p(c), _p(r) if r is not None else None, int(kind), _p(inter), OP, _p(out))
        return out

    def interpolate_wb(self, u, v, w, inter):
        inter = np.asfortranarray(inter, dtype=np.float64)
        OP = inter.shape[0]
        u, v, w = (np.asfortranarray(a, dtype=np.float64) for a in (u, v, w))
        out = self._cells(OP)
        lib().orc_interpolate_wb(self.h, _p(u), _p(v), _p(w), _p(inter), OP, _p(out))
        return out

    def interpolate_vort(self, U, inter):
        inter = np.asfortranarray(inter, dtype=np.float64)
        OP = inter.shape[0]
        U = np.asfortranarray(U, dtype=np.float64)
        out = self._cells(OP)
        lib().orc_interpolate_vort(self.h, _p(U), _p(inter), OP, _p(out))
        return out


def vtk_inter(OrdPoly, OrdPrint, xw):
    """vtkStruct's vtkInter (src/Outputs/vtkSphere.jl:199-219):
    (OrdPrint, OrdPrint, N, N), Fortran order."""
    N = OrdPoly + 1
    xw = np.ascontiguousarray(xw, dtype=np.float64)
    out = np.zeros(OrdPrint * OrdPrint * N * N)
    lib().orc_vtk_inter(int(OrdPoly), int(OrdPrint), _p(xw), _p(out))
    return out.reshape((OrdPrint, OrdPrint, N, N), order="F")


def cell_points_loops(X, xw, OrdPrint, Rad, RadPrint=1000.0, flat=False, H=1.0, dTol=1e-8):
    """Pure-Python loops over vtkStruct's corner points (src/Outputs/
    vtkSphere.jl:122-178) with TransSphereX! (src/Grids/Trans.jl:77-99):
    8 corners per sub-cell, cells ordered (iRef, jRef, iz, iF) fastest first.
    X (N*N, 2, 3, nz, NF).  For small grids only."""
    import math
    DoF, _, _, nz, NF = X.shape
    N = len(xw)
    xwZ = [-1.0, 1.0]

    def lag(x, xP, iP):
        f = 1.0
        for i in range(len(xP)):
            if i != iP:
                f = f * (x - xP[i]) / (xP[iP] - xP[i])
        return f

    def trans(ksi, eta, zeta, iz, iF):
        XP = [0.0, 0.0, 0.0]
        for j in range(N):
            Lj = lag(eta, xw, j)
            for i in range(N):
                Li = lag(ksi, xw, i) * Lj
                for k in range(2):
                    Fac = Li * lag(zeta, xwZ, k)
                    for l in range(3):
                        XP[l] += Fac * X[i + N * j, k, l, iz, iF]
        r = math.sqrt(XP[0] * XP[0] + XP[1] * XP[1] + XP[2] * XP[2])
        z = max(r - Rad, 0.0)
        return [x / r * (RadPrint + z) for x in XP]

    pts = []
    dd = 2.0 / OrdPrint
    for iF in range(NF):
        for iz in range(nz):
            eta0 = -1.0
            for jRef in range(OrdPrint):
                ksi0 = -1.0
                eta1 = eta0 + dd
                for iRef in range(OrdPrint):
                    ksi1 = ksi0 + dd
                    corners = [(ksi0, eta0, -1.0), (ksi1, eta0, -1.0), (ksi1, eta1, -1.0), (ksi0, eta1, -1.0),
                               (ksi0, eta0, 1.0), (ksi1, eta0, 1.0), (ksi1, eta1, 1.0), (ksi0, eta1, 1.0)]
                    x = [trans(a, b, c, iz, iF) for a, b, c in corners]
                    if flat:
                        sph = []
                        for (xx, yy, zz) in x:   # Grids.cart2sphere (src/Grids/Geometry.jl:65-75)
                            r = math.sqrt(xx * xx + yy * yy + zz * zz)
                            lam = math.atan2(yy, xx)
                            if yy < 0:
                                lam += 2 * math.pi
                            sph.append([lam, math.asin(zz / r), r])
                        lams = [q[0] for q in sph]
                        if abs(min(lams) - max(lams)) > 2 * math.pi - dTol:
                            for q in sph:
                                if q[0] > math.pi:
                                    q[0] -= 2 * math.pi
                                    if q[0] > 3 * math.pi:
                                        q[0] -= 2 * math.pi
                        x = [[q[0], q[1], max(q[2] - Rad, 0.0) / H * 3] for q in sph]
                    pts.extend(x)
                    ksi0 = ksi1
                eta0 = eta1
    return np.array(pts).T    # (3, 8 * cells)
