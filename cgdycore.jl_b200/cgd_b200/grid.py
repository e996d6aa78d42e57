"""Cubed-sphere grid, GLL element and metric for the hot path.

Host-side set-up that produces exactly the arrays the reference's hot path
consumes (CG.Glob, CG.DS/DW, Metric.X/dXdxI/J, CG.M/MMass, Metric.dz), built
from the same algorithms:

* topology + numbering: src/Grids/CubedGrid.jl:1-513 (nodes, edges, faces),
  src/Grids/Face.jl:48-167 (edge cycle, orientation flip),
  src/Grids/Orientation.jl:1-88, src/Grids/Renumbering.jl:10-93,
  src/Grids/SubGridGhost.jl:1-162 (single process: first-appearance
  renumbering), src/DyCore/NumberingFem.jl:21-105 (Glob, p <= 4);
* element: FastGaussQuadrature.gausslobatto (closed forms for p <= 4),
  src/DG/DLagrange.jl, src/DG/DerivativeMatrixSingle.jl:1-19;
* metric: src/Grids/JacobiSphere3GPU.jl:102-215 with the Sleve height
  (src/Grids/Adapt.jl:19-31, flat orography);
* lumped mass / dz: src/DyCore/MassCG.jl:61-75,
  src/DyCore/DiscretizationCG.jl:119-144.

The topology is held in flat integer arrays (0-based) rather than object
graphs.  The metric is evaluated vectorised with numpy in the reference's
operation order.
"""
from dataclasses import dataclass

import numpy as np

PI = np.float64(3.141592653589793)


# ---------------------------------------------------------------------------
# topology
# ---------------------------------------------------------------------------
class _Topo:
    def __init__(self, nnodes, nedges, nfaces):
        self.P = np.zeros((nnodes, 3))
        self.EN = np.zeros((nedges, 2), np.int64)       # edge -> nodes
        self.EF = np.full((nedges, 2), -1, np.int64)    # edge -> faces (creation order)
        self.ENF = np.zeros(nedges, np.int64)
        self.FN = np.zeros((nfaces, 4), np.int64)       # face -> nodes (cycle)
        self.FE = np.zeros((nfaces, 4), np.int64)       # face -> edges (cycle)
        self.FP = np.zeros((nfaces, 4, 3))               # face corner coordinates


def _cube_point(i1, i2, i3, n, x, y, z, rad):
    if i1 > 0:
        x = np.tan(np.float64(i1) * PI / np.float64(2 * n) - 0.25 * PI)
    if i2 > 0:
        y = np.tan(np.float64(i2) * PI / np.float64(2 * n) - 0.25 * PI)
    if i3 > 0:
        z = np.tan(np.float64(i3) * PI / np.float64(2 * n) - 0.25 * PI)
    x, y, z = np.float64(x), np.float64(y), np.float64(z)
    nrm = np.sqrt(x * x + y * y + z * z)
    return (x / nrm * rad, y / nrm * rad, z / nrm * rad)


def _cross(a, b):
    return (a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0])


def _build_face(T, E4, pos, rad):
    """Face constructor (src/Grids/Face.jl:48-167) for a quad."""
    ef = list(E4)
    for e in ef:
        T.EF[e, T.ENF[e]] = pos
        T.ENF[e] += 1
    FE = [ef[0], 0, 0, 0]
    n2 = T.EN[FE[0], 1]
    for i in range(1, 4):
        for i1 in range(i, 4):
            e = ef[i1]
            if n2 == T.EN[e, 0]:
                FE[i] = e
                n2 = T.EN[e, 1]
                ef[i1], ef[i] = ef[i], FE[i]
                break
            elif n2 == T.EN[e, 1]:
                FE[i] = e
                n2 = T.EN[e, 0]
                ef[i1], ef[i] = ef[i], FE[i]
                break
    FN = [T.EN[FE[0], 0], T.EN[FE[0], 1], 0, 0]
    for i in range(1, 3):
        FN[i + 1] = T.EN[FE[i], 1] if FN[i] == T.EN[FE[i], 0] else T.EN[FE[i], 0]
    P = [tuple(T.P[k]) for k in FN]
    mid = [0.0, 0.0, 0.0]
    for p in P:
        mid = [mid[c] + p[c] for c in range(3)]
    mid = [m / 4.0 for m in mid]
    nm = np.sqrt(mid[0] * mid[0] + mid[1] * mid[1] + mid[2] * mid[2])
    mid = [m / nm * rad for m in mid]
    nv = _cross(P[3], P[0])
    for i in range(3):
        t = _cross(P[i], P[i + 1])
        nv = tuple(nv[c] + t[c] for c in range(3))
    if nv[0] * mid[0] + nv[1] * mid[1] + nv[2] * mid[2] < 0:
        FN = FN[::-1]
        P = P[::-1]
        FE = [FE[2], FE[1], FE[0], FE[3]]
    T.FN[pos] = FN
    T.FE[pos] = FE
    T.FP[pos] = np.array(P)


def _cubed_topology(n, rad):
    nnodes = 6 * (n - 1) * (n - 1) + 12 * (n - 1) + 8
    nedges = 12 * (n - 1) * n + 12 * n
    nfaces = 6 * n * n
    T = _Topo(nnodes, nedges, nfaces)
    cnt = [0]

    def put(i1, i2, i3, x, y, z):
        T.P[cnt[0]] = _cube_point(i1, i2, i3, n, x, y, z, rad)
        cnt[0] += 1
        return cnt[0] - 1

    # node blocks in the order of src/Grids/CubedGrid.jl:16-234
    def block(gen):
        start = cnt[0]
        for args in gen:
            put(*args)
        return start

    m = n - 1
    W = block((-1, j, k, -1.0, 0.0, 0.0) for k in range(1, n) for j in range(1, n))
    E = block((-1, j, k, 1.0, 0.0, 0.0) for k in range(1, n) for j in range(1, n))
    S = block((i, -1, k, 0.0, -1.0, 0.0) for k in range(1, n) for i in range(1, n))
    Nn = block((i, -1, k, 0.0, 1.0, 0.0) for k in range(1, n) for i in range(1, n))
    B = block((i, j, -1, 0.0, 0.0, -1.0) for j in range(1, n) for i in range(1, n))
    Tp = block((i, j, -1, 0.0, 0.0, 1.0) for j in range(1, n) for i in range(1, n))
    WEmm = block((i, -1, -1, 0.0, -1.0, -1.0) for i in range(1, n))
    WEpm = block((i, -1, -1, 0.0, 1.0, -1.0) for i in range(1, n))
    WEmp = block((i, -1, -1, 0.0, -1.0, 1.0) for i in range(1, n))
    WEpp = block((i, -1, -1, 0.0, 1.0, 1.0) for i in range(1, n))
    SNmm = block((-1, j, -1, -1.0, 0.0, -1.0) for j in range(1, n))
    SNpm = block((-1, j, -1, 1.0, 0.0, -1.0) for j in range(1, n))
    SNmp = block((-1, j, -1, -1.0, 0.0, 1.0) for j in range(1, n))
    SNpp = block((-1, j, -1, 1.0, 0.0, 1.0) for j in range(1, n))
    BTmm = block((-1, -1, k, -1.0, -1.0, 0.0) for k in range(1, n))
    BTpm = block((-1, -1, k, 1.0, -1.0, 0.0) for k in range(1, n))
    BTmp = block((-1, -1, k, -1.0, 1.0, 0.0) for k in range(1, n))
    BTpp = block((-1, -1, k, 1.0, 1.0, 0.0) for k in range(1, n))
    corner = {}
    for key, xyz in [("mmm", (-1, -1, -1)), ("pmm", (1, -1, -1)), ("mpm", (-1, 1, -1)), ("ppm", (1, 1, -1)),
                     ("mmp", (-1, -1, 1)), ("pmp", (1, -1, 1)), ("mpp", (-1, 1, 1)), ("ppp", (1, 1, 1))]:
        corner[key] = put(-1, -1, -1, float(xyz[0]), float(xyz[1]), float(xyz[2]))
    assert cnt[0] == nnodes

    ecnt = [0]

    def edge(a, b):
        T.EN[ecnt[0]] = (a, b)
        ecnt[0] += 1

    def face_edges(start, e1a, e2a, e1b, e2b):
        """InsertFaceEdge (src/Grids/CubedGrid.jl:393-441); node ids 0-based,
        the reference's "NodeNumber - 1" becomes "nd - 1" on 1-based ids."""
        s1 = ecnt[0]
        nd, a, b = start + 1, e1a + 1, e2a + 1           # 1-based counters
        for _ in range(1, n):
            for i in range(1, n + 1):
                n1, n2 = nd - 1, nd
                if i == 1:
                    n1 = a; a += 1
                if i == n:
                    n2 = b; b += 1; nd -= 1
                edge(n1 - 1, n2 - 1)
                nd += 1
        s2 = ecnt[0]
        nd, a, b = start + 1, e1b + 1, e2b + 1
        for j in range(1, n + 1):
            for _ in range(1, n):
                n1, n2 = nd - (n - 1), nd
                if j == 1:
                    n1 = a; a += 1
                if j == n:
                    n2 = b; b += 1
                edge(n1 - 1, n2 - 1)
                nd += 1
        return s1, s2

    def edge_edges(start, c1, c2):
        s = ecnt[0]
        nd = start + 1
        for i in range(1, n + 1):
            n1, n2 = nd - 1, nd
            if i == 1:
                n1 = c1 + 1
            if i == n:
                n2 = c2 + 1
            edge(n1 - 1, n2 - 1)
            nd += 1
        return s

    fw = face_edges(W, BTmm, BTmp, SNmm, SNmp)
    fe = face_edges(E, BTpm, BTpp, SNpm, SNpp)
    fs = face_edges(S, BTmm, BTpm, WEmm, WEmp)
    fn = face_edges(Nn, BTmp, BTpp, WEpm, WEpp)
    fb = face_edges(B, SNmm, SNpm, WEmm, WEpm)
    ft = face_edges(Tp, SNmp, SNpp, WEmp, WEpp)
    c = corner
    eWEmm = edge_edges(WEmm, c["mmm"], c["pmm"])
    eWEpm = edge_edges(WEpm, c["mpm"], c["ppm"])
    eWEmp = edge_edges(WEmp, c["mmp"], c["pmp"])
    eWEpp = edge_edges(WEpp, c["mpp"], c["ppp"])
    eSNmm = edge_edges(SNmm, c["mmm"], c["mpm"])
    eSNpm = edge_edges(SNpm, c["pmm"], c["ppm"])
    eSNmp = edge_edges(SNmp, c["mmp"], c["mpp"])
    eSNpp = edge_edges(SNpp, c["pmp"], c["ppp"])
    eBTmm = edge_edges(BTmm, c["mmm"], c["mmp"])
    eBTpm = edge_edges(BTpm, c["pmm"], c["pmp"])
    eBTmp = edge_edges(BTmp, c["mpm"], c["mpp"])
    eBTpp = edge_edges(BTpp, c["ppm"], c["ppp"])
    assert ecnt[0] == nedges

    fcnt = [0]

    def face_faces(s12, ew1, ew2, sn1, sn2):
        """InsertFaceFace (src/Grids/CubedGrid.jl:464-513), 1-based counters."""
        e1, e2 = s12[0] + 1, s12[1] + 1
        ew1, ew2, sn1, sn2 = ew1 + 1, ew2 + 1, sn1 + 1, sn2 + 1
        for j in range(1, n + 1):
            for i in range(1, n + 1):
                E4 = [e1 - n, e1, e2 - 1, e2]
                if j == 1:
                    E4[0] = ew1; ew1 += 1
                if j == n:
                    E4[1] = ew2; ew2 += 1
                if i == 1:
                    E4[2] = sn1; sn1 += 1
                if i == n:
                    E4[3] = sn2; sn2 += 1; e2 -= 1
                e1 += 1
                e2 += 1
                _build_face(T, [x - 1 for x in E4], fcnt[0], rad)
                fcnt[0] += 1

    face_faces(fw, eSNmm, eSNmp, eBTmm, eBTmp)
    face_faces(fe, eSNpm, eSNpp, eBTpm, eBTpp)
    face_faces(fs, eWEmm, eWEmp, eBTmm, eBTpm)
    face_faces(fn, eWEpm, eWEpp, eBTmp, eBTpp)
    face_faces(fb, eWEmm, eWEpm, eSNmm, eSNpm)
    face_faces(ft, eWEmp, eWEpp, eSNmp, eSNpp)
    assert fcnt[0] == nfaces
    return T


def _orient(T):
    """Orientation! (src/Grids/Orientation.jl:1-88).  The while loop there runs
    once (size of a Vector along dim 2 is 1): each unvisited edge makes the
    opposite edge of its first face parallel to itself."""
    nedges = T.EN.shape[0]
    visit = np.zeros(nedges, bool)
    for e in range(nedges):
        if visit[e]:
            continue
        visit[e] = True
        f = T.EF[e, 0]
        fe = list(T.FE[f])
        i1 = fe.index(e) if e in fe else 3
        NF = list(T.FN[f]) + [T.FN[f, 0]]
        o = 1 if NF[i1] == T.EN[e, 0] else -1
        ip = (i1 + 2) % 4
        ep = fe[ip]
        op = 1 if NF[ip] == T.EN[ep, 0] else -1
        if op == o:
            if o == -1:
                T.EN[ep] = (NF[ip], NF[ip + 1])
            else:
                T.EN[ep] = (NF[ip + 1], NF[ip])
        visit[ep] = True


def _renumber_faces(T):
    """RenumberingFace4! (src/Grids/Renumbering.jl:48-93): rotate each face so
    that it starts at the first corner with two outgoing edges (or by three
    positions when no corner has two)."""
    starts = T.EN[T.FE, 0]                        # (nfaces, 4) start node of each edge
    for f in range(T.FN.shape[0]):
        iN = 3
        for k in range(4):
            iN = k
            if np.count_nonzero(starts[f] == T.FN[f, k]) >= 2:
                break
        if iN > 0:
            T.FN[f] = np.roll(T.FN[f], -iN)
            T.FE[f] = np.roll(T.FE[f], -iN)
            T.FP[f] = np.roll(T.FP[f], -iN, axis=0)


def build_topology(n, rad):
    """Global cubed-sphere topology after Orientation!/Renumbering! and the
    single-process sub-grid renumbering.  Returns (FN, FE, EN, FP, nnodes,
    nedges) with 0-based ids in the sub-grid numbering."""
    T = _cubed_topology(n, rad)
    _orient(T)
    _renumber_faces(T)
    # ConstructSubGridGhost, one process: nodes and edges by first appearance
    fn_flat = T.FN.ravel()
    fe_flat = T.FE.ravel()
    _, first_n = np.unique(fn_flat, return_index=True)
    node_order = fn_flat[np.sort(first_n)]
    _, first_e = np.unique(fe_flat, return_index=True)
    edge_order = fe_flat[np.sort(first_e)]
    node_new = np.empty(T.P.shape[0], np.int64)
    node_new[node_order] = np.arange(node_order.size)
    edge_new = np.empty(T.EN.shape[0], np.int64)
    edge_new[edge_order] = np.arange(edge_order.size)
    S = _Topo(0, 0, 0)
    S.P = T.P[node_order]
    S.EN = node_new[T.EN[edge_order]]
    S.FN = node_new[T.FN]
    S.FE = edge_new[T.FE]
    S.FP = T.FP.copy()
    _renumber_faces(S)
    return S.FN, S.FE, S.EN, S.FP, node_order.size, edge_order.size


_PER = {
    1: [1, 2, 4, 3],
    2: [1, 5, 2, 8, 9, 6, 4, 7, 3],
    3: [1, 5, 6, 2, 12, 13, 14, 7, 11, 15, 16, 8, 4, 10, 9, 3],
    4: [1, 5, 6, 7, 2, 16, 17, 18, 19, 8, 15, 20, 21, 22, 9, 14, 23, 24, 25, 10, 4, 13, 12, 11, 3],
}


def numbering_cg_quad(FN, FE, EN, nnodes, nedges, p):
    """Glob (1-based, shape (N*N, NF), Fortran order) and NumG:
    src/DyCore/NumberingFem.jl:21-105."""
    if p not in _PER:
        raise ValueError("OrdPoly must be 1..4 (the reference's NumberingFemCGQuad)")
    nf = FN.shape[0]
    m = p - 1
    ne_dofs = nedges * m
    numg = nnodes + ne_dofs + nf * m * m
    loc = np.zeros((nf, (p + 1) ** 2), np.int64)
    loc[:, 0:4] = FN + 1
    col = 4
    for i in range(4):
        e = FE[:, i]
        forward = EN[e, 0] == FN[:, i]
        j = np.arange(1, p)
        fwd = e[:, None] * m + j[None, :] + nnodes
        bwd = e[:, None] * m + j[::-1][None, :] + nnodes
        loc[:, col:col + m] = np.where(forward[:, None], fwd, bwd)
        col += m
    if m > 0:
        jj, ii = np.meshgrid(np.arange(1, p), np.arange(1, p), indexing="ij")
        inner = (ii + (jj - 1) * m).ravel()
        loc[:, col:] = nnodes + ne_dofs + inner[None, :] + (np.arange(nf)[:, None]) * m * m
    per = np.array(_PER[p]) - 1
    glob = loc[:, per].T.copy(order="F")       # (N*N, NF)
    return np.asfortranarray(glob), int(numg)


# ---------------------------------------------------------------------------
# element
# ---------------------------------------------------------------------------
def gauss_lobatto(p):
    if p == 1:
        return np.array([-1.0, 1.0]), np.array([1.0, 1.0])
    if p == 2:
        return np.array([-1.0, 0.0, 1.0]), np.array([1.0 / 3.0, 4.0 / 3.0, 1.0 / 3.0])
    if p == 3:
        a = np.sqrt(1.0 / 5.0)
        return np.array([-1.0, -a, a, 1.0]), np.array([1.0 / 6.0, 5.0 / 6.0, 5.0 / 6.0, 1.0 / 6.0])
    if p == 4:
        a = np.sqrt(3.0 / 7.0)
        return (np.array([-1.0, -a, 0.0, a, 1.0]),
                np.array([1.0 / 10.0, 49.0 / 90.0, 32.0 / 45.0, 49.0 / 90.0, 1.0 / 10.0]))
    raise ValueError("OrdPoly must be 1..4")


def derivative_matrices(p):
    """DS (strong) and DW = -W^-1 DS^T W (weak): src/DG/DerivativeMatrixSingle.jl:1-19."""
    xw, w = gauss_lobatto(p)
    N = p + 1
    DS = np.zeros((N, N))
    for i in range(N):
        for j in range(N):
            Df, f = 0.0, 1.0
            for k in range(N):
                if k != j:
                    Df = Df * (xw[i] - xw[k]) / (xw[j] - xw[k]) + f / (xw[j] - xw[k])
                    f = f * (xw[i] - xw[k]) / (xw[j] - xw[k])
            DS[i, j] = Df
    DW = np.zeros((N, N))
    for i in range(N):
        for j in range(N):
            DW[i, j] = -(1.0 / w[i]) * DS[j, i] * w[j]
    return xw, w, DS, DW


def vertical_uniform(nz, H):
    """AddVerticalGrid! (src/Grids/AddVerticalGrid.jl:1-16)."""
    z = np.zeros(nz + 1)
    d = H / nz
    for i in range(1, nz + 1):
        z[i] = z[i - 1] + d
    return z


def vertical_quadratic(nz, H):
    """z_k = H (k/nz)^2: levels stretched quadratically towards the surface."""
    k = np.arange(nz + 1, dtype=np.float64)
    return H * (k / nz) ** 2


# ---------------------------------------------------------------------------
# metric
# ---------------------------------------------------------------------------
def metric_sphere(FP, xw, DS, z, H, rad):
    """X (N*N,2,3,nz,NF), dXdxI (3,3,2,N*N,nz,NF), J (N*N,2,nz,NF):
    src/Grids/JacobiSphere3GPU.jl:102-215, shallow atmosphere, Sleve height
    with zero orography (src/Grids/Adapt.jl:19-31)."""
    NF = FP.shape[0]
    N = xw.size
    DoF = N * N
    nz = z.size - 1
    I = np.tile(np.arange(N), N)          # ID = I + N*J
    Jn = np.repeat(np.arange(N), N)
    k1 = xw[I][:, None]                     # (DoF, 1)
    k2 = xw[Jn][:, None]
    F = FP.transpose(1, 2, 0)               # (4 corners, 3, NF)
    one = 1.0
    Xc = [0.25 * (F[0, c][None, :] * (one - k1) * (one - k2) + F[1, c][None, :] * (one + k1) * (one - k2) +
                  F[2, c][None, :] * (one + k1) * (one + k2) + F[3, c][None, :] * (one - k1) * (one + k2))
          for c in range(3)]                # each (DoF, NF)
    r = np.sqrt(Xc[0] * Xc[0] + Xc[1] * Xc[1] + Xc[2] * Xc[2])
    f = rad / r
    # Sleve height with zs = 0 for the bottom (K=0) and top (K=1) node of each layer
    hR = np.zeros((2, nz))
    for K, ks in enumerate((-1.0, 1.0)):
        zl = 0.5 * ((one - ks) * z[:-1] + (one + ks) * z[1:])
        eta = zl / H
        hR[K] = np.where(eta <= 0.7, eta * H + 0.0, eta * H)
    X = np.empty((DoF, 2, 3, nz, NF))
    for c in range(3):
        base = Xc[c] / r                    # (DoF, NF)
        for K in range(2):
            X[:, K, c, :, :] = base[:, None, :] * (rad + hR[K])[None, :, None]
    theta = np.arcsin(Xc[2] / r)
    lam = np.arctan2(Xc[1], Xc[0])
    lam = np.where(Xc[1] < 0.0, lam + 2.0 * PI, lam)
    sl, cl, st, ct = np.sin(lam), np.cos(lam), np.sin(theta), np.cos(theta)
    A = np.empty((3, 3) + sl.shape)
    A[0, 0] = sl * sl * ct * ct + st * st
    A[0, 1] = -sl * cl * ct * ct
    A[0, 2] = -cl * st * ct
    A[1, 0] = A[0, 1]
    A[1, 1] = cl * cl * ct * ct + st * st
    A[1, 2] = -sl * st * ct
    A[2, 0] = -cl * st
    A[2, 1] = -sl * st
    A[2, 2] = ct
    DD = np.zeros((2, 3) + sl.shape)
    DD[0, 0] = -sl
    DD[0, 1] = cl
    DD[1, 2] = 1.0
    B = np.empty((3, 4) + sl.shape)
    for cc in range(3):
        for k in range(4):
            B[cc, k] = F[k, cc][None, :]
    kk1, kk2 = np.broadcast_to(k1, sl.shape), np.broadcast_to(k2, sl.shape)
    Cm = np.empty((4, 2) + sl.shape)
    Cm[0, 0], Cm[0, 1] = -one + kk2, -one + kk1
    Cm[1, 0], Cm[1, 1] = one - kk2, -one - kk1
    Cm[2, 0], Cm[2, 1] = one + kk2, one + kk1
    Cm[3, 0], Cm[3, 1] = -one - kk2, one - kk1
    t = 0.25 * f

    def mm(Lm, Rm):
        out = np.empty((Lm.shape[0], Rm.shape[1]) + sl.shape)
        for i in range(Lm.shape[0]):
            for j in range(Rm.shape[1]):
                acc = Lm[i, 0] * Rm[0, j]
                for k in range(1, Lm.shape[1]):
                    acc = acc + Lm[i, k] * Rm[k, j]
                out[i, j] = acc
        return out

    T1 = t[None, None] * DD
    T4 = mm(mm(mm(T1, A), B), Cm)           # (2, 2, DoF, NF)
    # vertical row: D * hR (constant over the element plane) and dz/2
    dXdxI = np.empty((3, 3, 2, DoF, nz, NF))
    J = np.empty((DoF, 2, nz, NF))
    for K in range(2):
        h = hR[K]                            # (nz,)
        Dx = DS[I, 0][:, None] * h[None, :]
        Dy = DS[Jn, 0][:, None] * h[None, :]
        for k in range(1, N):
            Dx = Dx + DS[I, k][:, None] * h[None, :]
            Dy = Dy + DS[Jn, k][:, None] * h[None, :]
        Dz = 0.5 * (hR[1] - hR[0])           # (nz,)
        a11 = T4[0, 0][:, None, :]
        a21 = T4[1, 0][:, None, :]
        a12 = T4[0, 1][:, None, :]
        a22 = T4[1, 1][:, None, :]
        a13 = 0.0
        a23 = 0.0
        a31 = Dx[:, :, None]
        a32 = Dy[:, :, None]
        a33 = Dz[None, :, None]
        J[:, K] = (a11 * (a22 * a33 - a23 * a32) - a12 * (a21 * a33 - a23 * a31) +
                   a13 * (a21 * a32 - a22 * a31))
        dXdxI[0, 0, K] = a22 * a33 - a23 * a32
        dXdxI[1, 0, K] = -(a21 * a33 - a23 * a31)
        dXdxI[2, 0, K] = a21 * a32 - a22 * a31
        dXdxI[0, 1, K] = -(a12 * a33 - a13 * a32)
        dXdxI[1, 1, K] = a11 * a33 - a13 * a31
        dXdxI[2, 1, K] = -(a11 * a32 - a12 * a31)
        dXdxI[0, 2, K] = a12 * a23 - a13 * a22
        dXdxI[1, 2, K] = -(a11 * a23 - a13 * a21)
        dXdxI[2, 2, K] = a11 * a22 - a12 * a21
    return np.asfortranarray(X), np.asfortranarray(dXdxI), np.asfortranarray(J)


def inverse_map(glob, numg):
    """Contributors (IF*DoF + ID) of each global DOF, ascending (CSR)."""
    DoF, NF = glob.shape
    g0 = (np.asarray(glob, order="F").T.ravel() - 1)          # index IF*DoF + ID
    order = np.argsort(g0, kind="stable")
    counts = np.bincount(g0, minlength=numg)
    ptr = np.zeros(numg + 1, np.int64)
    np.cumsum(counts, out=ptr[1:])
    return ptr, order


def mass_and_dz(glob, J, X, w, numg):
    """M (nz,NumG,2), MMass (nz,NumG) (src/DyCore/MassCG.jl:61-75) and dz
    (src/DyCore/DiscretizationCG.jl:119-144, last element written wins),
    summed over contributors in ascending (element, node) order."""
    DoF, _, nz, NF = J.shape
    N = int(round(np.sqrt(DoF)))
    ptr, order = inverse_map(glob, numg)
    IFs, IDs = order // DoF, order % DoF
    I, Jn = IDs % N, IDs // N
    J1 = J[IDs, 0, :, IFs]                 # (ncontrib, nz)
    J2 = J[IDs, 1, :, IFs]
    mm = 0.5 * (J1 + J2) * w[I][:, None] * w[Jn][:, None]
    M = np.zeros((nz, numg, 2), order="F")
    MM = np.zeros((nz, numg), order="F")
    maxc = int(np.max(np.diff(ptr)))
    for r in range(maxc):                  # sequential sum over the r-th contributor
        sel = np.nonzero(np.diff(ptr) > r)[0]
        q = ptr[sel] + r
        M[:, sel, 0] += J1[q].T
        M[:, sel, 1] += J2[q].T
        MM[:, sel] += mm[q].T
    last = ptr[1:] - 1                     # highest (element, node): written last
    xb = X[IDs[last], 0, :, :, IFs[last]]  # (numg, 3, nz)
    xt = X[IDs[last], 1, :, :, IFs[last]]
    r1 = np.sqrt(xb[:, 0] * xb[:, 0] + xb[:, 1] * xb[:, 1] + xb[:, 2] * xb[:, 2])
    r2 = np.sqrt(xt[:, 0] * xt[:, 0] + xt[:, 1] * xt[:, 1] + xt[:, 2] * xt[:, 2])
    dz = np.asfortranarray((r2 - r1).T)
    return M, MM, dz


@dataclass
class Grid:
    nPanel: int
    OrdPoly: int
    nz: int
    NF: int
    NumG: int
    NumNodes: int
    NumEdges: int
    Rad: float
    H: float
    z: np.ndarray
    glob: np.ndarray       # (N*N, NF) int64 1-based
    faces: np.ndarray      # (NF, 4, 3) corner coordinates
    xw: np.ndarray
    w: np.ndarray
    DS: np.ndarray
    DW: np.ndarray
    X: np.ndarray
    dXdxI: np.ndarray
    J: np.ndarray
    M: np.ndarray
    MMass: np.ndarray
    dz: np.ndarray


def init_grid_sphere(nPanel, OrdPoly, z, H, Rad):
    """Grid + element + metric for one process (InitGridSphere + InitSphere:
    src/Grids/InitGrid.jl:1-47, src/DyCore/InitDriver.jl:1-55)."""
    z = np.asarray(z, dtype=np.float64)
    FN, FE, EN, FP, nnodes, nedges = build_topology(nPanel, Rad)
    glob, numg = numbering_cg_quad(FN, FE, EN, nnodes, nedges, OrdPoly)
    xw, w, DS, DW = derivative_matrices(OrdPoly)
    X, dXdxI, J = metric_sphere(FP, xw, DS, z, H, Rad)
    M, MM, dz = mass_and_dz(glob, J, X, w, numg)
    return Grid(nPanel, OrdPoly, z.size - 1, FN.shape[0], numg, nnodes, nedges, Rad, H, z, glob, FP,
                xw, w, DS, DW, X, dXdxI, J, M, MM, dz)


def _fortran_tensor(shape, device):
    """A CUDA float64 tensor holding a Fortran-ordered array of `shape` (the
    tensor's own shape is reversed, contiguous)."""
    import torch
    return torch.empty(tuple(reversed(shape)), dtype=torch.float64, device=device)


def init_grid_sphere_device(nPanel, OrdPoly, z, H, Rad, device="cuda"):
    """init_grid_sphere with the floating-point arrays formed on the GPU: the
    topology and the Glob numbering on the host (integer work), the metric
    (cgd_metric_sphere) and the mass and dz (cgd_mass_dz) on the device.
    X, dXdxI, J, M, MMass and dz are CUDA tensors holding the reference's
    Fortran-ordered arrays (tensor shapes reversed).  The metric uses the
    device's trigonometric functions, so it agrees with init_grid_sphere to
    rounding."""
    from . import _lib
    z = np.asarray(z, dtype=np.float64)
    nz = z.size - 1
    FN, FE, EN, FP, nnodes, nedges = build_topology(nPanel, Rad)
    glob, numg = numbering_cg_quad(FN, FE, EN, nnodes, nedges, OrdPoly)
    xw, w, DS, DW = derivative_matrices(OrdPoly)
    NF, N = FN.shape[0], OrdPoly + 1
    DoF = N * N
    X = _fortran_tensor((DoF, 2, 3, nz, NF), device)
    dXdxI = _fortran_tensor((3, 3, 2, DoF, nz, NF), device)
    J = _fortran_tensor((DoF, 2, nz, NF), device)
    M = _fortran_tensor((nz, numg, 2), device)
    MM = _fortran_tensor((nz, numg), device)
    dz = _fortran_tensor((nz, numg), device)
    L = _lib.lib()
    fp = np.ascontiguousarray(FP, dtype=np.float64)
    dsf = np.asfortranarray(DS, dtype=np.float64)
    xw_, w_, z_ = (np.ascontiguousarray(a, dtype=np.float64) for a in (xw, w, z))
    _lib.check(L.cgd_metric_sphere(OrdPoly, nz, NF, fp.ctypes.data, xw_.ctypes.data, dsf.ctypes.data,
                                   z_.ctypes.data, float(H), float(Rad), X.data_ptr(), dXdxI.data_ptr(),
                                   J.data_ptr()), "cgd_metric_sphere")
    g64 = np.asfortranarray(glob, dtype=np.int64)
    _lib.check(L.cgd_mass_dz(OrdPoly, nz, NF, numg, g64.ctypes.data, w_.ctypes.data, J.data_ptr(), X.data_ptr(),
                             M.data_ptr(), MM.data_ptr(), dz.data_ptr()), "cgd_mass_dz")
    return Grid(nPanel, OrdPoly, nz, NF, numg, nnodes, nedges, Rad, H, z, glob, FP, xw, w, DS, DW,
                X, dXdxI, J, M, MM, dz)


def node_positions(grid):
    """(NumG, 2, 3, nz): the bottom and top positions of every column's nodes,
    taken from the highest-numbered element node holding the DOF (the one the
    reference's init kernels write last); works on host arrays and on the
    device tensors of init_grid_sphere_device."""
    DoF, numg = grid.glob.shape[0], grid.NumG
    g0 = np.asarray(grid.glob, order="F").T.ravel() - 1            # index IF*DoF + ID
    last = np.zeros(numg, np.int64)
    last[g0] = np.arange(g0.size)                                  # later writes overwrite
    IF, ID = last // DoF, last % DoF
    X = grid.X
    if isinstance(X, np.ndarray):
        return X[ID, :, :, :, IF]                                  # (numg, 2, 3, nz)
    import torch
    t = X[torch.as_tensor(IF, device=X.device), :, :, :, torch.as_tensor(ID, device=X.device)]   # (numg, nz, 3, 2)
    return t.permute(0, 3, 2, 1).cpu().numpy()
