// cgd_oracle.cpp - TEST INFRASTRUCTURE: FP64 CPU restatement of the
// CGDycore.jl nonhydrostatic spectral-element hot path.  Used only by the
// tests, by __graft_entry__.smoke() and by the CPU-baseline leg of bench.py,
// as the checker.  Never linked into the product library.
//
// Every function cites the reference file:line it restates (paths relative to
// the CGDycore.jl repository).  Floating-point operations are written in the
// reference's evaluation order (left-to-right, no contraction: build with
// -ffp-contract=off).  Where the reference sums through atomics in an
// unspecified order, this file uses one fixed order (documented at
// assemble_phase2) that the CUDA kernels reproduce.
//
// Pinning.  The global numbering (Glob) is pinned: it equals the reference's
// own golden file TestKernels/GlobInd (nPanel 30, p = 3) bit for bit
// (tests/golden/globind_n30_p3.json holds its digest).  The floating-point
// restatement (tendency, Jacobian, Schur solve, steps) is parity unpinned: the
// reference records no floating-point vectors for this path and cannot run
// here (no Julia), so it is checked by analytic invariants only (resting
// atmosphere, mass conservation, the Schur solve inverting its operator).
#include "cgd_oracle.h"
#include "../include/cgd_math.h"
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

const double PI = 3.141592653589793;

// ---------------------------------------------------------------------------
// Physical constants: src/DyCore/GlobalVariables.jl:188-230 (PhysParameters),
// with RadEarth taken from the configuration (the grid radius and
// Phys.RadEarth are one parameter here).
// ---------------------------------------------------------------------------
struct Phys {
  double RadEarth, Grav, Cpd, Cvd, Rd, p0, kappa, Omega;
  Phys(double rad) {
    RadEarth = rad;
    Grav = 9.80616;
    Cpd = 1004.0;
    Cvd = 717.0;
    Rd = Cpd - Cvd;
    p0 = 1.0e5;
    kappa = Rd / Cpd;
    Omega = 2.0 * PI / 24.0 / 3600.0;
  }
};

// ---------------------------------------------------------------------------
// Grid topology: restatement of src/Grids/{CubedGrid,Face,Edge,Orientation,
// Renumbering,SubGridGhost}.jl.  1-based indices throughout, as in Julia.
// ---------------------------------------------------------------------------
struct GNode { double P[3]; int N; };
struct GEdge { int N[2]; int E; int EI; int NumF; int F[2]; int FE[2]; };
struct GFace { int N[4]; int E[4]; double P[4][3]; int Orientation; int OrientE[4]; };

struct Topo {
  std::vector<GNode> nodes;  // 1..NumNodes
  std::vector<GEdge> edges;  // 1..NumEdges
  std::vector<GFace> faces;  // 1..NumFaces
};

// CubePoint: src/Grids/CubedGrid.jl:377-391
static void cube_point(int i1, int i2, int i3, int n, double x, double y, double z,
                       double Rad, double *P)
{
  if (i1 > 0) x = std::tan((double)i1 * PI / (double)(2 * n) - 0.25 * PI);
  if (i2 > 0) y = std::tan((double)i2 * PI / (double)(2 * n) - 0.25 * PI);
  if (i3 > 0) z = std::tan((double)i3 * PI / (double)(2 * n) - 0.25 * PI);
  double nrm = std::sqrt(x * x + y * y + z * z);
  P[0] = x / nrm * Rad;
  P[1] = y / nrm * Rad;
  P[2] = z / nrm * Rad;
}

// Edge constructor (topology part): src/Grids/Edge.jl:57-94
static void make_edge(Topo &T, int num, int N1, int N2)
{
  GEdge &e = T.edges[num];
  e.N[0] = N1; e.N[1] = N2;
  e.E = num; e.EI = num;
  e.NumF = 0; e.F[0] = e.F[1] = 0;
  e.FE[0] = e.FE[1] = 0;
}

static void cross3(const double *a, const double *b, double *c)
{
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}

// Face constructor: src/Grids/Face.jl:48-167 (quad, ChangeOrient = 3)
static void make_face(Topo &T, const int *Ein, int Pos, double Rad)
{
  int EdgesF[4] = {Ein[0], Ein[1], Ein[2], Ein[3]};
  GFace &F = T.faces[Pos];
  for (int iE = 0; iE < 4; ++iE) {       // Face.jl:59-62
    GEdge &e = T.edges[EdgesF[iE]];
    e.NumF += 1;
    e.F[e.NumF - 1] = Pos;
  }
  F.E[0] = EdgesF[0];                    // Face.jl:64-83 sort edges into a cycle
  int N2 = T.edges[F.E[0]].N[1];
  for (int iE = 1; iE < 4; ++iE) {
    for (int iE1 = iE; iE1 < 4; ++iE1) {
      const GEdge &e1 = T.edges[EdgesF[iE1]];
      if (N2 == e1.N[0]) {
        F.E[iE] = EdgesF[iE1];
        N2 = e1.N[1];
        EdgesF[iE1] = EdgesF[iE];
        EdgesF[iE] = F.E[iE];
        break;
      } else if (N2 == e1.N[1]) {
        F.E[iE] = EdgesF[iE1];
        N2 = e1.N[0];
        EdgesF[iE1] = EdgesF[iE];
        EdgesF[iE] = F.E[iE];
        break;
      }
    }
  }
  F.N[0] = T.edges[F.E[0]].N[0];          // Face.jl:84-92
  F.N[1] = T.edges[F.E[0]].N[1];
  for (int iE = 1; iE < 3; ++iE) {
    if (F.N[iE] == T.edges[F.E[iE]].N[0]) F.N[iE + 1] = T.edges[F.E[iE]].N[1];
    else F.N[iE + 1] = T.edges[F.E[iE]].N[0];
  }
  for (int i = 0; i < 4; ++i)
    for (int c = 0; c < 3; ++c) F.P[i][c] = T.nodes[F.N[i]].P[c];
  double Mid[3] = {0, 0, 0};              // Face.jl:114-126
  for (int i = 0; i < 4; ++i)
    for (int c = 0; c < 3; ++c) Mid[c] = Mid[c] + F.P[i][c];
  for (int c = 0; c < 3; ++c) Mid[c] = Mid[c] / 4.0;
  double nm = std::sqrt(Mid[0] * Mid[0] + Mid[1] * Mid[1] + Mid[2] * Mid[2]);
  for (int c = 0; c < 3; ++c) Mid[c] = Mid[c] / nm * Rad;
  double n[3], t[3];                      // Face.jl:133-138
  cross3(F.P[3], F.P[0], n);
  for (int i = 0; i < 3; ++i) {
    cross3(F.P[i], F.P[i + 1], t);
    for (int c = 0; c < 3; ++c) n[c] = n[c] + t[c];
  }
  double nn = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
  for (int c = 0; c < 3; ++c) n[c] = n[c] / nn;
  F.Orientation = 1;
  // OrientFaceSphere = dot(n, Mid): src/Grids/OrientFaceSphere.jl:1-4
  double orient = n[0] * Mid[0] + n[1] * Mid[1] + n[2] * Mid[2];
  if (orient < 0) {                       // Face.jl:139-156 (4 > ChangeOrient)
    int NT[4], ET[4];
    double PT[4][3];
    memcpy(NT, F.N, sizeof NT);
    memcpy(ET, F.E, sizeof ET);
    memcpy(PT, F.P, sizeof PT);
    for (int i = 0; i < 4; ++i) {
      F.N[i] = NT[3 - i];
      for (int c = 0; c < 3; ++c) F.P[i][c] = PT[3 - i][c];
    }
    for (int i = 0; i < 3; ++i) F.E[i] = ET[2 - i];
    F.Orientation = 1;
  }
  for (int i = 0; i < 4; ++i)
    F.OrientE[i] = (T.edges[F.E[i]].N[0] == F.N[i]) ? F.Orientation : -F.Orientation;
}

// InsertFaceEdge: src/Grids/CubedGrid.jl:393-441
static void insert_face_edge(Topo &T, int n, int &EdgeNumber, int NodeNumberStart,
                             int E1S1, int E2S1, int E1S2, int E2S2,
                             int &Start1, int &Start2)
{
  int NodeNumber = NodeNumberStart, NE1 = E1S1, NE2 = E2S1;
  Start1 = EdgeNumber;
  for (int j = 1; j <= n - 1; ++j)
    for (int i = 1; i <= n; ++i) {
      int N1 = NodeNumber - 1, N2 = NodeNumber;
      if (i == 1) { N1 = NE1; NE1 += 1; }
      if (i == n) { N2 = NE2; NE2 += 1; NodeNumber -= 1; }
      make_edge(T, EdgeNumber, N1, N2);
      EdgeNumber += 1;
      NodeNumber += 1;
    }
  NodeNumber = NodeNumberStart; NE1 = E1S2; NE2 = E2S2;
  Start2 = EdgeNumber;
  for (int j = 1; j <= n; ++j)
    for (int i = 1; i <= n - 1; ++i) {
      int N1 = NodeNumber - (n - 1), N2 = NodeNumber;
      if (j == 1) { N1 = NE1; NE1 += 1; }
      if (j == n) { N2 = NE2; NE2 += 1; }
      make_edge(T, EdgeNumber, N1, N2);
      EdgeNumber += 1;
      NodeNumber += 1;
    }
}

// InsertEdgeEdge: src/Grids/CubedGrid.jl:443-462
static int insert_edge_edge(Topo &T, int n, int &EdgeNumber, int NodeNumberStart, int E1, int E2)
{
  int NodeNumber = NodeNumberStart, start = EdgeNumber;
  for (int i = 1; i <= n; ++i) {
    int N1 = NodeNumber - 1, N2 = NodeNumber;
    if (i == 1) N1 = E1;
    if (i == n) N2 = E2;
    make_edge(T, EdgeNumber, N1, N2);
    EdgeNumber += 1;
    NodeNumber += 1;
  }
  return start;
}

// InsertFaceFace: src/Grids/CubedGrid.jl:464-513
static void insert_face_face(Topo &T, int n, int &FaceNumber, int S1, int S2,
                             int EW1, int EW2, int SN1, int SN2, double Rad)
{
  int EdgeNumber1 = S1, EdgeNumber2 = S2;
  for (int j = 1; j <= n; ++j)
    for (int i = 1; i <= n; ++i) {
      int E[4] = {EdgeNumber1 - n, EdgeNumber1, EdgeNumber2 - 1, EdgeNumber2};
      if (j == 1) { E[0] = EW1; EW1 += 1; }
      if (j == n) { E[1] = EW2; EW2 += 1; }
      if (i == 1) { E[2] = SN1; SN1 += 1; }
      if (i == n) { E[3] = SN2; SN2 += 1; EdgeNumber2 -= 1; }
      EdgeNumber1 += 1;
      EdgeNumber2 += 1;
      make_face(T, E, FaceNumber, Rad);
      FaceNumber += 1;
    }
}

static int edge_direction(int N1, int N2, const int *E)
{
  (void)N2;
  return (N1 == E[0]) ? 1 : -1;           // Orientation.jl:90-97
}

// Orientation!/Orient: src/Grids/Orientation.jl:1-88.  The edge face list is
// a Vector, so size(Edges[iE].F,2) == 1 and the while loop runs exactly once.
static void orientation(Topo &T)
{
  int NumEdges = (int)T.edges.size() - 1;
  std::vector<int> Visit(NumEdges + 1, 0);
  for (int iE0 = 1; iE0 <= NumEdges; ++iE0) {
    int iE = iE0;
    if (Visit[iE] == 1) continue;
    Visit[iE] = 1;
    int iF1 = T.edges[iE].F[0];
    int iE1 = 4;
    for (int l = 1; l <= 4; ++l) { iE1 = l; if (iE == T.faces[iF1].E[l - 1]) break; }
    int NF[5];
    for (int l = 0; l < 4; ++l) NF[l] = T.faces[iF1].N[l];
    NF[4] = NF[0];
    int o = edge_direction(NF[iE1 - 1], NF[iE1], T.edges[iE].N);
    int iEP1 = iE1 + 2;
    if (iEP1 > 4) iEP1 -= 4;
    int iEP = T.faces[iF1].E[iEP1 - 1];
    if (edge_direction(NF[iEP1 - 1], NF[iEP1], T.edges[iEP].N) == o) {
      if (o == -1) { T.edges[iEP].N[0] = NF[iEP1 - 1]; T.edges[iEP].N[1] = NF[iEP1]; }
      else { T.edges[iEP].N[0] = NF[iEP1]; T.edges[iEP].N[1] = NF[iEP1 - 1]; }
    }
    Visit[iEP] = 1;
  }
}

// RenumberingFace4! + PosEdgeInFace!: src/Grids/Renumbering.jl:10-93
static void renumbering(Topo &T)
{
  int NF = (int)T.faces.size() - 1, NE = (int)T.edges.size() - 1;
  for (int iF = 1; iF <= NF; ++iF) {
    GFace &F = T.faces[iF];
    int iN = 4, num = 0;
    for (int l = 1; l <= 4; ++l) {
      iN = l;
      int Nn = F.N[l - 1];
      num = 0;
      for (int iE = 0; iE < 4; ++iE) {
        if (Nn == T.edges[F.E[iE]].N[0]) num += 1;
        if (num == 2) break;
      }
      if (num == 2) break;
    }
    if (iN > 1) {
      int NT[8], ET[8];
      double PT[8][3];
      for (int l = 0; l < 8; ++l) {
        NT[l] = F.N[l % 4]; ET[l] = F.E[l % 4];
        for (int c = 0; c < 3; ++c) PT[l][c] = F.P[l % 4][c];
      }
      for (int l = 0; l < 4; ++l) {
        F.N[l] = NT[l + iN - 1]; F.E[l] = ET[l + iN - 1];
        for (int c = 0; c < 3; ++c) F.P[l][c] = PT[l + iN - 1][c];
      }
    }
    for (int l = 0; l < 4; ++l)
      F.OrientE[l] = (T.edges[F.E[l]].N[0] == F.N[l]) ? 1 : -1;
  }
  for (int iE = 1; iE <= NE; ++iE) {
    GEdge &e = T.edges[iE];
    e.FE[0] = e.FE[1] = 0;
    for (int i = 0; i < 2; ++i) {
      int iF = e.F[i];
      if (iF > 0)
        for (int l = 1; l <= 4; ++l)
          if (e.EI == T.edges[T.faces[iF].E[l - 1]].EI) { e.FE[i] = l; break; }
    }
    if (e.FE[0] > e.FE[1]) {
      std::swap(e.FE[0], e.FE[1]);
      std::swap(e.F[0], e.F[1]);
    }
  }
}

// CubedGrid: src/Grids/CubedGrid.jl:1-375 (order = true)
static Topo cubed_grid(int n, double Rad)
{
  Topo T;
  int NumNodes = 6 * (n - 1) * (n - 1) + 12 * (n - 1) + 8;
  int NumEdges = 12 * (n - 1) * n + 12 * n;
  int NumFaces = 6 * n * n;
  T.nodes.resize(NumNodes + 1);
  T.edges.resize(NumEdges + 1);
  T.faces.resize(NumFaces + 1);
  int NodeNumber = 1;
  auto put = [&](int i1, int i2, int i3, double x, double y, double z) {
    cube_point(i1, i2, i3, n, x, y, z, Rad, T.nodes[NodeNumber].P);
    T.nodes[NodeNumber].N = NodeNumber;
    NodeNumber += 1;
  };
  int W = NodeNumber;
  for (int k = 1; k <= n - 1; ++k) for (int j = 1; j <= n - 1; ++j) put(-1, j, k, -1.0, 0.0, 0.0);
  int E = NodeNumber;
  for (int k = 1; k <= n - 1; ++k) for (int j = 1; j <= n - 1; ++j) put(-1, j, k, 1.0, 0.0, 0.0);
  int S = NodeNumber;
  for (int k = 1; k <= n - 1; ++k) for (int i = 1; i <= n - 1; ++i) put(i, -1, k, 0.0, -1.0, 0.0);
  int Nn = NodeNumber;
  for (int k = 1; k <= n - 1; ++k) for (int i = 1; i <= n - 1; ++i) put(i, -1, k, 0.0, 1.0, 0.0);
  int B = NodeNumber;
  for (int j = 1; j <= n - 1; ++j) for (int i = 1; i <= n - 1; ++i) put(i, j, -1, 0.0, 0.0, -1.0);
  int Tp = NodeNumber;
  for (int j = 1; j <= n - 1; ++j) for (int i = 1; i <= n - 1; ++i) put(i, j, -1, 0.0, 0.0, 1.0);
  int WEmm = NodeNumber; for (int i = 1; i <= n - 1; ++i) put(i, -1, -1, 0.0, -1.0, -1.0);
  int WEpm = NodeNumber; for (int i = 1; i <= n - 1; ++i) put(i, -1, -1, 0.0, 1.0, -1.0);
  int WEmp = NodeNumber; for (int i = 1; i <= n - 1; ++i) put(i, -1, -1, 0.0, -1.0, 1.0);
  int WEpp = NodeNumber; for (int i = 1; i <= n - 1; ++i) put(i, -1, -1, 0.0, 1.0, 1.0);
  int SNmm = NodeNumber; for (int j = 1; j <= n - 1; ++j) put(-1, j, -1, -1.0, 0.0, -1.0);
  int SNpm = NodeNumber; for (int j = 1; j <= n - 1; ++j) put(-1, j, -1, 1.0, 0.0, -1.0);
  int SNmp = NodeNumber; for (int j = 1; j <= n - 1; ++j) put(-1, j, -1, -1.0, 0.0, 1.0);
  int SNpp = NodeNumber; for (int j = 1; j <= n - 1; ++j) put(-1, j, -1, 1.0, 0.0, 1.0);
  int BTmm = NodeNumber; for (int k = 1; k <= n - 1; ++k) put(-1, -1, k, -1.0, -1.0, 0.0);
  int BTpm = NodeNumber; for (int k = 1; k <= n - 1; ++k) put(-1, -1, k, 1.0, -1.0, 0.0);
  int BTmp = NodeNumber; for (int k = 1; k <= n - 1; ++k) put(-1, -1, k, -1.0, 1.0, 0.0);
  int BTpp = NodeNumber; for (int k = 1; k <= n - 1; ++k) put(-1, -1, k, 1.0, 1.0, 0.0);
  int mmm = NodeNumber; put(-1, -1, -1, -1.0, -1.0, -1.0);
  int pmm = NodeNumber; put(-1, -1, -1, 1.0, -1.0, -1.0);
  int mpm = NodeNumber; put(-1, -1, -1, -1.0, 1.0, -1.0);
  int ppm = NodeNumber; put(-1, -1, -1, 1.0, 1.0, -1.0);
  int mmp = NodeNumber; put(-1, -1, -1, -1.0, -1.0, 1.0);
  int pmp = NodeNumber; put(-1, -1, -1, 1.0, -1.0, 1.0);
  int mpp = NodeNumber; put(-1, -1, -1, -1.0, 1.0, 1.0);
  int ppp = NodeNumber; put(-1, -1, -1, 1.0, 1.0, 1.0);

  int EN = 1;
  int W1, W2, E1, E2, S1, S2, N1, N2, B1, B2, T1, T2;
  insert_face_edge(T, n, EN, W, BTmm, BTmp, SNmm, SNmp, W1, W2);
  insert_face_edge(T, n, EN, E, BTpm, BTpp, SNpm, SNpp, E1, E2);
  insert_face_edge(T, n, EN, S, BTmm, BTpm, WEmm, WEmp, S1, S2);
  insert_face_edge(T, n, EN, Nn, BTmp, BTpp, WEpm, WEpp, N1, N2);
  insert_face_edge(T, n, EN, B, SNmm, SNpm, WEmm, WEpm, B1, B2);
  insert_face_edge(T, n, EN, Tp, SNmp, SNpp, WEmp, WEpp, T1, T2);
  int eWEmm = insert_edge_edge(T, n, EN, WEmm, mmm, pmm);
  int eWEpm = insert_edge_edge(T, n, EN, WEpm, mpm, ppm);
  int eWEmp = insert_edge_edge(T, n, EN, WEmp, mmp, pmp);
  int eWEpp = insert_edge_edge(T, n, EN, WEpp, mpp, ppp);
  int eSNmm = insert_edge_edge(T, n, EN, SNmm, mmm, mpm);
  int eSNpm = insert_edge_edge(T, n, EN, SNpm, pmm, ppm);
  int eSNmp = insert_edge_edge(T, n, EN, SNmp, mmp, mpp);
  int eSNpp = insert_edge_edge(T, n, EN, SNpp, pmp, ppp);
  int eBTmm = insert_edge_edge(T, n, EN, BTmm, mmm, mmp);
  int eBTpm = insert_edge_edge(T, n, EN, BTpm, pmm, pmp);
  int eBTmp = insert_edge_edge(T, n, EN, BTmp, mpm, mpp);
  int eBTpp = insert_edge_edge(T, n, EN, BTpp, ppm, ppp);

  int FN = 1;
  insert_face_face(T, n, FN, W1, W2, eSNmm, eSNmp, eBTmm, eBTmp, Rad);
  insert_face_face(T, n, FN, E1, E2, eSNpm, eSNpp, eBTpm, eBTpp, Rad);
  insert_face_face(T, n, FN, S1, S2, eWEmm, eWEmp, eBTmm, eBTpm, Rad);
  insert_face_face(T, n, FN, N1, N2, eWEpm, eWEpp, eBTmp, eBTpp, Rad);
  insert_face_face(T, n, FN, B1, B2, eWEmm, eWEpm, eSNmm, eSNpm, Rad);
  insert_face_face(T, n, FN, T1, T2, eWEmp, eWEpp, eSNmp, eSNpp, Rad);

  orientation(T);
  renumbering(T);
  return T;
}

// ConstructSubGridGhost for a single process (all faces inner):
// src/Grids/SubGridGhost.jl:1-162.  Nodes and edges are renumbered in order of
// first appearance over the faces (unique/setdiff keep first appearance),
// faces keep their numbers, then Renumbering! runs again.
static Topo sub_grid_single(const Topo &G)
{
  int NF = (int)G.faces.size() - 1;
  int NN = (int)G.nodes.size() - 1, NE = (int)G.edges.size() - 1;
  std::vector<int> nodeNew(NN + 1, 0), edgeNew(NE + 1, 0);
  std::vector<int> nodeOrder, edgeOrder;
  for (int iF = 1; iF <= NF; ++iF)
    for (int i = 0; i < 4; ++i) {
      int e = G.faces[iF].E[i], nd = G.faces[iF].N[i];
      if (!edgeNew[e]) { edgeOrder.push_back(e); edgeNew[e] = (int)edgeOrder.size(); }
      if (!nodeNew[nd]) { nodeOrder.push_back(nd); nodeNew[nd] = (int)nodeOrder.size(); }
    }
  Topo S;
  S.nodes.resize(nodeOrder.size() + 1);
  S.edges.resize(edgeOrder.size() + 1);
  S.faces.resize(NF + 1);
  for (size_t i = 1; i <= nodeOrder.size(); ++i) {
    S.nodes[i] = G.nodes[nodeOrder[i - 1]];
    S.nodes[i].N = (int)i;
  }
  for (size_t i = 1; i <= edgeOrder.size(); ++i) {
    S.edges[i] = G.edges[edgeOrder[i - 1]];   // EI keeps the global number
    S.edges[i].E = (int)i;
    S.edges[i].N[0] = nodeNew[S.edges[i].N[0]];
    S.edges[i].N[1] = nodeNew[S.edges[i].N[1]];
  }
  for (int iF = 1; iF <= NF; ++iF) {
    S.faces[iF] = G.faces[iF];
    for (int j = 0; j < 4; ++j) {
      S.faces[iF].E[j] = edgeNew[S.faces[iF].E[j]];
      S.faces[iF].N[j] = nodeNew[S.faces[iF].N[j]];
    }
  }
  renumbering(S);
  return S;
}

// NumberingFemCGQuad: src/DyCore/NumberingFem.jl:21-105 (PolyOrd 1..4)
static std::vector<int> numbering_fem_cg_quad(const Topo &S, int p, int &NumG)
{
  static const int Per1[] = {1, 2, 4, 3};
  static const int Per2[] = {1, 5, 2, 8, 9, 6, 4, 7, 3};
  static const int Per3[] = {1, 5, 6, 2, 12, 13, 14, 7, 11, 15, 16, 8, 4, 10, 9, 3};
  static const int Per4[] = {1, 5, 6, 7, 2, 16, 17, 18, 19, 8, 15, 20, 21, 22, 9,
                             14, 23, 24, 25, 10, 4, 13, 12, 11, 3};
  const int *Per = p == 1 ? Per1 : p == 2 ? Per2 : p == 3 ? Per3 : Per4;
  int N = p + 1, DoF = N * N;
  int NF = (int)S.faces.size() - 1;
  int NumGlobN = (int)S.nodes.size() - 1;
  int NumGlobE = ((int)S.edges.size() - 1) * (p - 1);
  int NumGlobF = NF * (p - 1) * (p - 1);
  NumG = NumGlobN + NumGlobE + NumGlobF;
  std::vector<int> glob((size_t)DoF * NF);
  std::vector<int> loc(DoF);
  for (int iF = 1; iF <= NF; ++iF) {
    const GFace &F = S.faces[iF];
    int ii = 0;
    for (int i = 0; i < 4; ++i) loc[ii++] = S.nodes[F.N[i]].N;
    for (int i = 0; i < 4; ++i) {
      int iE = F.E[i];
      if (S.edges[iE].N[0] == F.N[i]) {
        for (int j = 1; j <= p - 1; ++j) loc[ii++] = (S.edges[iE].E - 1) * (p - 1) + j + NumGlobN;
      } else {
        for (int j = p - 1; j >= 1; --j) loc[ii++] = (S.edges[iE].E - 1) * (p - 1) + j + NumGlobN;
      }
    }
    for (int j = 1; j <= p - 1; ++j)
      for (int i = 1; i <= p - 1; ++i)
        loc[ii++] = NumGlobN + NumGlobE + i + (j - 1) * (p - 1) + (iF - 1) * (p - 1) * (p - 1);
    for (int ID = 0; ID < DoF; ++ID) glob[ID + (size_t)DoF * (iF - 1)] = loc[Per[ID] - 1];
  }
  return glob;
}

// GLL nodes/weights (FastGaussQuadrature.gausslobatto, closed forms for p<=4)
static void gll(int p, std::vector<double> &x, std::vector<double> &w)
{
  x.assign(p + 1, 0.0); w.assign(p + 1, 0.0);
  if (p == 1) { x = {-1.0, 1.0}; w = {1.0, 1.0}; }
  else if (p == 2) { x = {-1.0, 0.0, 1.0}; w = {1.0 / 3.0, 4.0 / 3.0, 1.0 / 3.0}; }
  else if (p == 3) {
    double a = std::sqrt(1.0 / 5.0);
    x = {-1.0, -a, a, 1.0}; w = {1.0 / 6.0, 5.0 / 6.0, 5.0 / 6.0, 1.0 / 6.0};
  } else {
    double a = std::sqrt(3.0 / 7.0);
    x = {-1.0, -a, 0.0, a, 1.0};
    w = {1.0 / 10.0, 49.0 / 90.0, 32.0 / 45.0, 49.0 / 90.0, 1.0 / 10.0};
  }
}

// DLagrange: src/DG/DLagrange.jl:1-10
static double dlagrange(double x, const std::vector<double> &xP, int iP)
{
  double Df = 0.0, f = 1.0;
  for (int i = 0; i < (int)xP.size(); ++i)
    if (i != iP) {
      Df = Df * (x - xP[i]) / (xP[iP] - xP[i]) + f / (xP[iP] - xP[i]);
      f = f * (x - xP[i]) / (xP[iP] - xP[i]);
    }
  return Df;
}

// ---------------------------------------------------------------------------
struct Model {
  int n, p, N, DoF, nz, NF, NumG, NumTr, NV, NumNodes, NumEdges;
  double Rad, H, nuCurl, nuGrad, nuDiv, Up;
  Phys phys{6.371e6};
  std::vector<double> z;
  std::vector<int> glob;                // 0-based global ids
  std::vector<double> xw, w, DS, DW;    // DS[i + N*j] = DS[i,j]
  std::vector<double> faceP;            // (4,3,NF)
  std::vector<double> X, dXdxI, J, M, MMass, dz;
  std::vector<double> fcor;             // (DoF, nz, NF) 2*Omega*sinlat at layer midpoints
  std::vector<int> inv_ptr, inv_idx;    // contributors (IF*DoF+ID) of each global id
  std::vector<double> bands;            // JRhoW, JWRho, JWRhoTh, JRhoThW (2, nz-1, NumG) each
  double rk_a[3][3], rk_c[3][3], rk_m[3], rk_gamma;
  // column physics in the tendency tail (off unless orc_set_physics)
  int held_suarez = 0, damping = 0;
  double hs[8] = {};                    // k_a, k_f, k_s, DeltaT_y, DeltaTh_z, T_equator, T_min, sigma_b
  std::vector<double> coslat, sinlat;   // (NumG) of the surface node
  std::vector<double> dampc;            // (nz, NumG) Relax sin^2(...) above H - StrideDamp, else 0
};

inline double &DXI(Model &m, int a, int b, int K, int ID, int Iz, int IF)
{
  return m.dXdxI[(size_t)(a - 1) + 3 * ((b - 1) + 3 * (K + 2 * (ID + (size_t)m.DoF * (Iz + (size_t)m.nz * IF))))];
}
inline double JJ(const Model &m, int ID, int K, int Iz, int IF)
{
  return m.J[ID + (size_t)m.DoF * (K + 2 * (Iz + (size_t)m.nz * IF))];
}
inline double XX(const Model &m, int ID, int K, int c, int Iz, int IF)
{
  return m.X[ID + (size_t)m.DoF * (K + 2 * (c + 3 * (Iz + (size_t)m.nz * IF)))];
}

// JacobiSphere3Kernel!: src/Grids/JacobiSphere3GPU.jl:102-215 with the Sleve
// height (src/Grids/Adapt.jl:19-31, zs = 0) and Det3 (JacobiSphere3GPU.jl:413).
static void build_metric(Model &m)
{
  int N = m.N, DoF = m.DoF, nz = m.nz, NF = m.NF;
  m.X.assign((size_t)DoF * 2 * 3 * nz * NF, 0.0);
  m.dXdxI.assign((size_t)9 * 2 * DoF * nz * NF, 0.0);
  m.J.assign((size_t)DoF * 2 * nz * NF, 0.0);
  double xwZ[2] = {-1.0, 1.0};
  double Rad = m.Rad, H = m.H;
  #pragma omp parallel for schedule(static)
  for (int IF = 0; IF < NF; ++IF) {
    const double *F = &m.faceP[(size_t)12 * IF];   // F[corner + 4*c]
    auto Fc = [&](int corner, int c) { return F[corner + 4 * c]; };
    std::vector<double> hR((size_t)2 * nz), dloc((size_t)DoF * 4);
    for (int Iz = 0; Iz < nz; ++Iz) {
      for (int K = 0; K < 2; ++K) {
        double zLoc = 0.5 * ((1.0 - xwZ[K]) * m.z[Iz] + (1.0 + xwZ[K]) * m.z[Iz + 1]);
        double eta = zLoc / H;
        double hh;
        if (eta <= 0.7) hh = eta * H + 0.0 * std::sinh((0.7 - eta) / 0.8 / 0.7) / std::sinh(1.0 / 0.8);
        else hh = eta * H;
        hR[K + 2 * Iz] = hh;
      }
    }
    for (int Jn = 0; Jn < N; ++Jn)
      for (int In = 0; In < N; ++In) {
        int ID = In + N * Jn;
        double ksi1 = m.xw[In], ksi2 = m.xw[Jn];
        double Xc[3];
        for (int c = 0; c < 3; ++c)
          Xc[c] = 0.25 * (Fc(0, c) * (1.0 - ksi1) * (1.0 - ksi2) + Fc(1, c) * (1.0 + ksi1) * (1.0 - ksi2) +
                          Fc(2, c) * (1.0 + ksi1) * (1.0 + ksi2) + Fc(3, c) * (1.0 - ksi1) * (1.0 + ksi2));
        double r = std::sqrt(Xc[0] * Xc[0] + Xc[1] * Xc[1] + Xc[2] * Xc[2]);
        double f = Rad / r;
        for (int Iz = 0; Iz < nz; ++Iz)
          for (int K = 0; K < 2; ++K)
            for (int c = 0; c < 3; ++c)
              m.X[ID + (size_t)DoF * (K + 2 * (c + 3 * (Iz + (size_t)nz * IF)))] = Xc[c] / r * (Rad + hR[K + 2 * Iz]);
        // cart2sphere: src/Grids/geometry_circle.jl:21-44
        double rr = std::sqrt(Xc[0] * Xc[0] + Xc[1] * Xc[1] + Xc[2] * Xc[2]);
        double theta = std::asin(Xc[2] / rr);
        double lam = std::atan2(Xc[1], Xc[0]);
        if (Xc[1] < 0.0) lam = lam + 2.0 * PI;
        double DD[2][3] = {{-std::sin(lam), std::cos(lam), 0.0}, {0.0, 0.0, 1.0}};
        double sinlam = std::sin(lam), coslam = std::cos(lam);
        double sinth = std::sin(theta), costh = std::cos(theta);
        double A[3][3];
        A[0][0] = sinlam * sinlam * costh * costh + sinth * sinth;
        A[0][1] = -sinlam * coslam * costh * costh;
        A[0][2] = -coslam * sinth * costh;
        A[1][0] = A[0][1];
        A[1][1] = coslam * coslam * costh * costh + sinth * sinth;
        A[1][2] = -sinlam * sinth * costh;
        A[2][0] = -coslam * sinth;
        A[2][1] = -sinlam * sinth;
        A[2][2] = costh;
        double Bm[3][4];
        for (int c = 0; c < 3; ++c)
          for (int k = 0; k < 4; ++k) Bm[c][k] = Fc(k, c);
        double C[4][2] = {{-1.0 + ksi2, -1.0 + ksi1}, {1.0 - ksi2, -1.0 - ksi1},
                          {1.0 + ksi2, 1.0 + ksi1}, {-1.0 - ksi2, 1.0 - ksi1}};
        // (((((1/4*f)*DD)*A)*B)*C), products summed left to right
        double t = 0.25 * f;
        double T1[2][3], T2[2][3], T3[2][4], T4[2][2];
        for (int i = 0; i < 2; ++i) for (int j = 0; j < 3; ++j) T1[i][j] = t * DD[i][j];
        for (int i = 0; i < 2; ++i) for (int j = 0; j < 3; ++j)
          T2[i][j] = T1[i][0] * A[0][j] + T1[i][1] * A[1][j] + T1[i][2] * A[2][j];
        for (int i = 0; i < 2; ++i) for (int j = 0; j < 4; ++j)
          T3[i][j] = T2[i][0] * Bm[0][j] + T2[i][1] * Bm[1][j] + T2[i][2] * Bm[2][j];
        for (int i = 0; i < 2; ++i) for (int j = 0; j < 2; ++j)
          T4[i][j] = T3[i][0] * C[0][j] + T3[i][1] * C[1][j] + T3[i][2] * C[2][j] + T3[i][3] * C[3][j];
        for (int i = 0; i < 2; ++i) for (int j = 0; j < 2; ++j) dloc[(size_t)ID * 4 + i + 2 * j] = T4[i][j];
      }
    for (int Iz = 0; Iz < nz; ++Iz)
      for (int K = 0; K < 2; ++K)
        for (int Jn = 0; Jn < N; ++Jn)
          for (int In = 0; In < N; ++In) {
            int ID = In + N * Jn;
            double h = hR[K + 2 * Iz];
            double DxhR = m.DS[In + N * 0] * h, DyhR = m.DS[Jn + N * 0] * h;
            for (int k = 1; k < N; ++k) {
              DxhR += m.DS[In + N * k] * h;
              DyhR += m.DS[Jn + N * k] * h;
            }
            double DzhR = 0.5 * (hR[1 + 2 * Iz] - hR[0 + 2 * Iz]);
            double A[3][3];
            A[0][0] = dloc[(size_t)ID * 4 + 0]; A[1][0] = dloc[(size_t)ID * 4 + 1];
            A[0][1] = dloc[(size_t)ID * 4 + 2]; A[1][1] = dloc[(size_t)ID * 4 + 3];
            A[0][2] = 0.0; A[1][2] = 0.0;
            A[2][0] = DxhR; A[2][1] = DyhR; A[2][2] = DzhR;
            double det = A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) -
                         A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
                         A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
            m.J[ID + (size_t)DoF * (K + 2 * (Iz + (size_t)nz * IF))] = det;
            DXI(m, 1, 1, K, ID, Iz, IF) = A[1][1] * A[2][2] - A[1][2] * A[2][1];
            DXI(m, 2, 1, K, ID, Iz, IF) = -(A[1][0] * A[2][2] - A[1][2] * A[2][0]);
            DXI(m, 3, 1, K, ID, Iz, IF) = A[1][0] * A[2][1] - A[1][1] * A[2][0];
            DXI(m, 1, 2, K, ID, Iz, IF) = -(A[0][1] * A[2][2] - A[0][2] * A[2][1]);
            DXI(m, 2, 2, K, ID, Iz, IF) = A[0][0] * A[2][2] - A[0][2] * A[2][0];
            DXI(m, 3, 2, K, ID, Iz, IF) = -(A[0][0] * A[2][1] - A[0][1] * A[2][0]);
            DXI(m, 1, 3, K, ID, Iz, IF) = A[0][1] * A[1][2] - A[0][2] * A[1][1];
            DXI(m, 2, 3, K, ID, Iz, IF) = -(A[0][0] * A[1][2] - A[0][2] * A[1][0]);
            DXI(m, 3, 3, K, ID, Iz, IF) = A[0][0] * A[1][1] - A[0][1] * A[1][0];
          }
  }
}

static void build_inverse_map(Model &m)
{
  m.inv_ptr.assign(m.NumG + 1, 0);
  for (int IF = 0; IF < m.NF; ++IF)
    for (int ID = 0; ID < m.DoF; ++ID) m.inv_ptr[m.glob[ID + (size_t)m.DoF * IF] + 1] += 1;
  for (int g = 0; g < m.NumG; ++g) m.inv_ptr[g + 1] += m.inv_ptr[g];
  m.inv_idx.assign(m.inv_ptr[m.NumG], 0);
  std::vector<int> fill(m.inv_ptr.begin(), m.inv_ptr.end() - 1);
  for (int IF = 0; IF < m.NF; ++IF)
    for (int ID = 0; ID < m.DoF; ++ID) {
      int g = m.glob[ID + (size_t)m.DoF * IF];
      m.inv_idx[fill[g]++] = IF * m.DoF + ID;    // ascending (IF, ID)
    }
}

// MassCGKernel!: src/DyCore/MassCG.jl:61-75 ; GridSizeSphereKernel!:
// src/DyCore/DiscretizationCG.jl:119-144 (dz: the last element writes).
static void build_mass_dz(Model &m)
{
  int nz = m.nz, N = m.N, DoF = m.DoF;
  m.M.assign((size_t)nz * m.NumG * 2, 0.0);
  m.MMass.assign((size_t)nz * m.NumG, 0.0);
  m.dz.assign((size_t)nz * m.NumG, 0.0);
  #pragma omp parallel for schedule(static)
  for (int g = 0; g < m.NumG; ++g)
    for (int q = m.inv_ptr[g]; q < m.inv_ptr[g + 1]; ++q) {
      int IF = m.inv_idx[q] / DoF, ID = m.inv_idx[q] % DoF;
      int I = ID % N, Jn = ID / N;
      for (int Iz = 0; Iz < nz; ++Iz) {
        double J1 = JJ(m, ID, 0, Iz, IF), J2 = JJ(m, ID, 1, Iz, IF);
        m.M[Iz + (size_t)nz * g] += J1;
        m.M[Iz + (size_t)nz * (g + (size_t)m.NumG)] += J2;
        m.MMass[Iz + (size_t)nz * g] += 0.5 * (J1 + J2) * m.w[I] * m.w[Jn];
        double x = XX(m, ID, 0, 0, Iz, IF), y = XX(m, ID, 0, 1, Iz, IF), zc = XX(m, ID, 0, 2, Iz, IF);
        double r1 = std::sqrt(x * x + y * y + zc * zc);
        x = XX(m, ID, 1, 0, Iz, IF); y = XX(m, ID, 1, 1, Iz, IF); zc = XX(m, ID, 1, 2, Iz, IF);
        double r2 = std::sqrt(x * x + y * y + zc * zc);
        m.dz[Iz + (size_t)nz * g] = r2 - r1;
      }
    }
}

// 2*Omega*sinlat at layer midpoints: CoriolisShallow (src/GPU/Coriolis.jl:18-28)
// evaluated at x = 0.5*(X_bottom + X_top) (MomentumKernel.jl:156-159).
static void build_fcor(Model &m)
{
  int DoF = m.DoF, nz = m.nz;
  m.fcor.assign((size_t)DoF * nz * m.NF, 0.0);
  #pragma omp parallel for schedule(static)
  for (int IF = 0; IF < m.NF; ++IF)
    for (int Iz = 0; Iz < nz; ++Iz)
      for (int ID = 0; ID < DoF; ++ID) {
        double x = 0.5 * (XX(m, ID, 0, 0, Iz, IF) + XX(m, ID, 1, 0, Iz, IF));
        double y = 0.5 * (XX(m, ID, 0, 1, Iz, IF) + XX(m, ID, 1, 1, Iz, IF));
        double zc = 0.5 * (XX(m, ID, 0, 2, Iz, IF) + XX(m, ID, 1, 2, Iz, IF));
        double sinlat = zc / std::sqrt(x * x + y * y + zc * zc);
        m.fcor[ID + (size_t)DoF * (Iz + (size_t)nz * IF)] = 2.0 * m.phys.Omega * sinlat;
      }
}

// SSP-Knoth tableau: src/Integration/RosenbrockMethod.jl:26-47
// a = alpha/Gamma, c = -inv(Gamma), m = Gamma'\b (exact in binary except m).
static void build_tableau(Model &m)
{
  memset(m.rk_a, 0, sizeof m.rk_a);
  memset(m.rk_c, 0, sizeof m.rk_c);
  m.rk_a[1][0] = 1.0; m.rk_a[2][0] = 0.25; m.rk_a[2][1] = 0.25;
  m.rk_c[1][0] = 0.0; m.rk_c[2][0] = -0.75; m.rk_c[2][1] = -0.75;
  double b1 = 1.0 / 6.0, b2 = 1.0 / 6.0, b3 = 2.0 / 3.0;
  // upper-triangular back substitution of Gamma' m = b
  double m3 = b3 / 1.0;
  double m2 = (b2 - (-0.75) * m3) / 1.0;
  double m1 = (b1 - (-0.75) * m3) / 1.0;
  m.rk_m[0] = m1; m.rk_m[1] = m2; m.rk_m[2] = m3;
  m.rk_gamma = 1.0;
}

// Dry pressure: src/Models/Equation.jl:25-38 with fast_powGPU (Equation.jl:79)
inline double pressure(const Phys &ph, double rhoth)
{
  return ph.p0 * cgd_exp(1.0 / (1.0 - ph.kappa) * cgd_log(ph.Rd * rhoth / ph.p0));
}

// ---------------------------------------------------------------------------
// RHS.  Element-node contributions are computed per element (parallel over
// elements), then summed per global DOF over the contributing element nodes
// in ascending (element, node) order (the owner gather that replaces the
// reference's atomic adds).
// ---------------------------------------------------------------------------
struct Ctx {
  Model &m;
  const double *U;
  int nz, NumG;
  explicit Ctx(Model &mm, const double *u) : m(mm), U(u), nz(mm.nz), NumG(mm.NumG) {}
  double u(int Iz, int g, int v) const { return U[Iz + (size_t)nz * (g + (size_t)NumG * v)]; }
  double Mk(int Iz, int g, int k) const { return m.M[Iz + (size_t)nz * (g + (size_t)NumG * k)]; }
};

static void gather(const Model &m, const std::vector<double> &C, int nf, double *out)
{
  // C layout: ((IF*nz + Iz)*nf + f)*DoF + ID ; out (nz, NumG, nf)
  int nz = m.nz, DoF = m.DoF;
  #pragma omp parallel for schedule(static)
  for (int g = 0; g < m.NumG; ++g)
    for (int f = 0; f < nf; ++f)
      for (int Iz = 0; Iz < nz; ++Iz) {
        double acc = 0.0;
        for (int q = m.inv_ptr[g]; q < m.inv_ptr[g + 1]; ++q) {
          int IF = m.inv_idx[q] / DoF, ID = m.inv_idx[q] % DoF;
          acc += C[(((size_t)IF * nz + Iz) * nf + f) * DoF + ID];
        }
        out[Iz + (size_t)nz * (g + (size_t)m.NumG * f)] = acc;
      }
}

// Phase 1 hyperviscosity: HyperViscKernel! (src/GPU/ViscKernel.jl:1-84) and
// HyperViscTracerKernel! (ViscKernel.jl:169-218), per element and level.
static void hypervisc1_element(Model &m, const Ctx &c, int IF, std::vector<double> &C1)
{
  int N = m.N, DoF = m.DoF, nz = m.nz, nf = 5 + m.NumTr;
  const double *D = m.DS.data(), *DW = m.DW.data();
  std::vector<double> uC(DoF), vC(DoF), uD(DoF), vD(DoF), Th(DoF), Curl(DoF), Div(DoF), Cx(DoF), Cy(DoF);
  for (int Iz = 0; Iz < nz; ++Iz) {
    double *out = &C1[((size_t)IF * nz + Iz) * nf * DoF];
    for (int ID = 0; ID < DoF; ++ID) {
      int g = m.glob[ID + (size_t)DoF * IF];
      double d11 = DXI(m, 1, 1, 0, ID, Iz, IF) + DXI(m, 1, 1, 1, ID, Iz, IF);
      double d12 = DXI(m, 1, 2, 0, ID, Iz, IF) + DXI(m, 1, 2, 1, ID, Iz, IF);
      double d21 = DXI(m, 2, 1, 0, ID, Iz, IF) + DXI(m, 2, 1, 1, ID, Iz, IF);
      double d22 = DXI(m, 2, 2, 0, ID, Iz, IF) + DXI(m, 2, 2, 1, ID, Iz, IF);
      double u = c.u(Iz, g, 1), v = c.u(Iz, g, 2);
      uC[ID] = d11 * v - d12 * u;                   // Curl12
      vC[ID] = d21 * v - d22 * u;
      uD[ID] = d11 * u + d12 * v;                   // Contra12
      vD[ID] = d21 * u + d22 * v;
      Th[ID] = c.u(Iz, g, 4) / c.u(Iz, g, 0);
    }
    for (int Jn = 0; Jn < N; ++Jn)
      for (int In = 0; In < N; ++In) {
        int ID = In + N * Jn;
        double Dxc = D[In] * Th[0 + N * Jn];
        double Dyc = D[Jn] * Th[In];
        double cu = D[In] * uC[0 + N * Jn] + D[Jn] * vC[In];
        double dv = D[In] * uD[0 + N * Jn] + D[Jn] * vD[In];
        for (int k = 1; k < N; ++k) {
          Dxc += D[In + N * k] * Th[k + N * Jn];
          Dyc += D[Jn + N * k] * Th[In + N * k];
          cu += D[In + N * k] * uC[k + N * Jn] + D[Jn + N * k] * vC[In + N * k];
          dv += D[In + N * k] * uD[k + N * Jn] + D[Jn + N * k] * vD[In + N * k];
        }
        double Js = JJ(m, ID, 0, Iz, IF) + JJ(m, ID, 1, Iz, IF);
        Curl[ID] = cu / Js;
        Div[ID] = dv / Js;
        double d11 = DXI(m, 1, 1, 0, ID, Iz, IF) + DXI(m, 1, 1, 1, ID, Iz, IF);
        double d12 = DXI(m, 1, 2, 0, ID, Iz, IF) + DXI(m, 1, 2, 1, ID, Iz, IF);
        double d21 = DXI(m, 2, 1, 0, ID, Iz, IF) + DXI(m, 2, 1, 1, ID, Iz, IF);
        double d22 = DXI(m, 2, 2, 0, ID, Iz, IF) + DXI(m, 2, 2, 1, ID, Iz, IF);
        double GradDx = (d11 * Dxc + d21 * Dyc) / Js;   // Grad12 (with J)
        double GradDy = (d12 * Dxc + d22 * Dyc) / Js;
        Cx[ID] = d11 * GradDx + d12 * GradDy;           // Contra12
        Cy[ID] = d21 * GradDx + d22 * GradDy;
      }
    for (int Jn = 0; Jn < N; ++Jn)
      for (int In = 0; In < N; ++In) {
        int ID = In + N * Jn;
        int g = m.glob[ID + (size_t)DoF * IF];
        double DxCurl = DW[In] * Curl[0 + N * Jn];
        double DyCurl = DW[Jn] * Curl[In];
        double DxDiv = DW[In] * Div[0 + N * Jn];
        double DyDiv = DW[Jn] * Div[In];
        double DivTh = DW[In] * Cx[0 + N * Jn] + DW[Jn] * Cy[In];
        for (int k = 1; k < N; ++k) {
          DxCurl += DW[In + N * k] * Curl[k + N * Jn];
          DyCurl += DW[Jn + N * k] * Curl[In + N * k];
          DxDiv += DW[In + N * k] * Div[k + N * Jn];
          DyDiv += DW[Jn + N * k] * Div[In + N * k];
          DivTh += DW[In + N * k] * Cx[k + N * Jn] + DW[Jn + N * k] * Cy[In + N * k];
        }
        double d11 = DXI(m, 1, 1, 0, ID, Iz, IF) + DXI(m, 1, 1, 1, ID, Iz, IF);
        double d12 = DXI(m, 1, 2, 0, ID, Iz, IF) + DXI(m, 1, 2, 1, ID, Iz, IF);
        double d21 = DXI(m, 2, 1, 0, ID, Iz, IF) + DXI(m, 2, 1, 1, ID, Iz, IF);
        double d22 = DXI(m, 2, 2, 0, ID, Iz, IF) + DXI(m, 2, 2, 1, ID, Iz, IF);
        double FuC = d12 * DxCurl + d22 * DyCurl;       // Rot12
        double FvC = -d11 * DxCurl - d21 * DyCurl;
        double FuD = d11 * DxDiv + d21 * DyDiv;         // Grad12 (no J)
        double FvD = d12 * DxDiv + d22 * DyDiv;
        double MC = c.Mk(Iz, g, 0) + c.Mk(Iz, g, 1);
        out[0 * DoF + ID] = -FuC / MC;
        out[1 * DoF + ID] = -FvC / MC;
        out[2 * DoF + ID] = FuD / MC;
        out[3 * DoF + ID] = FvD / MC;
        out[4 * DoF + ID] = DivTh / MC;
      }
    for (int iT = 0; iT < m.NumTr; ++iT) {
      for (int ID = 0; ID < DoF; ++ID) {
        int g = m.glob[ID + (size_t)DoF * IF];
        Th[ID] = c.u(Iz, g, 5 + iT) / c.u(Iz, g, 0);
      }
      for (int Jn = 0; Jn < N; ++Jn)
        for (int In = 0; In < N; ++In) {
          int ID = In + N * Jn;
          double Dxc = D[In] * Th[0 + N * Jn];
          double Dyc = D[Jn] * Th[In];
          for (int k = 1; k < N; ++k) {
            Dxc += D[In + N * k] * Th[k + N * Jn];
            Dyc += D[Jn + N * k] * Th[In + N * k];
          }
          double Js = JJ(m, ID, 0, Iz, IF) + JJ(m, ID, 1, Iz, IF);
          double d11 = DXI(m, 1, 1, 0, ID, Iz, IF) + DXI(m, 1, 1, 1, ID, Iz, IF);
          double d12 = DXI(m, 1, 2, 0, ID, Iz, IF) + DXI(m, 1, 2, 1, ID, Iz, IF);
          double d21 = DXI(m, 2, 1, 0, ID, Iz, IF) + DXI(m, 2, 1, 1, ID, Iz, IF);
          double d22 = DXI(m, 2, 2, 0, ID, Iz, IF) + DXI(m, 2, 2, 1, ID, Iz, IF);
          double GradDx = (d11 * Dxc + d21 * Dyc) / Js;
          double GradDy = (d12 * Dxc + d22 * Dyc) / Js;
          Cx[ID] = d11 * GradDx + d12 * GradDy;
          Cy[ID] = d21 * GradDx + d22 * GradDy;
        }
      for (int Jn = 0; Jn < N; ++Jn)
        for (int In = 0; In < N; ++In) {
          int ID = In + N * Jn;
          int g = m.glob[ID + (size_t)DoF * IF];
          double DivTr = DW[In] * Cx[0 + N * Jn] + DW[Jn] * Cy[In];
          for (int k = 1; k < N; ++k) DivTr += DW[In + N * k] * Cx[k + N * Jn] + DW[Jn + N * k] * Cy[In + N * k];
          double MC = c.Mk(Iz, g, 0) + c.Mk(Iz, g, 1);
          out[(5 + iT) * DoF + ID] = DivTr / MC;
        }
    }
  }
}

// RecU4: src/GPU/OperatorKernel.jl:1044-1059
static inline void recu4(double cLL, double cL, double cR, double cRR,
                         double JLL, double JL, double JR, double JRR, double &cFL, double &cFR)
{
  double kR = (JL / (JL + JR)) * ((JLL + JL) / (JLL + JL + JR));
  double kL = (JL / (JLL + JL)) * (JR / (JLL + JL + JR));
  double r = (cL - cLL) / (cR - cL + 1.e-20);
  cFL = cL + cgd_max(0.0, cgd_min(r, cgd_min(kL * r + kR, 1.0))) * (cR - cL);
  kL = (JR / (JR + JL)) * ((JRR + JR) / (JL + JR + JRR));
  kR = (JR / (JRR + JR)) * (JL / (JL + JR + JRR));
  r = (cR - cRR) / (cL - cR + 1.e-20);
  cFR = cR + cgd_max(0.0, cgd_min(r, cgd_min(kR * r + kL, 1.0))) * (cL - cR);
}

// Per-level terms of phase 2 at one element node (see assemble below).
struct P2Terms {
  double vu, vv, vth;           // HyperViscKoeffKernel!
  double mu, mv, mwlo, mwhi;    // MomentumVectorInvariantCoriolisKernel!
  double gu, gv, gwlo, gwhi;    // GradFullKernel!
  double fr_self, fr_up, hr;    // DivRhoTrUpwind3New2Kernel! (rho)
  double fth_self, fth_up, hth; // (rho*theta)
};

// Phase 2 for one element: HyperViscKoeffKernel! (ViscKernel.jl:86-167),
// HyperViscTracerKoeffKernel! (ViscKernel.jl:277-327),
// MomentumVectorInvariantCoriolisKernel! (MomentumKernel.jl:1-178),
// GradFullKernel! (GradKineticKernel.jl:1-129),
// DivRhoTrUpwind3New2Kernel! (OperatorKernel.jl:637-760).
static void phase2_element(Model &m, const Ctx &c, const double *T1, int IF, std::vector<double> &C2)
{
  int N = m.N, DoF = m.DoF, nz = m.nz, NT = m.NumTr, NV = 5 + NT;
  const double *D = m.DS.data(), *DW = m.DW.data();
  const Phys &ph = m.phys;
  auto t1 = [&](int Iz, int g, int f) { return T1[Iz + (size_t)nz * (g + (size_t)m.NumG * f)]; };
  std::vector<P2Terms> tm((size_t)nz * DoF);
  std::vector<double> tvtr((size_t)nz * DoF * (NT > 0 ? NT : 1));
  std::vector<double> tftr_self((size_t)nz * DoF * (NT > 0 ? NT : 1)), tftr_up((size_t)nz * DoF * (NT > 0 ? NT : 1));
  std::vector<double> thtr((size_t)nz * DoF * (NT > 0 ? NT : 1));
  std::vector<double> a1(DoF), a2(DoF), a3(DoF), a4(DoF), a5(DoF), a6(DoF), b1(DoF), b2(DoF), b3(DoF), b4(DoF);
  std::vector<double> cc(DoF), uc(DoF), vc(DoF), K1a(DoF), K2a(DoF), pa(DoF);
  std::vector<int> gl(DoF);
  for (int ID = 0; ID < DoF; ++ID) gl[ID] = m.glob[ID + (size_t)DoF * IF];
  auto dx = [&](int a, int b, int K, int ID, int Iz) { return DXI(m, a, b, K, ID, Iz, IF); };
  auto wsurf = [&](int ID) {
    int g = gl[ID];
    return -(dx(3, 1, 0, ID, 0) * c.u(0, g, 1) + dx(3, 2, 0, ID, 0) * c.u(0, g, 2)) / dx(3, 3, 0, ID, 0);
  };
  auto wlo = [&](int ID, int l) { return l == 0 ? wsurf(ID) : c.u(l - 1, gl[ID], 3); };
  auto whi = [&](int ID, int l) { return c.u(l, gl[ID], 3); };
  // vertical temps of the momentum kernel (MomentumKernel.jl:50-72)
  auto tuZ = [&](int K, int ID, int l) {
    double v = c.u(l, gl[ID], 2);
    return K == 0 ? dx(3, 3, 0, ID, l) * v - dx(3, 2, 0, ID, l) * wlo(ID, l)
                  : dx(3, 3, 1, ID, l) * v - dx(3, 2, 1, ID, l) * whi(ID, l);
  };
  auto tvZ = [&](int K, int ID, int l) {
    double u = c.u(l, gl[ID], 1);
    return K == 0 ? dx(3, 3, 0, ID, l) * u - dx(3, 1, 0, ID, l) * wlo(ID, l)
                  : dx(3, 3, 1, ID, l) * u - dx(3, 1, 1, ID, l) * whi(ID, l);
  };
  auto twZ = [&](int K, int ID, int l) {
    double u = c.u(l, gl[ID], 1), v = c.u(l, gl[ID], 2);
    return dx(3, 2, K, ID, l) * u - dx(3, 1, K, ID, l) * v;
  };
  // kinetic energy on the bottom/top node of level l (GradKineticKernel.jl:20-42)
  auto K1 = [&](int ID, int l) {
    int g = gl[ID];
    double u = c.u(l, g, 1), v = c.u(l, g, 2), wl = wlo(ID, l);
    return 0.5 * (u * u + v * v) + 0.5 * (wl * wl);
  };
  auto K2 = [&](int ID, int l) {
    int g = gl[ID];
    double u = c.u(l, g, 1), v = c.u(l, g, 2), wh = c.u(l, g, 3);
    return 0.5 * (u * u + v * v) + 0.5 * (wh * wh);
  };
  auto Js = [&](int ID, int l) { return JJ(m, ID, 0, l, IF) + JJ(m, ID, 1, l, IF); };
  auto cratio = [&](int ID, int l, int f) { return c.u(l, gl[ID], f) / c.u(l, gl[ID], 0); };

  for (int Iz = 0; Iz < nz; ++Iz) {
    P2Terms *T = &tm[(size_t)Iz * DoF];
    // ---- HyperViscKoeffKernel! ----
    for (int ID = 0; ID < DoF; ++ID) {
      int g = gl[ID];
      double d11 = dx(1, 1, 0, ID, Iz) + dx(1, 1, 1, ID, Iz);
      double d12 = dx(1, 2, 0, ID, Iz) + dx(1, 2, 1, ID, Iz);
      double d21 = dx(2, 1, 0, ID, Iz) + dx(2, 1, 1, ID, Iz);
      double d22 = dx(2, 2, 0, ID, Iz) + dx(2, 2, 1, ID, Iz);
      double c1 = t1(Iz, g, 0), c2 = t1(Iz, g, 1), c3 = t1(Iz, g, 2), c4 = t1(Iz, g, 3);
      a1[ID] = d11 * c2 - d12 * c1;     // Curl12(Cache1, Cache2)
      a2[ID] = d21 * c2 - d22 * c1;
      a3[ID] = d11 * c3 + d12 * c4;     // Contra12(Cache3, Cache4)
      a4[ID] = d21 * c3 + d22 * c4;
      a5[ID] = t1(Iz, g, 4);
    }
    for (int Jn = 0; Jn < N; ++Jn)
      for (int In = 0; In < N; ++In) {
        int ID = In + N * Jn, g = gl[ID];
        double Dxc = D[In] * a5[0 + N * Jn], Dyc = D[Jn] * a5[In];
        double cu = D[In] * a1[0 + N * Jn] + D[Jn] * a2[In];
        double dv = D[In] * a3[0 + N * Jn] + D[Jn] * a4[In];
        for (int k = 1; k < N; ++k) {
          Dxc += D[In + N * k] * a5[k + N * Jn];
          Dyc += D[Jn + N * k] * a5[In + N * k];
          cu += D[In + N * k] * a1[k + N * Jn] + D[Jn + N * k] * a2[In + N * k];
          dv += D[In + N * k] * a3[k + N * Jn] + D[Jn + N * k] * a4[In + N * k];
        }
        double js = Js(ID, Iz);
        b1[ID] = cu / js;
        b2[ID] = dv / js;
        double d11 = dx(1, 1, 0, ID, Iz) + dx(1, 1, 1, ID, Iz);
        double d12 = dx(1, 2, 0, ID, Iz) + dx(1, 2, 1, ID, Iz);
        double d21 = dx(2, 1, 0, ID, Iz) + dx(2, 1, 1, ID, Iz);
        double d22 = dx(2, 2, 0, ID, Iz) + dx(2, 2, 1, ID, Iz);
        double GradDx = (d11 * Dxc + d21 * Dyc) / js;
        double GradDy = (d12 * Dxc + d22 * Dyc) / js;
        double rho = c.u(Iz, g, 0);
        b3[ID] = rho * (d11 * GradDx + d12 * GradDy);   // Contra12(Rho, ...)
        b4[ID] = rho * (d21 * GradDx + d22 * GradDy);
      }
    for (int Jn = 0; Jn < N; ++Jn)
      for (int In = 0; In < N; ++In) {
        int ID = In + N * Jn, g = gl[ID];
        double DxCurl = DW[In] * b1[0 + N * Jn], DyCurl = DW[Jn] * b1[In];
        double DxDiv = DW[In] * b2[0 + N * Jn], DyDiv = DW[Jn] * b2[In];
        double DivTh = DW[In] * b3[0 + N * Jn] + DW[Jn] * b4[In];
        for (int k = 1; k < N; ++k) {
          DxCurl += DW[In + N * k] * b1[k + N * Jn];
          DyCurl += DW[Jn + N * k] * b1[In + N * k];
          DxDiv += DW[In + N * k] * b2[k + N * Jn];
          DyDiv += DW[Jn + N * k] * b2[In + N * k];
          DivTh += DW[In + N * k] * b3[k + N * Jn] + DW[Jn + N * k] * b4[In + N * k];
        }
        double d11 = dx(1, 1, 0, ID, Iz) + dx(1, 1, 1, ID, Iz);
        double d12 = dx(1, 2, 0, ID, Iz) + dx(1, 2, 1, ID, Iz);
        double d21 = dx(2, 1, 0, ID, Iz) + dx(2, 1, 1, ID, Iz);
        double d22 = dx(2, 2, 0, ID, Iz) + dx(2, 2, 1, ID, Iz);
        double FuC = d12 * DxCurl + d22 * DyCurl;
        double FvC = -d11 * DxCurl - d21 * DyCurl;
        double FuD = d11 * DxDiv + d21 * DyDiv;
        double FvD = d12 * DxDiv + d22 * DyDiv;
        double MC = c.Mk(Iz, g, 0) + c.Mk(Iz, g, 1);
        T[ID].vu = -(-m.nuCurl * FuC + m.nuGrad * FuD) / MC;
        T[ID].vv = -(-m.nuCurl * FvC + m.nuGrad * FvD) / MC;
        T[ID].vth = -m.nuDiv * DivTh / MC;
      }
    // ---- HyperViscTracerKoeffKernel! ----
    for (int iT = 0; iT < NT; ++iT) {
      for (int ID = 0; ID < DoF; ++ID) a5[ID] = t1(Iz, gl[ID], 5 + iT);
      for (int Jn = 0; Jn < N; ++Jn)
        for (int In = 0; In < N; ++In) {
          int ID = In + N * Jn, g = gl[ID];
          double Dxc = D[In] * a5[0 + N * Jn], Dyc = D[Jn] * a5[In];
          for (int k = 1; k < N; ++k) {
            Dxc += D[In + N * k] * a5[k + N * Jn];
            Dyc += D[Jn + N * k] * a5[In + N * k];
          }
          double js = Js(ID, Iz);
          double d11 = dx(1, 1, 0, ID, Iz) + dx(1, 1, 1, ID, Iz);
          double d12 = dx(1, 2, 0, ID, Iz) + dx(1, 2, 1, ID, Iz);
          double d21 = dx(2, 1, 0, ID, Iz) + dx(2, 1, 1, ID, Iz);
          double d22 = dx(2, 2, 0, ID, Iz) + dx(2, 2, 1, ID, Iz);
          double GradDx = (d11 * Dxc + d21 * Dyc) / js;
          double GradDy = (d12 * Dxc + d22 * Dyc) / js;
          double rho = c.u(Iz, g, 0);
          b3[ID] = rho * (d11 * GradDx + d12 * GradDy);
          b4[ID] = rho * (d21 * GradDx + d22 * GradDy);
        }
      for (int Jn = 0; Jn < N; ++Jn)
        for (int In = 0; In < N; ++In) {
          int ID = In + N * Jn, g = gl[ID];
          double DivTr = DW[In] * b3[0 + N * Jn] + DW[Jn] * b4[In];
          for (int k = 1; k < N; ++k) DivTr += DW[In + N * k] * b3[k + N * Jn] + DW[Jn + N * k] * b4[In + N * k];
          double MC = c.Mk(Iz, g, 0) + c.Mk(Iz, g, 1);
          tvtr[((size_t)Iz * DoF + ID) * NT + iT] = -m.nuDiv * DivTr / MC;
        }
    }
    // ---- MomentumVectorInvariantCoriolisKernel! ----
    for (int ID = 0; ID < DoF; ++ID) {
      int g = gl[ID];
      double u = c.u(Iz, g, 1), v = c.u(Iz, g, 2);
      double wl = wlo(ID, Iz), wh = whi(ID, Iz);
      // (K=0 -> arrays a*, K=1 -> arrays b*)
      a1[ID] = -dx(1, 2, 0, ID, Iz) * wl;  b1[ID] = -dx(1, 2, 1, ID, Iz) * wh;   // tempuZ1
      a2[ID] = -dx(2, 2, 0, ID, Iz) * wl;  b2[ID] = -dx(2, 2, 1, ID, Iz) * wh;   // tempuZ2
      a3[ID] = -dx(1, 1, 0, ID, Iz) * wl;  b3[ID] = -dx(1, 1, 1, ID, Iz) * wh;   // tempvZ1
      a4[ID] = -dx(2, 1, 0, ID, Iz) * wl;  b4[ID] = -dx(2, 1, 1, ID, Iz) * wh;   // tempvZ2
      a5[ID] = dx(1, 2, 0, ID, Iz) * u - dx(1, 1, 0, ID, Iz) * v;                 // tempwZ1 K=0
      a6[ID] = dx(2, 2, 0, ID, Iz) * u - dx(2, 1, 0, ID, Iz) * v;                 // tempwZ2 K=0
      uc[ID] = dx(1, 2, 1, ID, Iz) * u - dx(1, 1, 1, ID, Iz) * v;                 // tempwZ1 K=1
      vc[ID] = dx(2, 2, 1, ID, Iz) * u - dx(2, 1, 1, ID, Iz) * v;                 // tempwZ2 K=1
    }
    for (int Jn = 0; Jn < N; ++Jn)
      for (int In = 0; In < N; ++In) {
        int ID = In + N * Jn, g = gl[ID];
        double u = c.u(Iz, g, 1), v = c.u(Iz, g, 2), rho = c.u(Iz, g, 0);
        double wl = wlo(ID, Iz), wh = whi(ID, Iz);
        double FU = 0.0, FV = 0.0, FW1 = 0.0, FW2 = 0.0;
        if (Iz > 0) {
          double FluxUZ = 0.5 * (tuZ(0, ID, Iz) - tuZ(1, ID, Iz - 1));
          double FluxVZ = 0.5 * (tvZ(0, ID, Iz) - tvZ(1, ID, Iz - 1));
          double FluxWZ = 0.5 * (twZ(0, ID, Iz) - twZ(1, ID, Iz - 1));
          FU += (-v * FluxWZ - wl * FluxVZ);
          FV += (u * FluxWZ - wl * FluxUZ);
          FW1 += (u * FluxVZ + v * FluxUZ);
        }
        if (Iz < nz - 1) {
          double FluxUZ = 0.5 * (tuZ(0, ID, Iz + 1) - tuZ(1, ID, Iz));
          double FluxVZ = 0.5 * (tvZ(0, ID, Iz + 1) - tvZ(1, ID, Iz));
          double FluxWZ = 0.5 * (twZ(0, ID, Iz + 1) - twZ(1, ID, Iz));
          FU += (-v * FluxWZ - wh * FluxVZ);
          FV += (u * FluxWZ - wh * FluxUZ);
          FW2 += (u * FluxVZ + v * FluxUZ);
        }
        double U1 = 0.5 * (tuZ(1, ID, Iz) - tuZ(0, ID, Iz)), U2 = U1;
        double V1 = 0.5 * (tvZ(1, ID, Iz) - tvZ(0, ID, Iz)), V2 = V1;
        double W1 = 0.5 * (twZ(1, ID, Iz) - twZ(0, ID, Iz)), W2 = W1;
        U1 += D[In] * a1[0 + N * Jn] + D[Jn] * a2[In];
        U2 += D[In] * b1[0 + N * Jn] + D[Jn] * b2[In];
        V1 += D[In] * a3[0 + N * Jn] + D[Jn] * a4[In];
        V2 += D[In] * b3[0 + N * Jn] + D[Jn] * b4[In];
        W1 += D[In] * a5[0 + N * Jn] + D[Jn] * a6[In];
        W2 += D[In] * uc[0 + N * Jn] + D[Jn] * vc[In];
        for (int k = 1; k < N; ++k) {
          U1 += D[In + N * k] * a1[k + N * Jn] + D[Jn + N * k] * a2[In + N * k];
          U2 += D[In + N * k] * b1[k + N * Jn] + D[Jn + N * k] * b2[In + N * k];
          V1 += D[In + N * k] * a3[k + N * Jn] + D[Jn + N * k] * a4[In + N * k];
          V2 += D[In + N * k] * b3[k + N * Jn] + D[Jn + N * k] * b4[In + N * k];
          W1 += D[In + N * k] * a5[k + N * Jn] + D[Jn + N * k] * a6[In + N * k];
          W2 += D[In + N * k] * uc[k + N * Jn] + D[Jn + N * k] * vc[In + N * k];
        }
        double fc = m.fcor[ID + (size_t)DoF * (Iz + (size_t)nz * IF)];
        double FuCor = v * fc, FvCor = -u * fc, FwCor = 0.0;
        double J1 = JJ(m, ID, 0, Iz, IF), J2 = JJ(m, ID, 1, Iz, IF);
        FU += FuCor * (J1 + J2);
        FV += FvCor * (J1 + J2);
        FW1 += FwCor * J1;
        FW2 += FwCor * J2;
        double MC = c.Mk(Iz, g, 0) + c.Mk(Iz, g, 1);
        T[ID].mu = (-v * W1 - wl * V1 - v * W2 - wh * V2 + FU) / MC;
        T[ID].mv = (u * W1 - wl * U1 + u * W2 - wh * U2 + FV) / MC;
        T[ID].mwlo = 0.0; T[ID].mwhi = 0.0;
        if (Iz > 0)
          T[ID].mwlo = rho * (u * V1 + v * U1 + FW1) /
                       (c.u(Iz - 1, g, 0) * c.Mk(Iz - 1, g, 1) + rho * c.Mk(Iz, g, 0));
        if (Iz < nz - 1)
          T[ID].mwhi = rho * (u * V2 + v * U2 + FW2) /
                       (c.u(Iz + 1, g, 0) * c.Mk(Iz + 1, g, 0) + rho * c.Mk(Iz, g, 1));
      }
    // ---- GradFullKernel! ----
    for (int ID = 0; ID < DoF; ++ID) {
      K1a[ID] = K1(ID, Iz);
      K2a[ID] = K2(ID, Iz);
      pa[ID] = pressure(ph, c.u(Iz, gl[ID], 4));
    }
    for (int Jn = 0; Jn < N; ++Jn)
      for (int In = 0; In < N; ++In) {
        int ID = In + N * Jn, g = gl[ID];
        double rho = c.u(Iz, g, 0);
        double DXp = D[In] * pa[0 + N * Jn], DYp = D[Jn] * pa[In];
        double DXK1 = D[In] * K1a[0 + N * Jn], DYK1 = D[Jn] * K1a[In];
        double DXK2 = D[In] * K2a[0 + N * Jn], DYK2 = D[Jn] * K2a[In];
        for (int k = 1; k < N; ++k) {
          DXK1 += D[In + N * k] * K1a[k + N * Jn];
          DYK1 += D[Jn + N * k] * K1a[In + N * k];
          DXK2 += D[In + N * k] * K2a[k + N * Jn];
          DYK2 += D[Jn + N * k] * K2a[In + N * k];
          DXp += D[In + N * k] * pa[k + N * Jn];
          DYp += D[Jn + N * k] * pa[In + N * k];
        }
        double GuF1 = -(dx(1, 1, 0, ID, Iz) * DXK1 + dx(2, 1, 0, ID, Iz) * DYK1);
        double GvF1 = -(dx(1, 2, 0, ID, Iz) * DXK1 + dx(2, 2, 0, ID, Iz) * DYK1);
        double GuF2 = -(dx(1, 1, 1, ID, Iz) * DXK2 + dx(2, 1, 1, ID, Iz) * DYK2);
        double GvF2 = -(dx(1, 2, 1, ID, Iz) * DXK2 + dx(2, 2, 1, ID, Iz) * DYK2);
        double d11 = dx(1, 1, 0, ID, Iz) + dx(1, 1, 1, ID, Iz);
        double d12 = dx(1, 2, 0, ID, Iz) + dx(1, 2, 1, ID, Iz);
        double d21 = dx(2, 1, 0, ID, Iz) + dx(2, 1, 1, ID, Iz);
        double d22 = dx(2, 2, 0, ID, Iz) + dx(2, 2, 1, ID, Iz);
        double Gradu = d11 * DXp + d21 * DYp;     // Grad12 (no J)
        double Gradv = d12 * DXp + d22 * DYp;
        double GwF1 = 0.0, GwF2 = 0.0, GZ;
        if (Iz > 0) {
          GZ = 0.5 * (K1a[ID] - K2(ID, Iz - 1));
          GuF1 += -GZ * dx(3, 1, 0, ID, Iz);
          GvF1 += -GZ * dx(3, 2, 0, ID, Iz);
          GwF1 += -rho * GZ * dx(3, 3, 0, ID, Iz);
        }
        if (Iz < nz - 1) {
          GZ = 0.5 * (K1(ID, Iz + 1) - K2a[ID]);
          GuF2 += -GZ * dx(3, 1, 1, ID, Iz);
          GvF2 += -GZ * dx(3, 2, 1, ID, Iz);
          GwF2 += -rho * GZ * dx(3, 3, 1, ID, Iz);
        }
        GZ = 0.5 * (K2a[ID] - K1a[ID]);
        GuF2 += -GZ * dx(3, 1, 1, ID, Iz);
        GuF1 += -GZ * dx(3, 1, 0, ID, Iz);
        GvF2 += -GZ * dx(3, 2, 1, ID, Iz);
        GvF1 += -GZ * dx(3, 2, 0, ID, Iz);
        GwF2 += -rho * GZ * dx(3, 3, 1, ID, Iz);
        GwF1 += -rho * GZ * dx(3, 3, 0, ID, Iz);
        double Grav = ph.Grav;
        GZ = -Grav * rho * (JJ(m, ID, 0, Iz, IF) + JJ(m, ID, 1, Iz, IF)) /
             (dx(3, 3, 0, ID, Iz) + dx(3, 3, 1, ID, Iz));
        Gradu += GZ * (dx(3, 1, 0, ID, Iz) + dx(3, 1, 1, ID, Iz));
        Gradv += GZ * (dx(3, 2, 0, ID, Iz) + dx(3, 2, 1, ID, Iz));
        double MC = c.Mk(Iz, g, 0) + c.Mk(Iz, g, 1);
        T[ID].gu = (GuF1 + GuF2 - Gradu / rho) / MC;
        T[ID].gv = (GvF1 + GvF2 - Gradv / rho) / MC;
        T[ID].gwlo = 0.0; T[ID].gwhi = 0.0;
        if (Iz < nz - 1) {
          double rhop = c.u(Iz + 1, g, 0);
          GZ = 0.5 * (pressure(ph, c.u(Iz + 1, g, 4)) - pa[ID]);
          double Gradw = GZ * (dx(3, 3, 1, ID, Iz) + dx(3, 3, 0, ID, Iz + 1));
          double Gradp = -(Gradw + Grav * (rho * JJ(m, ID, 1, Iz, IF) + rhop * JJ(m, ID, 0, Iz + 1, IF)));
          T[ID].gwhi = (GwF2 + Gradp) / (rhop * c.Mk(Iz + 1, g, 0) + rho * c.Mk(Iz, g, 1));
        }
        if (Iz > 0)
          T[ID].gwlo = GwF1 / (c.u(Iz - 1, g, 0) * c.Mk(Iz - 1, g, 1) + rho * c.Mk(Iz, g, 0));
      }
    // ---- DivRhoTrUpwind3New2Kernel! ----
    int Izm1 = Iz > 0 ? Iz - 1 : 0;
    int Izp1 = Iz + 1 < nz ? Iz + 1 : nz - 1;
    int Izp2 = Iz + 2 < nz ? Iz + 2 : nz - 1;
    for (int ID = 0; ID < DoF; ++ID) {
      int g = gl[ID];
      double rho = c.u(Iz, g, 0), u = c.u(Iz, g, 1), v = c.u(Iz, g, 2);
      double MC = c.Mk(Iz, g, 0) + c.Mk(Iz, g, 1);
      T[ID].fr_self = 0.0; T[ID].fr_up = 0.0; T[ID].fth_self = 0.0; T[ID].fth_up = 0.0;
      double wCon = 0.0;
      if (Iz < nz - 1) {
        double rhop = c.u(Iz + 1, g, 0), up = c.u(Iz + 1, g, 1), vp = c.u(Iz + 1, g, 2);
        double w = c.u(Iz, g, 3);
        wCon = rho * (dx(3, 1, 1, ID, Iz) * u + dx(3, 2, 1, ID, Iz) * v + dx(3, 3, 1, ID, Iz) * w) +
               rhop * (dx(3, 1, 0, ID, Iz + 1) * up + dx(3, 2, 0, ID, Iz + 1) * vp + dx(3, 3, 0, ID, Iz + 1) * w);
        double MCp = c.Mk(Iz + 1, g, 0) + c.Mk(Iz + 1, g, 1);
        double cFL, cFR;
        recu4(cratio(ID, Izm1, 4), cratio(ID, Iz, 4), cratio(ID, Izp1, 4), cratio(ID, Izp2, 4),
              Js(ID, Izm1), Js(ID, Iz), Js(ID, Izp1), Js(ID, Izp2), cFL, cFR);
        double Flux = 0.25 * ((std::fabs(wCon) + wCon) * cFL + (-std::fabs(wCon) + wCon) * cFR);
        T[ID].fth_self = -Flux / MC;
        T[ID].fth_up = Flux / MCp;
        Flux = 0.5 * wCon;
        T[ID].fr_self = -Flux / MC;
        T[ID].fr_up = Flux / MCp;
        for (int iT = 0; iT < NT; ++iT) {
          recu4(cratio(ID, Izm1, 5 + iT), cratio(ID, Iz, 5 + iT), cratio(ID, Izp1, 5 + iT), cratio(ID, Izp2, 5 + iT),
                Js(ID, Izm1), Js(ID, Iz), Js(ID, Izp1), Js(ID, Izp2), cFL, cFR);
          double Fl = 0.25 * ((std::fabs(wCon) + wCon) * cFL + (-std::fabs(wCon) + wCon) * cFR);
          tftr_self[((size_t)Iz * DoF + ID) * NT + iT] = -Fl / MC;
          tftr_up[((size_t)Iz * DoF + ID) * NT + iT] = Fl / MCp;
        }
      } else {
        for (int iT = 0; iT < NT; ++iT) {
          tftr_self[((size_t)Iz * DoF + ID) * NT + iT] = 0.0;
          tftr_up[((size_t)Iz * DoF + ID) * NT + iT] = 0.0;
        }
      }
      double d11 = dx(1, 1, 0, ID, Iz) + dx(1, 1, 1, ID, Iz);
      double d12 = dx(1, 2, 0, ID, Iz) + dx(1, 2, 1, ID, Iz);
      double d21 = dx(2, 1, 0, ID, Iz) + dx(2, 1, 1, ID, Iz);
      double d22 = dx(2, 2, 0, ID, Iz) + dx(2, 2, 1, ID, Iz);
      uc[ID] = -rho * (d11 * u + d12 * v);       // Contra12(-Rho, u, v)
      vc[ID] = -rho * (d21 * u + d22 * v);
      cc[ID] = cratio(ID, Iz, 4);
    }
    for (int Jn = 0; Jn < N; ++Jn)
      for (int In = 0; In < N; ++In) {
        int ID = In + N * Jn, g = gl[ID];
        double DivRhoTr = D[In] * uc[0 + N * Jn] * cc[0 + N * Jn] + D[Jn] * vc[In] * cc[In];
        double DivRho = D[In] * uc[0 + N * Jn] + D[Jn] * vc[In];
        for (int k = 1; k < N; ++k) {
          DivRhoTr += D[In + N * k] * uc[k + N * Jn] * cc[k + N * Jn] + D[Jn + N * k] * vc[In + N * k] * cc[In + N * k];
          DivRho += D[In + N * k] * uc[k + N * Jn] + D[Jn + N * k] * vc[In + N * k];
        }
        double MC = c.Mk(Iz, g, 0) + c.Mk(Iz, g, 1);
        T[ID].hth = DivRhoTr / MC;
        T[ID].hr = DivRho / MC;
      }
    for (int iT = 0; iT < NT; ++iT) {
      for (int ID = 0; ID < DoF; ++ID) cc[ID] = cratio(ID, Iz, 5 + iT);
      for (int Jn = 0; Jn < N; ++Jn)
        for (int In = 0; In < N; ++In) {
          int ID = In + N * Jn, g = gl[ID];
          double DivRhoTr = D[In] * uc[0 + N * Jn] * cc[0 + N * Jn] + D[Jn] * vc[In] * cc[In];
          for (int k = 1; k < N; ++k)
            DivRhoTr += D[In + N * k] * uc[k + N * Jn] * cc[k + N * Jn] + D[Jn + N * k] * vc[In + N * k] * cc[In + N * k];
          double MC = c.Mk(Iz, g, 0) + c.Mk(Iz, g, 1);
          thtr[((size_t)Iz * DoF + ID) * NT + iT] = DivRhoTr / MC;
        }
    }
  }
  // ---- assemble the element-node contributions (fixed order) ----
  //  rho   : vflux(top of Iz) , vflux(top of Iz-1) , horizontal divergence
  //  u, v  : hyperviscosity , momentum , pressure/kinetic gradient
  //  w(Iz) : (momentum(Iz, upper node) + gradient(Iz, upper node)) +
  //          (momentum(Iz+1, lower node) + gradient(Iz+1, lower node))
  //  rho*theta, rho*q : hyperviscosity , vflux(top of Iz) , vflux(top of Iz-1) ,
  //          horizontal divergence
  for (int Iz = 0; Iz < nz; ++Iz) {
    double *out = &C2[((size_t)IF * nz + Iz) * NV * DoF];
    for (int ID = 0; ID < DoF; ++ID) {
      const P2Terms &t = tm[(size_t)Iz * DoF + ID];
      double acc = 0.0;
      if (Iz < nz - 1) acc += t.fr_self;
      if (Iz > 0) acc += tm[(size_t)(Iz - 1) * DoF + ID].fr_up;
      acc += t.hr;
      out[0 * DoF + ID] = acc;
      acc = 0.0; acc += t.vu; acc += t.mu; acc += t.gu;
      out[1 * DoF + ID] = acc;
      acc = 0.0; acc += t.vv; acc += t.mv; acc += t.gv;
      out[2 * DoF + ID] = acc;
      acc = 0.0;
      if (Iz < nz - 1) {
        const P2Terms &tu = tm[(size_t)(Iz + 1) * DoF + ID];
        double hi = t.mwhi + t.gwhi;
        double lo = tu.mwlo + tu.gwlo;
        acc = hi + lo;
      }
      out[3 * DoF + ID] = acc;
      acc = 0.0; acc += t.vth;
      if (Iz < nz - 1) acc += t.fth_self;
      if (Iz > 0) acc += tm[(size_t)(Iz - 1) * DoF + ID].fth_up;
      acc += t.hth;
      out[4 * DoF + ID] = acc;
      for (int iT = 0; iT < NT; ++iT) {
        size_t q = ((size_t)Iz * DoF + ID) * NT + iT;
        acc = 0.0; acc += tvtr[q];
        if (Iz < nz - 1) acc += tftr_self[q];
        if (Iz > 0) acc += tftr_up[((size_t)(Iz - 1) * DoF + ID) * NT + iT];
        acc += thtr[q];
        out[(5 + iT) * DoF + ID] = acc;
      }
    }
  }
}

// The column physics of the tendency tail (src/GPU/FcnGPU.jl:953-966), after
// the DSS: ForceKernel! with the dry Held-Suarez Force
// (src/GPU/OperatorKernel.jl:1073-1080, src/Examples/initial.jl:513-531,
// parameters src/Examples/parameters.jl:122-131) and DampKernel! with
// DampingW (src/GPU/OperatorKernel.jl:1061-1071, src/GPU/dampingGPU.jl:1-19).
// fast_powGPU(x, y) = exp(y log x) (src/Models/Equation.jl:79).
static void physics_tail(const Model &m, const double *U, double *F)
{
  if (!m.held_suarez && !m.damping) return;
  const int nz = m.nz, NumG = m.NumG;
  const size_t S = (size_t)nz * NumG;
  const Phys &ph = m.phys;
  #pragma omp parallel for schedule(static)
  for (int g = 0; g < NumG; ++g)
    for (int Iz = 0; Iz < nz; ++Iz) {
      const size_t o = Iz + (size_t)nz * g;
      if (m.held_suarez) {
        const double k_a = m.hs[0], k_f = m.hs[1], k_s = m.hs[2], DeltaT_y = m.hs[3], DeltaTh_z = m.hs[4];
        const double T_equator = m.hs[5], T_min = m.hs[6], sigma_b = m.hs[7];
        const double p = pressure(ph, U[o + 4 * S]);
        const double Sigma = p / ph.p0;
        const double SigmaPowKappa = cgd_exp(ph.kappa * cgd_log(Sigma));
        const double height_factor = std::max(0.0, (Sigma - sigma_b) / (1.0 - sigma_b));
        const double coslat = m.coslat[g], sinlat = m.sinlat[g];
        F[o + S] += -(k_f * height_factor) * U[o + S];
        F[o + 2 * S] += -(k_f * height_factor) * U[o + 2 * S];
        const double kT = k_a + (k_s - k_a) * height_factor * coslat * coslat * coslat * coslat;
        double Teq = (T_equator - DeltaT_y * sinlat * sinlat - DeltaTh_z * cgd_log(Sigma) * coslat * coslat) *
                     SigmaPowKappa;
        Teq = std::max(T_min, Teq);
        const double T = p / (U[o] * ph.Rd);
        const double DeltaT = kT * (T - Teq);
        F[o + 4 * S] += -U[o + 4 * S] / T * DeltaT;
      }
      if (m.damping) F[o + 3 * S] += -m.dampc[o] * U[o + 3 * S];
    }
}

static void rhs(Model &m, const double *U, double *F)
{
  Ctx c(m, U);
  int nf1 = 5 + m.NumTr, NV = m.NV;
  std::vector<double> C1((size_t)m.NF * m.nz * nf1 * m.DoF);
  #pragma omp parallel for schedule(dynamic, 4)
  for (int IF = 0; IF < m.NF; ++IF) hypervisc1_element(m, c, IF, C1);
  std::vector<double> T1((size_t)m.nz * m.NumG * nf1);
  gather(m, C1, nf1, T1.data());
  C1.clear(); C1.shrink_to_fit();
  std::vector<double> C2((size_t)m.NF * m.nz * NV * m.DoF);
  #pragma omp parallel for schedule(dynamic, 4)
  for (int IF = 0; IF < m.NF; ++IF) phase2_element(m, c, T1.data(), IF, C2);
  gather(m, C2, NV, F);
  physics_tail(m, U, F);
}

// JacSchurKernel!: src/DyCore/JacSchur.jl:29-75 (AuxG[:,:,4] == 0 for Dry),
// dPresdRhoTh: src/Models/Equation.jl:33-36
static void jac(Model &m, const double *U)
{
  int nz = m.nz, NumG = m.NumG;
  size_t bs = (size_t)2 * (nz - 1) * NumG;
  m.bands.assign(4 * bs, 0.0);
  double *JRhoW = m.bands.data(), *JWRho = JRhoW + bs, *JWRhoTh = JWRho + bs, *JRhoThW = JWRhoTh + bs;
  const Phys &ph = m.phys;
  double expo = ph.kappa / (1.0 - ph.kappa);
  #pragma omp parallel for schedule(static)
  for (int IC = 0; IC < NumG; ++IC)
    for (int Iz = 0; Iz < nz - 1; ++Iz) {
      double RhoL = U[Iz + (size_t)nz * IC], RhoR = U[Iz + 1 + (size_t)nz * IC];
      double RhoThL = U[Iz + (size_t)nz * (IC + (size_t)NumG * 4)] + 0.0;
      double RhoThR = U[Iz + 1 + (size_t)nz * (IC + (size_t)NumG * 4)] + 0.0;
      double dzL = m.dz[Iz + (size_t)nz * IC], dzR = m.dz[Iz + 1 + (size_t)nz * IC];
      size_t o = 2 * (Iz + (size_t)(nz - 1) * IC);
      double RhoF = (RhoL * dzL + RhoR * dzR) / (dzL + dzR);
      JRhoW[o] = -RhoF / dzL;
      JRhoW[o + 1] = RhoF / dzR;
      double dPdThL = ph.Rd * cgd_pow(ph.Rd * RhoThL / ph.p0, expo);
      double dPdThR = ph.Rd * cgd_pow(ph.Rd * RhoThR / ph.p0, expo);
      JWRhoTh[o] = -dPdThR / RhoF / (0.5 * (dzL + dzR));
      JWRhoTh[o + 1] = dPdThL / RhoF / (0.5 * (dzL + dzR));
      JWRho[o] = -ph.Grav * dzR / RhoF / (dzL + dzR);
      JWRho[o + 1] = -ph.Grav * dzL / RhoF / (dzL + dzR);
      double RhoThF = (RhoThL * dzL + RhoThR * dzR) / (dzL + dzR);
      JRhoThW[o] = -RhoThF / dzL;
      JRhoThW[o + 1] = RhoThF / dzR;
    }
}

// SchurSolveGPU!: src/Integration/SchurSolve.jl:45-177 (TriDiagKernel!,
// SchurSolveFKernel!, SchurSolveTriKernel!/triSolve!, SchurSolveBKernel!)
static void schur(Model &m, double *k, double *v, double fac)
{
  int nz = m.nz, NumG = m.NumG, NV = m.NV;
  size_t bs = (size_t)2 * (nz - 1) * NumG;
  const double *JRhoW = m.bands.data(), *JWRho = JRhoW + bs, *JWRhoTh = JWRho + bs, *JRhoThW = JWRhoTh + bs;
  int n = nz - 1;
  #pragma omp parallel for schedule(static)
  for (int IC = 0; IC < NumG; ++IC) {
    std::vector<double> tri((size_t)3 * n), x(n), b(n);
    auto B = [&](const double *arr, int r, int Iz) { return arr[r + 2 * (Iz + (size_t)(nz - 1) * IC)]; };
    auto V = [&](int Iz, int f) -> double & { return v[Iz + (size_t)nz * (IC + (size_t)NumG * f)]; };
    auto Kk = [&](int Iz, int f) -> double & { return k[Iz + (size_t)nz * (IC + (size_t)NumG * f)]; };
    double invfac = 1.0 / fac;
    double invfac2 = invfac / fac;
    for (int Iz = 0; Iz < n; ++Iz) {                       // TriDiagKernel!
      double t0, t1, t2;
      if (Iz == 0) {
        t0 = 0.0;
        t1 = invfac2 - B(JWRho, 1, Iz) * B(JRhoW, 0, Iz) - B(JWRho, 0, Iz) * B(JRhoW, 1, Iz) -
             B(JWRhoTh, 1, Iz) * B(JRhoThW, 0, Iz) - B(JWRhoTh, 0, Iz) * B(JRhoThW, 1, Iz);
        t2 = -B(JWRho, 1, Iz + 1) * B(JRhoW, 1, Iz) - B(JWRhoTh, 1, Iz + 1) * B(JRhoThW, 1, Iz);
      } else if (Iz == n - 1) {
        t0 = -B(JWRho, 0, Iz - 1) * B(JRhoW, 0, Iz) - B(JWRhoTh, 0, Iz - 1) * B(JRhoThW, 0, Iz);
        t1 = invfac2 - B(JWRho, 1, Iz) * B(JRhoW, 0, Iz) - B(JWRho, 0, Iz) * B(JRhoW, 1, Iz) -
             B(JWRhoTh, 1, Iz) * B(JRhoThW, 0, Iz) - B(JWRhoTh, 0, Iz) * B(JRhoThW, 1, Iz);
        t2 = 0.0;
      } else {
        t0 = -B(JWRho, 0, Iz - 1) * B(JRhoW, 0, Iz) - B(JWRhoTh, 0, Iz - 1) * B(JRhoThW, 0, Iz);
        t1 = invfac2 - B(JWRho, 1, Iz) * B(JRhoW, 0, Iz) - B(JWRho, 0, Iz) * B(JRhoW, 1, Iz) -
             B(JWRhoTh, 1, Iz) * B(JRhoThW, 0, Iz) - B(JWRhoTh, 0, Iz) * B(JRhoThW, 1, Iz);
        t2 = -B(JWRho, 1, Iz + 1) * B(JRhoW, 1, Iz) - B(JWRhoTh, 1, Iz + 1) * B(JRhoThW, 1, Iz);
      }
      tri[3 * Iz] = t0; tri[3 * Iz + 1] = t1; tri[3 * Iz + 2] = t2;
    }
    for (int Iz = 0; Iz < nz; ++Iz) {                      // SchurSolveFKernel!
      if (Iz < nz - 1)
        V(Iz, 3) = V(Iz, 3) / fac + B(JWRho, 1, Iz) * V(Iz, 0) + B(JWRho, 0, Iz) * V(Iz + 1, 0) +
                   B(JWRhoTh, 1, Iz) * V(Iz, 4) + B(JWRhoTh, 0, Iz) * V(Iz + 1, 4);
      else
        Kk(Iz, 3) = 0.0;
    }
    for (int i = 0; i < n; ++i) b[i] = V(i, 3);            // triSolve!
    x[0] = tri[1];
    for (int i = 0; i < n - 1; ++i) {
      x[i + 1] = tri[3 * (i + 1) + 1] - tri[3 * i + 2] / x[i] * tri[3 * (i + 1)];
      b[i + 1] = b[i + 1] - tri[3 * i + 2] / x[i] * b[i];
    }
    x[n - 1] = b[n - 1] / x[n - 1];
    for (int i = n - 2; i >= 0; --i) x[i] = (b[i] - tri[3 * (i + 1)] * x[i + 1]) / x[i];
    for (int i = 0; i < n; ++i) Kk(i, 3) = x[i];
    for (int Iz = 0; Iz < nz; ++Iz) {                      // SchurSolveBKernel!
      if (Iz == 0) {
        V(Iz, 0) += B(JRhoW, 0, Iz) * Kk(Iz, 3);
        V(Iz, 4) += B(JRhoThW, 0, Iz) * Kk(Iz, 3);
      } else if (Iz == nz - 1) {
        V(Iz, 0) += B(JRhoW, 1, Iz - 1) * Kk(Iz - 1, 3);
        V(Iz, 4) += B(JRhoThW, 1, Iz - 1) * Kk(Iz - 1, 3);
      } else {
        V(Iz, 0) += B(JRhoW, 0, Iz) * Kk(Iz, 3) + B(JRhoW, 1, Iz - 1) * Kk(Iz - 1, 3);
        V(Iz, 4) += B(JRhoThW, 0, Iz) * Kk(Iz, 3) + B(JRhoThW, 1, Iz - 1) * Kk(Iz - 1, 3);
      }
      Kk(Iz, 0) = fac * V(Iz, 0);
      Kk(Iz, 1) = fac * V(Iz, 1);
      Kk(Iz, 2) = fac * V(Iz, 2);
      Kk(Iz, 4) = fac * V(Iz, 4);
      for (int iT = 5; iT < NV; ++iT) Kk(Iz, iT) = fac * V(Iz, iT);
    }
  }
}

// RosenbrockSchur!: src/Integration/RosenbrockSchur.jl:1-33
static void ros_step(Model &m, double *V, double dt)
{
  size_t S = (size_t)m.nz * m.NumG * m.NV;
  std::vector<double> Vn(V, V + S), fV(S), k(3 * S);
  for (int i = 0; i < 3; ++i) {
    #pragma omp parallel for schedule(static)
    for (size_t q = 0; q < S; ++q) {
      double x = Vn[q];
      for (int j = 0; j < i; ++j) x = x + m.rk_a[i][j] * k[j * S + q];
      V[q] = x;
    }
    rhs(m, V, fV.data());
    if (i == 0) jac(m, V);
    for (int j = 0; j < i; ++j) {
      double fac = m.rk_c[i][j] / dt;
      #pragma omp parallel for schedule(static)
      for (size_t q = 0; q < S; ++q) fV[q] = fV[q] + fac * k[j * S + q];
    }
    schur(m, &k[i * S], fV.data(), dt * m.rk_gamma);
  }
  #pragma omp parallel for schedule(static)
  for (size_t q = 0; q < S; ++q) {
    double x = Vn[q];
    for (int i = 0; i < 3; ++i) x = x + m.rk_m[i] * k[i * S + q];
    V[q] = x;
  }
}

// BaroWaveExample: src/Examples/initial.jl:386-462 with
// ParamBaroWaveDrySphere (src/Examples/parameters.jl:48-83), Deep = false.
static void barowave(const Model &m, const double *x, double &Rho, double &uS, double &vS, double &w, double &Th)
{
  const Phys &ph = m.phys;
  double T0E = 310.0, T0P = 240.0, Bp = 2.0, Kp = 3.0, Lapse = 0.005;
  double PertExpR = 0.1, PertLon = PI / 9.0, PertLat = 2.0 * PI / 9.0, PertZ = 15000.0;
  double r = std::sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
  double Lat = std::asin(x[2] / r);
  double Lon = std::atan2(x[1], x[0]);
  if (x[1] < 0.0) Lon = Lon + 2.0 * PI;
  double Z = std::max(r - ph.RadEarth, 0.0);
  double T0 = 0.5 * (T0E + T0P);
  double ConstA = 1.0 / Lapse;
  double ConstB = (T0 - T0P) / (T0 * T0P);
  double ConstC = 0.5 * (Kp + 2.0) * (T0E - T0P) / (T0E * T0P);
  double ConstH = ph.Rd * T0 / ph.Grav;
  double ScaledZ = Z / (Bp * ConstH);
  double Tau1 = ConstA * Lapse / T0 * std::exp(Lapse / T0 * Z) +
                ConstB * (1.0 - 2.0 * ScaledZ * ScaledZ) * std::exp(-ScaledZ * ScaledZ);
  double Tau2 = ConstC * (1.0 - 2.0 * ScaledZ * ScaledZ) * std::exp(-ScaledZ * ScaledZ);
  double IntTau1 = ConstA * (std::exp(Lapse / T0 * Z) - 1.0) + ConstB * Z * std::exp(-ScaledZ * ScaledZ);
  double IntTau2 = ConstC * Z * std::exp(-ScaledZ * ScaledZ);
  double RRatio = 1.0;
  double InteriorTerm = std::pow(RRatio * std::cos(Lat), Kp) -
                        Kp / (Kp + 2.0) * std::pow(RRatio * std::cos(Lat), Kp + 2.0);
  double Temperature = 1.0 / (RRatio * RRatio) / (Tau1 - Tau2 * InteriorTerm);
  double Pressure = ph.p0 * std::exp(-ph.Grav / ph.Rd * (IntTau1 - IntTau2 * InteriorTerm));
  Rho = Pressure / (ph.Rd * Temperature);
  Th = Temperature * std::pow(ph.p0 / Pressure, ph.Rd / ph.Cpd);
  double InteriorTermU = std::pow(RRatio * std::cos(Lat), Kp - 1.0) - std::pow(RRatio * std::cos(Lat), Kp + 1.0);
  double BigU = ph.Grav / ph.RadEarth * Kp * IntTau2 * InteriorTermU * Temperature;
  double RCosLat = ph.RadEarth * std::cos(Lat);
  double OmegaRCosLat = ph.Omega * RCosLat;
  uS = -OmegaRCosLat + std::sqrt(OmegaRCosLat * OmegaRCosLat + RCosLat * BigU);
  vS = 0.0;
  double GreatCircleR = std::acos(std::sin(PertLat) * std::sin(Lat) +
                                  std::cos(PertLat) * std::cos(Lat) * std::cos(Lon - PertLon));
  GreatCircleR = GreatCircleR / PertExpR;
  double PertTaper;
  if (Z < PertZ)
    PertTaper = 1.0 - 3.0 * Z * Z / (PertZ * PertZ) + 2.0 * Z * Z * Z / (PertZ * PertZ * PertZ);
  else
    PertTaper = 0.0;
  double uSPert = GreatCircleR < 1.0 ? m.Up * PertTaper * std::exp(-GreatCircleR * GreatCircleR) : 0.0;
  uS = uS + uSPert;
  w = 0.0;
}

} // namespace

// ===========================================================================
extern "C" {

int orc_set_threads(int n)
{
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}

void *orc_create(const orc_cfg *cfg, const double *zlev)
{
  if (!cfg || !zlev || cfg->OrdPoly < 1 || cfg->OrdPoly > 4 || cfg->nPanel < 1 || cfg->nz < 2) return nullptr;
  Model *m = new Model();
  m->n = cfg->nPanel; m->p = cfg->OrdPoly; m->N = m->p + 1; m->DoF = m->N * m->N;
  m->nz = cfg->nz; m->NumTr = cfg->NumTr; m->NV = 5 + cfg->NumTr;
  m->Rad = cfg->Rad; m->H = cfg->H; m->phys = Phys(cfg->Rad);
  m->nuCurl = cfg->HyperDCurl; m->nuGrad = cfg->HyperDGrad; m->nuDiv = cfg->HyperDDiv; m->Up = cfg->Up;
  m->z.assign(zlev, zlev + m->nz + 1);
  Topo G = cubed_grid(m->n, m->Rad);
  Topo S = sub_grid_single(G);
  m->NF = (int)S.faces.size() - 1;
  m->NumNodes = (int)S.nodes.size() - 1;
  m->NumEdges = (int)S.edges.size() - 1;
  int NumG = 0;
  std::vector<int> g1 = numbering_fem_cg_quad(S, m->p, NumG);
  m->NumG = NumG;
  m->glob.resize(g1.size());
  for (size_t i = 0; i < g1.size(); ++i) m->glob[i] = g1[i] - 1;
  m->faceP.assign((size_t)12 * m->NF, 0.0);
  for (int iF = 1; iF <= m->NF; ++iF)
    for (int k = 0; k < 4; ++k)
      for (int c = 0; c < 3; ++c) m->faceP[k + 4 * (c + 3 * (size_t)(iF - 1))] = S.faces[iF].P[k][c];
  gll(m->p, m->xw, m->w);
  int N = m->N;
  m->DS.assign(N * N, 0.0);
  m->DW.assign(N * N, 0.0);
  for (int i = 0; i < N; ++i)
    for (int j = 0; j < N; ++j) m->DS[i + N * j] = dlagrange(m->xw[i], m->xw, j);
  // DW = -inv(diagm(w)) * DS' * diagm(w): src/DG/DerivativeMatrixSingle.jl:10
  for (int i = 0; i < N; ++i)
    for (int j = 0; j < N; ++j) m->DW[i + N * j] = -(1.0 / m->w[i]) * m->DS[j + N * i] * m->w[j];
  build_metric(*m);
  build_inverse_map(*m);
  build_mass_dz(*m);
  build_fcor(*m);
  build_tableau(*m);
  return m;
}

void orc_destroy(void *h) { delete static_cast<Model *>(h); }

int orc_sizes(void *h, int64_t *out)
{
  Model *m = static_cast<Model *>(h);
  out[0] = m->NF; out[1] = m->NumG; out[2] = m->DoF; out[3] = m->N;
  out[4] = m->NumNodes; out[5] = m->NumEdges;
  return 0;
}

int orc_get_glob(void *h, int64_t *glob1)
{
  Model *m = static_cast<Model *>(h);
  for (size_t i = 0; i < m->glob.size(); ++i) glob1[i] = m->glob[i] + 1;
  return 0;
}

int orc_get_gll(void *h, double *xw, double *w, double *DS, double *DW)
{
  Model *m = static_cast<Model *>(h);
  memcpy(xw, m->xw.data(), m->N * sizeof(double));
  memcpy(w, m->w.data(), m->N * sizeof(double));
  memcpy(DS, m->DS.data(), m->N * m->N * sizeof(double));
  memcpy(DW, m->DW.data(), m->N * m->N * sizeof(double));
  return 0;
}

int orc_get_faces(void *h, double *F)
{
  Model *m = static_cast<Model *>(h);
  memcpy(F, m->faceP.data(), m->faceP.size() * sizeof(double));
  return 0;
}

int orc_get_metric(void *h, double *X, double *dXdxI, double *J)
{
  Model *m = static_cast<Model *>(h);
  if (X) memcpy(X, m->X.data(), m->X.size() * sizeof(double));
  if (dXdxI) memcpy(dXdxI, m->dXdxI.data(), m->dXdxI.size() * sizeof(double));
  if (J) memcpy(J, m->J.data(), m->J.size() * sizeof(double));
  return 0;
}

int orc_get_mass(void *h, double *M, double *MMass)
{
  Model *m = static_cast<Model *>(h);
  if (M) memcpy(M, m->M.data(), m->M.size() * sizeof(double));
  if (MMass) memcpy(MMass, m->MMass.data(), m->MMass.size() * sizeof(double));
  return 0;
}

int orc_get_dz(void *h, double *dz)
{
  Model *m = static_cast<Model *>(h);
  memcpy(dz, m->dz.data(), m->dz.size() * sizeof(double));
  return 0;
}

int orc_set_metric(void *h, const double *X, const double *dXdxI, const double *J,
                   const double *M, const double *dz)
{
  Model *m = static_cast<Model *>(h);
  if (X) { memcpy(m->X.data(), X, m->X.size() * sizeof(double)); build_fcor(*m); }
  if (dXdxI) memcpy(m->dXdxI.data(), dXdxI, m->dXdxI.size() * sizeof(double));
  if (J) memcpy(m->J.data(), J, m->J.size() * sizeof(double));
  if (M) memcpy(m->M.data(), M, m->M.size() * sizeof(double));
  if (dz) memcpy(m->dz.data(), dz, m->dz.size() * sizeof(double));
  return 0;
}

// InitialConditions (src/GPU/InitialConditions.jl:1-68) with the init kernels
// of src/GPU/InitialKernel.jl:1-116: each element writes every global node it
// holds, so the element written last (highest index) wins.  Tracers: Gaussian
// blobs q = exp(-(d/1e6 m)^2) (d great-circle distance on the sphere), slot rho*q.
int orc_init_state(void *h, double *U, const double *tracer_lonlat)
{
  Model *m = static_cast<Model *>(h);
  int nz = m->nz, DoF = m->DoF, NumG = m->NumG;
  size_t S = (size_t)nz * NumG * m->NV;
  std::fill(U, U + S, 0.0);
  auto Uv = [&](int Iz, int g, int v) -> double & { return U[Iz + (size_t)nz * (g + (size_t)NumG * v)]; };
  for (int IF = 0; IF < m->NF; ++IF)
    for (int Iz = 0; Iz < nz; ++Iz)
      for (int ID = 0; ID < DoF; ++ID) {
        int g = m->glob[ID + (size_t)DoF * IF];
        double x[3];
        for (int c = 0; c < 3; ++c) x[c] = 0.5 * (XX(*m, ID, 0, c, Iz, IF) + XX(*m, ID, 1, c, Iz, IF));
        double Rho, uS, vS, w, Th;
        barowave(*m, x, Rho, uS, vS, w, Th);
        Uv(Iz, g, 0) = Rho;
        Uv(Iz, g, 1) = uS;
        Uv(Iz, g, 2) = vS;
        Uv(Iz, g, 4) = Rho * Th;
        double r = std::sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
        for (int iT = 0; iT < m->NumTr; ++iT) {
          double lon = tracer_lonlat[2 * iT], lat = tracer_lonlat[2 * iT + 1];
          double cx = std::cos(lat) * std::cos(lon), cy = std::cos(lat) * std::sin(lon), cz = std::sin(lat);
          double d = (x[0] * cx + x[1] * cy + x[2] * cz) / r;
          d = std::min(1.0, std::max(-1.0, d));
          double dist = m->phys.RadEarth * std::acos(d) / 1.0e6;
          Uv(Iz, g, 5 + iT) = Rho * std::exp(-dist * dist);
        }
        if (Iz <= nz - 2) {
          for (int c = 0; c < 3; ++c) x[c] = 0.5 * (XX(*m, ID, 1, c, Iz, IF) + XX(*m, ID, 0, c, Iz + 1, IF));
          barowave(*m, x, Rho, uS, vS, w, Th);
          Uv(Iz, g, 3) = w;
        }
      }
  return 0;
}

int orc_pressure(void *h, const double *U, double *p)
{
  Model *m = static_cast<Model *>(h);
  size_t S = (size_t)m->nz * m->NumG;
  for (size_t q = 0; q < S; ++q) p[q] = pressure(m->phys, U[q + 4 * S]);
  return 0;
}

int orc_hypervisc1(void *h, const double *U, double *Temp1)
{
  Model *m = static_cast<Model *>(h);
  Ctx c(*m, U);
  int nf1 = 5 + m->NumTr;
  std::vector<double> C1((size_t)m->NF * m->nz * nf1 * m->DoF);
  #pragma omp parallel for schedule(dynamic, 4)
  for (int IF = 0; IF < m->NF; ++IF) hypervisc1_element(*m, c, IF, C1);
  gather(*m, C1, nf1, Temp1);
  return 0;
}

// The element-node contributions before their DSS, layout
// ((IF*nz + Iz)*nf + f)*DoF + ID: phase 1 (T1 == NULL, nf = 5 + NumTr) or
// phase 2 at the DSS'd phase-1 cache T1 (nf = NV).  orc_hypervisc1 and
// orc_rhs are these summed per global DOF in ascending (element, node) order.
int orc_contributions(void *h, const double *U, const double *T1, double *C)
{
  Model *m = static_cast<Model *>(h);
  Ctx c(*m, U);
  const int nf = T1 ? m->NV : 5 + m->NumTr;
  std::vector<double> Cv((size_t)m->NF * m->nz * nf * m->DoF);
  #pragma omp parallel for schedule(dynamic, 4)
  for (int IF = 0; IF < m->NF; ++IF) {
    if (T1) phase2_element(*m, c, T1, IF, Cv);
    else hypervisc1_element(*m, c, IF, Cv);
  }
  memcpy(C, Cv.data(), Cv.size() * sizeof(double));
  return 0;
}

// Column physics: the surface latitude of every column from the bottom node
// of its highest-numbered element node (MetricLowerBoundaryKernel!,
// src/DyCore/DiscretizationCG.jl:159-178, cart2sphere src/Grids/Geometry.jl:65-73),
// the layer-midpoint height zP (GridSizeSphereKernel!, DiscretizationCG.jl:119-144)
// and the damping coefficient there.
int orc_set_physics(void *h, int held_suarez, const double *hs8, int damping, double damp_H, double damp_stride,
                    double damp_relax)
{
  Model *m = static_cast<Model *>(h);
  m->held_suarez = held_suarez;
  m->damping = damping;
  for (int i = 0; i < 8; ++i) m->hs[i] = hs8 ? hs8[i] : 0.0;
  const int nz = m->nz, NumG = m->NumG, DoF = m->DoF;
  m->coslat.assign(NumG, 0.0);
  m->sinlat.assign(NumG, 0.0);
  m->dampc.assign((size_t)nz * NumG, 0.0);
  const double pi = 3.141592653589793;
  for (int IF = 0; IF < m->NF; ++IF)
    for (int ID = 0; ID < DoF; ++ID) {
      const int g = m->glob[ID + (size_t)DoF * IF];
      const double x = XX(*m, ID, 0, 0, 0, IF), y = XX(*m, ID, 0, 1, 0, IF), z = XX(*m, ID, 0, 2, 0, IF);
      const double r = std::sqrt(x * x + y * y + z * z);
      const double lat = std::asin(z / r);
      m->coslat[g] = std::cos(lat);
      m->sinlat[g] = std::sin(lat);
      for (int Iz = 0; Iz < nz; ++Iz) {
        const double xm = 0.5 * (XX(*m, ID, 0, 0, Iz, IF) + XX(*m, ID, 1, 0, Iz, IF));
        const double ym = 0.5 * (XX(*m, ID, 0, 1, Iz, IF) + XX(*m, ID, 1, 1, Iz, IF));
        const double zm = 0.5 * (XX(*m, ID, 0, 2, Iz, IF) + XX(*m, ID, 1, 2, Iz, IF));
        const double rm = std::sqrt(xm * xm + ym * ym + zm * zm);
        const double zP = std::max(rm - m->Rad, 0.0);
        double c = 0.0;
        if (zP >= damp_H - damp_stride) {
          const double sn = std::sin(0.5 * pi * (1.0 - (damp_H - zP) / damp_stride));
          c = damp_relax * (sn * sn);
        }
        m->dampc[Iz + (size_t)nz * g] = c;
      }
    }
  return 0;
}

int orc_rhs(void *h, const double *U, double *F)
{
  rhs(*static_cast<Model *>(h), U, F);
  return 0;
}

int orc_jac(void *h, const double *U, double *bands)
{
  Model *m = static_cast<Model *>(h);
  jac(*m, U);
  if (bands) memcpy(bands, m->bands.data(), m->bands.size() * sizeof(double));
  return 0;
}

int orc_schur(void *h, double *k, double *v, double fac)
{
  Model *m = static_cast<Model *>(h);
  if (m->bands.empty()) return -1;
  schur(*m, k, v, fac);
  return 0;
}

int orc_ros_step(void *h, double *U, double dt, int nsteps)
{
  Model *m = static_cast<Model *>(h);
  for (int s = 0; s < nsteps; ++s) ros_step(*m, U, dt);
  return 0;
}

double orc_mass_integral(void *h, const double *U)
{
  Model *m = static_cast<Model *>(h);
  size_t S = (size_t)m->nz * m->NumG;
  double acc = 0.0;
  for (size_t q = 0; q < S; ++q) acc += U[q] * m->MMass[q];
  return acc;
}

// ---------------------------------------------------------------------------
// Output interpolation (src/Outputs).  Cell (I,J) of element IF, layer Iz:
// the GLL interpolant at the sub-cell centre, Inter[I,J,iP,jP] summed over
// the element's nodes in the reference's loop order (jP outer, iP inner).
// ---------------------------------------------------------------------------
// DG.Lagrange: src/DG/Lagrange.jl:1-9
static double lagrange(double x, const double *xP, int n, int iP)
{
  double f = 1;
  for (int i = 0; i < n; ++i)
    if (i != iP) f = f * (x - xP[i]) / (xP[iP] - xP[i]);
  return f;
}

int orc_vtk_inter(int OrdPoly, int OrdPrint, const double *xw, double *inter)
{
  // vtkStruct's vtkInter: src/Outputs/vtkSphere.jl:199-219
  const int N = OrdPoly + 1, OP = OrdPrint;
  std::fill(inter, inter + (size_t)OP * OP * N * N, 0.0);
  const double dd = 2.0 / OP;
  double eta0 = -1;
  for (int jRef = 1; jRef <= OP; ++jRef) {
    double ksi0 = -1;
    const double eta1 = eta0 + dd;
    for (int iRef = 1; iRef <= OP; ++iRef) {
      const double ksi1 = ksi0 + dd;
      for (int j = 1; j <= N; ++j)
        for (int i = 1; i <= N; ++i) {
          double &v = inter[(iRef - 1) + OP * ((jRef - 1) + OP * ((i - 1) + N * (j - 1)))];
          v = v + lagrange(0.5 * (ksi0 + ksi1), xw, N, i - 1) * lagrange(0.5 * (eta0 + eta1), xw, N, j - 1);
        }
      ksi0 = ksi1;
    }
    eta0 = eta1;
  }
  return 0;
}

// kind 0: InterpolateKernel! (src/Outputs/vtkOutputKernel.jl:49-74), or with
// rhoc InterpolateRhoKernel! (:97-121); kind 1: of the dry pressure, kind 2:
// of the dry potential temperature (p, T, PotT of src/Models/Equation.jl:24-32,
// c = rho*theta, rhoc = rho).
int orc_interpolate(void *h, const double *c, const double *rhoc, int kind, const double *inter, int OP,
                    double *cell)
{
  Model *m = static_cast<Model *>(h);
  const int N = m->N, nz = m->nz, OP2 = OP * OP;
  const Phys &ph = m->phys;
  for (int IF = 0; IF < m->NF; ++IF)
    for (int Iz = 0; Iz < nz; ++Iz)
      for (int J = 0; J < OP; ++J)
        for (int I = 0; I < OP; ++I) {
          double acc = 0;
          for (int jP = 0; jP < N; ++jP)
            for (int iP = 0; iP < N; ++iP) {
              const int iD = iP + N * jP;
              const size_t o = Iz + (size_t)nz * m->glob[iD + (size_t)m->DoF * IF];
              const double w = inter[I + OP * J + (size_t)OP2 * iD];
              if (kind == 1) {
                acc += w * pressure(ph, c[o]);
              } else if (kind == 2) {
                const double p = pressure(ph, c[o]);
                const double T = p / (ph.Rd * rhoc[o]);
                acc += w * (std::pow(ph.p0 / p, ph.Rd / ph.Cpd) * T);
              } else if (rhoc) {
                acc += w * c[o] / rhoc[o];
              } else {
                acc += w * c[o];
              }
            }
          cell[I + OP * (J + (size_t)OP * (Iz + (size_t)nz * IF))] = acc;
        }
  return 0;
}

// InterpolateWBKernel!: src/Outputs/vtkOutputKernel.jl:123-159
int orc_interpolate_wb(void *h, const double *u, const double *v, const double *w, const double *inter, int OP,
                       double *cell)
{
  Model *m = static_cast<Model *>(h);
  const int N = m->N, nz = m->nz, OP2 = OP * OP;
  for (int IF = 0; IF < m->NF; ++IF)
    for (int Iz = 0; Iz < nz; ++Iz)
      for (int J = 0; J < OP; ++J)
        for (int I = 0; I < OP; ++I) {
          double acc = 0;
          for (int jP = 0; jP < N; ++jP)
            for (int iP = 0; iP < N; ++iP) {
              const int iD = iP + N * jP;
              const size_t o = Iz + (size_t)nz * m->glob[iD + (size_t)m->DoF * IF];
              const double wi = 0.5 * inter[I + OP * J + (size_t)OP2 * iD];
              if (Iz == 0) {
                const double w0 = -(u[o] * DXI(*m, 3, 1, 0, iD, Iz, IF) + v[o] * DXI(*m, 3, 2, 0, iD, Iz, IF)) /
                                  DXI(*m, 3, 3, 0, iD, Iz, IF);
                acc += wi * (w[o] + w0);
              } else {
                acc += wi * (w[o] + w[o - 1]);
              }
            }
          cell[I + OP * (J + (size_t)OP * (Iz + (size_t)nz * IF))] = acc;
        }
  return 0;
}

// InterpolateRotKernel!: src/Outputs/vtkOutputKernel.jl:1-47 (its atomic
// sums in ascending node order: the xi sum, then the eta sum, from 0).
int orc_interpolate_vort(void *h, const double *U, const double *inter, int OP, double *cell)
{
  Model *m = static_cast<Model *>(h);
  const int N = m->N, DoF = m->DoF, nz = m->nz, OP2 = OP * OP;
  const size_t S = (size_t)nz * m->NumG;
  std::vector<double> tx(DoF), ty(DoF), rot(DoF);
  for (int IF = 0; IF < m->NF; ++IF)
    for (int Iz = 0; Iz < nz; ++Iz) {
      for (int ID = 0; ID < DoF; ++ID) {
        const size_t o = Iz + (size_t)nz * m->glob[ID + (size_t)DoF * IF];
        const double uu = U[o + S], vv = U[o + 2 * S];
        tx[ID] = (DXI(*m, 1, 1, 0, ID, Iz, IF) + DXI(*m, 1, 1, 1, ID, Iz, IF)) * vv -
                 (DXI(*m, 1, 2, 0, ID, Iz, IF) + DXI(*m, 1, 2, 1, ID, Iz, IF)) * uu;
        ty[ID] = (DXI(*m, 2, 1, 0, ID, Iz, IF) + DXI(*m, 2, 1, 1, ID, Iz, IF)) * vv -
                 (DXI(*m, 2, 2, 0, ID, Iz, IF) + DXI(*m, 2, 2, 1, ID, Iz, IF)) * uu;
      }
      for (int j = 0; j < N; ++j)
        for (int i = 0; i < N; ++i) {
          double acc = 0;
          for (int I = 0; I < N; ++I) acc += m->DS[i + N * I] * tx[I + N * j];
          for (int J = 0; J < N; ++J) acc += m->DS[j + N * J] * ty[i + N * J];
          rot[i + N * j] = acc / (JJ(*m, i + N * j, 0, Iz, IF) + JJ(*m, i + N * j, 1, Iz, IF));
        }
      for (int J = 0; J < OP; ++J)
        for (int I = 0; I < OP; ++I) {
          double acc = 0;
          for (int iD = 0; iD < DoF; ++iD) acc += inter[I + OP * J + (size_t)OP2 * iD] * rot[iD];
          cell[I + OP * (J + (size_t)OP * (Iz + (size_t)nz * IF))] = acc;
        }
    }
  return 0;
}

} // extern "C"
