// cgd_phase2.cuh - the fused tendency kernel (phase 2 of the RHS).
//
// One CTA per (element, chunk of LC levels); inside it one warp per level
// (N = 5: lanes 0..24 are the 25 nodes; for smaller N a warp holds
// LPW = 32 / N^2 levels).  Grid: (chunks, elements), chunks fastest so the
// chunks of one element, which share their halo planes, run together.
//
// The number of tracers NT is a template parameter.
//
//   1. The CTA stages the pointwise quantities of its LC levels plus two halo
//      planes on each side (state, vertical metric, lumped mass, pressure -
//      computed beforehand, once per column-level, by the kernel that forms
//      the state - theta and tracer ratios) in shared memory.  One barrier.
//   2. One thread per (node, interface) forms the vertical mass flux and the
//      limited upwind fluxes of the interfaces L0-1 .. L0+LC-1 (the one below
//      the chunk is formed by both neighbouring chunks, with identical
//      operations).  One barrier.
//   3. Each warp then works on its own level alone.  Every horizontal D/DW
//      derivative sum goes through a per-warp scratch with __syncwarp only;
//      the terms that couple levels read the neighbour planes staged in 1.
//
// The vertical momentum equation lives on interfaces: the contribution of
// the element node to w at interface l is hi(l) + lo(l+1), hi from the upper
// node of level l and lo from the lower node of level l+1.  Each level writes
// its hi into field 3 of the contribution buffer and its lo into the extra
// slot NV, one level down; the owner gather adds the pair per contributor.
//
// Expressions are the reference's (ViscKernel.jl:86-167,277-327,
// MomentumKernel.jl:1-178, GradKineticKernel.jl:1-129,
// OperatorKernel.jl:637-760) evaluated in the same order as the CPU
// restatement, with the same per-node contribution order.
#pragma once
#include "cgd_kernels.cuh"

namespace cgd {

// pointwise quantities per (plane, node)
enum {
  Q_RHO = 0, Q_U, Q_V, Q_W, Q_D310, Q_D311, Q_D320, Q_D321, Q_D330, Q_D331,
  Q_M0, Q_M1, Q_P, Q_J0, Q_CTH,
  Q_TR0   // + one per tracer: rho*q / rho
};


// quantities of the CTA's own levels per (level, node)
enum {
  O_D110 = 0, O_D111, O_D120, O_D121, O_D210, O_D211, O_D220, O_D221, O_J1, O_FC,
  O_N     // the DSS'd hyperviscosity cache (5 + NumTr fields) is staged into the warps' scratch
};

// Warps (levels for p = 4) per CTA: 8, two 256-thread CTAs per SM at 128
// registers a thread, so that one CTA's staging overlaps the other's
// arithmetic (at nPanel 30, nz 45: 1.415 ms against 1.533 ms for one
// 512-thread CTA of 16 levels, which re-stages fewer halo planes).  W > 0
// sets the warps instead (the batched ensemble's autotuner also tries 16).
template <int N, int NT, typename R, int W = 0>
struct P2Cfg {
  static constexpr int WARPS = W > 0 ? W : 8;
  static constexpr int DoF = N * N;
  static constexpr int LPW = 32 / DoF;           // levels per warp
  static constexpr int LC = WARPS * LPW;         // levels per CTA
  static constexpr int RP = LC + 4;              // staged planes
  static constexpr int THREADS = 32 * WARPS;
  // scratch quantities per warp (the largest derivative round: 5+NT, 4+2NT,
  // 6 for each half of the momentum round, 6+NT) and the scratch row length;
  // before round 1 the scratch holds the warp's levels of the DSS'd phase-1
  // cache (5 + NT fields, stored as R), staged with the rest
  static constexpr int NSCR = (4 + 2 * NT) > (6 + NT) ? (4 + 2 * NT) : (6 + NT);
  static_assert(NSCR >= 5 + NT, "the scratch holds the phase-1 cache");
  static constexpr int SCS = LPW * DoF;
  // warp stride of the scratch, odd in elements: the staging copies of the
  // cache (consecutive threads, consecutive levels, so consecutive warps'
  // regions) then fall into different shared-memory banks
  static constexpr int SCW = NSCR * SCS + ((NSCR * SCS) % 2 == 0 ? 1 : 0);
  // the own levels' phase-1 cache: float in the mixed form (as stored), else double
  using CT = typename std::conditional<sizeof(R) == sizeof(float), float, double>::type;
  static_assert(sizeof(CT) == sizeof(R), "cache and scratch share their type");
  static constexpr size_t SMEM = ((size_t)(Q_TR0 + NT) * RP * DoF + (size_t)O_N * LC * DoF +
                                   (size_t)(2 + NT) * (LC + 1) * DoF) * sizeof(double) +
                                  (size_t)WARPS * SCW * sizeof(R);
  // CTAs per SM the registers are sized for (128 registers a thread).  At
  // p = 4 with two tracers two CTAs take 154 KB of shared memory and leave
  // about 92 KB of the SM's unified array to L1, which the 8-byte cp.async
  // copies of the staging share sectors through: 1.347 ms per launch on the
  // drop-in grid, against 1.656 ms with the array carved out as shared
  // memory (28 KB of L1) and 1.901 ms with three CTAs of 80 registers.
  static constexpr int MINB = WARPS >= 16 ? 1 : 2;
};

template <int N, int NT, typename R, int W = 0>
__device__ __forceinline__ void phase2_body(const GP &P, const double *__restrict__ U, const double *__restrict__ Pr,
                                            const double *__restrict__ T1, double *__restrict__ C, const int chunk,
                                            const int IF)
{
  using CF = P2Cfg<N, NT, R, W>;
  constexpr bool MIX = sizeof(R) == sizeof(float);
  constexpr int DoF = CF::DoF, LPW = CF::LPW, LC = CF::LC, RP = CF::RP;
  extern __shared__ double sm[];
  const int nz = P.nz, NumG = P.NumG;
  const int L0 = chunk * LC;
  const size_t cs = (size_t)DoF * nz, fs = (size_t)nz * NumG;
  double *pw = sm;                                             // [Q][R][DoF]
  using CTc = typename CF::CT;
  double *ow = pw + (size_t)(Q_TR0 + NT) * RP * DoF;             // [O][LC][DoF]
  double *fx = ow + (size_t)O_N * LC * DoF;                     // [2+NT][LC+1][DoF] interface fluxes
  R *scr = reinterpret_cast<R *>(fx + (size_t)(2 + NT) * (LC + 1) * DoF);   // [warp][SCW >= NSCR*SCS]
  const double *mte = P.met + (size_t)IF * NCOMP * cs;
#define PW(q, p, id) pw[((size_t)(q) * RP + (p)) * DoF + (id)]

  // ---------------- 1. stage the pointwise planes L0-2 .. L0+LC+1 ----------------
  // (level fastest: every load is a run of consecutive levels of one column
  // or one metric row) and the own levels' metric and cache
  // at most two slots per thread (DoF * RP <= 2 * THREADS); every value is
  // copied with cp.async, so all of a thread's copies are in flight at once
  static_assert(DoF * RP <= 2 * CF::THREADS, "two staging slots per thread");
#pragma unroll
  for (int r = 0; r < 2; ++r) {
    const int s = threadIdx.x + r * CF::THREADS;
    if (s >= DoF * RP) continue;
    const int ID = s / RP, p = s % RP;
    const int lev = L0 - 2 + p;
    if (lev < 0 || lev >= nz) continue;
    const int g = P.glob[IF * DoF + ID];
    const double *Ug = U + (size_t)nz * g + lev;
    const double *mt = mte + (size_t)ID * nz + lev;
    if (p >= 2 && p <= LC + 1) {
      double *o = ow + (size_t)(p - 2) * DoF + ID;
      constexpr size_t os = (size_t)LC * DoF;
      cp_async8(o + O_D110 * os, mt + C_D11_0 * cs); cp_async8(o + O_D111 * os, mt + C_D11_1 * cs);
      cp_async8(o + O_D120 * os, mt + C_D12_0 * cs); cp_async8(o + O_D121 * os, mt + C_D12_1 * cs);
      cp_async8(o + O_D210 * os, mt + C_D21_0 * cs); cp_async8(o + O_D211 * os, mt + C_D21_1 * cs);
      cp_async8(o + O_D220 * os, mt + C_D22_0 * cs); cp_async8(o + O_D221 * os, mt + C_D22_1 * cs);
      cp_async8(o + O_J1 * os, mt + C_J1 * cs);
      cp_async8(o + O_FC * os, mt + C_FCOR * cs);
      // the cache goes to the scratch slots SC(f, ID) of the level's warp
      const int li = p - 2;
      CTc *oc = reinterpret_cast<CTc *>(scr) + ((size_t)(li / LPW) * CF::SCW + (li % LPW) * DoF + ID);
      if (MIX) {   // the mixed form's phase-1 cache is stored as float, and staged as float
        const float *T = reinterpret_cast<const float *>(T1) + (size_t)nz * g + lev;
#pragma unroll
        for (int f = 0; f < 5 + NT; ++f) cp_async4(reinterpret_cast<float *>(oc) + f * CF::SCS, T + f * fs);
      } else {
        const double *T = T1 + (size_t)nz * g + lev;
#pragma unroll
        for (int f = 0; f < 5 + NT; ++f) cp_async8(reinterpret_cast<double *>(oc) + f * CF::SCS, T + f * fs);
      }
    }
    cp_async8(&PW(Q_RHO, p, ID), Ug);
    cp_async8(&PW(Q_CTH, p, ID), Ug + 4 * fs);   // rho*theta for now
#pragma unroll
    for (int q = 0; q < NT; ++q) cp_async8(&PW(Q_TR0 + q, p, ID), Ug + (5 + q) * fs);   // rho*q for now
    if (p == 0 || p == RP - 1) continue;   // the outer halo planes feed the upwind stencil only
    cp_async8(&PW(Q_U, p, ID), Ug + fs);
    cp_async8(&PW(Q_V, p, ID), Ug + 2 * fs);
    cp_async8(&PW(Q_W, p, ID), Ug + 3 * fs);
    cp_async8(&PW(Q_D310, p, ID), mt + C_D31_0 * cs); cp_async8(&PW(Q_D311, p, ID), mt + C_D31_1 * cs);
    cp_async8(&PW(Q_D320, p, ID), mt + C_D32_0 * cs); cp_async8(&PW(Q_D321, p, ID), mt + C_D32_1 * cs);
    cp_async8(&PW(Q_D330, p, ID), mt + C_D33_0 * cs); cp_async8(&PW(Q_D331, p, ID), mt + C_D33_1 * cs);
    cp_async8(&PW(Q_J0, p, ID), mt + C_J0 * cs);
    cp_async8(&PW(Q_M0, p, ID), P.M + lev + (size_t)nz * g);
    cp_async8(&PW(Q_M1, p, ID), P.M + lev + (size_t)nz * (g + (size_t)NumG));
    cp_async8(&PW(Q_P, p, ID), Pr + lev + (size_t)nz * g);
  }
  // theta and the tracer ratios of the staged planes, each formed by the
  // thread that copied its rho*theta, rho*q and rho (its own copies have
  // landed after its wait), then one barrier
  cp_async_wait_all();
#pragma unroll
  for (int r = 0; r < 2; ++r) {
    const int s = threadIdx.x + r * CF::THREADS;
    if (s >= DoF * RP) continue;
    const int ID = s / RP, p = s % RP;
    const int lev = L0 - 2 + p;
    if (lev < 0 || lev >= nz) continue;
    const double rho = PW(Q_RHO, p, ID);
    PW(Q_CTH, p, ID) = PW(Q_CTH, p, ID) / rho;
#pragma unroll
    for (int q = 0; q < NT; ++q) PW(Q_TR0 + q, p, ID) = PW(Q_TR0 + q, p, ID) / rho;
  }
  __syncthreads();

  // ---------------- 2. interface fluxes ----------------
  // wCon and the limited upwind fluxes (RecU4, OperatorKernel.jl:1044-1059,
  // J-only coefficients precomputed) of the interface il between levels il
  // and il+1, stored unscaled per interface
  for (int s = threadIdx.x; s < DoF * (LC + 1); s += CF::THREADS) {
    const int ID = s / (LC + 1), i = s % (LC + 1);
    const int il = L0 - 1 + i;
    if (il < 0 || il >= nz - 1) continue;
    const int pl = i + 1;   // plane of level il
    const double wI = PW(Q_W, pl, ID);
    const double wCon =
        PW(Q_RHO, pl, ID) * (PW(Q_D311, pl, ID) * PW(Q_U, pl, ID) + PW(Q_D321, pl, ID) * PW(Q_V, pl, ID) +
                             PW(Q_D331, pl, ID) * wI) +
        PW(Q_RHO, pl + 1, ID) * (PW(Q_D310, pl + 1, ID) * PW(Q_U, pl + 1, ID) +
                                 PW(Q_D320, pl + 1, ID) * PW(Q_V, pl + 1, ID) + PW(Q_D330, pl + 1, ID) * wI);
    const double *mt = mte + (size_t)ID * nz + il;
    const double kR1 = mt[C_RK0 * cs], kL1 = mt[C_RK1 * cs], kL2 = mt[C_RK2 * cs], kR2 = mt[C_RK3 * cs];
    const int pm = il > 0 ? pl - 1 : pl, pp2 = il + 2 < nz ? pl + 2 : pl + 1;
    const double aw = fabs(wCon);
    auto upwind = [&](int q) {
      const double cLL = PW(q, pm, ID), cL = PW(q, pl, ID), cR = PW(q, pl + 1, ID), cRR = PW(q, pp2, ID);
      double r = (cL - cLL) / (cR - cL + 1.e-20);
      const double cFL = cL + cgd_max(0.0, cgd_min(r, cgd_min(kL1 * r + kR1, 1.0))) * (cR - cL);
      r = (cR - cRR) / (cL - cR + 1.e-20);
      const double cFR = cR + cgd_max(0.0, cgd_min(r, cgd_min(kR2 * r + kL2, 1.0))) * (cL - cR);
      return 0.25 * ((aw + wCon) * cFL + (-aw + wCon) * cFR);
    };
    double *f = fx + (size_t)i * DoF + ID;
    f[0] = wCon;
    f[(LC + 1) * DoF] = upwind(Q_CTH);
#pragma unroll
    for (int q = 0; q < NT; ++q) f[(2 + q) * (LC + 1) * DoF] = upwind(Q_TR0 + q);
  }
  __syncthreads();

  // ---------------- 3. one level per warp (LPW levels for N < 5) ----------------
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int sub = lane / DoF, ID = lane - sub * DoF;
  const int lv = L0 + warp * LPW + sub;
  const bool act = sub < LPW && lv < nz;
  const int I = ID % N, Jn = ID / N;
  const int p0 = lv - (L0 - 2);          // own plane
  constexpr int SCS = CF::SCS;
  R *sw = scr + (size_t)warp * CF::SCW + sub * DoF;     // this level's scratch row base
#define SC(q, id) sw[(q) * SCS + (id)]

  // derivative coefficients of this node
  R DI[N], DJ[N];
#pragma unroll
  for (int k = 0; k < N; ++k) {
    DI[k] = (R)P.D[I + N * k];
    DJ[k] = (R)P.D[Jn + N * k];
  }
  // own quantities
  const int li = lv - L0;                // own row of the per-level arrays
#define OW(q) ow[((size_t)(q) * LC + li) * DoF + ID]
#define OT(f) SC(f, ID)   // own level's DSS'd phase-1 cache, in the scratch until round 1 overwrites it
  double rho = 1, u = 0, v = 0, wl = 0, wh = 0, M0 = 1, M1 = 0, MC = 1, Js = 1, J0 = 0, J1 = 0;
  double e310 = 0, e311 = 0, e320 = 0, e321 = 0, e330 = 1, e331 = 1;
  if (act) {
    J1 = OW(O_J1);
    rho = PW(Q_RHO, p0, ID); u = PW(Q_U, p0, ID); v = PW(Q_V, p0, ID); wh = PW(Q_W, p0, ID);
    e310 = PW(Q_D310, p0, ID); e311 = PW(Q_D311, p0, ID); e320 = PW(Q_D320, p0, ID);
    e321 = PW(Q_D321, p0, ID); e330 = PW(Q_D330, p0, ID); e331 = PW(Q_D331, p0, ID);
    J0 = PW(Q_J0, p0, ID);
    M0 = PW(Q_M0, p0, ID); M1 = PW(Q_M1, p0, ID);
    Js = J0 + J1;
    MC = M0 + M1;
    // surface w from no normal flow (MomentumKernel.jl:35-36)
    wl = lv == 0 ? -(e310 * u + e320 * v) / e330 : PW(Q_W, p0 - 1, ID);
  }
  const double rJs = 1.0 / Js, rMC = 1.0 / MC;
  (void)rJs; (void)rMC;
  // the horizontal metric of the own level, held in registers through the
  // rounds (each __syncwarp would otherwise make the compiler re-read it from
  // shared memory): the components and the sums over the two nodes
  double c110 = 0.0, c111 = 0.0, c120 = 0.0, c121 = 0.0, c210 = 0.0, c211 = 0.0, c220 = 0.0, c221 = 0.0;
  if (act) {
    c110 = OW(O_D110); c111 = OW(O_D111); c120 = OW(O_D120); c121 = OW(O_D121);
    c210 = OW(O_D210); c211 = OW(O_D211); c220 = OW(O_D220); c221 = OW(O_D221);
  }
  const double d11s = c110 + c111, d12s = c120 + c121, d21s = c210 + c211, d22s = c220 + c221;

  // ---- round 1: first derivatives of the DSS'd hyperviscosity cache ----
  if (act) {
    const R d11 = (R)d11s, d12 = (R)d12s, d21 = (R)d21s, d22 = (R)d22s;
    // each lane reads and writes only its own column ID of the scratch; the
    // tracer caches stay in place as SC(5 + q)
    const R c1 = OT(0), c2 = OT(1), c3 = OT(2), c4 = OT(3), c5 = OT(4);
    SC(0, ID) = d11 * c2 - d12 * c1;       // Curl12(Cache1, Cache2)
    SC(1, ID) = d21 * c2 - d22 * c1;
    SC(2, ID) = d11 * c3 + d12 * c4;       // Contra12(Cache3, Cache4)
    SC(3, ID) = d21 * c3 + d22 * c4;
    SC(4, ID) = c5;
  }
  __syncwarp();
  R b1 = 0, b2 = 0, b3 = 0, b4 = 0;
  R e3t[NT > 0 ? NT : 1], e4t[NT > 0 ? NT : 1];
  if (act) {
    const R d11 = (R)d11s, d12 = (R)d12s, d21 = (R)d21s, d22 = (R)d22s;
    {
      R Dxc = DI[0] * SC(4, N * Jn), Dyc = DJ[0] * SC(4, I);
      R cu = DI[0] * SC(0, N * Jn) + DJ[0] * SC(1, I);
      R dv = DI[0] * SC(2, N * Jn) + DJ[0] * SC(3, I);
#pragma unroll
      for (int k = 1; k < N; ++k) {
        Dxc = rsum1(Dxc, DI[k], SC(4, k + N * Jn));
        Dyc = rsum1(Dyc, DJ[k], SC(4, I + N * k));
        cu = rsum2(cu, DI[k], SC(0, k + N * Jn), DJ[k], SC(1, I + N * k));
        dv = rsum2(dv, DI[k], SC(2, k + N * Jn), DJ[k], SC(3, I + N * k));
      }
      b1 = CGD_DIVJ(cu);
      b2 = CGD_DIVJ(dv);
      const R GradDx = CGD_DIVJ(d11 * Dxc + d21 * Dyc);
      const R GradDy = CGD_DIVJ(d12 * Dxc + d22 * Dyc);
      b3 = rho * (d11 * GradDx + d12 * GradDy);
      b4 = rho * (d21 * GradDx + d22 * GradDy);
    }
#pragma unroll
    for (int q = 0; q < NT; ++q) {
      {
        R Dxc = DI[0] * SC(5 + q, N * Jn), Dyc = DJ[0] * SC(5 + q, I);
#pragma unroll
        for (int k = 1; k < N; ++k) {
          Dxc = rsum1(Dxc, DI[k], SC(5 + q, k + N * Jn));
          Dyc = rsum1(Dyc, DJ[k], SC(5 + q, I + N * k));
        }
        const R GradDx = CGD_DIVJ(d11 * Dxc + d21 * Dyc);
        const R GradDy = CGD_DIVJ(d12 * Dxc + d22 * Dyc);
        e3t[q] = rho * (d11 * GradDx + d12 * GradDy);
        e4t[q] = rho * (d21 * GradDx + d22 * GradDy);
      }
    }
  }
  __syncwarp();
  // ---- round 2: second (weak) derivatives -> hyperviscosity tendencies ----
  if (act) {
    SC(0, ID) = b1; SC(1, ID) = b2; SC(2, ID) = b3; SC(3, ID) = b4;
#pragma unroll
    for (int q = 0; q < NT; ++q) { SC(4 + 2 * q, ID) = e3t[q]; SC(5 + 2 * q, ID) = e4t[q]; }
  }
  __syncwarp();
  // The element-node contributions are accumulated in the restatement's order
  // (rho: flux top, flux bottom, horizontal divergence; u, v: hyperviscosity,
  // momentum, gradient; rho*theta and tracers: hyperviscosity, flux top, flux
  // bottom, horizontal divergence) as soon as each term is available.
  double acc_r = 0.0, acc_u = 0.0, acc_v = 0.0, acc_th = 0.0, acc_tr[NT > 0 ? NT : 1];
  if (act) {
    R WI[N], WJ[N];
#pragma unroll
    for (int k = 0; k < N; ++k) {
      WI[k] = (R)P.DW[I + N * k];
      WJ[k] = (R)P.DW[Jn + N * k];
    }
    R DxCurl = WI[0] * SC(0, N * Jn), DyCurl = WJ[0] * SC(0, I);
    R DxDiv = WI[0] * SC(1, N * Jn), DyDiv = WJ[0] * SC(1, I);
    R DivTh = WI[0] * SC(2, N * Jn) + WJ[0] * SC(3, I);
#pragma unroll
    for (int k = 1; k < N; ++k) {
      DxCurl = rsum1(DxCurl, WI[k], SC(0, k + N * Jn));
      DyCurl = rsum1(DyCurl, WJ[k], SC(0, I + N * k));
      DxDiv = rsum1(DxDiv, WI[k], SC(1, k + N * Jn));
      DyDiv = rsum1(DyDiv, WJ[k], SC(1, I + N * k));
      DivTh = rsum2(DivTh, WI[k], SC(2, k + N * Jn), WJ[k], SC(3, I + N * k));
    }
    const R d11 = (R)d11s, d12 = (R)d12s, d21 = (R)d21s, d22 = (R)d22s;
    const R FuC = d12 * DxCurl + d22 * DyCurl;
    const R FvC = -d11 * DxCurl - d21 * DyCurl;
    const R FuD = d11 * DxDiv + d21 * DyDiv;
    const R FvD = d12 * DxDiv + d22 * DyDiv;
    acc_u += CGD_DIVM(-(-P.nuCurl * FuC + P.nuGrad * FuD));
    acc_v += CGD_DIVM(-(-P.nuCurl * FvC + P.nuGrad * FvD));
    acc_th += CGD_DIVM(-P.nuDiv * DivTh);
#pragma unroll
    for (int q = 0; q < NT; ++q) {
      {
        R DivTr = WI[0] * SC(4 + 2 * q, N * Jn) + WJ[0] * SC(5 + 2 * q, I);
#pragma unroll
        for (int k = 1; k < N; ++k)
          DivTr = rsum2(DivTr, WI[k], SC(4 + 2 * q, k + N * Jn), WJ[k], SC(5 + 2 * q, I + N * k));
        acc_tr[q] = 0.0;
        acc_tr[q] += CGD_DIVM(-P.nuDiv * DivTr);
      }
    }
  }
  __syncwarp();
  const bool top = act && lv < nz - 1, bot = act && lv > 0;
  // ---- vertical fluxes of the two interfaces of the level
#define FX(k, il) fx[((size_t)(k) * (LC + 1) + (il) - (L0 - 1)) * DoF + ID]
  if (top) {
    acc_r += CGD_DIVM(-(0.5 * FX(0, lv)));
    acc_th += CGD_DIVM(-FX(1, lv));
#pragma unroll
    for (int q = 0; q < NT; ++q) acc_tr[q] += CGD_DIVM(-FX(2 + q, lv));
  }
  if (bot) {
    acc_r += CGD_DIVM(0.5 * FX(0, lv - 1));
    acc_th += CGD_DIVM(FX(1, lv - 1));
#pragma unroll
    for (int q = 0; q < NT; ++q) acc_tr[q] += CGD_DIVM(FX(2 + q, lv - 1));
  }
  // ---- round 3: vector-invariant momentum, in two halves of six quantities ----
  const double tu0 = e330 * v - e320 * wl, tu1 = e331 * v - e321 * wh;
  const double tv0 = e330 * u - e310 * wl, tv1 = e331 * u - e311 * wh;
  const double tw0 = e320 * u - e310 * v, tw1 = e321 * u - e311 * v;
  R U1 = 0, U2 = 0, V1 = 0, V2 = 0, W1 = 0, W2 = 0;
  if (act) {
    const R d110 = (R)c110, d111 = (R)c111, d120 = (R)c120, d121 = (R)c121;
    const R d210 = (R)c210, d220 = (R)c220, d221 = (R)c221;
    const R wlR = (R)wl, whR = (R)wh;
    SC(0, ID) = -d120 * wlR;  SC(1, ID) = -d121 * whR;    // tempuZ1
    SC(2, ID) = -d220 * wlR;  SC(3, ID) = -d221 * whR;    // tempuZ2
    SC(4, ID) = -d110 * wlR;                              // tempvZ1 (lower)
    SC(5, ID) = -d210 * wlR;                              // tempvZ2 (lower)
    (void)d111;
  }
  __syncwarp();
  if (act) {
    U1 = (R)(0.5 * (tu1 - tu0)); U2 = U1;
    V1 = (R)(0.5 * (tv1 - tv0)); V2 = V1;
    W1 = (R)(0.5 * (tw1 - tw0)); W2 = W1;
#pragma unroll
    for (int k = 0; k < N; ++k) {
      U1 = rsum2(U1, DI[k], SC(0, k + N * Jn), DJ[k], SC(2, I + N * k));
      U2 = rsum2(U2, DI[k], SC(1, k + N * Jn), DJ[k], SC(3, I + N * k));
      V1 = rsum2(V1, DI[k], SC(4, k + N * Jn), DJ[k], SC(5, I + N * k));
    }
  }
  __syncwarp();
  if (act) {
    const R d110 = (R)c110, d111 = (R)c111, d120 = (R)c120, d121 = (R)c121;
    const R d210 = (R)c210, d211 = (R)c211, d220 = (R)c220, d221 = (R)c221;
    const R uR = (R)u, vR = (R)v, whR = (R)wh;
    SC(0, ID) = -d111 * whR;                              // tempvZ1 (upper)
    SC(1, ID) = -d211 * whR;                              // tempvZ2 (upper)
    SC(2, ID) = d120 * uR - d110 * vR;                    // tempwZ1
    SC(3, ID) = d121 * uR - d111 * vR;
    SC(4, ID) = d220 * uR - d210 * vR;                    // tempwZ2
    SC(5, ID) = d221 * uR - d211 * vR;
  }
  __syncwarp();
  // the w denominators (rho_l M1_l + rho_l+1 M0_l+1 at the interface); the fast
  // build multiplies by their reciprocals
  double mwhi = 0.0, mwlo = 0.0, den_hi = 1.0, den_lo = 1.0, rho1 = 0.0;
#ifdef CGD_FAST
#define CGD_DIVW(x, d) ((x) * (1.0 / (d)))
#else
#define CGD_DIVW(x, d) ((x) / (d))
#endif
  if (act) {
#pragma unroll
    for (int k = 0; k < N; ++k) {
      V2 = rsum2(V2, DI[k], SC(0, k + N * Jn), DJ[k], SC(1, I + N * k));
      W1 = rsum2(W1, DI[k], SC(2, k + N * Jn), DJ[k], SC(4, I + N * k));
      W2 = rsum2(W2, DI[k], SC(3, k + N * Jn), DJ[k], SC(5, I + N * k));
    }
    // vertical parts from the neighbour levels
    double FU = 0.0, FV = 0.0, FW1 = 0.0, FW2 = 0.0;
    if (bot) {
      const int pb = p0 - 1;
      const double ub = PW(Q_U, pb, ID), vb = PW(Q_V, pb, ID), wb = PW(Q_W, pb, ID);
      const double tu1b = PW(Q_D331, pb, ID) * vb - PW(Q_D321, pb, ID) * wb;
      const double tv1b = PW(Q_D331, pb, ID) * ub - PW(Q_D311, pb, ID) * wb;
      const double tw1b = PW(Q_D321, pb, ID) * ub - PW(Q_D311, pb, ID) * vb;
      const double FluxUZ = 0.5 * (tu0 - tu1b);
      const double FluxVZ = 0.5 * (tv0 - tv1b);
      const double FluxWZ = 0.5 * (tw0 - tw1b);
      FU += (-v * FluxWZ - wl * FluxVZ);
      FV += (u * FluxWZ - wl * FluxUZ);
      FW1 += (u * FluxVZ + v * FluxUZ);
      den_lo = PW(Q_RHO, pb, ID) * PW(Q_M1, pb, ID) + rho * M0;
    }
    if (top) {
      const int pa = p0 + 1;
      rho1 = PW(Q_RHO, pa, ID);
      const double u1 = PW(Q_U, pa, ID), v1 = PW(Q_V, pa, ID);
      const double wl1 = wh;   // the lower w of level lv+1 is the upper w of lv
      const double tu0a = PW(Q_D330, pa, ID) * v1 - PW(Q_D320, pa, ID) * wl1;
      const double tv0a = PW(Q_D330, pa, ID) * u1 - PW(Q_D310, pa, ID) * wl1;
      const double tw0a = PW(Q_D320, pa, ID) * u1 - PW(Q_D310, pa, ID) * v1;
      const double FluxUZt = 0.5 * (tu0a - tu1);
      const double FluxVZt = 0.5 * (tv0a - tv1);
      const double FluxWZt = 0.5 * (tw0a - tw1);
      FU += (-v * FluxWZt - wh * FluxVZt);
      FV += (u * FluxWZt - wh * FluxUZt);
      FW2 += (u * FluxVZt + v * FluxUZt);
      den_hi = rho1 * PW(Q_M0, pa, ID) + rho * M1;
    }
    const double fc = OW(O_FC);
    const double FuCor = v * fc, FvCor = -u * fc, FwCor = 0.0;
    FU += FuCor * (J0 + J1);
    FV += FvCor * (J0 + J1);
    FW1 += FwCor * J0;
    FW2 += FwCor * J1;
    acc_u += CGD_DIVM(-v * W1 - wl * V1 - v * W2 - wh * V2 + FU);
    acc_v += CGD_DIVM(u * W1 - wl * U1 + u * W2 - wh * U2 + FV);
    if (top) mwhi = CGD_DIVW(rho * (u * V2 + v * U2 + FW2), den_hi);
    if (bot) mwlo = CGD_DIVW(rho * (u * V1 + v * U1 + FW1), den_lo);
  }
  __syncwarp();
  // ---- round 4: kinetic-energy and pressure gradients, flux divergences ----
  const double K1s = 0.5 * (u * u + v * v) + 0.5 * (wl * wl);   // K on the bottom node
  const double K2s = 0.5 * (u * u + v * v) + 0.5 * (wh * wh);   // K on the top node
  if (act) {
    const double d11 = d11s, d12 = d12s, d21 = d21s, d22 = d22s;
    SC(0, ID) = (R)K1s;
    SC(1, ID) = (R)K2s;
    SC(2, ID) = (R)(-rho * (d11 * u + d12 * v));           // Contra12(-Rho, u, v)
    SC(3, ID) = (R)(-rho * (d21 * u + d22 * v));
    // pressure (the mixed form: its perturbation from the level's FP64
    // reference), theta and the tracer ratios of the own plane
    SC(4, ID) = (R)(PW(Q_P, p0, ID) - (MIX ? P.pref[lv] : 0.0));
    SC(5, ID) = (R)PW(Q_CTH, p0, ID);
#pragma unroll
    for (int q = 0; q < NT; ++q) SC(6 + q, ID) = (R)PW(Q_TR0 + q, p0, ID);
  }
  __syncwarp();
  if (!act) return;   // no warp-level synchronisation below
#ifdef CGD_FAST
  const double rrho = 1.0 / rho;
#define CGD_DIVR(x) ((x) * rrho)
#else
#define CGD_DIVR(x) ((x) / rho)
#endif
  double whi = 0.0, wlo = 0.0;
  {
    const R *pa = &SC(4, 0);
    R DXp = DI[0] * pa[N * Jn], DYp = DJ[0] * pa[I];
    R DXK1 = DI[0] * SC(0, N * Jn), DYK1 = DJ[0] * SC(0, I);
    R DXK2 = DI[0] * SC(1, N * Jn), DYK2 = DJ[0] * SC(1, I);
#pragma unroll
    for (int k = 1; k < N; ++k) {
      DXK1 = rsum1(DXK1, DI[k], SC(0, k + N * Jn));
      DYK1 = rsum1(DYK1, DJ[k], SC(0, I + N * k));
      DXK2 = rsum1(DXK2, DI[k], SC(1, k + N * Jn));
      DYK2 = rsum1(DYK2, DJ[k], SC(1, I + N * k));
      DXp = rsum1(DXp, DI[k], pa[k + N * Jn]);
      DYp = rsum1(DYp, DJ[k], pa[I + N * k]);
    }
    const double d110 = c110, d111 = c111, d120 = c120, d121 = c121;
    const double d210 = c210, d211 = c211, d220 = c220, d221 = c221;
    const double d11 = d110 + d111, d12 = d120 + d121, d21 = d210 + d211, d22 = d220 + d221;
    double GuF1 = -(d110 * DXK1 + d210 * DYK1);
    double GvF1 = -(d120 * DXK1 + d220 * DYK1);
    double GuF2 = -(d111 * DXK2 + d211 * DYK2);
    double GvF2 = -(d121 * DXK2 + d221 * DYK2);
    double Gradu = d11 * DXp + d21 * DYp;
    double Gradv = d12 * DXp + d22 * DYp;
    double GZ = -P.Grav * rho * (J0 + J1) / (e330 + e331);
    Gradu += GZ * (e310 + e311);
    Gradv += GZ * (e320 + e321);
    // kinetic-energy jumps to the neighbour levels
    double GwF2 = 0.0, K2b = 0.0, K1a = 0.0;
    if (bot) {
      const int pb = p0 - 1;
      const double ub = PW(Q_U, pb, ID), vb = PW(Q_V, pb, ID), wb = PW(Q_W, pb, ID);
      K2b = 0.5 * (ub * ub + vb * vb) + 0.5 * (wb * wb);
      GZ = 0.5 * (K1s - K2b);
      GuF1 += -GZ * e310;
      GvF1 += -GZ * e320;
    }
    if (top) {
      const int pa1 = p0 + 1;
      const double u1 = PW(Q_U, pa1, ID), v1 = PW(Q_V, pa1, ID);
      K1a = 0.5 * (u1 * u1 + v1 * v1) + 0.5 * (wh * wh);
      GZ = 0.5 * (K1a - K2s);
      GuF2 += -GZ * e311;
      GvF2 += -GZ * e321;
      GwF2 += -rho * GZ * e331;
    }
    GZ = 0.5 * (K2s - K1s);
    GuF2 += -GZ * e311;
    GuF1 += -GZ * e310;
    GvF2 += -GZ * e321;
    GvF1 += -GZ * e320;
    GwF2 += -rho * GZ * e331;
    acc_u += CGD_DIVM(GuF1 + GuF2 - CGD_DIVR(Gradu));
    acc_v += CGD_DIVM(GvF1 + GvF2 - CGD_DIVR(Gradv));
    // w: upper node of lv (interface lv) and lower node of lv (interface lv-1)
    if (top) {
      const int pa1 = p0 + 1;
      GZ = 0.5 * (PW(Q_P, pa1, ID) - PW(Q_P, p0, ID));
      const double Gradw = GZ * (e331 + PW(Q_D330, pa1, ID));
      const double Gradp = -(Gradw + P.Grav * (rho * J1 + rho1 * PW(Q_J0, pa1, ID)));
      whi = mwhi + CGD_DIVW(GwF2 + Gradp, den_hi);
    }
    if (bot) {
      double GwF1 = 0.0;
      double GZa = 0.5 * (K1s - K2b);
      GwF1 += -rho * GZa * e330;
      GZa = 0.5 * (K2s - K1s);
      GwF1 += -rho * GZa * e330;
      wlo = mwlo + CGD_DIVW(GwF1, den_lo);
    }
    // horizontal flux divergences
    const R *cc = &SC(5, 0);
    R DivRhoTr = DI[0] * SC(2, N * Jn) * cc[N * Jn] + DJ[0] * SC(3, I) * cc[I];
    R DivRho = DI[0] * SC(2, N * Jn) + DJ[0] * SC(3, I);
#pragma unroll
    for (int k = 1; k < N; ++k) {
      DivRhoTr = rsum2(DivRhoTr, DI[k] * SC(2, k + N * Jn), cc[k + N * Jn], DJ[k] * SC(3, I + N * k), cc[I + N * k]);
      DivRho = rsum2(DivRho, DI[k], SC(2, k + N * Jn), DJ[k], SC(3, I + N * k));
    }
    acc_th += CGD_DIVM(DivRhoTr);
    acc_r += CGD_DIVM(DivRho);
#pragma unroll
    for (int q = 0; q < NT; ++q) {
      {
        const R *ct = &SC(6 + q, 0);
        R Dv = DI[0] * SC(2, N * Jn) * ct[N * Jn] + DJ[0] * SC(3, I) * ct[I];
#pragma unroll
        for (int k = 1; k < N; ++k)
          Dv = rsum2(Dv, DI[k] * SC(2, k + N * Jn), ct[k + N * Jn], DJ[k] * SC(3, I + N * k), ct[I + N * k]);
        acc_tr[q] += CGD_DIVM(Dv);
      }
    }
  }
  // --- store the contributions
  using CT = typename std::conditional<MIX, float, double>::type;   // stored contributions
  CT *out = reinterpret_cast<CT *>(C) + ((size_t)IF * P.NC * DoF + ID) * nz + lv;
  out[0] = (CT)acc_r;
  out[cs] = (CT)acc_u;
  out[2 * cs] = (CT)acc_v;
  out[3 * cs] = (CT)whi;
  if (bot) out[(size_t)P.NV * cs - 1] = (CT)wlo;   // slot NV, one level down
  out[4 * cs] = (CT)acc_th;
#pragma unroll
  for (int q = 0; q < NT; ++q) out[(5 + q) * cs] = (CT)acc_tr[q];
#undef CGD_DIVR
#undef FX
#undef CGD_DIVW
#undef OW
#undef OT
#undef SC
#undef PW
}

template <int N, int NT, typename R>
__global__ void __launch_bounds__(P2Cfg<N, NT, R>::THREADS, P2Cfg<N, NT, R>::MINB)
    k_phase2(const GP P, const double *__restrict__ U, const double *__restrict__ Pr, const double *__restrict__ T1,
             double *__restrict__ C)
{
  phase2_body<N, NT, R>(P, U, Pr, T1, C, blockIdx.x, P.IF0 + blockIdx.y);
}

}  // namespace cgd
