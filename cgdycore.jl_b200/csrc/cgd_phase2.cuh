// cgd_phase2.cuh - the fused tendency kernel as a vertical sweep.
//
// One CTA per element column.  The CTA walks up the column in chunks of LC
// levels; thread t works on node ID = t / LC and chunk level t % LC (level
// fastest, so a warp's global loads are runs of consecutive levels).  Each
// chunk iteration runs three passes separated by barriers:
//
//   P (levels L0 .. L0+LC-1): load the level's state, hyperviscosity cache,
//     lumped mass and metric; compute everything that is local to the
//     (element, level) plane - pointwise quantities and the horizontal D/DW
//     derivative sums - and store it in a ring of planes in shared memory.
//   F (interfaces L0-2 .. L0+LC-3): contravariant vertical mass flux and the
//     limited third-order upwind fluxes (RecU4) of rho*theta and tracers;
//     each interface is computed once and kept in its lower level's plane.
//   V (levels L0-3 .. L0+LC-4): everything that couples neighbouring levels
//     (vertical momentum fluxes, kinetic-energy jumps, the vertical pressure
//     gradient and the interface fluxes) and the assembly of the element
//     node's contributions, written to the DSS contribution buffer.
//
// V lags P by three levels, so every neighbour plane it touches is already in
// the ring (R = LC + 4 planes).  Expressions are the reference's
// (ViscKernel.jl:86-167,277-327, MomentumKernel.jl:1-178,
// GradKineticKernel.jl:1-129, OperatorKernel.jl:637-760) evaluated in the same
// order as the CPU restatement, with the same contribution order.
#pragma once
#include "cgd_kernels.cuh"

namespace cgd {

// ring quantities per (plane, node)
enum {
  R_RHO = 0, R_U, R_V, R_W, R_WLO, R_MC, R_M0, R_M1,
  R_D310, R_D311, R_D320, R_D321, R_D330, R_D331, R_J0, R_J1, R_FC,
  R_U1, R_U2, R_V1, R_V2, R_W1, R_W2, R_P,
  R_GUF1, R_GVF1, R_GUF2, R_GVF2, R_GRADU, R_GRADV,
  R_CTH, R_VU, R_VV, R_VTH, R_HR, R_HTH, R_WCON, R_FTH,
  R_TR0   // + 4 per tracer: c, visc, horizontal divergence, interface flux
};
constexpr int RQ = R_TR0 + 4 * MAXTR;
constexpr int NTMP = 21;   // plane temporaries for the derivative sums

template <int N, int LC>
struct SweepCfg {
  static constexpr int DoF = N * N;
  static constexpr int R = LC + 4;
  static constexpr int THREADS = ((LC * DoF + 31) / 32) * 32;
  static size_t smem(int NT)
  {
    return (size_t)(R_TR0 + 4 * NT) * R * DoF * 8 + (size_t)NTMP * LC * DoF * 8;
  }
};

template <int N, int LC>
__global__ void __launch_bounds__(SweepCfg<N, LC>::THREADS)
    k_phase2_sweep(const GP P, const double *__restrict__ U, const double *__restrict__ T1,
                   double *__restrict__ C)
{
  using CF = SweepCfg<N, LC>;
  constexpr int DoF = CF::DoF;
  constexpr int R = CF::R;
  extern __shared__ double sm[];
  const int NT = P.NumTr;
  const int Q = R_TR0 + 4 * NT;
  double *ring = sm;
  double *tmp = sm + (size_t)Q * R * DoF;
  const int IF = blockIdx.x;
  const int t = threadIdx.x;
  const int lvl = t % LC, ID = t / LC;
  const bool active = ID < DoF;
  const int I = ID % N, Jn = ID / N;
  const int nz = P.nz, NumG = P.NumG;
  const size_t cs = (size_t)DoF * nz, fs = (size_t)nz * NumG;
  const int g = active ? P.glob[IF * DoF + ID] : 0;
  const double *mtb = P.met + ((size_t)IF * NCOMP * DoF + ID) * nz;
  const double *Ug = U + (size_t)nz * g;
#define RG(q, lev, id) ring[((size_t)(q) * R + ((lev) % R)) * DoF + (id)]
#define TP(k, id) tmp[((size_t)(k) * LC + lvl) * DoF + (id)]
  const int rowT = lvl;   // tmp plane row of this thread

  const int niter = (nz + 3 + LC - 1) / LC;
  for (int it = 0; it < niter; ++it) {
    const int L0 = it * LC;
    // ======================= pass P =======================
    const int l = L0 + lvl;
    const bool pact = active && l < nz;
    double rho = 1, u = 0, v = 0, wl = 0, wh = 0, MC = 1, Js = 1;
    double d11 = 0, d12 = 0, d21 = 0, d22 = 0;
    double d110 = 0, d111 = 0, d120 = 0, d121 = 0, d210 = 0, d211 = 0, d220 = 0, d221 = 0;
    double d310 = 0, d311 = 0, d320 = 0, d321 = 0, d330 = 0, d331 = 0;
    if (pact) {
      d110 = mtb[C_D11_0 * cs + l]; d111 = mtb[C_D11_1 * cs + l];
      d120 = mtb[C_D12_0 * cs + l]; d121 = mtb[C_D12_1 * cs + l];
      d210 = mtb[C_D21_0 * cs + l]; d211 = mtb[C_D21_1 * cs + l];
      d220 = mtb[C_D22_0 * cs + l]; d221 = mtb[C_D22_1 * cs + l];
      d310 = mtb[C_D31_0 * cs + l]; d311 = mtb[C_D31_1 * cs + l];
      d320 = mtb[C_D32_0 * cs + l]; d321 = mtb[C_D32_1 * cs + l];
      d330 = mtb[C_D33_0 * cs + l]; d331 = mtb[C_D33_1 * cs + l];
      const double J0 = mtb[C_J0 * cs + l], J1 = mtb[C_J1 * cs + l];
      const double fc = mtb[C_FCOR * cs + l];
      rho = Ug[l]; u = Ug[fs + l]; v = Ug[2 * fs + l];
      const double w = Ug[3 * fs + l], rth = Ug[4 * fs + l];
      const double wm1 = l > 0 ? Ug[3 * fs + l - 1] : 0.0;
      const double M0 = P.M[l + (size_t)nz * g], M1 = P.M[l + (size_t)nz * (g + (size_t)NumG)];
      const double *T = T1 + l + (size_t)nz * g;
      const double c1 = T[0], c2 = T[fs], c3 = T[2 * fs], c4 = T[3 * fs], c5 = T[4 * fs];
      d11 = d110 + d111; d12 = d120 + d121; d21 = d210 + d211; d22 = d220 + d221;
      Js = J0 + J1;
      MC = M0 + M1;
      // surface w from no normal flow (MomentumKernel.jl:35-36)
      wl = l == 0 ? -(d310 * u + d320 * v) / d330 : wm1;
      wh = w;
      RG(R_RHO, l, ID) = rho; RG(R_U, l, ID) = u; RG(R_V, l, ID) = v; RG(R_W, l, ID) = wh;
      RG(R_WLO, l, ID) = wl; RG(R_MC, l, ID) = MC; RG(R_M0, l, ID) = M0; RG(R_M1, l, ID) = M1;
      RG(R_D310, l, ID) = d310; RG(R_D311, l, ID) = d311; RG(R_D320, l, ID) = d320;
      RG(R_D321, l, ID) = d321; RG(R_D330, l, ID) = d330; RG(R_D331, l, ID) = d331;
      RG(R_J0, l, ID) = J0; RG(R_J1, l, ID) = J1; RG(R_FC, l, ID) = fc;
      RG(R_P, l, ID) = pressure_dry(P, rth);
      RG(R_CTH, l, ID) = rth / rho;
      for (int q = 0; q < NT; ++q) RG(R_TR0 + 4 * q, l, ID) = Ug[(5 + q) * fs + l] / rho;
      // plane temporaries
      TP(0, ID) = d11 * c2 - d12 * c1;       // Curl12(Cache1, Cache2)
      TP(1, ID) = d21 * c2 - d22 * c1;
      TP(2, ID) = d11 * c3 + d12 * c4;       // Contra12(Cache3, Cache4)
      TP(3, ID) = d21 * c3 + d22 * c4;
      TP(4, ID) = c5;
      TP(5, ID) = -d120 * wl;  TP(6, ID) = -d121 * wh;    // tempuZ1
      TP(7, ID) = -d220 * wl;  TP(8, ID) = -d221 * wh;    // tempuZ2
      TP(9, ID) = -d110 * wl;  TP(10, ID) = -d111 * wh;   // tempvZ1
      TP(11, ID) = -d210 * wl; TP(12, ID) = -d211 * wh;   // tempvZ2
      TP(13, ID) = d120 * u - d110 * v;                    // tempwZ1
      TP(14, ID) = d121 * u - d111 * v;
      TP(15, ID) = d220 * u - d210 * v;                    // tempwZ2
      TP(16, ID) = d221 * u - d211 * v;
      TP(17, ID) = 0.5 * (u * u + v * v) + 0.5 * (wl * wl);   // K on the bottom node
      TP(18, ID) = 0.5 * (u * u + v * v) + 0.5 * (wh * wh);   // K on the top node
      TP(19, ID) = -rho * (d11 * u + d12 * v);                // Contra12(-Rho, u, v)
      TP(20, ID) = -rho * (d21 * u + d22 * v);
    }
    const double rJs = 1.0 / Js, rMC = 1.0 / MC;
    (void)rJs; (void)rMC;
    __syncthreads();
    double b1 = 0, b2 = 0, b3 = 0, b4 = 0;
    if (pact) {
      const double *D = P.D;
      // hyperviscosity: first derivatives of the DSS'd cache
      {
        const double *a1 = &TP(0, 0), *a2 = &TP(1, 0), *a3 = &TP(2, 0), *a4 = &TP(3, 0), *a5 = &TP(4, 0);
        double Dxc = D[I] * a5[N * Jn], Dyc = D[Jn] * a5[I];
        double cu = D[I] * a1[N * Jn] + D[Jn] * a2[I];
        double dv = D[I] * a3[N * Jn] + D[Jn] * a4[I];
#pragma unroll
        for (int k = 1; k < N; ++k) {
          Dxc += D[I + N * k] * a5[k + N * Jn];
          Dyc += D[Jn + N * k] * a5[I + N * k];
          cu += D[I + N * k] * a1[k + N * Jn] + D[Jn + N * k] * a2[I + N * k];
          dv += D[I + N * k] * a3[k + N * Jn] + D[Jn + N * k] * a4[I + N * k];
        }
        b1 = CGD_DIVJ(cu);
        b2 = CGD_DIVJ(dv);
        double GradDx = CGD_DIVJ(d11 * Dxc + d21 * Dyc);
        double GradDy = CGD_DIVJ(d12 * Dxc + d22 * Dyc);
        b3 = rho * (d11 * GradDx + d12 * GradDy);
        b4 = rho * (d21 * GradDx + d22 * GradDy);
      }
      // momentum: horizontal parts of U1..W2
      {
        const double tu0 = d330 * v - d320 * wl, tu1 = d331 * v - d321 * wh;
        const double tv0 = d330 * u - d310 * wl, tv1 = d331 * u - d311 * wh;
        const double tw0 = d320 * u - d310 * v, tw1 = d321 * u - d311 * v;
        double U1 = 0.5 * (tu1 - tu0), U2 = U1;
        double V1 = 0.5 * (tv1 - tv0), V2 = V1;
        double W1 = 0.5 * (tw1 - tw0), W2 = W1;
        const double *a1 = &TP(5, 0), *b1p = &TP(6, 0), *a2 = &TP(7, 0), *b2p = &TP(8, 0);
        const double *a3 = &TP(9, 0), *b3p = &TP(10, 0), *a4 = &TP(11, 0), *b4p = &TP(12, 0);
        const double *a5 = &TP(13, 0), *b5p = &TP(14, 0), *a6 = &TP(15, 0), *b6p = &TP(16, 0);
        U1 += D[I] * a1[N * Jn] + D[Jn] * a2[I];
        U2 += D[I] * b1p[N * Jn] + D[Jn] * b2p[I];
        V1 += D[I] * a3[N * Jn] + D[Jn] * a4[I];
        V2 += D[I] * b3p[N * Jn] + D[Jn] * b4p[I];
        W1 += D[I] * a5[N * Jn] + D[Jn] * a6[I];
        W2 += D[I] * b5p[N * Jn] + D[Jn] * b6p[I];
#pragma unroll
        for (int k = 1; k < N; ++k) {
          U1 += D[I + N * k] * a1[k + N * Jn] + D[Jn + N * k] * a2[I + N * k];
          U2 += D[I + N * k] * b1p[k + N * Jn] + D[Jn + N * k] * b2p[I + N * k];
          V1 += D[I + N * k] * a3[k + N * Jn] + D[Jn + N * k] * a4[I + N * k];
          V2 += D[I + N * k] * b3p[k + N * Jn] + D[Jn + N * k] * b4p[I + N * k];
          W1 += D[I + N * k] * a5[k + N * Jn] + D[Jn + N * k] * a6[I + N * k];
          W2 += D[I + N * k] * b5p[k + N * Jn] + D[Jn + N * k] * b6p[I + N * k];
        }
        RG(R_U1, l, ID) = U1; RG(R_U2, l, ID) = U2; RG(R_V1, l, ID) = V1;
        RG(R_V2, l, ID) = V2; RG(R_W1, l, ID) = W1; RG(R_W2, l, ID) = W2;
      }
      // kinetic-energy and pressure gradients (plane part) + gravity
      {
        const double *Ka = &TP(17, 0), *Kb = &TP(18, 0);
        const double *pa = &RG(R_P, l, 0);
        double DXp = D[I] * pa[N * Jn], DYp = D[Jn] * pa[I];
        double DXK1 = D[I] * Ka[N * Jn], DYK1 = D[Jn] * Ka[I];
        double DXK2 = D[I] * Kb[N * Jn], DYK2 = D[Jn] * Kb[I];
#pragma unroll
        for (int k = 1; k < N; ++k) {
          DXK1 += D[I + N * k] * Ka[k + N * Jn];
          DYK1 += D[Jn + N * k] * Ka[I + N * k];
          DXK2 += D[I + N * k] * Kb[k + N * Jn];
          DYK2 += D[Jn + N * k] * Kb[I + N * k];
          DXp += D[I + N * k] * pa[k + N * Jn];
          DYp += D[Jn + N * k] * pa[I + N * k];
        }
        RG(R_GUF1, l, ID) = -(d110 * DXK1 + d210 * DYK1);
        RG(R_GVF1, l, ID) = -(d120 * DXK1 + d220 * DYK1);
        RG(R_GUF2, l, ID) = -(d111 * DXK2 + d211 * DYK2);
        RG(R_GVF2, l, ID) = -(d121 * DXK2 + d221 * DYK2);
        double Gradu = d11 * DXp + d21 * DYp;
        double Gradv = d12 * DXp + d22 * DYp;
        const double GZ = -P.Grav * rho * (RG(R_J0, l, ID) + RG(R_J1, l, ID)) / (d330 + d331);
        Gradu += GZ * (d310 + d311);
        Gradv += GZ * (d320 + d321);
        RG(R_GRADU, l, ID) = Gradu;
        RG(R_GRADV, l, ID) = Gradv;
      }
      // horizontal flux divergence of rho, rho*theta, rho*q
      {
        const double *uc = &TP(19, 0), *vc = &TP(20, 0);
        const double *cc = &RG(R_CTH, l, 0);
        double DivRhoTr = D[I] * uc[N * Jn] * cc[N * Jn] + D[Jn] * vc[I] * cc[I];
        double DivRho = D[I] * uc[N * Jn] + D[Jn] * vc[I];
#pragma unroll
        for (int k = 1; k < N; ++k) {
          DivRhoTr += D[I + N * k] * uc[k + N * Jn] * cc[k + N * Jn] + D[Jn + N * k] * vc[I + N * k] * cc[I + N * k];
          DivRho += D[I + N * k] * uc[k + N * Jn] + D[Jn + N * k] * vc[I + N * k];
        }
        RG(R_HTH, l, ID) = CGD_DIVM(DivRhoTr);
        RG(R_HR, l, ID) = CGD_DIVM(DivRho);
        for (int q = 0; q < NT; ++q) {
          const double *ct = &RG(R_TR0 + 4 * q, l, 0);
          double Dv = D[I] * uc[N * Jn] * ct[N * Jn] + D[Jn] * vc[I] * ct[I];
#pragma unroll
          for (int k = 1; k < N; ++k)
            Dv += D[I + N * k] * uc[k + N * Jn] * ct[k + N * Jn] + D[Jn + N * k] * vc[I + N * k] * ct[I + N * k];
          RG(R_TR0 + 4 * q + 2, l, ID) = CGD_DIVM(Dv);
        }
      }
    }
    __syncthreads();
    // hyperviscosity: second (weak) derivatives
    if (pact) { TP(0, ID) = b1; TP(1, ID) = b2; TP(2, ID) = b3; TP(3, ID) = b4; }
    __syncthreads();
    if (pact) {
      const double *DW = P.DW;
      const double *e1 = &TP(0, 0), *e2 = &TP(1, 0), *e3 = &TP(2, 0), *e4 = &TP(3, 0);
      double DxCurl = DW[I] * e1[N * Jn], DyCurl = DW[Jn] * e1[I];
      double DxDiv = DW[I] * e2[N * Jn], DyDiv = DW[Jn] * e2[I];
      double DivTh = DW[I] * e3[N * Jn] + DW[Jn] * e4[I];
#pragma unroll
      for (int k = 1; k < N; ++k) {
        DxCurl += DW[I + N * k] * e1[k + N * Jn];
        DyCurl += DW[Jn + N * k] * e1[I + N * k];
        DxDiv += DW[I + N * k] * e2[k + N * Jn];
        DyDiv += DW[Jn + N * k] * e2[I + N * k];
        DivTh += DW[I + N * k] * e3[k + N * Jn] + DW[Jn + N * k] * e4[I + N * k];
      }
      double FuC = d12 * DxCurl + d22 * DyCurl;
      double FvC = -d11 * DxCurl - d21 * DyCurl;
      double FuD = d11 * DxDiv + d21 * DyDiv;
      double FvD = d12 * DxDiv + d22 * DyDiv;
      RG(R_VU, l, ID) = CGD_DIVM(-(-P.nuCurl * FuC + P.nuGrad * FuD));
      RG(R_VV, l, ID) = CGD_DIVM(-(-P.nuCurl * FvC + P.nuGrad * FvD));
      RG(R_VTH, l, ID) = CGD_DIVM(-P.nuDiv * DivTh);
    }
    for (int q = 0; q < NT; ++q) {   // tracer hyperviscosity
      __syncthreads();
      if (pact) TP(4, ID) = T1[l + (size_t)nz * g + (5 + q) * fs];
      __syncthreads();
      double e3v = 0, e4v = 0;
      if (pact) {
        const double *D = P.D;
        const double *a5 = &TP(4, 0);
        double Dxc = D[I] * a5[N * Jn], Dyc = D[Jn] * a5[I];
#pragma unroll
        for (int k = 1; k < N; ++k) {
          Dxc += D[I + N * k] * a5[k + N * Jn];
          Dyc += D[Jn + N * k] * a5[I + N * k];
        }
        double GradDx = CGD_DIVJ(d11 * Dxc + d21 * Dyc);
        double GradDy = CGD_DIVJ(d12 * Dxc + d22 * Dyc);
        e3v = rho * (d11 * GradDx + d12 * GradDy);
        e4v = rho * (d21 * GradDx + d22 * GradDy);
        TP(5, ID) = e3v;
        TP(6, ID) = e4v;
      }
      __syncthreads();
      if (pact) {
        const double *DW = P.DW;
        const double *e3 = &TP(5, 0), *e4 = &TP(6, 0);
        double DivTr = DW[I] * e3[N * Jn] + DW[Jn] * e4[I];
#pragma unroll
        for (int k = 1; k < N; ++k) DivTr += DW[I + N * k] * e3[k + N * Jn] + DW[Jn + N * k] * e4[I + N * k];
        RG(R_TR0 + 4 * q + 1, l, ID) = CGD_DIVM(-P.nuDiv * DivTr);
      }
    }
    __syncthreads();

    // ======================= pass F =======================
    {
      const int il = L0 - 2 + lvl;
      if (active && il >= 0 && il < nz - 1) {
        const int lm = il > 0 ? il - 1 : 0, lp1 = il + 1, lp2 = il + 2 < nz ? il + 2 : nz - 1;
        const double wI = RG(R_W, il, ID);
        const double wCon =
            RG(R_RHO, il, ID) * (RG(R_D311, il, ID) * RG(R_U, il, ID) + RG(R_D321, il, ID) * RG(R_V, il, ID) +
                                 RG(R_D331, il, ID) * wI) +
            RG(R_RHO, lp1, ID) * (RG(R_D310, lp1, ID) * RG(R_U, lp1, ID) + RG(R_D320, lp1, ID) * RG(R_V, lp1, ID) +
                                  RG(R_D330, lp1, ID) * wI);
        const double kR1 = mtb[C_RK0 * cs + il], kL1 = mtb[C_RK1 * cs + il];
        const double kL2 = mtb[C_RK2 * cs + il], kR2 = mtb[C_RK3 * cs + il];
        const double aw = fabs(wCon);
        auto upwind = [&](int q) {
          const double cLL = RG(q, lm, ID), cL = RG(q, il, ID), cR = RG(q, lp1, ID), cRR = RG(q, lp2, ID);
          // RecU4 (OperatorKernel.jl:1044-1059) with its J-only coefficients precomputed
          double r = (cL - cLL) / (cR - cL + 1.e-20);
          const double cFL = cL + cgd_max(0.0, cgd_min(r, cgd_min(kL1 * r + kR1, 1.0))) * (cR - cL);
          r = (cR - cRR) / (cL - cR + 1.e-20);
          const double cFR = cR + cgd_max(0.0, cgd_min(r, cgd_min(kR2 * r + kL2, 1.0))) * (cL - cR);
          return 0.25 * ((aw + wCon) * cFL + (-aw + wCon) * cFR);
        };
        RG(R_WCON, il, ID) = wCon;
        RG(R_FTH, il, ID) = upwind(R_CTH);
        for (int q = 0; q < NT; ++q) RG(R_TR0 + 4 * q + 3, il, ID) = upwind(R_TR0 + 4 * q);
      }
    }
    __syncthreads();

    // ======================= pass V =======================
    {
      const int lv = L0 - 3 + lvl;
      if (active && lv >= 0 && lv < nz) {
        const double rho_ = RG(R_RHO, lv, ID), u_ = RG(R_U, lv, ID), v_ = RG(R_V, lv, ID);
        const double wl_ = RG(R_WLO, lv, ID), wh_ = RG(R_W, lv, ID);
        const double MC = RG(R_MC, lv, ID);
#ifdef CGD_FAST
        const double rMC = 1.0 / MC, rrho = 1.0 / rho_;
#define CGD_DIVR(x) ((x) * rrho)
#else
#define CGD_DIVR(x) ((x) / rho_)
#endif
        const double e310 = RG(R_D310, lv, ID), e311 = RG(R_D311, lv, ID), e320 = RG(R_D320, lv, ID);
        const double e321 = RG(R_D321, lv, ID), e330 = RG(R_D330, lv, ID), e331 = RG(R_D331, lv, ID);
        const bool top = lv < nz - 1, bot = lv > 0;
        // --- momentum
        const double tu0 = e330 * v_ - e320 * wl_, tu1 = e331 * v_ - e321 * wh_;
        const double tv0 = e330 * u_ - e310 * wl_, tv1 = e331 * u_ - e311 * wh_;
        const double tw0 = e320 * u_ - e310 * v_, tw1 = e321 * u_ - e311 * v_;
        double FU = 0.0, FV = 0.0, FW1 = 0.0, FW2 = 0.0;
        if (bot) {
          const int lb = lv - 1;
          const double ub = RG(R_U, lb, ID), vb = RG(R_V, lb, ID), wb = RG(R_W, lb, ID);
          const double tu1b = RG(R_D331, lb, ID) * vb - RG(R_D321, lb, ID) * wb;
          const double tv1b = RG(R_D331, lb, ID) * ub - RG(R_D311, lb, ID) * wb;
          const double tw1b = RG(R_D321, lb, ID) * ub - RG(R_D311, lb, ID) * vb;
          const double FluxUZ = 0.5 * (tu0 - tu1b);
          const double FluxVZ = 0.5 * (tv0 - tv1b);
          const double FluxWZ = 0.5 * (tw0 - tw1b);
          FU += (-v_ * FluxWZ - wl_ * FluxVZ);
          FV += (u_ * FluxWZ - wl_ * FluxUZ);
          FW1 += (u_ * FluxVZ + v_ * FluxUZ);
        }
        // upper neighbour (level lv+1) quantities shared by several terms
        double rho1 = 0, u1 = 0, v1 = 0, w1 = 0, wl1 = 0, tu0a = 0, tv0a = 0, tw0a = 0;
        double FluxUZt = 0, FluxVZt = 0, FluxWZt = 0;
        if (top) {
          const int la = lv + 1;
          rho1 = RG(R_RHO, la, ID); u1 = RG(R_U, la, ID); v1 = RG(R_V, la, ID);
          w1 = RG(R_W, la, ID); wl1 = RG(R_WLO, la, ID);
          tu0a = RG(R_D330, la, ID) * v1 - RG(R_D320, la, ID) * wl1;
          tv0a = RG(R_D330, la, ID) * u1 - RG(R_D310, la, ID) * wl1;
          tw0a = RG(R_D320, la, ID) * u1 - RG(R_D310, la, ID) * v1;
          FluxUZt = 0.5 * (tu0a - tu1);
          FluxVZt = 0.5 * (tv0a - tv1);
          FluxWZt = 0.5 * (tw0a - tw1);
          FU += (-v_ * FluxWZt - wh_ * FluxVZt);
          FV += (u_ * FluxWZt - wh_ * FluxUZt);
          FW2 += (u_ * FluxVZt + v_ * FluxUZt);
        }
        const double J0_ = RG(R_J0, lv, ID), J1_ = RG(R_J1, lv, ID), fc = RG(R_FC, lv, ID);
        const double FuCor = v_ * fc, FvCor = -u_ * fc, FwCor = 0.0;
        FU += FuCor * (J0_ + J1_);
        FV += FvCor * (J0_ + J1_);
        FW1 += FwCor * J0_;
        FW2 += FwCor * J1_;
        const double U1 = RG(R_U1, lv, ID), U2 = RG(R_U2, lv, ID), V1 = RG(R_V1, lv, ID);
        const double V2 = RG(R_V2, lv, ID), W1 = RG(R_W1, lv, ID), W2 = RG(R_W2, lv, ID);
        const double mu = CGD_DIVM(-v_ * W1 - wl_ * V1 - v_ * W2 - wh_ * V2 + FU);
        const double mv = CGD_DIVM(u_ * W1 - wl_ * U1 + u_ * W2 - wh_ * U2 + FV);
        (void)FW1;
        // --- kinetic energy / pressure gradient
        const double K1s = 0.5 * (u_ * u_ + v_ * v_) + 0.5 * (wl_ * wl_);
        const double K2s = 0.5 * (u_ * u_ + v_ * v_) + 0.5 * (wh_ * wh_);
        double GuF1 = RG(R_GUF1, lv, ID), GvF1 = RG(R_GVF1, lv, ID);
        double GuF2 = RG(R_GUF2, lv, ID), GvF2 = RG(R_GVF2, lv, ID);
        double GwF2 = 0.0, GZ;
        if (bot) {
          const int lb = lv - 1;
          const double ub = RG(R_U, lb, ID), vb = RG(R_V, lb, ID), wb = RG(R_W, lb, ID);
          const double K2b = 0.5 * (ub * ub + vb * vb) + 0.5 * (wb * wb);
          GZ = 0.5 * (K1s - K2b);
          GuF1 += -GZ * e310;
          GvF1 += -GZ * e320;
        }
        double K1a = 0;
        if (top) {
          K1a = 0.5 * (u1 * u1 + v1 * v1) + 0.5 * (wl1 * wl1);
          GZ = 0.5 * (K1a - K2s);
          GuF2 += -GZ * e311;
          GvF2 += -GZ * e321;
          GwF2 += -rho_ * GZ * e331;
        }
        GZ = 0.5 * (K2s - K1s);
        GuF2 += -GZ * e311;
        GuF1 += -GZ * e310;
        GvF2 += -GZ * e321;
        GvF1 += -GZ * e320;
        GwF2 += -rho_ * GZ * e331;
        const double gu = CGD_DIVM(GuF1 + GuF2 - CGD_DIVR(RG(R_GRADU, lv, ID)));
        const double gv = CGD_DIVM(GvF1 + GvF2 - CGD_DIVR(RG(R_GRADV, lv, ID)));
        // --- w at the top interface: upper node of lv + lower node of lv+1
        double wcontrib = 0.0;
        if (top) {
          const double M1_ = RG(R_M1, lv, ID), M0a = RG(R_M0, lv + 1, ID);
          const double mwhi = rho_ * (u_ * V2 + v_ * U2 + FW2) / (rho1 * M0a + rho_ * M1_);
          const double pl = RG(R_P, lv, ID), pa = RG(R_P, lv + 1, ID);
          GZ = 0.5 * (pa - pl);
          const double Gradw = GZ * (e331 + RG(R_D330, lv + 1, ID));
          const double Gradp = -(Gradw + P.Grav * (rho_ * J1_ + rho1 * RG(R_J0, lv + 1, ID)));
          const double gwhi = (GwF2 + Gradp) / (rho1 * M0a + rho_ * M1_);
          // lower node of level lv+1 (its bottom interface is this one)
          double FW1a = 0.0;
          FW1a += (u1 * FluxVZt + v1 * FluxUZt);
          FW1a += FwCor * RG(R_J0, lv + 1, ID);
          const double mwlo = rho1 * (u1 * RG(R_V1, lv + 1, ID) + v1 * RG(R_U1, lv + 1, ID) + FW1a) /
                              (rho_ * M1_ + rho1 * M0a);
          const double K2a = 0.5 * (u1 * u1 + v1 * v1) + 0.5 * (w1 * w1);
          double GwF1a = 0.0;
          double GZa = 0.5 * (K1a - K2s);
          GwF1a += -rho1 * GZa * RG(R_D330, lv + 1, ID);
          GZa = 0.5 * (K2a - K1a);
          GwF1a += -rho1 * GZa * RG(R_D330, lv + 1, ID);
          const double gwlo = GwF1a / (rho_ * M1_ + rho1 * M0a);
          const double hi = mwhi + gwhi;
          const double lo = mwlo + gwlo;
          wcontrib = hi + lo;
        }
        // --- interface fluxes of this layer
        double fr_top = 0, fr_bot = 0, fth_top = 0, fth_bot = 0;
        if (top) {
          const double Flr = 0.5 * RG(R_WCON, lv, ID);
          fr_top = CGD_DIVM(-Flr);
          fth_top = CGD_DIVM(-RG(R_FTH, lv, ID));
        }
        if (bot) {
          const double Flr = 0.5 * RG(R_WCON, lv - 1, ID);
          fr_bot = CGD_DIVM(Flr);
          fth_bot = CGD_DIVM(RG(R_FTH, lv - 1, ID));
        }
        // --- assemble (same order as the CPU restatement)
        double *out = C + ((size_t)IF * P.NV * DoF + ID) * nz + lv;
        double acc = 0.0;
        if (top) acc += fr_top;
        if (bot) acc += fr_bot;
        acc += RG(R_HR, lv, ID);
        out[0] = acc;
        acc = 0.0; acc += RG(R_VU, lv, ID); acc += mu; acc += gu;
        out[cs] = acc;
        acc = 0.0; acc += RG(R_VV, lv, ID); acc += mv; acc += gv;
        out[2 * cs] = acc;
        out[3 * cs] = wcontrib;
        acc = 0.0; acc += RG(R_VTH, lv, ID);
        if (top) acc += fth_top;
        if (bot) acc += fth_bot;
        acc += RG(R_HTH, lv, ID);
        out[4 * cs] = acc;
        for (int q = 0; q < NT; ++q) {
          acc = 0.0; acc += RG(R_TR0 + 4 * q + 1, lv, ID);
          if (top) acc += CGD_DIVM(-RG(R_TR0 + 4 * q + 3, lv, ID));
          if (bot) acc += CGD_DIVM(RG(R_TR0 + 4 * q + 3, lv - 1, ID));
          acc += RG(R_TR0 + 4 * q + 2, lv, ID);
          out[(5 + q) * cs] = acc;
        }
#undef CGD_DIVR
      }
    }
    __syncthreads();
  }
#undef RG
#undef TP
  (void)rowT;
}

}  // namespace cgd
