// cgd_kernels.cuh - sm_100a kernels of the FP64 hot path.
//
// Layouts in HBM
//   state U, Temp1, F, k   (nz, NumG, NV) level fastest (the reference layout)
//   met                    [IF][comp][ID][nz]  17 components per element node
//                          and level (14 used dXdxI entries, J bottom/top,
//                          2*Omega*sin(lat) at the layer midpoint)
//   C  (contributions)     [IF][field][ID][nz]  element-local DSS inputs
//   M                      (nz, NumG, 2)
//
// Direct-stiffness summation is an owner gather: the element kernels write
// every element-node contribution to C, and one thread per (global DOF,
// level) sums the contributions of the element nodes that share the DOF in
// ascending (element, node) order.  No atomics: results are bit-reproducible
// and equal to the CPU restatement's.
//
// Every floating-point expression below is written in the reference's
// evaluation order; the file is compiled with -fmad=false so that no
// multiply-add is contracted (the bit-exactness contract with the oracle).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/cgd_math.h"

namespace cgd {

constexpr int NCOMP = 17;
enum {
  C_D11_0 = 0, C_D11_1, C_D12_0, C_D12_1, C_D21_0, C_D21_1, C_D22_0, C_D22_1,
  C_D31_0, C_D31_1, C_D32_0, C_D32_1, C_D33_0, C_D33_1, C_J0, C_J1, C_FCOR
};
constexpr int MAXTR = 4;
constexpr int MAXNV = 5 + MAXTR;

// Everything a kernel needs about the grid, passed by value.
struct GP {
  int N, DoF, nz, NF, NumG, NumTr, NV;
  const double *met;        // [IF][comp][ID][nz]
  const double *M;          // (nz, NumG, 2)
  const double *dz;         // (nz, NumG)
  const int *glob;          // [IF*DoF + ID], 0-based
  const int *inv_ptr;       // NumG + 1
  const long long *inv_off; // (IF*NV*DoF + ID)*nz for every contributor
  double D[25], DW[25];     // D[i + N*j] = DS[i,j]
  double Grav, Rd, p0, kappa, nuCurl, nuGrad, nuDiv;
};

// Rosenbrock-W coefficients (src/Integration/RosenbrockMethod.jl:26-47).
struct RK {
  double a[3][3], c[3][3], m[3], gamma;
};

__device__ __forceinline__ double pressure_dry(const GP &P, double rhoth)
{
  // src/Models/Equation.jl:25-38, fast_powGPU (Equation.jl:79)
  return P.p0 * cgd_exp(1.0 / (1.0 - P.kappa) * cgd_log(P.Rd * rhoth / P.p0));
}

// RecU4: src/GPU/OperatorKernel.jl:1044-1059
__device__ __forceinline__ void recu4(double cLL, double cL, double cR, double cRR, double JLL,
                                      double JL, double JR, double JRR, double &cFL, double &cFR)
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

// ---------------------------------------------------------------------------
// Phase 1: HyperViscKernel! + HyperViscTracerKernel!
// (src/GPU/ViscKernel.jl:1-84,169-218).  One CTA per (element, tile of LT
// levels); thread (node, level).  Purely horizontal: no vertical halo.
// ---------------------------------------------------------------------------
template <int N>
__global__ void __launch_bounds__(256) k_hypervisc1(const GP P, const double *__restrict__ U,
                                                    double *__restrict__ C)
{
  constexpr int DoF = N * N;
  constexpr int LT = 256 / DoF;
  __shared__ double s[9][LT * DoF];
  const int IF = blockIdx.x;
  const int t = threadIdx.x;
  const int lvl = t % LT, ID = t / LT;
  const int I = ID % N, Jn = ID / N;
  const int l = blockIdx.y * LT + lvl;
  const int nz = P.nz, NumG = P.NumG;
  const bool act = (ID < DoF) && (l < nz);
  const int si = lvl * DoF + ID, row = lvl * DoF;
  const size_t cs = (size_t)DoF * nz;
  int g = 0;
  double d11 = 0, d12 = 0, d21 = 0, d22 = 0, Js = 1, MC = 1;
  const double *mt = P.met + ((size_t)IF * NCOMP * DoF + ID) * nz + l;
  if (act) {
    g = P.glob[IF * DoF + ID];
    d11 = mt[C_D11_0 * cs] + mt[C_D11_1 * cs];
    d12 = mt[C_D12_0 * cs] + mt[C_D12_1 * cs];
    d21 = mt[C_D21_0 * cs] + mt[C_D21_1 * cs];
    d22 = mt[C_D22_0 * cs] + mt[C_D22_1 * cs];
    Js = mt[C_J0 * cs] + mt[C_J1 * cs];
    const double *Ug = U + l + (size_t)nz * g;
    const size_t fs = (size_t)nz * NumG;
    double u = Ug[1 * fs], v = Ug[2 * fs];
    s[0][si] = d11 * v - d12 * u;   // Curl12
    s[1][si] = d21 * v - d22 * u;
    s[2][si] = d11 * u + d12 * v;   // Contra12
    s[3][si] = d21 * u + d22 * v;
    s[4][si] = Ug[4 * fs] / Ug[0];
    MC = P.M[l + (size_t)nz * g] + P.M[l + (size_t)nz * (g + (size_t)NumG)];
  }
  __syncthreads();
  if (act) {
    const double *uC = s[0] + row, *vC = s[1] + row, *uD = s[2] + row, *vD = s[3] + row, *Th = s[4] + row;
    double Dxc = P.D[I] * Th[N * Jn];
    double Dyc = P.D[Jn] * Th[I];
    double cu = P.D[I] * uC[N * Jn] + P.D[Jn] * vC[I];
    double dv = P.D[I] * uD[N * Jn] + P.D[Jn] * vD[I];
#pragma unroll
    for (int k = 1; k < N; ++k) {
      Dxc += P.D[I + N * k] * Th[k + N * Jn];
      Dyc += P.D[Jn + N * k] * Th[I + N * k];
      cu += P.D[I + N * k] * uC[k + N * Jn] + P.D[Jn + N * k] * vC[I + N * k];
      dv += P.D[I + N * k] * uD[k + N * Jn] + P.D[Jn + N * k] * vD[I + N * k];
    }
    s[5][si] = cu / Js;
    s[6][si] = dv / Js;
    double GradDx = (d11 * Dxc + d21 * Dyc) / Js;   // Grad12 with J
    double GradDy = (d12 * Dxc + d22 * Dyc) / Js;
    s[7][si] = d11 * GradDx + d12 * GradDy;         // Contra12
    s[8][si] = d21 * GradDx + d22 * GradDy;
  }
  __syncthreads();
  double *out = C + ((size_t)IF * P.NV * DoF + ID) * nz + l;
  if (act) {
    const double *Cu = s[5] + row, *Dv = s[6] + row, *Cx = s[7] + row, *Cy = s[8] + row;
    double DxCurl = P.DW[I] * Cu[N * Jn], DyCurl = P.DW[Jn] * Cu[I];
    double DxDiv = P.DW[I] * Dv[N * Jn], DyDiv = P.DW[Jn] * Dv[I];
    double DivTh = P.DW[I] * Cx[N * Jn] + P.DW[Jn] * Cy[I];
#pragma unroll
    for (int k = 1; k < N; ++k) {
      DxCurl += P.DW[I + N * k] * Cu[k + N * Jn];
      DyCurl += P.DW[Jn + N * k] * Cu[I + N * k];
      DxDiv += P.DW[I + N * k] * Dv[k + N * Jn];
      DyDiv += P.DW[Jn + N * k] * Dv[I + N * k];
      DivTh += P.DW[I + N * k] * Cx[k + N * Jn] + P.DW[Jn + N * k] * Cy[I + N * k];
    }
    double FuC = d12 * DxCurl + d22 * DyCurl;       // Rot12
    double FvC = -d11 * DxCurl - d21 * DyCurl;
    double FuD = d11 * DxDiv + d21 * DyDiv;         // Grad12
    double FvD = d12 * DxDiv + d22 * DyDiv;
    out[0 * cs] = -FuC / MC;
    out[1 * cs] = -FvC / MC;
    out[2 * cs] = FuD / MC;
    out[3 * cs] = FvD / MC;
    out[4 * cs] = DivTh / MC;
  }
  for (int iT = 0; iT < P.NumTr; ++iT) {
    if (act) {
      const size_t fs = (size_t)nz * NumG;
      const double *Ug = U + l + (size_t)nz * g;
      s[4][si] = Ug[(5 + iT) * fs] / Ug[0];
    }
    __syncthreads();
    if (act) {
      const double *Tr = s[4] + row;
      double Dxc = P.D[I] * Tr[N * Jn];
      double Dyc = P.D[Jn] * Tr[I];
#pragma unroll
      for (int k = 1; k < N; ++k) {
        Dxc += P.D[I + N * k] * Tr[k + N * Jn];
        Dyc += P.D[Jn + N * k] * Tr[I + N * k];
      }
      double GradDx = (d11 * Dxc + d21 * Dyc) / Js;
      double GradDy = (d12 * Dxc + d22 * Dyc) / Js;
      s[7][si] = d11 * GradDx + d12 * GradDy;
      s[8][si] = d21 * GradDx + d22 * GradDy;
    }
    __syncthreads();
    if (act) {
      const double *Cx = s[7] + row, *Cy = s[8] + row;
      double DivTr = P.DW[I] * Cx[N * Jn] + P.DW[Jn] * Cy[I];
#pragma unroll
      for (int k = 1; k < N; ++k) DivTr += P.DW[I + N * k] * Cx[k + N * Jn] + P.DW[Jn + N * k] * Cy[I + N * k];
      out[(5 + iT) * cs] = DivTr / MC;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Owner gather (DSS): out(l, g, f) = sum over contributors in ascending
// (element, node) order.  Thread per (g, l), level fastest.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_gather(const GP P, const double *__restrict__ C,
                                                double *__restrict__ out)
{
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int nz = P.nz;
  if (tid >= (long long)nz * P.NumG) return;
  const int g = (int)(tid / nz), l = (int)(tid % nz);
  const int q0 = P.inv_ptr[g], q1 = P.inv_ptr[g + 1];
  const size_t fstr = (size_t)P.DoF * nz;
  for (int f = 0; f < P.NV; ++f) {
    double acc = 0.0;
    for (int q = q0; q < q1; ++q) acc += C[P.inv_off[q] + f * fstr + l];
    out[l + (size_t)nz * (g + (size_t)P.NumG * f)] = acc;
  }
}

// ---------------------------------------------------------------------------
// Phase 2: HyperViscKoeffKernel! + HyperViscTracerKoeffKernel!
// (ViscKernel.jl:86-167,277-327), MomentumVectorInvariantCoriolisKernel!
// (MomentumKernel.jl:1-178), GradFullKernel! (GradKineticKernel.jl:1-129) and
// DivRhoTrUpwind3New2Kernel! (OperatorKernel.jl:637-760) fused; the pressure
// (DiagnosticKernel.jl:96-115) is recomputed in registers.
// One CTA per (element, tile of LT levels); threads cover LT + 1 levels: the
// extra level above the tile only produces the lower-node w contributions
// that belong to the tile's top interface.
// Element-node contribution order (the oracle uses the same):
//   rho   : -flux(top)/MC + flux(bottom)/MC + horizontal divergence
//   u, v  : hyperviscosity + momentum + gradient
//   w(l)  : (momentum_hi(l) + gradient_hi(l)) + (momentum_lo(l+1) + gradient_lo(l+1))
//   rho*theta, rho*q : hyperviscosity - flux(top) + flux(bottom) + divergence
// ---------------------------------------------------------------------------
template <int N>
__global__ void __launch_bounds__(256) k_phase2(const GP P, const double *__restrict__ U,
                                                const double *__restrict__ T1, double *__restrict__ C)
{
  constexpr int DoF = N * N;
  constexpr int LTP = 256 / DoF;
  constexpr int LT = LTP - 1;
  __shared__ double s[12][LTP * DoF];
  __shared__ double slo[2][LTP * DoF];
  const int IF = blockIdx.x;
  const int t = threadIdx.x;
  const int lvl = t % LTP, ID = t / LTP;
  const int I = ID % N, Jn = ID / N;
  const int l = blockIdx.y * LT + lvl;
  const int nz = P.nz, NumG = P.NumG, NT = P.NumTr;
  const bool act = (ID < DoF) && (l < nz);
  const bool own = act && (lvl < LT);
  const int si = lvl * DoF + ID, row = lvl * DoF;
  const size_t cs = (size_t)DoF * nz, fs = (size_t)nz * NumG;
  const int g = act ? P.glob[IF * DoF + ID] : 0;
  const double *mtb = P.met + ((size_t)IF * NCOMP * DoF + ID) * nz;   // + comp*cs + level
  const double *Ug = U + (size_t)nz * g;                              // + f*fs + level
  auto mt = [&](int comp, int lev) { return mtb[comp * cs + lev]; };
  auto Uv = [&](int f, int lev) { return Ug[f * fs + lev]; };
  auto MCat = [&](int lev) { return P.M[lev + (size_t)nz * g] + P.M[lev + (size_t)nz * (g + (size_t)NumG)]; };
  auto Jsum = [&](int lev) { return mt(C_J0, lev) + mt(C_J1, lev); };

  double d11 = 0, d12 = 0, d21 = 0, d22 = 0, Js = 1, MC = 1, rho = 1, u = 0, v = 0;
  if (act) {
    d11 = mt(C_D11_0, l) + mt(C_D11_1, l);
    d12 = mt(C_D12_0, l) + mt(C_D12_1, l);
    d21 = mt(C_D21_0, l) + mt(C_D21_1, l);
    d22 = mt(C_D22_0, l) + mt(C_D22_1, l);
    Js = Jsum(l);
    MC = MCat(l);
    rho = Uv(0, l); u = Uv(1, l); v = Uv(2, l);
  }

  // ---------------- hyperviscosity, second application ----------------
  double vu = 0, vv = 0, vth = 0, vtr[MAXTR] = {0, 0, 0, 0};
  if (own) {
    const double *T = T1 + l + (size_t)nz * g;
    double c1 = T[0], c2 = T[fs], c3 = T[2 * fs], c4 = T[3 * fs];
    s[0][si] = d11 * c2 - d12 * c1;   // Curl12(Cache1, Cache2)
    s[1][si] = d21 * c2 - d22 * c1;
    s[2][si] = d11 * c3 + d12 * c4;   // Contra12(Cache3, Cache4)
    s[3][si] = d21 * c3 + d22 * c4;
    s[4][si] = T[4 * fs];
  }
  __syncthreads();
  if (own) {
    const double *a1 = s[0] + row, *a2 = s[1] + row, *a3 = s[2] + row, *a4 = s[3] + row, *a5 = s[4] + row;
    double Dxc = P.D[I] * a5[N * Jn], Dyc = P.D[Jn] * a5[I];
    double cu = P.D[I] * a1[N * Jn] + P.D[Jn] * a2[I];
    double dv = P.D[I] * a3[N * Jn] + P.D[Jn] * a4[I];
#pragma unroll
    for (int k = 1; k < N; ++k) {
      Dxc += P.D[I + N * k] * a5[k + N * Jn];
      Dyc += P.D[Jn + N * k] * a5[I + N * k];
      cu += P.D[I + N * k] * a1[k + N * Jn] + P.D[Jn + N * k] * a2[I + N * k];
      dv += P.D[I + N * k] * a3[k + N * Jn] + P.D[Jn + N * k] * a4[I + N * k];
    }
    s[5][si] = cu / Js;
    s[6][si] = dv / Js;
    double GradDx = (d11 * Dxc + d21 * Dyc) / Js;
    double GradDy = (d12 * Dxc + d22 * Dyc) / Js;
    s[7][si] = rho * (d11 * GradDx + d12 * GradDy);   // Contra12(Rho, ...)
    s[8][si] = rho * (d21 * GradDx + d22 * GradDy);
  }
  __syncthreads();
  if (own) {
    const double *b1 = s[5] + row, *b2 = s[6] + row, *b3 = s[7] + row, *b4 = s[8] + row;
    double DxCurl = P.DW[I] * b1[N * Jn], DyCurl = P.DW[Jn] * b1[I];
    double DxDiv = P.DW[I] * b2[N * Jn], DyDiv = P.DW[Jn] * b2[I];
    double DivTh = P.DW[I] * b3[N * Jn] + P.DW[Jn] * b4[I];
#pragma unroll
    for (int k = 1; k < N; ++k) {
      DxCurl += P.DW[I + N * k] * b1[k + N * Jn];
      DyCurl += P.DW[Jn + N * k] * b1[I + N * k];
      DxDiv += P.DW[I + N * k] * b2[k + N * Jn];
      DyDiv += P.DW[Jn + N * k] * b2[I + N * k];
      DivTh += P.DW[I + N * k] * b3[k + N * Jn] + P.DW[Jn + N * k] * b4[I + N * k];
    }
    double FuC = d12 * DxCurl + d22 * DyCurl;
    double FvC = -d11 * DxCurl - d21 * DyCurl;
    double FuD = d11 * DxDiv + d21 * DyDiv;
    double FvD = d12 * DxDiv + d22 * DyDiv;
    vu = -(-P.nuCurl * FuC + P.nuGrad * FuD) / MC;
    vv = -(-P.nuCurl * FvC + P.nuGrad * FvD) / MC;
    vth = -P.nuDiv * DivTh / MC;
  }
  for (int iT = 0; iT < NT; ++iT) {
    __syncthreads();
    if (own) s[4][si] = T1[l + (size_t)nz * g + (5 + iT) * fs];
    __syncthreads();
    if (own) {
      const double *a5 = s[4] + row;
      double Dxc = P.D[I] * a5[N * Jn], Dyc = P.D[Jn] * a5[I];
#pragma unroll
      for (int k = 1; k < N; ++k) {
        Dxc += P.D[I + N * k] * a5[k + N * Jn];
        Dyc += P.D[Jn + N * k] * a5[I + N * k];
      }
      double GradDx = (d11 * Dxc + d21 * Dyc) / Js;
      double GradDy = (d12 * Dxc + d22 * Dyc) / Js;
      s[7][si] = rho * (d11 * GradDx + d12 * GradDy);
      s[8][si] = rho * (d21 * GradDx + d22 * GradDy);
    }
    __syncthreads();
    if (own) {
      const double *b3 = s[7] + row, *b4 = s[8] + row;
      double DivTr = P.DW[I] * b3[N * Jn] + P.DW[Jn] * b4[I];
#pragma unroll
      for (int k = 1; k < N; ++k) DivTr += P.DW[I + N * k] * b3[k + N * Jn] + P.DW[Jn + N * k] * b4[I + N * k];
#pragma unroll
      for (int q = 0; q < MAXTR; ++q)
        if (q == iT) vtr[q] = -P.nuDiv * DivTr / MC;
    }
  }
  __syncthreads();

  // ---------------- vector-invariant momentum + Coriolis ----------------
  // surface w from no normal flow (MomentumKernel.jl:35-36)
  auto wsurf = [&]() {
    return -(mt(C_D31_0, 0) * Uv(1, 0) + mt(C_D32_0, 0) * Uv(2, 0)) / mt(C_D33_0, 0);
  };
  auto wlo = [&](int lev) { return lev == 0 ? wsurf() : Uv(3, lev - 1); };
  double wl = 0, wh = 0;
  if (act) {
    wl = wlo(l);
    wh = Uv(3, l);
    s[0][si] = -mt(C_D12_0, l) * wl;   s[1][si] = -mt(C_D12_1, l) * wh;    // tempuZ1
    s[2][si] = -mt(C_D22_0, l) * wl;   s[3][si] = -mt(C_D22_1, l) * wh;    // tempuZ2
    s[4][si] = -mt(C_D11_0, l) * wl;   s[5][si] = -mt(C_D11_1, l) * wh;    // tempvZ1
    s[6][si] = -mt(C_D21_0, l) * wl;   s[7][si] = -mt(C_D21_1, l) * wh;    // tempvZ2
    s[8][si] = mt(C_D12_0, l) * u - mt(C_D11_0, l) * v;                     // tempwZ1
    s[9][si] = mt(C_D12_1, l) * u - mt(C_D11_1, l) * v;
    s[10][si] = mt(C_D22_0, l) * u - mt(C_D21_0, l) * v;                    // tempwZ2
    s[11][si] = mt(C_D22_1, l) * u - mt(C_D21_1, l) * v;
  }
  __syncthreads();
  double mu = 0, mv = 0, mwhi = 0;
  if (act) {
    // vertical temps of level lev (MomentumKernel.jl:50-72)
    auto tuZ0 = [&](int lev) { return mt(C_D33_0, lev) * Uv(2, lev) - mt(C_D32_0, lev) * wlo(lev); };
    auto tuZ1 = [&](int lev) { return mt(C_D33_1, lev) * Uv(2, lev) - mt(C_D32_1, lev) * Uv(3, lev); };
    auto tvZ0 = [&](int lev) { return mt(C_D33_0, lev) * Uv(1, lev) - mt(C_D31_0, lev) * wlo(lev); };
    auto tvZ1 = [&](int lev) { return mt(C_D33_1, lev) * Uv(1, lev) - mt(C_D31_1, lev) * Uv(3, lev); };
    auto twZ0 = [&](int lev) { return mt(C_D32_0, lev) * Uv(1, lev) - mt(C_D31_0, lev) * Uv(2, lev); };
    auto twZ1 = [&](int lev) { return mt(C_D32_1, lev) * Uv(1, lev) - mt(C_D31_1, lev) * Uv(2, lev); };
    double FU = 0.0, FV = 0.0, FW1 = 0.0, FW2 = 0.0;
    double tu0 = tuZ0(l), tu1 = tuZ1(l), tv0 = tvZ0(l), tv1 = tvZ1(l), tw0 = twZ0(l), tw1 = twZ1(l);
    if (l > 0) {
      double FluxUZ = 0.5 * (tu0 - tuZ1(l - 1));
      double FluxVZ = 0.5 * (tv0 - tvZ1(l - 1));
      double FluxWZ = 0.5 * (tw0 - twZ1(l - 1));
      FU += (-v * FluxWZ - wl * FluxVZ);
      FV += (u * FluxWZ - wl * FluxUZ);
      FW1 += (u * FluxVZ + v * FluxUZ);
    }
    if (l < nz - 1) {
      double FluxUZ = 0.5 * (tuZ0(l + 1) - tu1);
      double FluxVZ = 0.5 * (tvZ0(l + 1) - tv1);
      double FluxWZ = 0.5 * (twZ0(l + 1) - tw1);
      FU += (-v * FluxWZ - wh * FluxVZ);
      FV += (u * FluxWZ - wh * FluxUZ);
      FW2 += (u * FluxVZ + v * FluxUZ);
    }
    double U1 = 0.5 * (tu1 - tu0), U2 = U1;
    double V1 = 0.5 * (tv1 - tv0), V2 = V1;
    double W1 = 0.5 * (tw1 - tw0), W2 = W1;
    const double *a1 = s[0] + row, *b1 = s[1] + row, *a2 = s[2] + row, *b2 = s[3] + row;
    const double *a3 = s[4] + row, *b3 = s[5] + row, *a4 = s[6] + row, *b4 = s[7] + row;
    const double *a5 = s[8] + row, *b5 = s[9] + row, *a6 = s[10] + row, *b6 = s[11] + row;
    U1 += P.D[I] * a1[N * Jn] + P.D[Jn] * a2[I];
    U2 += P.D[I] * b1[N * Jn] + P.D[Jn] * b2[I];
    V1 += P.D[I] * a3[N * Jn] + P.D[Jn] * a4[I];
    V2 += P.D[I] * b3[N * Jn] + P.D[Jn] * b4[I];
    W1 += P.D[I] * a5[N * Jn] + P.D[Jn] * a6[I];
    W2 += P.D[I] * b5[N * Jn] + P.D[Jn] * b6[I];
#pragma unroll
    for (int k = 1; k < N; ++k) {
      U1 += P.D[I + N * k] * a1[k + N * Jn] + P.D[Jn + N * k] * a2[I + N * k];
      U2 += P.D[I + N * k] * b1[k + N * Jn] + P.D[Jn + N * k] * b2[I + N * k];
      V1 += P.D[I + N * k] * a3[k + N * Jn] + P.D[Jn + N * k] * a4[I + N * k];
      V2 += P.D[I + N * k] * b3[k + N * Jn] + P.D[Jn + N * k] * b4[I + N * k];
      W1 += P.D[I + N * k] * a5[k + N * Jn] + P.D[Jn + N * k] * a6[I + N * k];
      W2 += P.D[I + N * k] * b5[k + N * Jn] + P.D[Jn + N * k] * b6[I + N * k];
    }
    double fc = mt(C_FCOR, l);
    double FuCor = v * fc, FvCor = -u * fc, FwCor = 0.0;
    double J1 = mt(C_J0, l), J2 = mt(C_J1, l);
    FU += FuCor * (J1 + J2);
    FV += FvCor * (J1 + J2);
    FW1 += FwCor * J1;
    FW2 += FwCor * J2;
    mu = (-v * W1 - wl * V1 - v * W2 - wh * V2 + FU) / MC;
    mv = (u * W1 - wl * U1 + u * W2 - wh * U2 + FV) / MC;
    double mwlo = 0.0;
    if (l > 0)
      mwlo = rho * (u * V1 + v * U1 + FW1) / (Uv(0, l - 1) * P.M[l - 1 + (size_t)nz * (g + (size_t)NumG)] +
                                               rho * P.M[l + (size_t)nz * g]);
    if (l < nz - 1)
      mwhi = rho * (u * V2 + v * U2 + FW2) / (Uv(0, l + 1) * P.M[l + 1 + (size_t)nz * g] +
                                               rho * P.M[l + (size_t)nz * (g + (size_t)NumG)]);
    slo[0][si] = mwlo;
  }
  __syncthreads();

  // ---------------- kinetic-energy and pressure gradient, gravity ----------------
  auto K1 = [&](int lev) {
    double uu = Uv(1, lev), vvv = Uv(2, lev), w0 = wlo(lev);
    return 0.5 * (uu * uu + vvv * vvv) + 0.5 * (w0 * w0);
  };
  auto K2 = [&](int lev) {
    double uu = Uv(1, lev), vvv = Uv(2, lev), w1 = Uv(3, lev);
    return 0.5 * (uu * uu + vvv * vvv) + 0.5 * (w1 * w1);
  };
  double pl = 0;
  if (act) {
    pl = pressure_dry(P, Uv(4, l));
    s[0][si] = K1(l);
    s[1][si] = K2(l);
    s[2][si] = pl;
  }
  __syncthreads();
  double gu = 0, gv = 0, gwhi = 0;
  if (act) {
    const double *Ka = s[0] + row, *Kb = s[1] + row, *pa = s[2] + row;
    double DXp = P.D[I] * pa[N * Jn], DYp = P.D[Jn] * pa[I];
    double DXK1 = P.D[I] * Ka[N * Jn], DYK1 = P.D[Jn] * Ka[I];
    double DXK2 = P.D[I] * Kb[N * Jn], DYK2 = P.D[Jn] * Kb[I];
#pragma unroll
    for (int k = 1; k < N; ++k) {
      DXK1 += P.D[I + N * k] * Ka[k + N * Jn];
      DYK1 += P.D[Jn + N * k] * Ka[I + N * k];
      DXK2 += P.D[I + N * k] * Kb[k + N * Jn];
      DYK2 += P.D[Jn + N * k] * Kb[I + N * k];
      DXp += P.D[I + N * k] * pa[k + N * Jn];
      DYp += P.D[Jn + N * k] * pa[I + N * k];
    }
    double GuF1 = -(mt(C_D11_0, l) * DXK1 + mt(C_D21_0, l) * DYK1);
    double GvF1 = -(mt(C_D12_0, l) * DXK1 + mt(C_D22_0, l) * DYK1);
    double GuF2 = -(mt(C_D11_1, l) * DXK2 + mt(C_D21_1, l) * DYK2);
    double GvF2 = -(mt(C_D12_1, l) * DXK2 + mt(C_D22_1, l) * DYK2);
    double Gradu = d11 * DXp + d21 * DYp;
    double Gradv = d12 * DXp + d22 * DYp;
    double GwF1 = 0.0, GwF2 = 0.0, GZ;
    double k1l = Ka[ID], k2l = Kb[ID];
    if (l > 0) {
      GZ = 0.5 * (k1l - K2(l - 1));
      GuF1 += -GZ * mt(C_D31_0, l);
      GvF1 += -GZ * mt(C_D32_0, l);
      GwF1 += -rho * GZ * mt(C_D33_0, l);
    }
    if (l < nz - 1) {
      GZ = 0.5 * (K1(l + 1) - k2l);
      GuF2 += -GZ * mt(C_D31_1, l);
      GvF2 += -GZ * mt(C_D32_1, l);
      GwF2 += -rho * GZ * mt(C_D33_1, l);
    }
    GZ = 0.5 * (k2l - k1l);
    GuF2 += -GZ * mt(C_D31_1, l);
    GuF1 += -GZ * mt(C_D31_0, l);
    GvF2 += -GZ * mt(C_D32_1, l);
    GvF1 += -GZ * mt(C_D32_0, l);
    GwF2 += -rho * GZ * mt(C_D33_1, l);
    GwF1 += -rho * GZ * mt(C_D33_0, l);
    const double Grav = P.Grav;
    GZ = -Grav * rho * (mt(C_J0, l) + mt(C_J1, l)) / (mt(C_D33_0, l) + mt(C_D33_1, l));
    Gradu += GZ * (mt(C_D31_0, l) + mt(C_D31_1, l));
    Gradv += GZ * (mt(C_D32_0, l) + mt(C_D32_1, l));
    gu = (GuF1 + GuF2 - Gradu / rho) / MC;
    gv = (GvF1 + GvF2 - Gradv / rho) / MC;
    if (l < nz - 1) {
      double rhop = Uv(0, l + 1);
      GZ = 0.5 * (pressure_dry(P, Uv(4, l + 1)) - pl);
      double Gradw = GZ * (mt(C_D33_1, l) + mt(C_D33_0, l + 1));
      double Gradp = -(Gradw + Grav * (rho * mt(C_J1, l) + rhop * mt(C_J0, l + 1)));
      gwhi = (GwF2 + Gradp) / (rhop * P.M[l + 1 + (size_t)nz * g] + rho * P.M[l + (size_t)nz * (g + (size_t)NumG)]);
    }
    double gwlo = 0.0;
    if (l > 0)
      gwlo = GwF1 / (Uv(0, l - 1) * P.M[l - 1 + (size_t)nz * (g + (size_t)NumG)] + rho * P.M[l + (size_t)nz * g]);
    slo[1][si] = gwlo;
  }
  __syncthreads();

  // ---------------- continuity, rho*theta and tracer fluxes ----------------
  double hr = 0, hth = 0, htr[MAXTR] = {0, 0, 0, 0};
  if (own) {
    s[0][si] = -rho * (d11 * u + d12 * v);   // Contra12(-Rho, u, v)
    s[1][si] = -rho * (d21 * u + d22 * v);
    s[2][si] = Uv(4, l) / rho;
  }
  __syncthreads();
  if (own) {
    const double *uc = s[0] + row, *vc = s[1] + row, *cc = s[2] + row;
    double DivRhoTr = P.D[I] * uc[N * Jn] * cc[N * Jn] + P.D[Jn] * vc[I] * cc[I];
    double DivRho = P.D[I] * uc[N * Jn] + P.D[Jn] * vc[I];
#pragma unroll
    for (int k = 1; k < N; ++k) {
      DivRhoTr += P.D[I + N * k] * uc[k + N * Jn] * cc[k + N * Jn] + P.D[Jn + N * k] * vc[I + N * k] * cc[I + N * k];
      DivRho += P.D[I + N * k] * uc[k + N * Jn] + P.D[Jn + N * k] * vc[I + N * k];
    }
    hth = DivRhoTr / MC;
    hr = DivRho / MC;
  }
  for (int iT = 0; iT < NT; ++iT) {
    __syncthreads();
    if (own) s[2][si] = Uv(5 + iT, l) / rho;
    __syncthreads();
    if (own) {
      const double *uc = s[0] + row, *vc = s[1] + row, *cc = s[2] + row;
      double DivRhoTr = P.D[I] * uc[N * Jn] * cc[N * Jn] + P.D[Jn] * vc[I] * cc[I];
#pragma unroll
      for (int k = 1; k < N; ++k)
        DivRhoTr += P.D[I + N * k] * uc[k + N * Jn] * cc[k + N * Jn] + P.D[Jn + N * k] * vc[I + N * k] * cc[I + N * k];
#pragma unroll
      for (int q = 0; q < MAXTR; ++q)
        if (q == iT) htr[q] = DivRhoTr / MC;
    }
  }
  if (!own) return;   // no further __syncthreads below

  // vertical upwind fluxes through the top (interface l) and bottom
  // (interface l-1) of this layer; each is the reference's per-interface flux
  // (OperatorKernel.jl:689-702) divided by this layer's MC.
  double fr_top = 0, fr_bot = 0, fth_top = 0, fth_bot = 0;
  double ftr_top[MAXTR] = {0, 0, 0, 0}, ftr_bot[MAXTR] = {0, 0, 0, 0};
  auto cr = [&](int f, int lev) { return Uv(f, lev) / Uv(0, lev); };
  auto wcon_at = [&](int il) {   // interface il between layers il and il+1
    double w = Uv(3, il);
    return Uv(0, il) * (mt(C_D31_1, il) * Uv(1, il) + mt(C_D32_1, il) * Uv(2, il) + mt(C_D33_1, il) * w) +
           Uv(0, il + 1) * (mt(C_D31_0, il + 1) * Uv(1, il + 1) + mt(C_D32_0, il + 1) * Uv(2, il + 1) +
                            mt(C_D33_0, il + 1) * w);
  };
  for (int side = 0; side < 2; ++side) {
    int il = side == 0 ? l : l - 1;
    if (il < 0 || il >= nz - 1) continue;
    double wCon = wcon_at(il);
    int lm = il > 0 ? il - 1 : 0, lp1 = il + 1, lp2 = il + 2 < nz ? il + 2 : nz - 1;
    double JLL = Jsum(lm), JL = Jsum(il), JR = Jsum(lp1), JRR = Jsum(lp2);
    double cFL, cFR;
    recu4(cr(4, lm), cr(4, il), cr(4, lp1), cr(4, lp2), JLL, JL, JR, JRR, cFL, cFR);
    double Flux = 0.25 * ((fabs(wCon) + wCon) * cFL + (-fabs(wCon) + wCon) * cFR);
    double Flr = 0.5 * wCon;
    if (side == 0) { fth_top = -Flux / MC; fr_top = -Flr / MC; }
    else { fth_bot = Flux / MC; fr_bot = Flr / MC; }
    for (int iT = 0; iT < NT; ++iT) {
      recu4(cr(5 + iT, lm), cr(5 + iT, il), cr(5 + iT, lp1), cr(5 + iT, lp2), JLL, JL, JR, JRR, cFL, cFR);
      double Fl = 0.25 * ((fabs(wCon) + wCon) * cFL + (-fabs(wCon) + wCon) * cFR);
#pragma unroll
      for (int q = 0; q < MAXTR; ++q)
        if (q == iT) { if (side == 0) ftr_top[q] = -Fl / MC; else ftr_bot[q] = Fl / MC; }
    }
  }

  // ---------------- assemble this element node's contributions ----------------
  double *out = C + ((size_t)IF * P.NV * DoF + ID) * nz + l;
  double acc = 0.0;
  if (l < nz - 1) acc += fr_top;
  if (l > 0) acc += fr_bot;
  acc += hr;
  out[0] = acc;
  acc = 0.0; acc += vu; acc += mu; acc += gu;
  out[cs] = acc;
  acc = 0.0; acc += vv; acc += mv; acc += gv;
  out[2 * cs] = acc;
  acc = 0.0;
  if (l < nz - 1) {
    double hi = mwhi + gwhi;
    double lo = slo[0][si + DoF] + slo[1][si + DoF];
    acc = hi + lo;
  }
  out[3 * cs] = acc;
  acc = 0.0; acc += vth;
  if (l < nz - 1) acc += fth_top;
  if (l > 0) acc += fth_bot;
  acc += hth;
  out[4 * cs] = acc;
#pragma unroll
  for (int q = 0; q < MAXTR; ++q)
    if (q < NT) {
      acc = 0.0; acc += vtr[q];
      if (l < nz - 1) acc += ftr_top[q];
      if (l > 0) acc += ftr_bot[q];
      acc += htr[q];
      out[(5 + q) * cs] = acc;
    }
}

// ---------------------------------------------------------------------------
// Column part of a Rosenbrock-W stage, fused (one warp per column, lanes over
// levels): owner gather of the tendency, stage corrections
// fV = F + sum_j c_ij/dt k_j, vertical acoustic Jacobian from the step's
// initial state (JacSchurKernel!, src/DyCore/JacSchur.jl:29-75), the Schur
// tridiagonal system (TriDiagKernel!, SchurSolveFKernel!, triSolve!,
// SchurSolveBKernel!: src/Integration/SchurSolve.jl:1-114) and the stage
// update of RosenbrockSchur! (src/Integration/RosenbrockSchur.jl:13-32).
// MODE 0: stage 1 -> k1, Vst = Vn + a21 k1
// MODE 1: stage 2 -> k2, Vst = (Vn + a31 k1) + a32 k2
// MODE 2: stage 3 -> Vout = ((Vn + m1 k1) + m2 k2) + m3 k3   (Vout may alias Vn)
// MODE 3: standalone Schur solve with stored bands: k, v updated (cgd_schur_solve)
// ---------------------------------------------------------------------------
struct ColArgs {
  const double *C;       // contributions of phase 2 (MODE 0..2)
  const double *Vn;      // step initial state (MODE 0..2)
  const double *k1, *k2;
  double *kout;          // MODE 0,1,3
  double *Vout;          // MODE 0,1 (stage state), 2 (new state)
  double *v;             // MODE 3: right-hand side (overwritten)
  const double *bands;   // MODE 3: (2, nz-1, NumG) x 4
  double dt, fac;
  RK rk;
};

constexpr int COL_WARPS = 4;
constexpr int COL_NARR = MAXNV + 8 + 3 + 1;   // fv[NV], 8 bands, tri[3], x

__device__ __forceinline__ void jac_at(const GP &P, double RhoL, double RhoR, double RhoThL0, double RhoThR0,
                                       double dzL, double dzR, double *jb)
{
  // JacSchurKernel! (src/DyCore/JacSchur.jl:40-73); AuxG[:,:,4] == 0 for Dry
  double RhoThL = RhoThL0 + 0.0, RhoThR = RhoThR0 + 0.0;
  double RhoF = (RhoL * dzL + RhoR * dzR) / (dzL + dzR);
  jb[0] = -RhoF / dzL;             // JRhoW[1]
  jb[1] = RhoF / dzR;              // JRhoW[2]
  double expo = P.kappa / (1.0 - P.kappa);
  double dPdThL = P.Rd * cgd_pow(P.Rd * RhoThL / P.p0, expo);
  double dPdThR = P.Rd * cgd_pow(P.Rd * RhoThR / P.p0, expo);
  jb[4] = -dPdThR / RhoF / (0.5 * (dzL + dzR));   // JWRhoTh[1]
  jb[5] = dPdThL / RhoF / (0.5 * (dzL + dzR));    // JWRhoTh[2]
  jb[2] = -P.Grav * dzR / RhoF / (dzL + dzR);     // JWRho[1]
  jb[3] = -P.Grav * dzL / RhoF / (dzL + dzR);     // JWRho[2]
  double RhoThF = (RhoThL * dzL + RhoThR * dzR) / (dzL + dzR);
  jb[6] = -RhoThF / dzL;           // JRhoThW[1]
  jb[7] = RhoThF / dzR;            // JRhoThW[2]
}

template <int MODE>
__global__ void __launch_bounds__(32 * COL_WARPS) k_column(const GP P, const ColArgs A)
{
  extern __shared__ double csm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = blockIdx.x * COL_WARPS + warp;
  if (g >= P.NumG) return;
  const int nz = P.nz, n = nz - 1, NV = P.NV, NumG = P.NumG;
  double *sw = csm + (size_t)warp * COL_NARR * 64;
  double *fv = sw;                      // [NV][64]
  double *jb = sw + MAXNV * 64;         // [8][64]
  double *tri = jb + 8 * 64;            // [3][64]
  double *xs = tri + 3 * 64;            // [64]
  const size_t fs = (size_t)nz * NumG;
  const double fac = A.fac;

  // 1. tendency (owner gather) + stage corrections ; bands
  for (int l = lane; l < nz; l += 32) {
    if (MODE <= 2) {
      const int q0 = P.inv_ptr[g], q1 = P.inv_ptr[g + 1];
      const size_t fstr = (size_t)P.DoF * nz;
      for (int f = 0; f < NV; ++f) {
        double acc = 0.0;
        for (int q = q0; q < q1; ++q) acc += A.C[P.inv_off[q] + f * fstr + l];
        double x = acc;
        if (MODE >= 1) x = x + A.rk.c[MODE][0] / A.dt * A.k1[l + (size_t)nz * g + f * fs];
        if (MODE >= 2) x = x + A.rk.c[MODE][1] / A.dt * A.k2[l + (size_t)nz * g + f * fs];
        fv[f * 64 + l] = x;
      }
      if (l < n) {
        double b[8];
        const double *V0 = A.Vn + (size_t)nz * g;
        jac_at(P, V0[l], V0[l + 1], V0[l + 4 * fs], V0[l + 1 + 4 * fs],
               P.dz[l + (size_t)nz * g], P.dz[l + 1 + (size_t)nz * g], b);
        for (int r = 0; r < 8; ++r) jb[r * 64 + l] = b[r];
      }
    } else {
      for (int f = 0; f < NV; ++f) fv[f * 64 + l] = A.v[l + (size_t)nz * g + f * fs];
      if (l < n) {
        const size_t bs = (size_t)2 * n * NumG;
        for (int arr = 0; arr < 4; ++arr)
          for (int r = 0; r < 2; ++r) jb[(2 * arr + r) * 64 + l] = A.bands[arr * bs + r + 2 * (l + (size_t)n * g)];
      }
    }
  }
  __syncwarp();
  // jb rows: 0,1 JRhoW ; 2,3 JWRho ; 4,5 JWRhoTh ; 6,7 JRhoThW  (row r = Julia index r%2+1)
#define JB(arr, r, i) jb[((arr) * 2 + (r)) * 64 + (i)]
  const double invfac = 1.0 / fac;
  const double invfac2 = invfac / fac;
  double v3new[2];
  for (int it = 0, l = lane; l < nz; l += 32, ++it) {
    if (l < n) {   // TriDiagKernel!
      double t0, t1, t2;
      t1 = invfac2 - JB(1, 1, l) * JB(0, 0, l) - JB(1, 0, l) * JB(0, 1, l) -
           JB(2, 1, l) * JB(3, 0, l) - JB(2, 0, l) * JB(3, 1, l);
      if (l == 0) t0 = 0.0;
      else t0 = -JB(1, 0, l - 1) * JB(0, 0, l) - JB(2, 0, l - 1) * JB(3, 0, l);
      if (l == n - 1) t2 = 0.0;
      else t2 = -JB(1, 1, l + 1) * JB(0, 1, l) - JB(2, 1, l + 1) * JB(3, 1, l);
      tri[l] = t0; tri[64 + l] = t1; tri[128 + l] = t2;
      // SchurSolveFKernel!
      v3new[it] = fv[3 * 64 + l] / fac + JB(1, 1, l) * fv[l] + JB(1, 0, l) * fv[l + 1] +
                  JB(2, 1, l) * fv[4 * 64 + l] + JB(2, 0, l) * fv[4 * 64 + l + 1];
    }
  }
  __syncwarp();
  for (int it = 0, l = lane; l < n; l += 32, ++it) fv[3 * 64 + l] = v3new[it];
  __syncwarp();
  if (lane == 0) {   // triSolve! (Thomas), b = fv[3], x = xs
    double *b = fv + 3 * 64;
    xs[0] = tri[64 + 0];
    for (int i = 0; i < n - 1; ++i) {
      xs[i + 1] = tri[64 + i + 1] - tri[128 + i] / xs[i] * tri[i + 1];
      b[i + 1] = b[i + 1] - tri[128 + i] / xs[i] * b[i];
    }
    xs[n - 1] = b[n - 1] / xs[n - 1];
    for (int i = n - 2; i >= 0; --i) xs[i] = (b[i] - tri[i + 1] * xs[i + 1]) / xs[i];
  }
  __syncwarp();
  // SchurSolveBKernel! and the stage update
  double res[2][MAXNV];
  for (int it = 0, l = lane; l < nz; l += 32, ++it) {
    double kw = l < n ? xs[l] : 0.0;
    double v0 = fv[l], v4 = fv[4 * 64 + l];
    if (l == 0) {
      v0 += JB(0, 0, l) * xs[l];
      v4 += JB(3, 0, l) * xs[l];
    } else if (l == nz - 1) {
      v0 += JB(0, 1, l - 1) * xs[l - 1];
      v4 += JB(3, 1, l - 1) * xs[l - 1];
    } else {
      v0 += JB(0, 0, l) * xs[l] + JB(0, 1, l - 1) * xs[l - 1];
      v4 += JB(3, 0, l) * xs[l] + JB(3, 1, l - 1) * xs[l - 1];
    }
    for (int f = 0; f < NV; ++f) {
      double k;
      if (f == 3) k = kw;
      else if (f == 0) k = fac * v0;
      else if (f == 4) k = fac * v4;
      else k = fac * fv[f * 64 + l];
      res[it][f] = k;
    }
    if (MODE == 3) {
      // v after SchurSolveF/B (the Thomas sweep works on a copy, as in
      // SchurSolveTriKernel!'s shared-memory vCol)
      A.v[l + (size_t)nz * g] = v0;
      A.v[l + (size_t)nz * g + 4 * fs] = v4;
      if (l < n) A.v[l + (size_t)nz * g + 3 * fs] = v3new[it];
    }
  }
#undef JB
  // all lanes have finished reading Vn (for the bands) before anything is written
  __syncwarp();
  for (int it = 0, l = lane; l < nz; l += 32, ++it) {
    for (int f = 0; f < NV; ++f) {
      const size_t o = l + (size_t)nz * g + f * fs;
      double k = res[it][f];
      if (MODE == 0) {
        A.kout[o] = k;
        A.Vout[o] = A.Vn[o] + A.rk.a[1][0] * k;
      } else if (MODE == 1) {
        A.kout[o] = k;
        A.Vout[o] = A.Vn[o] + A.rk.a[2][0] * A.k1[o] + A.rk.a[2][1] * k;
      } else if (MODE == 2) {
        A.Vout[o] = A.Vn[o] + A.rk.m[0] * A.k1[o] + A.rk.m[1] * A.k2[o] + A.rk.m[2] * k;
      } else {
        A.kout[o] = k;
      }
    }
  }
}

// Jacobian bands into memory (cgd_jac): one thread per (interface, column)
__global__ void k_jac(const GP P, const double *__restrict__ U, double *__restrict__ bands)
{
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int n = P.nz - 1;
  if (tid >= (long long)n * P.NumG) return;
  const int g = (int)(tid / n), l = (int)(tid % n);
  const int nz = P.nz;
  const size_t fs = (size_t)nz * P.NumG;
  const double *V0 = U + (size_t)nz * g;
  double b[8];
  jac_at(P, V0[l], V0[l + 1], V0[l + 4 * fs], V0[l + 1 + 4 * fs], P.dz[l + (size_t)nz * g],
         P.dz[l + 1 + (size_t)nz * g], b);
  const size_t bs = (size_t)2 * n * P.NumG;
  for (int arr = 0; arr < 4; ++arr)
    for (int r = 0; r < 2; ++r) bands[arr * bs + r + 2 * (l + (size_t)n * g)] = b[arr * 2 + r];
}

__global__ void k_pressure(const GP P, const double *__restrict__ U, double *__restrict__ p)
{
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long S = (long long)P.nz * P.NumG;
  if (tid >= S) return;
  p[tid] = pressure_dry(P, U[tid + 4 * S]);
}

// 1 if any entry is not finite
__global__ void k_nonfinite(const double *__restrict__ x, long long n, int *__restrict__ flag)
{
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long stride = (long long)gridDim.x * blockDim.x;
  int bad = 0;
  for (; i < n; i += stride) {
    double v = x[i];
    if (!(v - v == 0.0)) bad = 1;
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(flag, 1);
}

// deterministic two-level reduction of sum(rho*MMass): per-block partials in
// fixed order, then one block sums the partials in order
__global__ void k_mass_partial(const double *__restrict__ rho, const double *__restrict__ mm, long long n,
                               double *__restrict__ part)
{
  __shared__ double sh[256];
  long long chunk = (n + gridDim.x - 1) / gridDim.x;
  long long b0 = blockIdx.x * chunk, b1 = b0 + chunk < n ? b0 + chunk : n;
  double acc = 0.0;
  for (long long i = b0 + threadIdx.x; i < b1; i += blockDim.x) acc += rho[i] * mm[i];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__global__ void k_mass_final(const double *__restrict__ part, int nb, double *__restrict__ out)
{
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double acc = 0.0;
    for (int i = 0; i < nb; ++i) acc += part[i];
    out[0] = acc;
  }
}

} // namespace cgd
