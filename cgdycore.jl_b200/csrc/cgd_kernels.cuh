// cgd_kernels.cuh - sm_100a kernels of the FP64 hot path.
//
// Layouts in HBM
//   state U, Temp1, F, k   (nz, NumG, NV) level fastest (the reference layout)
//   met                    [IF][comp][ID][nz]  21 components per element node
//                          and level (14 used dXdxI entries, J bottom/top,
//                          2*Omega*sin(lat) at the layer midpoint, the four
//                          J-only coefficients of RecU4 at the interface above)
//   C  (contributions)     [IF][slot][ID][nz]  element-local DSS inputs; NV + 1
//                          slots (the tendency fields, then the lower-node
//                          part of the phase-2 w contribution, one level down)
//   M                      (nz, NumG, 2)
//
// Direct-stiffness summation is an owner gather: the element kernels write
// every element-node contribution to C, and one thread per (global DOF,
// level) sums the contributions of the element nodes that share the DOF in
// ascending (element, node) order.  No atomics: results are bit-reproducible
// and equal to the CPU restatement's.
//
// Every floating-point expression below is written in the reference's
// evaluation order (see CGD_FAST below for the two builds).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <type_traits>
#include "../../include/cgd_math.h"

// Two builds come from this source, both compiled without multiply-add
// contraction (-fmad=false).  The exact build evaluates the reference's
// expressions literally - every division is a division - so results are
// bit-identical to the CPU restatement.  The fast build (CGD_FAST) replaces
// the final division of a chain by the time-invariant sums J0+J1 (element
// Jacobian) and M0+M1 (lumped mass), or by rho, with a multiply by a
// reciprocal computed once per node and level (one rounding more, at the
// end of the chain).
#ifdef CGD_FAST
#define CGD_DIVJ(x) ((x) * rJs)
#define CGD_DIVM(x) ((x) * rMC)
#else
#define CGD_DIVJ(x) ((x) / Js)
#define CGD_DIVM(x) ((x) / MC)
#endif

namespace cgd {

// Arithmetic of the horizontal derivative sums, generic in the compute type R.
// For R = double the expressions are the reference's, unfused, in its order
// (acc + c*x; acc + (c1*x1 + c2*x2)); for R = float (the mixed form) they are
// fused multiply-adds.
__device__ __forceinline__ double rsum1(double acc, double c, double x) { return acc + c * x; }
__device__ __forceinline__ double rsum2(double acc, double c1, double x1, double c2, double x2)
{
  return acc + (c1 * x1 + c2 * x2);
}
__device__ __forceinline__ float rsum1(float acc, float c, float x) { return __fmaf_rn(c, x, acc); }
__device__ __forceinline__ float rsum2(float acc, float c1, float x1, float c2, float x2)
{
  return __fmaf_rn(c1, x1, __fmaf_rn(c2, x2, acc));
}

// 8- and 4-byte asynchronous copies global -> shared (cp.async, sm_80 and
// later) and the wait for all of a thread's copies
__device__ __forceinline__ void cp_async8(double *smem_dst, const double *gsrc)
{
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async4(float *smem_dst, const float *gsrc)
{
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

constexpr int NCOMP = 21;
enum {
  C_D11_0 = 0, C_D11_1, C_D12_0, C_D12_1, C_D21_0, C_D21_1, C_D22_0, C_D22_1,
  C_D31_0, C_D31_1, C_D32_0, C_D32_1, C_D33_0, C_D33_1, C_J0, C_J1, C_FCOR,
  // RecU4 coefficients of the interface above the level (they depend on J only):
  // kR, kL of the left state and kL, kR of the right state
  C_RK0, C_RK1, C_RK2, C_RK3
};
constexpr int MAXTR = 4;
constexpr int MAXNV = 5 + MAXTR;

// Everything a kernel needs about the grid, passed by value.
struct GP {
  int N, DoF, nz, NF, NumG, NumTr, NV;
  int NC;                   // contribution slots per element node: NV fields + the lower-node w of phase 2
  int IF0;                  // first element of a launch over a range of elements (k_hypervisc1, k_phase2)
  const double *met;        // [IF][comp][ID][nz]
  const double *M;          // (nz, NumG, 2)
  const double *dz;         // (nz, NumG)
  const int *glob;          // [IF*DoF + ID], 0-based
  const int *inv_ptr;       // NumG + 1
  const long long *inv_off; // (IF*NC*DoF + ID)*nz for every contributor
  const long long *inv_tab; // 4 per DOF: its first four inv_off entries, -1 past the count (-1 first: > 4)
  double D[25], DW[25];     // D[i + N*j] = DS[i,j]
  const double *pref;       // mixed form: per-level FP64 reference pressure and theta
  const double *thref;
  double Grav, Rd, p0, kappa, nuCurl, nuGrad, nuDiv;
  // column physics of the tendency tail (cgd_set_physics): the dry
  // Held-Suarez forcing and the Rayleigh damping of w near the top
  int held_suarez, damping;
  double hs[8];             // k_a, k_f, k_s, DeltaT_y, DeltaTh_z, T_equator, T_min, sigma_b
  const double *coslat, *sinlat;   // (NumG) latitude of each column's surface node
  const double *dampc;             // (nz, NumG) damping rate at the layer midpoint
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

// The column physics of the tendency tail at level l of column g
// (src/GPU/FcnGPU.jl:953-966): ForceKernel! with the dry Held-Suarez Force
// (src/GPU/OperatorKernel.jl:1073-1080, src/Examples/initial.jl:513-531) and
// DampKernel! with DampingW (OperatorKernel.jl:1061-1071,
// src/GPU/dampingGPU.jl:1-19), for the state values rho, u, v, w, rho*theta
// and the pressure p there: adds to f[1] (u), f[2] (v), f[3] (w), f[4]
// (rho*theta).  fast_powGPU(x, y) = exp(y log x) (src/Models/Equation.jl:79).
__device__ __forceinline__ void physics_terms(const GP &P, int l, int g, double rho, double u, double v, double w,
                                              double rhoth, double p, double *f)
{
  if (P.held_suarez) {
    const double k_a = P.hs[0], k_f = P.hs[1], k_s = P.hs[2], DeltaT_y = P.hs[3], DeltaTh_z = P.hs[4];
    const double T_equator = P.hs[5], T_min = P.hs[6], sigma_b = P.hs[7];
    const double Sigma = p / P.p0;
    const double SigmaPowKappa = cgd_exp(P.kappa * cgd_log(Sigma));
    const double height_factor = cgd_max(0.0, (Sigma - sigma_b) / (1.0 - sigma_b));
    const double coslat = P.coslat[g], sinlat = P.sinlat[g];
    f[1] += -(k_f * height_factor) * u;
    f[2] += -(k_f * height_factor) * v;
    const double kT = k_a + (k_s - k_a) * height_factor * coslat * coslat * coslat * coslat;
    double Teq = (T_equator - DeltaT_y * sinlat * sinlat - DeltaTh_z * cgd_log(Sigma) * coslat * coslat) *
                 SigmaPowKappa;
    Teq = cgd_max(T_min, Teq);
    const double T = p / (rho * P.Rd);
    const double DeltaT = kT * (T - Teq);
    f[4] += -rhoth / T * DeltaT;
  }
  if (P.damping) f[3] += -P.dampc[l + (size_t)P.nz * g] * w;
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
// R is the compute type of the derivative sums: double, or float for the
// mixed form, where theta enters as its perturbation from the level's FP64
// reference value.
// ---------------------------------------------------------------------------
// shared arrays of phase 1: planes 0-3 curl/contra of (u,v), 4 theta, 5-8
// the first derivatives, then per tracer its ratio and the two components of
// its gradient, each LT levels x DoF nodes
template <int N, int NT, typename R, int LT_ = 256 / (N * N)>
struct HV1Smem {
  static constexpr int DoF = N * N, LT = LT_;
  static constexpr int PLANES = 9 + 3 * NT;
  static constexpr size_t BYTES = (size_t)PLANES * LT * DoF * sizeof(R);
};

// Level tile of k_hypervisc1.  At p = 4 in FP64, 16 levels (400 threads,
// three CTAs per SM): a warp then reads runs of 16 consecutive levels of two
// nodes instead of 10 levels of three or four, so the metric and state loads
// touch fewer L1 lines: 0.416 -> 0.310 ms on the drop-in grid.  Elsewhere 256 / N^2 levels (256
// threads, four CTAs per SM), which the FP32 form also keeps (0.286 ms against
// 0.316 ms with 16 levels).
template <int N, typename R>
struct HV1Tile {
  static constexpr bool WIDE = N == 5 && sizeof(R) == sizeof(double);
  static constexpr int LT = WIDE ? 16 : 256 / (N * N);
  static constexpr int THREADS = WIDE ? LT * N * N : 256;
  static constexpr int MINB = WIDE ? 3 : 4;
};
template <int N, int NT, typename R>
__device__ __forceinline__ R *hv1_static_smem()
{
  using S = HV1Smem<N, NT, R>;
  __shared__ R s[S::PLANES * S::LT * S::DoF];
  return s;
}

// sbuf: the shared arrays (hv1_static_smem, or a kernel's dynamic buffer)
template <int N, int NT, typename R, int LT = 256 / (N * N)>
__device__ __forceinline__ void hypervisc1_body(const GP &P, const double *__restrict__ U, double *__restrict__ C,
                                                const int tile, const int IF, R *sbuf)
{
  constexpr bool MIX = sizeof(R) == sizeof(float);
  constexpr int DoF = N * N;
  R(*s)[LT * DoF] = reinterpret_cast<R(*)[LT * DoF]>(sbuf);
  const int t = threadIdx.x;
  const int lvl = t % LT, ID = t / LT;
  const int I = ID % N, Jn = ID / N;
  const int l = tile * LT + lvl;
  const int nz = P.nz, NumG = P.NumG;
  const bool act = (ID < DoF) && (l < nz);
  const int si = lvl * DoF + ID, row = lvl * DoF;
  const size_t cs = (size_t)DoF * nz;
  int g = 0;
  R d11 = 0, d12 = 0, d21 = 0, d22 = 0;
  double JsD = 1, MCD = 1;
  R DI[N], DJ[N];
#pragma unroll
  for (int k = 0; k < N; ++k) {
    DI[k] = (R)P.D[I + N * k];
    DJ[k] = (R)P.D[Jn + N * k];
  }
  const double *mt = P.met + ((size_t)IF * NCOMP * DoF + ID) * nz + l;
  if (act) {
    g = P.glob[IF * DoF + ID];
    d11 = (R)(mt[C_D11_0 * cs] + mt[C_D11_1 * cs]);
    d12 = (R)(mt[C_D12_0 * cs] + mt[C_D12_1 * cs]);
    d21 = (R)(mt[C_D21_0 * cs] + mt[C_D21_1 * cs]);
    d22 = (R)(mt[C_D22_0 * cs] + mt[C_D22_1 * cs]);
    JsD = mt[C_J0 * cs] + mt[C_J1 * cs];
    const double *Ug = U + l + (size_t)nz * g;
    const size_t fs = (size_t)nz * NumG;
    const R u = (R)Ug[1 * fs], v = (R)Ug[2 * fs];
    s[0][si] = d11 * v - d12 * u;   // Curl12
    s[1][si] = d21 * v - d22 * u;
    s[2][si] = d11 * u + d12 * v;   // Contra12
    s[3][si] = d21 * u + d22 * v;
    if (MIX) s[4][si] = (R)(Ug[4 * fs] / Ug[0] - P.thref[l]);
    else s[4][si] = (R)(Ug[4 * fs] / Ug[0]);
#pragma unroll
    for (int q = 0; q < NT; ++q) s[9 + 3 * q][si] = (R)(Ug[(5 + q) * fs] / Ug[0]);
    MCD = P.M[l + (size_t)nz * g] + P.M[l + (size_t)nz * (g + (size_t)NumG)];
  }
  const R Js = (R)JsD, MC = (R)MCD;
  const R rJs = (R)(1.0 / JsD), rMC = (R)(1.0 / MCD);
  (void)rJs; (void)rMC; (void)Js; (void)MC;
  __syncthreads();
  if (act) {
    const R *uC = s[0] + row, *vC = s[1] + row, *uD = s[2] + row, *vD = s[3] + row, *Th = s[4] + row;
    R Dxc = DI[0] * Th[N * Jn];
    R Dyc = DJ[0] * Th[I];
    R cu = DI[0] * uC[N * Jn] + DJ[0] * vC[I];
    R dv = DI[0] * uD[N * Jn] + DJ[0] * vD[I];
#pragma unroll
    for (int k = 1; k < N; ++k) {
      Dxc = rsum1(Dxc, DI[k], Th[k + N * Jn]);
      Dyc = rsum1(Dyc, DJ[k], Th[I + N * k]);
      cu = rsum2(cu, DI[k], uC[k + N * Jn], DJ[k], vC[I + N * k]);
      dv = rsum2(dv, DI[k], uD[k + N * Jn], DJ[k], vD[I + N * k]);
    }
    s[5][si] = CGD_DIVJ(cu);
    s[6][si] = CGD_DIVJ(dv);
    R GradDx = CGD_DIVJ(d11 * Dxc + d21 * Dyc);   // Grad12 with J
    R GradDy = CGD_DIVJ(d12 * Dxc + d22 * Dyc);
    s[7][si] = d11 * GradDx + d12 * GradDy;         // Contra12
    s[8][si] = d21 * GradDx + d22 * GradDy;
#pragma unroll
    for (int q = 0; q < NT; ++q) {
      const R *Tr = s[9 + 3 * q] + row;
      R Dxt = DI[0] * Tr[N * Jn];
      R Dyt = DJ[0] * Tr[I];
#pragma unroll
      for (int k = 1; k < N; ++k) {
        Dxt = rsum1(Dxt, DI[k], Tr[k + N * Jn]);
        Dyt = rsum1(Dyt, DJ[k], Tr[I + N * k]);
      }
      R GDx = CGD_DIVJ(d11 * Dxt + d21 * Dyt);
      R GDy = CGD_DIVJ(d12 * Dxt + d22 * Dyt);
      s[10 + 3 * q][si] = d11 * GDx + d12 * GDy;
      s[11 + 3 * q][si] = d21 * GDx + d22 * GDy;
    }
  }
  __syncthreads();
  using CT = typename std::conditional<MIX, float, double>::type;   // stored contributions
  CT *out = reinterpret_cast<CT *>(C) + ((size_t)IF * P.NC * DoF + ID) * nz + l;
  R WI[N], WJ[N];
#pragma unroll
  for (int k = 0; k < N; ++k) {
    WI[k] = (R)P.DW[I + N * k];
    WJ[k] = (R)P.DW[Jn + N * k];
  }
  if (act) {
    const R *Cu = s[5] + row, *Dv = s[6] + row, *Cx = s[7] + row, *Cy = s[8] + row;
    R DxCurl = WI[0] * Cu[N * Jn], DyCurl = WJ[0] * Cu[I];
    R DxDiv = WI[0] * Dv[N * Jn], DyDiv = WJ[0] * Dv[I];
    R DivTh = WI[0] * Cx[N * Jn] + WJ[0] * Cy[I];
#pragma unroll
    for (int k = 1; k < N; ++k) {
      DxCurl = rsum1(DxCurl, WI[k], Cu[k + N * Jn]);
      DyCurl = rsum1(DyCurl, WJ[k], Cu[I + N * k]);
      DxDiv = rsum1(DxDiv, WI[k], Dv[k + N * Jn]);
      DyDiv = rsum1(DyDiv, WJ[k], Dv[I + N * k]);
      DivTh = rsum2(DivTh, WI[k], Cx[k + N * Jn], WJ[k], Cy[I + N * k]);
    }
    R FuC = d12 * DxCurl + d22 * DyCurl;       // Rot12
    R FvC = -d11 * DxCurl - d21 * DyCurl;
    R FuD = d11 * DxDiv + d21 * DyDiv;         // Grad12
    R FvD = d12 * DxDiv + d22 * DyDiv;
    out[0 * cs] = (CT)CGD_DIVM(-FuC);
    out[1 * cs] = (CT)CGD_DIVM(-FvC);
    out[2 * cs] = (CT)CGD_DIVM(FuD);
    out[3 * cs] = (CT)CGD_DIVM(FvD);
    out[4 * cs] = (CT)CGD_DIVM(DivTh);
#pragma unroll
    for (int q = 0; q < NT; ++q) {
      const R *Tx = s[10 + 3 * q] + row, *Ty = s[11 + 3 * q] + row;
      R DivTr = WI[0] * Tx[N * Jn] + WJ[0] * Ty[I];
#pragma unroll
      for (int k = 1; k < N; ++k) DivTr = rsum2(DivTr, WI[k], Tx[k + N * Jn], WJ[k], Ty[I + N * k]);
      out[(5 + q) * cs] = (CT)CGD_DIVM(DivTr);
    }
  }
}

// Shared arrays: HV1Smem<N, NT, R, HV1Tile<N, R>::LT>::BYTES of dynamic shared memory.
template <int N, int NT, typename R>
__global__ void __launch_bounds__(HV1Tile<N, R>::THREADS, HV1Tile<N, R>::MINB)
    k_hypervisc1(const GP P, const double *__restrict__ U, double *__restrict__ C)
{
  extern __shared__ __align__(16) unsigned char hv1_dyn[];
  hypervisc1_body<N, NT, R, HV1Tile<N, R>::LT>(P, U, C, blockIdx.x, P.IF0 + blockIdx.y,
                                               reinterpret_cast<R *>(hv1_dyn));
}

// Contributions and the phase-1 cache: double, or float in the mixed form
// (C32, a compile-time choice of every kernel that reads or writes them).
template <bool C32>
__device__ __forceinline__ double cload(const double *C, long long i)
{
  return C32 ? (double)reinterpret_cast<const float *>(C)[i] : C[i];
}
template <bool C32>
__device__ __forceinline__ void cstore(double *C, long long i, double v)
{
  if (C32) reinterpret_cast<float *>(C)[i] = (float)v;
  else C[i] = v;
}

// Sum over the NQ contributors (element-node offsets o) of one global DOF at
// one level, for every field, each sum from 0.0 in ascending order.
// WSPLIT (the phase-2 tendency): a node's contribution to w at interface l is
// its upper part (slot 3, level l) plus its lower part (slot NV, stored at
// level l), zero at the top level.
template <int NQ, bool WSPLIT, bool C32>
__device__ __forceinline__ void gather_nq(const GP &P, const double *__restrict__ C, const long long *o, bool wtop,
                                          size_t fstr, double *acc)
{
  double wlo[NQ];
  if (WSPLIT) {
#pragma unroll
    for (int j = 0; j < NQ; ++j) wlo[j] = !wtop ? cload<C32>(C, o[j] + P.NV * fstr) : 0.0;
  }
#pragma unroll
  for (int f = 0; f < MAXNV; ++f) {
    if (f < P.NV) {
      double x[NQ];
#pragma unroll
      for (int j = 0; j < NQ; ++j) x[j] = !(WSPLIT && f == 3 && wtop) ? cload<C32>(C, o[j] + f * fstr) : 0.0;
      if (WSPLIT && f == 3) {
#pragma unroll
        for (int j = 0; j < NQ; ++j) x[j] = wtop ? 0.0 : x[j] + wlo[j];
      }
      double a = 0.0;
#pragma unroll
      for (int j = 0; j < NQ; ++j) a += x[j];
      acc[f] = a;
    }
  }
}

// Sum the contributions of the element nodes sharing global DOF g at level l
// (ascending element, node order) for every field.  Every cubed-sphere node
// has 1 to 4 contributors; each count has its own fully unrolled path (the
// count is uniform over a column, so over a warp of the column kernel), whose
// loads are all independent.
template <bool WSPLIT, bool C32>
__device__ __forceinline__ void gather_node(const GP &P, const double *__restrict__ C, int g, int l, size_t fstr,
                                            double *acc)
{
  // one 32-byte row of the table gives the count and the offsets, so the
  // contribution loads wait on a single index load
  const longlong2 *t = reinterpret_cast<const longlong2 *>(P.inv_tab) + 2 * (size_t)g;
  const longlong2 ta = t[0], tb = t[1];
  const bool wtop = WSPLIT && l == P.nz - 1;
  long long o[4] = {ta.x + l, ta.y + l, tb.x + l, tb.y + l};
  const int nq = ta.x < 0 ? 0 : 1 + (ta.y >= 0) + (tb.x >= 0) + (tb.y >= 0);
  switch (nq) {
    case 1:
      gather_nq<1, WSPLIT, C32>(P, C, o, wtop, fstr, acc);
      return;
    case 2:
      gather_nq<2, WSPLIT, C32>(P, C, o, wtop, fstr, acc);
      return;
    case 3:
      gather_nq<3, WSPLIT, C32>(P, C, o, wtop, fstr, acc);
      return;
    case 4:
      gather_nq<4, WSPLIT, C32>(P, C, o, wtop, fstr, acc);
      return;
    default:
      break;
  }
  const int q0 = P.inv_ptr[g], q1 = P.inv_ptr[g + 1];
#pragma unroll
  for (int f = 0; f < MAXNV; ++f) {
    if (f < P.NV) {
      double a = 0.0;
      for (int q = q0; q < q1; ++q) {
        const long long oq = P.inv_off[q] + l;
        double x = cload<C32>(C, oq + f * fstr);
        if (WSPLIT && f == 3) x = wtop ? 0.0 : x + cload<C32>(C, oq + P.NV * fstr);
        a += x;
      }
      acc[f] = a;
    }
  }
}

// ---------------------------------------------------------------------------
// Owner gather (DSS): out(l, g, f) = sum over contributors in ascending
// (element, node) order.  Thread per (g, l), level fastest.
// ---------------------------------------------------------------------------
// OUTC: the output is the phase-1 cache (stored like the contributions),
// otherwise an FP64 tendency.
template <bool WSPLIT, bool OUTC, bool C32>
__device__ __forceinline__ void gather_body(const GP &P, const double *__restrict__ C, double *__restrict__ out,
                                            const long long tid)
{
  const int nz = P.nz;
  if (tid >= (long long)nz * P.NumG) return;
  const int g = (int)(tid / nz), l = (int)(tid % nz);
  const size_t fstr = (size_t)P.DoF * nz;
  double acc[MAXNV];
  gather_node<WSPLIT, C32>(P, C, g, l, fstr, acc);
#pragma unroll
  for (int f = 0; f < MAXNV; ++f)
    if (f < P.NV) {
      const long long o = l + (long long)nz * (g + (long long)P.NumG * f);
      if (OUTC) cstore<C32>(out, o, acc[f]);
      else out[o] = acc[f];
    }
}

template <bool WSPLIT, bool OUTC, bool C32>
__global__ void __launch_bounds__(256) k_gather(const GP P, const double *__restrict__ C,
                                                double *__restrict__ out)
{
  gather_body<WSPLIT, OUTC, C32>(P, C, out, (long long)blockIdx.x * blockDim.x + threadIdx.x);
}

// ---------------------------------------------------------------------------
// Column part of a Rosenbrock-W stage, fused (one warp per column, lanes over
// levels): owner gather of the tendency, stage corrections
// fV = F + sum_j c_ij/dt k_j, the vertical acoustic Jacobian of the step's
// initial state (JacSchurKernel!, src/DyCore/JacSchur.jl:29-75), the Schur
// tridiagonal system (TriDiagKernel!, SchurSolveFKernel!, triSolve!,
// SchurSolveBKernel!: src/Integration/SchurSolve.jl:1-114) and the stage
// update of RosenbrockSchur! (src/Integration/RosenbrockSchur.jl:13-32).
// MODE 0: stage 1 -> k1, Vst = Vn + a21 k1; the Jacobian bands are formed
//         and kept (level fastest) for stages 2 and 3
// MODE 1: stage 2 -> k2, Vst = (Vn + a31 k1) + a32 k2
// MODE 2: stage 3 -> Vout = ((Vn + m1 k1) + m2 k2) + m3 k3   (Vout may alias Vn)
// MODE 3: standalone Schur solve with stored bands: k, v updated (cgd_schur_solve)
// Only rho, w and rho*theta enter the Schur system; every other field has
// k = fac * fV and is finished right after its gather.
// ---------------------------------------------------------------------------
struct ColArgs {
  const double *C;       // contributions of phase 2 (MODE 0..2)
  const double *Vn;      // step initial state (MODE 0..2)
  const double *k1, *k2;
  double *kout;          // MODE 0,1,3
  double *Vout;          // MODE 0,1 (stage state), 2 (new state)
  double *v;             // MODE 3: right-hand side (overwritten)
  // MODE 3: the four Jacobian bands JRhoW, JWRho, JWRhoTh, JRhoThW, each
  // (2, nz-1, NumG) in the reference layout (the JCache arrays)
  const double *jb4[4];
  double *jbg;           // MODE 0 writes, 1-2 read: [8][NumG][nz-1] bands of the step
  // MODE 0..2 with column physics: the stage state the tendency is of and its
  // pressure (Vs may be Vout: each lane reads its own levels before writing them)
  const double *Vs, *ps;
  double dt, fac;
  RK rk;
};

constexpr int COL_WARPS = 8;
// per warp: fv of rho, w, rho*theta, 8 bands, tri[3], x; each nz long.  (The
// step's initial rho, w, rho*theta were once copied into three more arrays
// by cp.async at the start for the update at the end; reading them at the
// update instead is faster: 0.426/0.449 -> 0.411/0.427 ms for the second and
// third stage on the drop-in grid, the smaller arrays leaving more L1.)
constexpr int COL_ARR = 15;
// CTAs per SM the column kernel's registers are sized for: five for the first
// stage (48 registers; 0.474 -> 0.464 ms on the drop-in grid), four for the
// others (64 registers; five cost them 4-20 %)
template <int MODE>
constexpr int col_min_blocks() { return MODE == 0 ? 5 : 4; }

// dPresdRhoTh (src/Models/Equation.jl:33-36) of one level
__device__ __forceinline__ double dpdrhoth(const GP &P, double RhoTh0)
{
  const double RhoTh = RhoTh0 + 0.0;
  return P.Rd * cgd_pow(P.Rd * RhoTh / P.p0, P.kappa / (1.0 - P.kappa));
}

__device__ __forceinline__ void jac_bands(const GP &P, double RhoL, double RhoR, double RhoThL0, double RhoThR0,
                                          double dPdThL, double dPdThR, double dzL, double dzR, double *jb)
{
  // JacSchurKernel! (src/DyCore/JacSchur.jl:40-73); AuxG[:,:,4] == 0 for Dry
  double RhoThL = RhoThL0 + 0.0, RhoThR = RhoThR0 + 0.0;
  double RhoF = (RhoL * dzL + RhoR * dzR) / (dzL + dzR);
  jb[0] = -RhoF / dzL;             // JRhoW[1]
  jb[1] = RhoF / dzR;              // JRhoW[2]
  jb[4] = -dPdThR / RhoF / (0.5 * (dzL + dzR));   // JWRhoTh[1]
  jb[5] = dPdThL / RhoF / (0.5 * (dzL + dzR));    // JWRhoTh[2]
  jb[2] = -P.Grav * dzR / RhoF / (dzL + dzR);     // JWRho[1]
  jb[3] = -P.Grav * dzL / RhoF / (dzL + dzR);     // JWRho[2]
  double RhoThF = (RhoThL * dzL + RhoThR * dzR) / (dzL + dzR);
  jb[6] = -RhoThF / dzL;           // JRhoThW[1]
  jb[7] = RhoThF / dzR;            // JRhoThW[2]
}

__device__ __forceinline__ void jac_at(const GP &P, double RhoL, double RhoR, double RhoThL0, double RhoThR0,
                                       double dzL, double dzR, double *jb)
{
  jac_bands(P, RhoL, RhoR, RhoThL0, RhoThR0, dpdrhoth(P, RhoThL0), dpdrhoth(P, RhoThR0), dzL, dzR, jb);
}

// Solve M x = b for one column with the warp's 32 lanes (the fast build's
// triSolve!).  M(i,i) = t1(i), M(i+1,i) = t2(i), M(i,i+1) = t0(i+1), n <= 64
// rows; lane L holds rows 2L and 2L+1.  The Thomas recurrences become scans:
//   pivots d(i) = t1(i) - t2(i-1) t0(i) / d(i-1) = p(i)/q(i), (p, q) the first
//     column of the product M_i ... M_0 with M_i = [[t1(i), -t2(i-1) t0(i)], [1, 0]]
//     (products rescaled by powers of two, which is exact);
//   forward b'(i) = b(i) - t2(i-1)/d(i-1) b'(i-1), an affine prefix scan;
//   back x(i) = (b'(i) - t0(i+1) x(i+1)) / d(i), an affine suffix scan.
struct Mat2 {
  double a, b, c, d;
};
__device__ __forceinline__ Mat2 mat2_mul(const Mat2 &x, const Mat2 &y)
{
  return {x.a * y.a + x.b * y.c, x.a * y.b + x.b * y.d, x.c * y.a + x.d * y.c, x.c * y.b + x.d * y.d};
}
// m scaled by 2^-e, e the binary exponent of its largest entry (largest |entry|
// = f 2^e, 0.5 <= f < 1).  When that entry is a normal number whose 2^-e is
// normal too (biased exponent 1 .. 2044), the scaling is one multiply by 2^-e,
// assembled from the exponent bits: a multiply by an exact power of two is
// the single correctly rounded x 2^-e, so it equals ldexp(x, -e) bit for bit.
// Other magnitudes (zero, subnormal, near overflow, not finite) take
// frexp/ldexp.
__device__ __forceinline__ Mat2 mat2_scaled(Mat2 m)
{
  const double mx = fmax(fmax(fabs(m.a), fabs(m.b)), fmax(fabs(m.c), fabs(m.d)));
  const int be = (int)((unsigned long long)__double_as_longlong(mx) >> 52);   // mx >= 0: no sign bit
  if (be >= 1 && be <= 2044) {
    // e = be - 1022; 2^-e has the biased exponent 1023 - e = 2045 - be
    const double sc = __longlong_as_double((long long)(2045 - be) << 52);
    m.a *= sc; m.b *= sc; m.c *= sc; m.d *= sc;
  } else if (mx > 0.0) {
    int e;
    frexp(mx, &e);
    m.a = ldexp(m.a, -e); m.b = ldexp(m.b, -e); m.c = ldexp(m.c, -e); m.d = ldexp(m.d, -e);
  }
  return m;
}
__device__ __forceinline__ Mat2 mat2_shfl_up(const Mat2 &m, int k)
{
  return {__shfl_up_sync(0xffffffffu, m.a, k), __shfl_up_sync(0xffffffffu, m.b, k),
          __shfl_up_sync(0xffffffffu, m.c, k), __shfl_up_sync(0xffffffffu, m.d, k)};
}
__device__ __forceinline__ void warp_tri_solve(const double *t0, const double *t1, const double *t2,
                                               const double *b, double *x, int n, int lane)
{
  constexpr unsigned FULL = 0xffffffffu;
  const Mat2 I2 = {1.0, 0.0, 0.0, 1.0};
  const int i0 = 2 * lane, i1 = i0 + 1;
  auto mi = [&](int i) -> Mat2 {
    if (i >= n) return I2;
    return {t1[i], i > 0 ? -t2[i - 1] * t0[i] : 0.0, 1.0, 0.0};
  };
  const Mat2 A0 = mi(i0), A1 = mi(i1);
  // pivots
  Mat2 S = mat2_scaled(mat2_mul(A1, A0));
#pragma unroll
  for (int k = 1; k < 32; k <<= 1) {
    Mat2 Sp = mat2_shfl_up(S, k);
    if (lane < k) Sp = I2;
    S = mat2_scaled(mat2_mul(S, Sp));
  }
  Mat2 E = mat2_shfl_up(S, 1);
  if (lane == 0) E = I2;
  const Mat2 P0 = mat2_scaled(mat2_mul(A0, E));
  const Mat2 P1 = mat2_scaled(mat2_mul(A1, P0));
  const double r0 = i0 < n ? P0.c / P0.a : 0.0;   // 1 / d(i0)
  const double r1 = i1 < n ? P1.c / P1.a : 0.0;   // 1 / d(i1)
  // forward substitution
  const double rprev = __shfl_up_sync(FULL, r1, 1);   // 1 / d(i0 - 1)
  const double a0 = i0 < n ? (i0 > 0 ? -t2[i0 - 1] * rprev : 0.0) : 1.0;
  const double a1 = i1 < n ? -t2[i0] * r0 : 1.0;
  const double c0 = i0 < n ? b[i0] : 0.0, c1 = i1 < n ? b[i1] : 0.0;
  double CA = a1 * a0, CB = a1 * c0 + c1;
#pragma unroll
  for (int k = 1; k < 32; k <<= 1) {
    double pA = __shfl_up_sync(FULL, CA, k), pB = __shfl_up_sync(FULL, CB, k);
    if (lane < k) { pA = 1.0; pB = 0.0; }
    CB = CA * pB + CB;
    CA = CA * pA;
  }
  double yprev = __shfl_up_sync(FULL, CB, 1);
  if (lane == 0) yprev = 0.0;
  const double bp0 = a0 * yprev + c0, bp1 = a1 * bp0 + c1;
  // back substitution
  const double al0 = i0 + 1 < n ? -t0[i0 + 1] * r0 : 0.0, be0 = bp0 * r0;
  const double al1 = i1 + 1 < n ? -t0[i1 + 1] * r1 : 0.0, be1 = bp1 * r1;
  CA = al0 * al1;
  CB = al0 * be1 + be0;
#pragma unroll
  for (int k = 1; k < 32; k <<= 1) {
    double nA = __shfl_down_sync(FULL, CA, k), nB = __shfl_down_sync(FULL, CB, k);
    if (lane + k >= 32) { nA = 1.0; nB = 0.0; }
    CB = CA * nB + CB;
    CA = CA * nA;
  }
  double xnext = __shfl_down_sync(FULL, CB, 1);
  if (lane == 31) xnext = 0.0;
  const double x1v = al1 * xnext + be1, x0v = al0 * x1v + be0;
  if (i0 < n) x[i0] = x0v;
  if (i1 < n) x[i1] = x1v;
}

template <int MODE, bool C32>
__device__ __forceinline__ void column_body(const GP &P, const ColArgs &A, const int bx)
{
  extern __shared__ double csm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g0 = bx * COL_WARPS;
  const int g = g0 + warp;
  const int nz = P.nz, n = nz - 1, NV = P.NV, NumG = P.NumG;
  const bool valid = g < NumG;   // no early return: the block synchronises below
  const int LS = nz;                    // per-warp arrays of nz entries
  double *sw = csm + (size_t)warp * COL_ARR * LS;
  double *fv = sw;                      // [3][nz]: rho, w, rho*theta
  double *jb = sw + 3 * LS;             // [8][nz]
  double *tri = jb + 8 * LS;            // [3][nz]
  double *xs = tri + 3 * LS;            // [nz]
  const size_t fs = (size_t)nz * NumG;
  const double fac = A.fac;
  // k1, k2 of the Schur fields (rho, w, rho*theta), kept for the update
  double s1[2][3], s2[2][3];

  // stages 2 and 3: the stored bands of the step are copied into the warp's
  // band rows first, so that they are in flight with the gather's loads
  if ((MODE == 1 || MODE == 2) && valid) {
    const size_t js = (size_t)NumG * n;
#pragma unroll
    for (int it = 0; it < 2; ++it) {
      const int l = lane + 32 * it;
      if (l >= n) continue;
      const double *jg = A.jbg + (size_t)g * n + l;
#pragma unroll
      for (int r = 0; r < 8; ++r) cp_async8(jb + r * LS + l, jg + r * js);
    }
  }

  // 1. tendency (owner gather) + stage corrections; fields outside the Schur
  //    system finished here; bands
#pragma unroll
  for (int it = 0; it < 2; ++it) {
    const int l = lane + 32 * it;
    if (!valid || l >= nz) continue;
    const size_t o0 = l + (size_t)nz * g;
    if (MODE <= 2) {
      const size_t fstr = (size_t)P.DoF * nz;
      double gacc[MAXNV];
      gather_node<true, C32>(P, A.C, g, l, fstr, gacc);
      if (P.held_suarez || P.damping) {   // the tendency tail, at the stage state
        const double *vs = A.Vs + o0;
        physics_terms(P, l, g, vs[0], vs[fs], vs[2 * fs], vs[3 * fs], vs[4 * fs], A.ps[o0], gacc);
      }
#pragma unroll
      for (int f = 0; f < MAXNV; ++f) {
        if (f >= NV) break;
        const size_t o = o0 + f * fs;
        double x = gacc[f];
        double x1 = 0.0, x2 = 0.0;
        if (MODE >= 1) {
          x1 = A.k1[o];
          x = x + A.rk.c[MODE][0] / A.dt * x1;
        }
        if (MODE >= 2) {
          x2 = A.k2[o];
          x = x + A.rk.c[MODE][1] / A.dt * x2;
        }
        if (f == 0 || f == 3 || f == 4) {
          const int sf = f == 0 ? 0 : f - 2;   // 0, 1, 2
          fv[sf * LS + l] = x;
          s1[it][sf] = x1;
          s2[it][sf] = x2;
        } else {
          const double k = fac * x;
          const double vn = A.Vn[o];
          if (MODE == 0) {
            A.kout[o] = k;
            A.Vout[o] = vn + A.rk.a[1][0] * k;
          } else if (MODE == 1) {
            A.kout[o] = k;
            A.Vout[o] = vn + A.rk.a[2][0] * x1 + A.rk.a[2][1] * k;
          } else {
            A.Vout[o] = vn + A.rk.m[0] * x1 + A.rk.m[1] * x2 + A.rk.m[2] * k;
          }
        }
      }
      if (MODE == 0) {
        // dPresdRhoTh once per level, shared with the interface below
        xs[l] = dpdrhoth(P, A.Vn[o0 + 4 * fs]);
      }
    } else {
      fv[l] = A.v[o0];
      fv[LS + l] = A.v[o0 + 3 * fs];
      fv[2 * LS + l] = A.v[o0 + 4 * fs];
      for (int f = 1; f < NV; ++f)
        if (f != 3 && f != 4) A.kout[o0 + f * fs] = fac * A.v[o0 + f * fs];
      if (l < n) {
        for (int arr = 0; arr < 4; ++arr)
          for (int r = 0; r < 2; ++r) jb[(2 * arr + r) * LS + l] = A.jb4[arr][r + 2 * (l + (size_t)n * g)];
      }
    }
  }
  if (MODE == 1 || MODE == 2) cp_async_wait_all();   // this lane's band copies; the warp sync below publishes them
  if (MODE == 0) {
    __syncwarp();
#pragma unroll
    for (int it = 0; it < 2; ++it) {
      const int l = lane + 32 * it;
      if (!valid || l >= n) continue;
      double *jg = A.jbg + (size_t)g * n + l;
      const size_t js = (size_t)NumG * n;
      if (MODE == 0) {
        double b[8];
        const double *V0 = A.Vn + (size_t)nz * g;
        jac_bands(P, V0[l], V0[l + 1], V0[l + 4 * fs], V0[l + 1 + 4 * fs], xs[l], xs[l + 1],
                  P.dz[l + (size_t)nz * g], P.dz[l + 1 + (size_t)nz * g], b);
#pragma unroll
        for (int r = 0; r < 8; ++r) {
          jb[r * LS + l] = b[r];
          jg[r * js] = b[r];
        }
      }
    }
  }
  __syncwarp();
  // jb rows: 0,1 JRhoW ; 2,3 JWRho ; 4,5 JWRhoTh ; 6,7 JRhoThW  (row r = Julia index r%2+1)
#define JB(arr, r, i) jb[((arr) * 2 + (r)) * LS + (i)]
#define FV0(i) fv[(i)]
#define FV3(i) fv[LS + (i)]
#define FV4(i) fv[2 * LS + (i)]
  const double invfac = 1.0 / fac;
  const double invfac2 = invfac / fac;
  double v3new[2] = {0.0, 0.0};
#pragma unroll
  for (int it = 0; it < 2; ++it) {
    const int l = lane + 32 * it;
    if (valid && l < n) {   // TriDiagKernel!
      double t0, t1, t2;
      t1 = invfac2 - JB(1, 1, l) * JB(0, 0, l) - JB(1, 0, l) * JB(0, 1, l) -
           JB(2, 1, l) * JB(3, 0, l) - JB(2, 0, l) * JB(3, 1, l);
      if (l == 0) t0 = 0.0;
      else t0 = -JB(1, 0, l - 1) * JB(0, 0, l) - JB(2, 0, l - 1) * JB(3, 0, l);
      if (l == n - 1) t2 = 0.0;
      else t2 = -JB(1, 1, l + 1) * JB(0, 1, l) - JB(2, 1, l + 1) * JB(3, 1, l);
      tri[l] = t0; tri[LS + l] = t1; tri[2 * LS + l] = t2;
      // SchurSolveFKernel!
      v3new[it] = FV3(l) / fac + JB(1, 1, l) * FV0(l) + JB(1, 0, l) * FV0(l + 1) +
                  JB(2, 1, l) * FV4(l) + JB(2, 0, l) * FV4(l + 1);
    }
  }
  __syncwarp();
#pragma unroll
  for (int it = 0; it < 2; ++it)
    if (valid && lane + 32 * it < n) FV3(lane + 32 * it) = v3new[it];
#ifdef CGD_FAST
  // triSolve! as three warp scans over the column's levels (fast build);
  // the result differs from the sequential sweep by rounding only
  __syncwarp();
  if (!valid) return;   // warp-uniform; nothing below synchronises the block
  warp_tri_solve(tri, tri + LS, tri + 2 * LS, fv + LS, xs, n, lane);
  __syncwarp();
#else
  __syncthreads();
  // triSolve! (Thomas), b = FV3, x = xs: the serial sweeps of the block's
  // columns run concurrently, one per lane of the first warp
  if (threadIdx.x < COL_WARPS && g0 + (int)threadIdx.x < NumG) {
    double *sc = csm + (size_t)threadIdx.x * COL_ARR * LS;
    double *b = sc + LS;
    const double *tr = sc + 11 * LS;
    double *x = sc + 14 * LS;
    x[0] = tr[LS + 0];
    for (int i = 0; i < n - 1; ++i) {
      const double m = tr[2 * LS + i] / x[i];   // the reference's tri[3,i]/x[i], used twice
      x[i + 1] = tr[LS + i + 1] - m * tr[i + 1];
      b[i + 1] = b[i + 1] - m * b[i];
    }
    x[n - 1] = b[n - 1] / x[n - 1];
    for (int i = n - 2; i >= 0; --i) x[i] = (b[i] - tr[i + 1] * x[i + 1]) / x[i];
  }
  __syncthreads();
#endif
  if (!valid) return;
  // SchurSolveBKernel! and the stage update of rho, w, rho*theta; each lane
  // owns levels lane and lane + 32
#pragma unroll
  for (int it = 0; it < 2; ++it) {
    const int l = lane + 32 * it;
    if (l >= nz) continue;
    const double kw = l < n ? xs[l] : 0.0;
    double v0 = FV0(l), v4 = FV4(l);
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
    const size_t o0 = l + (size_t)nz * g;
    if (MODE == 3) {
      // v after SchurSolveF/B (the Thomas sweep works on a copy, as in
      // SchurSolveTriKernel!'s shared-memory vCol)
      A.v[o0] = v0;
      A.v[o0 + 4 * fs] = v4;
      if (l < n) A.v[o0 + 3 * fs] = it == 0 ? v3new[0] : v3new[1];
    }
    const double kk[3] = {fac * v0, kw, fac * v4};
#pragma unroll
    for (int sf = 0; sf < 3; ++sf) {
      const int f = sf == 0 ? 0 : sf + 2;
      const size_t o = o0 + f * fs;
      const double k = kk[sf];
      if (MODE == 0) {
        const double vn = A.Vn[o];
        A.kout[o] = k;
        A.Vout[o] = vn + A.rk.a[1][0] * k;
      } else if (MODE == 1) {
        const double vn = A.Vn[o];
        A.kout[o] = k;
        A.Vout[o] = vn + A.rk.a[2][0] * s1[it][sf] + A.rk.a[2][1] * k;
      } else if (MODE == 2) {
        // Vout may alias Vn: this lane alone reads index o and then writes it
        const double vn = A.Vn[o];
        A.Vout[o] = vn + A.rk.m[0] * s1[it][sf] + A.rk.m[1] * s2[it][sf] + A.rk.m[2] * k;
        if (A.kout) A.kout[o] = k;   // the last stage's k of rho, w, rho*theta (adjoint replay only)
      } else {
        A.kout[o] = k;
      }
    }
  }
#undef JB
#undef FV0
#undef FV3
#undef FV4
}

template <int MODE, bool C32>
__global__ void __launch_bounds__(32 * COL_WARPS, col_min_blocks<MODE>()) k_column(const GP P, const ColArgs A)
{
  column_body<MODE, C32>(P, A, blockIdx.x);
}

// The kernels below are defined by the forward translation unit only (the
// adjoint's, cgd_adjoint.cu, includes this header for its device functions).
#ifndef CGD_ADJOINT_TU
// Mixed form: the FP64 reference profile of pressure and theta, the
// horizontal mean of each level of a state (one CTA per level, fixed-order
// tree reduction, so the profile is reproducible).
__global__ void __launch_bounds__(256) k_refprof(const GP P, const double *__restrict__ U, double *__restrict__ pref,
                                                 double *__restrict__ thref)
{
  __shared__ double sp[256], st[256];
  const int l = blockIdx.x, nz = P.nz, NumG = P.NumG;
  const size_t fs = (size_t)nz * NumG;
  double a = 0.0, b = 0.0;
  for (int g = threadIdx.x; g < NumG; g += blockDim.x) {
    const double rho = U[l + (size_t)nz * g], rth = U[l + (size_t)nz * g + 4 * fs];
    a += pressure_dry(P, rth);
    b += rth / rho;
  }
  sp[threadIdx.x] = a;
  st[threadIdx.x] = b;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      sp[threadIdx.x] += sp[threadIdx.x + w];
      st[threadIdx.x] += st[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    pref[l] = sp[0] / NumG;
    thref[l] = st[0] / NumG;
  }
}

// The four band arrays of the reference's JCache (JRhoW, JWRho, JWRhoTh,
// JRhoThW), each (2, nz-1, NumG).
struct Bands4 {
  double *b[4];
};

// The column physics added to a tendency F of the state U with pressure p
// (cgd_rhs): one thread per column-level.
__global__ void __launch_bounds__(256) k_physics(const GP P, const double *__restrict__ U,
                                                 const double *__restrict__ p, double *__restrict__ F)
{
  const long long S = (long long)P.nz * P.NumG;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= S) return;
  const int g = (int)(t / P.nz), l = (int)(t - (long long)g * P.nz);
  double f[5] = {0.0, F[t + S], F[t + 2 * S], F[t + 3 * S], F[t + 4 * S]};
  physics_terms(P, l, g, U[t], U[t + S], U[t + 2 * S], U[t + 3 * S], U[t + 4 * S], p[t], f);
  F[t + S] = f[1];
  F[t + 2 * S] = f[2];
  F[t + 3 * S] = f[3];
  F[t + 4 * S] = f[4];
}

// Jacobian bands into memory (cgd_jac): one thread per (interface, column)
__global__ void k_jac(const GP P, const double *__restrict__ U, const Bands4 out)
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
  for (int arr = 0; arr < 4; ++arr)
    for (int r = 0; r < 2; ++r) out.b[arr][r + 2 * (l + (size_t)n * g)] = b[arr * 2 + r];
}

__device__ __forceinline__ void pressure_body(const GP &P, const double *__restrict__ U, double *__restrict__ p,
                                              const long long tid)
{
  const long long S = (long long)P.nz * P.NumG;
  if (tid >= S) return;
  p[tid] = pressure_dry(P, U[tid + 4 * S]);
}

__global__ void __launch_bounds__(256) k_pressure(const GP P, const double *__restrict__ U, double *__restrict__ p)
{
  pressure_body(P, U, p, (long long)blockIdx.x * blockDim.x + threadIdx.x);
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

#endif  // CGD_ADJOINT_TU

} // namespace cgd
