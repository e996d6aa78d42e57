// cgd_output.cuh - interpolation of the state to the output sub-cells.
//
// The reference writes its VTK output from OrdPrint x OrdPrint sub-cells per
// element and layer: each cell value is the element's GLL interpolant at the
// cell centre, Inter[I,J,iP,jP] = L_iP(xi_I) L_jP(eta_J)
// (src/Outputs/vtkSphere.jl:199-219), applied to the nodal values gathered
// through Glob (InterpolateKernel!, src/Outputs/vtkOutputKernel.jl:49-74).
// The kernels below evaluate the same sums in the same order:
//
//   k_interp      cCell = sum_(jP,iP) Inter * c            (InterpolateKernel!)
//                 cCell = sum_(jP,iP) Inter * c / rhoc     (InterpolateRhoKernel!, :97-121)
//                 of pressure or potential temperature     (the "Pres" and "Th" outputs)
//   k_interp_wb   layer-mean w, the surface w from no normal flow
//                                                          (InterpolateWBKernel!, :123-159)
//   k_interp_vort element-local vertical vorticity         (InterpolateRotKernel!, :1-47)
//
// The reference's vorticity kernel accumulates with atomics (unordered); here
// every sum runs in ascending node order: the curl at node (i,j) is
// sum_I D(i,I) tx(I,j) followed by sum_J D(j,J) ty(i,J), from 0.
// Inter is Fortran-ordered (OrdPrint, OrdPrint, N, N); cCell is
// (OrdPrint, OrdPrint, nz, NF).  Thread order: level fastest, so the gathered
// state columns are read contiguously.
#pragma once
#include "cgd_kernels.cuh"

namespace cgd {

constexpr int OUT_MAX_PRINT = 8;   // OrdPrint <= 8

// The nodal value the interpolation reads at state offset o: c itself
// (INTERP_C, divided by rhoc as in InterpolateRhoKernel! when rhoc is not
// null), or, with c = rho*theta and rhoc = rho, the pressure (INTERP_PRES)
// or the potential temperature (INTERP_POTT) of the dry model's Pressure
// (src/Models/Equation.jl:24-32, evaluated by PressureKernel! into
// Cache.AuxG[:,:,1] and [:,:,3]).
enum { INTERP_C = 0, INTERP_PRES = 1, INTERP_POTT = 2 };

__device__ __forceinline__ double pott_dry(const GP &P, double rho, double rhoth)
{
  const double p = pressure_dry(P, rhoth);
  const double T = p / (P.Rd * rho);
  return pow(P.p0 / p, P.kappa) * T;   // (p0/p)^(Rd/Cpd) * T
}

__global__ void __launch_bounds__(256) k_interp(const GP P, const double *__restrict__ c,
                                                const double *__restrict__ rhoc, int kind,
                                                const double *__restrict__ inter, int OP, double *__restrict__ cell)
{
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int nz = P.nz, N = P.N, OP2 = OP * OP;
  if (t >= (long long)nz * OP2 * P.NF) return;
  const int Iz = (int)(t % nz);
  const long long r = t / nz;
  const int cI = (int)(r % OP2), IF = (int)(r / OP2);
  const int *gl = P.glob + (size_t)IF * P.DoF;
  double acc = 0.0;
  for (int jP = 0; jP < N; ++jP)
    for (int iP = 0; iP < N; ++iP) {
      const int iD = iP + N * jP;
      const size_t o = Iz + (size_t)nz * gl[iD];
      const double w = inter[cI + (size_t)OP2 * iD];
      if (kind == INTERP_PRES) acc += w * pressure_dry(P, c[o]);
      else if (kind == INTERP_POTT) acc += w * pott_dry(P, rhoc[o], c[o]);
      else if (rhoc) acc += w * c[o] / rhoc[o];
      else acc += w * c[o];
    }
  const int I = cI % OP, J = cI / OP;
  cell[I + (size_t)OP * (J + (size_t)OP * (Iz + (size_t)nz * IF))] = acc;
}

// Layer-mean vertical velocity: 0.5 (w(Iz) + w(Iz-1)) per node, and in the
// lowest layer 0.5 (w(1) + w0) with w0 = -(u d31 + v d32) / d33 of the lower
// node (no normal flow through the surface).
__global__ void __launch_bounds__(256) k_interp_wb(const GP P, const double *__restrict__ u,
                                                   const double *__restrict__ v, const double *__restrict__ w,
                                                   const double *__restrict__ inter, int OP,
                                                   double *__restrict__ cell)
{
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int nz = P.nz, N = P.N, DoF = P.DoF, OP2 = OP * OP;
  if (t >= (long long)nz * OP2 * P.NF) return;
  const int Iz = (int)(t % nz);
  const long long r = t / nz;
  const int cI = (int)(r % OP2), IF = (int)(r / OP2);
  const int *gl = P.glob + (size_t)IF * DoF;
  const size_t cs = (size_t)DoF * nz;
  double acc = 0.0;
  for (int jP = 0; jP < N; ++jP)
    for (int iP = 0; iP < N; ++iP) {
      const int iD = iP + N * jP;
      const size_t o = Iz + (size_t)nz * gl[iD];
      const double wi = 0.5 * inter[cI + (size_t)OP2 * iD];
      double wb;
      if (Iz == 0) {
        const double *mt = P.met + ((size_t)IF * NCOMP * DoF + iD) * nz;   // level 0
        const double w0 = -(u[o] * mt[C_D31_0 * cs] + v[o] * mt[C_D32_0 * cs]) / mt[C_D33_0 * cs];
        wb = w[o] + w0;
      } else {
        wb = w[o] + w[o - 1];
      }
      acc += wi * wb;
    }
  const int I = cI % OP, J = cI / OP;
  cell[I + (size_t)OP * (J + (size_t)OP * (Iz + (size_t)nz * IF))] = acc;
}

// Vertical vorticity of (u, v) per element (no direct-stiffness summation):
// tx = D11 v - D12 u, ty = D21 v - D22 u at every node, the curl
// D_xi tx + D_eta ty, divided by J, interpolated to the cells.
// One CTA per (element, tile of LT levels); threads (node, level).
template <int N>
__global__ void __launch_bounds__(256) k_interp_vort(const GP P, const double *__restrict__ U,
                                                     const double *__restrict__ inter, int OP,
                                                     double *__restrict__ cell)
{
  constexpr int DoF = N * N, LT = 256 / DoF;
  __shared__ double tx[LT][DoF], ty[LT][DoF], rot[LT][DoF];
  const int nz = P.nz, NumG = P.NumG, OP2 = OP * OP;
  const int IF = blockIdx.y, l0 = blockIdx.x * LT;
  const int iz = threadIdx.x / DoF, ID = threadIdx.x % DoF;
  const int Iz = l0 + iz;
  const bool act = iz < LT && Iz < nz;
  const size_t cs = (size_t)DoF * nz;
  const double *mt = P.met + ((size_t)IF * NCOMP * DoF + ID) * nz + Iz;
  if (act) {
    const size_t o = Iz + (size_t)nz * P.glob[(size_t)IF * DoF + ID];
    const double u = U[o + (size_t)nz * NumG], v = U[o + 2 * (size_t)nz * NumG];
    tx[iz][ID] = (mt[C_D11_0 * cs] + mt[C_D11_1 * cs]) * v - (mt[C_D12_0 * cs] + mt[C_D12_1 * cs]) * u;
    ty[iz][ID] = (mt[C_D21_0 * cs] + mt[C_D21_1 * cs]) * v - (mt[C_D22_0 * cs] + mt[C_D22_1 * cs]) * u;
  }
  __syncthreads();
  if (act) {
    const int i = ID % N, j = ID / N;
    double acc = 0.0;
#pragma unroll
    for (int I = 0; I < N; ++I) acc += P.D[i + N * I] * tx[iz][I + N * j];
#pragma unroll
    for (int J = 0; J < N; ++J) acc += P.D[j + N * J] * ty[iz][i + N * J];
    rot[iz][ID] = acc / (mt[C_J0 * cs] + mt[C_J1 * cs]);
  }
  __syncthreads();
  for (int s = threadIdx.x; s < LT * OP2; s += blockDim.x) {
    const int lz = s / OP2, cI = s % OP2;
    const int Lz = l0 + lz;
    if (Lz >= nz) continue;
    double acc = 0.0;
    for (int iD = 0; iD < DoF; ++iD) acc += inter[cI + (size_t)OP2 * iD] * rot[lz][iD];
    const int I = cI % OP, J = cI / OP;
    cell[I + (size_t)OP * (J + (size_t)OP * (Lz + (size_t)nz * IF))] = acc;
  }
}

}  // namespace cgd
