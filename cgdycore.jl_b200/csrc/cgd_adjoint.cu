// cgd_adjoint.cu - the adjoint kernels (cgd_adjoint.cuh) and their launchers.
//
// A translation unit of its own so that it can be compiled with multiply-add
// contraction: the adjoint is checked against finite differences (to 1e-6
// and 1e-7 relative), not bit for bit, and fused multiply-adds take out most
// of its separate FP64 multiplies and adds.  The forward kernels, whose
// results match the CPU restatement's rounding, stay in cgd_b200.cu, built
// without contraction.
#define CGD_ADJOINT_TU
#include "cgd_adjoint.cuh"
#include "cgd_adjoint_launch.h"

namespace cgd {

namespace {

template <int N>
cudaError_t rhs_adjoint_t(const GP &gp, const double *U, const double *T1, const double *pres, const double *LF,
                          double *LU, double *LT1, cudaStream_t stream)
{
  using CF = AdjCfg<N>;
  cudaError_t e = cudaFuncSetAttribute(k_phase2_adj<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CF::SMEM);
  if (e != cudaSuccess) return e;
  const dim3 grid((gp.nz + CF::LC - 1) / CF::LC, gp.NF);
  k_phase2_adj<N><<<grid, CF::THREADS, CF::SMEM, stream>>>(gp, U, pres, T1, LF, LU, LT1);
  using HT = AdjHV1Tile<N>;
  const dim3 grid1((gp.nz + HT::LT - 1) / HT::LT, gp.NF);
  k_hypervisc1_adj<N><<<grid1, HT::THREADS, 0, stream>>>(gp, U, LT1, LU);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_rhs_adjoint(const GP &gp, const double *U, const double *T1, const double *pres,
                               const double *LF, double *LU, double *LT1, cudaStream_t stream)
{
  switch (gp.N) {
    case 2: return rhs_adjoint_t<2>(gp, U, T1, pres, LF, LU, LT1, stream);
    case 3: return rhs_adjoint_t<3>(gp, U, T1, pres, LF, LU, LT1, stream);
    case 4: return rhs_adjoint_t<4>(gp, U, T1, pres, LF, LU, LT1, stream);
    default: return rhs_adjoint_t<5>(gp, U, T1, pres, LF, LU, LT1, stream);
  }
}

cudaError_t launch_column_adjoint(const GP &gp, const double *mu, double mus, const double *kx, const double *jbg,
                                  const double *Vn, double fac, double *AR, double *LV, cudaStream_t stream)
{
  cudaError_t e = cudaFuncSetAttribute(k_column_adj, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       COL_WARPS * CA_ARR * 64 * (int)sizeof(double));
  if (e != cudaSuccess) return e;
  const size_t smem = (size_t)COL_WARPS * CA_ARR * gp.nz * sizeof(double);
  k_column_adj<<<(gp.NumG + COL_WARPS - 1) / COL_WARPS, 32 * COL_WARPS, smem, stream>>>(gp, mu, mus, kx, jbg, Vn,
                                                                                        fac, AR, LV);
  return cudaGetLastError();
}

cudaError_t launch_adjoint_update(long long n, const double *L, const double *AR, const double *Lt, double *LV,
                                  double *Lk0, double *Lk1, double m0, double m1, double cA, double cB, double a0,
                                  double a1, cudaStream_t stream)
{
  const unsigned nb = (unsigned)((n + 255) / 256);
  k_adj_update<<<nb, 256, 0, stream>>>(n, L, AR, Lt, LV, Lk0, Lk1, m0, m1, cA, cB, a0, a1);
  return cudaGetLastError();
}

}  // namespace cgd
