// cgd_adjoint_launch.h - launchers of the adjoint kernels, defined in
// cgd_adjoint.cu (its own translation unit) and called by cgd_b200.cu.
#pragma once
#include <cuda_runtime.h>

namespace cgd {

struct GP;

// Reverse of the tendency on one state (no tracers, FP64): phase 2 into LU
// and LT1 (both zeroed by the caller), then phase 1 from LT1 into LU.
cudaError_t launch_rhs_adjoint(const GP &gp, const double *U, const double *T1, const double *pres,
                               const double *LF, double *LU, double *LT1, cudaStream_t stream);
// Reverse of one stage's column Schur solve.
cudaError_t launch_column_adjoint(const GP &gp, const double *mu, double mus, const double *kx, const double *jbg,
                                  const double *Vn, double fac, double *AR, double *LV, cudaStream_t stream);
// The stage-combination sweep of the step adjoint (k_adj_update).
cudaError_t launch_adjoint_update(long long n, const double *L, const double *AR, const double *Lt, double *LV,
                                  double *Lk0, double *Lk1, double m0, double m1, double cA, double cB, double a0,
                                  double a1, cudaStream_t stream);

}  // namespace cgd
