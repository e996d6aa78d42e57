// cgd_mixed.cuh - mixed-precision form (FP32 perturbations around an FP64
// hydrostatic reference state).
#pragma once
#include "cgd_kernels.cuh"

namespace cgd {

struct MixedState;

inline int mixed_create(MixedState *&m, const GP &, cudaStream_t, const double *, const double *)
{
  m = nullptr;
  return CGD_ERR_UNSUPPORTED;
}
inline void mixed_destroy(MixedState *) {}
inline int mixed_rhs(MixedState *, const GP &, const double *, double *, double *, double *) { return 1; }
inline int mixed_ros_step(MixedState *, const GP &, double *, double, int, double *) { return CGD_ERR_UNSUPPORTED; }

}  // namespace cgd
