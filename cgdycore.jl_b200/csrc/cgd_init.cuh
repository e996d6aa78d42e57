// cgd_init.cuh - the grid set-up on the device: the metric of the cubed
// sphere (JacobiSphere3Kernel!), the lumped mass and dz (MassCGKernel!,
// GridSizeSphereKernel!), and the compaction of the reference-layout metric
// into the element metric the tendency kernels read.
//
// The host set-up (grid topology and the Glob numbering, integer work) stays
// on the host; the floating-point arrays of the grid, which grow with
// NF * N^2 * nz, are formed here in the reference's evaluation order.  The
// metric uses the device's sin/cos/asin/atan2, which may differ from the
// host's libm in the last bit, so it agrees with the host metric to rounding,
// not bit for bit; the mass, dz and the compaction are bit for bit the host
// code's on the same metric.
#pragma once
#include "cgd_kernels.cuh"

namespace cgd {

// X (N*N,2,3,nz,NF), dXdxI (3,3,2,N*N,nz,NF), J (N*N,2,nz,NF): one thread
// per element node, every level.  src/Grids/JacobiSphere3GPU.jl:102-215
// (shallow atmosphere) with the Sleve height at zero orography
// (src/Grids/Adapt.jl:19-31).  FP (NF,4,3) corner points, xw the GLL nodes,
// DS (N,N) column-major, z (nz+1) level heights.
template <int N>
__global__ void __launch_bounds__(256) k_metric_sphere(int nz, int NF, const double *__restrict__ FP,
                                                       const double *__restrict__ xw, const double *__restrict__ DS,
                                                       const double *__restrict__ z, double H, double rad,
                                                       double *__restrict__ X, double *__restrict__ dXdxI,
                                                       double *__restrict__ J)
{
  constexpr int DoF = N * N;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)NF * DoF) return;
  const int IF = (int)(t / DoF), ID = (int)(t - (long long)IF * DoF);
  const int I = ID % N, Jn = ID / N;
  const double one = 1.0;
  const double k1 = xw[I], k2 = xw[Jn];
  double F[4][3];
  for (int k = 0; k < 4; ++k)
    for (int c = 0; c < 3; ++c) F[k][c] = FP[((size_t)IF * 4 + k) * 3 + c];
  double Xc[3];
  for (int c = 0; c < 3; ++c)
    Xc[c] = 0.25 * (F[0][c] * (one - k1) * (one - k2) + F[1][c] * (one + k1) * (one - k2) +
                    F[2][c] * (one + k1) * (one + k2) + F[3][c] * (one - k1) * (one + k2));
  const double r = sqrt(Xc[0] * Xc[0] + Xc[1] * Xc[1] + Xc[2] * Xc[2]);
  const double f = rad / r;
  const double theta = asin(Xc[2] / r);
  double lam = atan2(Xc[1], Xc[0]);
  if (Xc[1] < 0.0) lam = lam + 2.0 * 3.141592653589793;
  const double sl = sin(lam), cl = cos(lam), st = sin(theta), ct = cos(theta);
  double A[3][3];
  A[0][0] = sl * sl * ct * ct + st * st;
  A[0][1] = -sl * cl * ct * ct;
  A[0][2] = -cl * st * ct;
  A[1][0] = A[0][1];
  A[1][1] = cl * cl * ct * ct + st * st;
  A[1][2] = -sl * st * ct;
  A[2][0] = -cl * st;
  A[2][1] = -sl * st;
  A[2][2] = ct;
  const double DD[2][3] = {{-sl, cl, 0.0}, {0.0, 0.0, 1.0}};
  double B[3][4];
  for (int cc = 0; cc < 3; ++cc)
    for (int k = 0; k < 4; ++k) B[cc][k] = F[k][cc];
  const double Cm[4][2] = {{-one + k2, -one + k1}, {one - k2, -one - k1}, {one + k2, one + k1}, {-one - k2, one - k1}};
  const double tt = 0.25 * f;
  // T4 = ((tt DD) A) B Cm, each product summed left to right from its first term
  double T1[2][3], T2[2][3], T3[2][4], T4[2][2];
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 3; ++j) T1[i][j] = tt * DD[i][j];
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 3; ++j) {
      double acc = T1[i][0] * A[0][j];
      for (int k = 1; k < 3; ++k) acc = acc + T1[i][k] * A[k][j];
      T2[i][j] = acc;
    }
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 4; ++j) {
      double acc = T2[i][0] * B[0][j];
      for (int k = 1; k < 3; ++k) acc = acc + T2[i][k] * B[k][j];
      T3[i][j] = acc;
    }
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 2; ++j) {
      double acc = T3[i][0] * Cm[0][j];
      for (int k = 1; k < 4; ++k) acc = acc + T3[i][k] * Cm[k][j];
      T4[i][j] = acc;
    }
  const double a11 = T4[0][0], a21 = T4[1][0], a12 = T4[0][1], a22 = T4[1][1], a13 = 0.0, a23 = 0.0;
  for (int Iz = 0; Iz < nz; ++Iz) {
    double hR[2];
    for (int K = 0; K < 2; ++K) {
      const double ks = K == 0 ? -1.0 : 1.0;
      const double zl = 0.5 * ((one - ks) * z[Iz] + (one + ks) * z[Iz + 1]);
      const double eta = zl / H;
      hR[K] = eta <= 0.7 ? eta * H + 0.0 : eta * H;
    }
    const double Dz = 0.5 * (hR[1] - hR[0]);
    for (int K = 0; K < 2; ++K) {
      const double h = hR[K];
      for (int c = 0; c < 3; ++c)
        X[ID + (size_t)DoF * (K + 2 * (c + 3 * (Iz + (size_t)nz * IF)))] = Xc[c] / r * (rad + h);
      double Dx = DS[I] * h, Dy = DS[Jn] * h;
      for (int k = 1; k < N; ++k) {
        Dx = Dx + DS[I + N * k] * h;
        Dy = Dy + DS[Jn + N * k] * h;
      }
      const double a31 = Dx, a32 = Dy, a33 = Dz;
      J[ID + (size_t)DoF * (K + 2 * (Iz + (size_t)nz * IF))] =
          a11 * (a22 * a33 - a23 * a32) - a12 * (a21 * a33 - a23 * a31) + a13 * (a21 * a32 - a22 * a31);
      double *d = dXdxI + 9 * (K + 2 * (ID + (size_t)DoF * (Iz + (size_t)nz * IF)));
      d[0 + 3 * 0] = a22 * a33 - a23 * a32;
      d[1 + 3 * 0] = -(a21 * a33 - a23 * a31);
      d[2 + 3 * 0] = a21 * a32 - a22 * a31;
      d[0 + 3 * 1] = -(a12 * a33 - a13 * a32);
      d[1 + 3 * 1] = a11 * a33 - a13 * a31;
      d[2 + 3 * 1] = -(a11 * a32 - a12 * a31);
      d[0 + 3 * 2] = a12 * a23 - a13 * a22;
      d[1 + 3 * 2] = -(a11 * a23 - a13 * a21);
      d[2 + 3 * 2] = a11 * a22 - a12 * a21;
    }
  }
}

// M (nz,NumG,2), MMass (nz,NumG) and dz (nz,NumG): one thread per (DOF,
// level), the contributors (inv_ptr/inv_idx: IF*DoF+ID ascending) summed in
// order from 0.0.  src/DyCore/MassCG.jl:61-75; dz from the highest
// contributing element node (the last to write it), as in
// GridSizeSphereKernel! (src/DyCore/DiscretizationCG.jl:119-144).
__global__ void __launch_bounds__(256) k_mass_dz(int N, int nz, int NumG, const int *__restrict__ inv_ptr,
                                                 const int *__restrict__ inv_idx, const double *__restrict__ w,
                                                 const double *__restrict__ J, const double *__restrict__ X,
                                                 double *__restrict__ M, double *__restrict__ MMass,
                                                 double *__restrict__ dz)
{
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nz * NumG) return;
  const int g = (int)(t / nz), l = (int)(t - (long long)g * nz);
  const int DoF = N * N;
  double m0 = 0.0, m1 = 0.0, mm = 0.0;
  int last = -1;
  for (int q = inv_ptr[g]; q < inv_ptr[g + 1]; ++q) {
    const int c = inv_idx[q], IF = c / DoF, ID = c - IF * DoF;
    const double J1 = J[ID + (size_t)DoF * (0 + 2 * (l + (size_t)nz * IF))];
    const double J2 = J[ID + (size_t)DoF * (1 + 2 * (l + (size_t)nz * IF))];
    m0 += J1;
    m1 += J2;
    mm += 0.5 * (J1 + J2) * w[ID % N] * w[ID / N];
    last = c;
  }
  const size_t o = l + (size_t)nz * g;
  M[o] = m0;
  M[o + (size_t)nz * NumG] = m1;
  MMass[o] = mm;
  const int IF = last / DoF, ID = last - IF * DoF;
  double rr[2];
  for (int K = 0; K < 2; ++K) {
    const double *x = X + ID + (size_t)DoF * (K + 2 * (3 * (l + (size_t)nz * IF)));
    const double x0 = x[0], x1 = x[2 * (size_t)DoF], x2 = x[4 * (size_t)DoF];
    rr[K] = sqrt(x0 * x0 + x1 * x1 + x2 * x2);
  }
  dz[o] = rr[1] - rr[0];
}

// The compact element metric [IF][comp][ID][nz] from the reference-layout
// arrays on the device: one thread per element-node-level, the expressions
// of the host path (Coriolis at the layer midpoint, the J-only RecU4
// coefficients of the interface above).
__global__ void __launch_bounds__(256) k_compact_metric(int DoF, int nz, int NF, double Omega2,
                                                        const double *__restrict__ dXdxI,
                                                        const double *__restrict__ J,
                                                        const double *__restrict__ X, double *__restrict__ met)
{
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)NF * DoF * nz) return;
  const int Iz = (int)(t % nz);
  const long long r = t / nz;
  const int ID = (int)(r % DoF), IF = (int)(r / DoF);
  auto dx = [&](int a, int b, int K) {
    return dXdxI[(size_t)(a - 1) + 3 * ((b - 1) + 3 * (K + 2 * (ID + (size_t)DoF * (Iz + (size_t)nz * IF))))];
  };
  auto jj = [&](int K, int lev) { return J[ID + (size_t)DoF * (K + 2 * (lev + (size_t)nz * IF))]; };
  auto xx = [&](int K, int c) { return X[ID + (size_t)DoF * (K + 2 * (c + 3 * (Iz + (size_t)nz * IF)))]; };
  double v[NCOMP];
  v[C_D11_0] = dx(1, 1, 0); v[C_D11_1] = dx(1, 1, 1);
  v[C_D12_0] = dx(1, 2, 0); v[C_D12_1] = dx(1, 2, 1);
  v[C_D21_0] = dx(2, 1, 0); v[C_D21_1] = dx(2, 1, 1);
  v[C_D22_0] = dx(2, 2, 0); v[C_D22_1] = dx(2, 2, 1);
  v[C_D31_0] = dx(3, 1, 0); v[C_D31_1] = dx(3, 1, 1);
  v[C_D32_0] = dx(3, 2, 0); v[C_D32_1] = dx(3, 2, 1);
  v[C_D33_0] = dx(3, 3, 0); v[C_D33_1] = dx(3, 3, 1);
  v[C_J0] = jj(0, Iz); v[C_J1] = jj(1, Iz);
  const double x = 0.5 * (xx(0, 0) + xx(1, 0));
  const double y = 0.5 * (xx(0, 1) + xx(1, 1));
  const double zc = 0.5 * (xx(0, 2) + xx(1, 2));
  const double sinlat = zc / sqrt(x * x + y * y + zc * zc);
  v[C_FCOR] = Omega2 * sinlat;
  v[C_RK0] = v[C_RK1] = v[C_RK2] = v[C_RK3] = 0.0;
  if (Iz < nz - 1) {
    auto js = [&](int lev) { return jj(0, lev) + jj(1, lev); };
    const double JLL = js(Iz > 0 ? Iz - 1 : 0), JL = js(Iz), JR = js(Iz + 1), JRR = js(Iz + 2 < nz ? Iz + 2 : nz - 1);
    v[C_RK0] = (JL / (JL + JR)) * ((JLL + JL) / (JLL + JL + JR));
    v[C_RK1] = (JL / (JLL + JL)) * (JR / (JLL + JL + JR));
    v[C_RK2] = (JR / (JR + JL)) * ((JRR + JR) / (JL + JR + JRR));
    v[C_RK3] = (JR / (JRR + JR)) * (JL / (JL + JR + JRR));
  }
  for (int c = 0; c < NCOMP; ++c) met[(((size_t)IF * NCOMP + c) * DoF + ID) * nz + Iz] = v[c];
}

}  // namespace cgd
