// cgd_adjoint.cuh - hand-written adjoint (reverse mode) of the FP64 tendency
// F(U) (FcnGPU!, src/GPU/FcnGPU.jl:552-968) without tracers.
//
// Given lambda_F (nz, NumG, 5) the kernels accumulate lambda_U = (dF/dU)^T
// lambda_F.  The tendency is F = DSS2(phase2(U, T1)) with T1 = DSS1(phase1(U)):
//
//   * the adjoint of a DSS (owner gather, F_g = sum of the contributions of
//     the element nodes sharing g) is a broadcast: every contribution's
//     adjoint is lambda at its global DOF;
//   * k_phase2_adj recomputes the forward quantities of one (element, chunk
//     of levels) and runs phase 2 in reverse, one warp per level; the
//     horizontal D/DW sums are transposed through the per-warp scratch;
//   * k_hypervisc1_adj does the same for phase 1, given lambda_T1.
//
// Contributions to lambda_U and lambda_T1 are accumulated with FP64 atomics
// (several elements and neighbouring levels feed the same entry), so the
// adjoint is not bit-reproducible; it is checked against finite differences
// of the forward path.
#pragma once
#include "cgd_phase2.cuh"

namespace cgd {

// phi = max(0, min(r, min(k r + c, 1))) with the branches of cgd_min/cgd_max,
// and its derivative in r
__device__ __forceinline__ double lim_phi(double r, double k, double c, double &dphi)
{
  const double lin = k * r + c;
  double m2 = lin, dm2 = k;
  if (1.0 < lin) { m2 = 1.0; dm2 = 0.0; }
  double m1 = r, dm1 = 1.0;
  if (m2 < r) { m1 = m2; dm1 = dm2; }
  if (m1 > 0.0) { dphi = dm1; return m1; }
  dphi = 0.0;
  return 0.0;
}

// Reverse of the limited upwind flux (RecU4, OperatorKernel.jl:1044-1059) of
// one interface: F = 0.25 ((|w| + w) cFL + (-|w| + w) cFR).  Given aF, the
// adjoint of F, returns the adjoints of w and of the four stencil values.
__device__ __forceinline__ void upwind_adj(double cLL, double cL, double cR, double cRR, double kR1, double kL1,
                                           double kL2, double kR2, double w, double aF, double &aw, double &aLL,
                                           double &aL, double &aR, double &aRR)
{
  const double den1 = cR - cL + 1.e-20, num1 = cL - cLL, r1 = num1 / den1;
  double dphi1;
  const double phi1 = lim_phi(r1, kL1, kR1, dphi1);
  const double cFL = cL + phi1 * (cR - cL);
  const double den2 = cL - cR + 1.e-20, num2 = cR - cRR, r2 = num2 / den2;
  double dphi2;
  const double phi2 = lim_phi(r2, kR2, kL2, dphi2);
  const double cFR = cR + phi2 * (cL - cR);
  const double absw = fabs(w), sg = w > 0.0 ? 1.0 : (w < 0.0 ? -1.0 : 0.0);
  aw = 0.25 * ((sg + 1.0) * cFL + (1.0 - sg) * cFR) * aF;
  const double acFL = 0.25 * (absw + w) * aF, acFR = 0.25 * (-absw + w) * aF;
  aLL = 0.0;
  aRR = 0.0;
  aL = (1.0 - phi1) * acFL;
  aR = phi1 * acFL;
  const double ar1 = dphi1 * (cR - cL) * acFL;
  const double an1 = ar1 / den1, ad1 = -an1 * r1;
  aL += an1 - ad1;
  aLL -= an1;
  aR += ad1;
  aR += (1.0 - phi2) * acFR;
  aL += phi2 * acFR;
  const double ar2 = dphi2 * (cL - cR) * acFR;
  const double an2 = ar2 / den2, ad2 = -an2 * r2;
  aR += an2 - ad2;
  aRR -= an2;
  aL += ad2;
}


// staged quantities of the adjoint kernels
enum {
  A_RHO = 0, A_U, A_V, A_W, A_TH, A_IR, A_DPD, A_P, A_D310, A_D311, A_D320, A_D321, A_D330, A_D331, A_J0, A_M0, A_M1,
  A_NQ
};
enum { B_D110 = 0, B_D111, B_D120, B_D121, B_D210, B_D211, B_D220, B_D221, B_J1, B_FC, B_C1, B_NQ = B_C1 + 5 };
constexpr int ADJ_WARPS = 8;
constexpr int ADJ_NS = 6;   // scratch quantities per warp (the largest transposed round)

template <int N>
struct AdjCfg {
  static constexpr int DoF = N * N;
  static constexpr int LPW = 32 / DoF;
  static constexpr int LC = ADJ_WARPS * LPW;
  static constexpr int RP = LC + 4;
  static constexpr int THREADS = 32 * ADJ_WARPS;
  // staged planes, own-level quantities, per-warp scratch, the limiter
  // coefficients of the LC + 1 interfaces L0-1 .. L0+LC-1, and the CTA's sums
  // of its state-adjoint contributions (5 fields of the RP planes)
  static constexpr size_t SMEM = ((size_t)A_NQ * RP * DoF + (size_t)B_NQ * LC * DoF + (size_t)ADJ_WARPS * ADJ_NS * 32 +
                                  (size_t)4 * (LC + 1) * DoF + (size_t)5 * RP * DoF) * sizeof(double);
};

// Stage the planes L0-2 .. L0+LC+1 of one element (as the forward kernel):
// every value is copied with cp.async, so all of a thread's copies are in
// flight at once; after its own copies land, the thread forms 1/rho, theta
// and dp/d(rho*theta) of its slots.  The caller's barrier follows.
template <int N>
__device__ __forceinline__ void adj_stage(const GP &P, const double *__restrict__ U, const double *__restrict__ Pr,
                                          const double *__restrict__ T1, double *pw, double *ow, double *rk, int IF,
                                          int L0)
{
  using CF = AdjCfg<N>;
  constexpr int DoF = CF::DoF, LC = CF::LC, RP = CF::RP;
  const int nz = P.nz, NumG = P.NumG;
  const size_t cs = (size_t)DoF * nz, fs = (size_t)nz * NumG;
  const double *mte = P.met + (size_t)IF * NCOMP * cs;
#define AWs(q) pw[((q) * RP + p) * DoF + ID]
  for (int s = threadIdx.x; s < DoF * RP; s += CF::THREADS) {
    const int ID = s / RP, p = s % RP;
    const int lev = L0 - 2 + p;
    if (lev < 0 || lev >= nz) continue;
    const int g = P.glob[IF * DoF + ID];
    const double *Ug = U + (size_t)nz * g + lev;
    const double *mt = mte + (size_t)ID * nz + lev;
    cp_async8(&AWs(A_RHO), Ug);
    cp_async8(&AWs(A_TH), Ug + 4 * fs);   // rho*theta for now
    if (p >= 1 && p <= LC + 1 && lev < nz - 1) {   // interface lev, between levels lev and lev + 1
      double *r = rk + (size_t)(p - 1) * DoF + ID;
      constexpr size_t rs = (size_t)(LC + 1) * DoF;
      cp_async8(r, mt + C_RK0 * cs); cp_async8(r + rs, mt + C_RK1 * cs);
      cp_async8(r + 2 * rs, mt + C_RK2 * cs); cp_async8(r + 3 * rs, mt + C_RK3 * cs);
    }
    if (p >= 2 && p <= LC + 1) {
      double *o = ow + (size_t)(p - 2) * DoF + ID;
      constexpr size_t os = (size_t)LC * DoF;
      cp_async8(o + B_D110 * os, mt + C_D11_0 * cs); cp_async8(o + B_D111 * os, mt + C_D11_1 * cs);
      cp_async8(o + B_D120 * os, mt + C_D12_0 * cs); cp_async8(o + B_D121 * os, mt + C_D12_1 * cs);
      cp_async8(o + B_D210 * os, mt + C_D21_0 * cs); cp_async8(o + B_D211 * os, mt + C_D21_1 * cs);
      cp_async8(o + B_D220 * os, mt + C_D22_0 * cs); cp_async8(o + B_D221 * os, mt + C_D22_1 * cs);
      cp_async8(o + B_J1 * os, mt + C_J1 * cs);
      cp_async8(o + B_FC * os, mt + C_FCOR * cs);
      if (T1) {
        const double *T = T1 + (size_t)nz * g + lev;
        for (int f = 0; f < 5; ++f) cp_async8(o + (B_C1 + f) * os, T + f * fs);
      }
    }
    if (p == 0 || p == RP - 1) continue;
    cp_async8(&AWs(A_U), Ug + fs);
    cp_async8(&AWs(A_V), Ug + 2 * fs);
    cp_async8(&AWs(A_W), Ug + 3 * fs);
    cp_async8(&AWs(A_D310), mt + C_D31_0 * cs); cp_async8(&AWs(A_D311), mt + C_D31_1 * cs);
    cp_async8(&AWs(A_D320), mt + C_D32_0 * cs); cp_async8(&AWs(A_D321), mt + C_D32_1 * cs);
    cp_async8(&AWs(A_D330), mt + C_D33_0 * cs); cp_async8(&AWs(A_D331), mt + C_D33_1 * cs);
    cp_async8(&AWs(A_J0), mt + C_J0 * cs);
    cp_async8(&AWs(A_M0), P.M + lev + (size_t)nz * g);
    cp_async8(&AWs(A_M1), P.M + lev + (size_t)nz * (g + (size_t)NumG));
    if (Pr) cp_async8(&AWs(A_P), Pr + lev + (size_t)nz * g);
    else AWs(A_P) = 0.0;
  }
  cp_async_wait_all();
  for (int s = threadIdx.x; s < DoF * RP; s += CF::THREADS) {
    const int ID = s / RP, p = s % RP;
    const int lev = L0 - 2 + p;
    if (lev < 0 || lev >= nz) continue;
    const double rho = AWs(A_RHO), rth = AWs(A_TH);
    AWs(A_IR) = 1.0 / rho;
    AWs(A_TH) = rth / rho;
    if (p == 0 || p == RP - 1) continue;
    AWs(A_DPD) = AWs(A_P) / ((1.0 - P.kappa) * rth);   // dp/d(rho*theta)
  }
#undef AWs
}

// Reverse of phase 2 (no tracers): LU += (d phase2 / d U)^T lambda and
// LT1 += (d phase2 / d T1)^T lambda, lambda being lambda_F broadcast to the
// element nodes.  One CTA per (element, chunk of LC levels), one warp per level.
// Two blocks per SM (128 registers, a few hundred bytes of spills) run this
// latency-bound kernel faster than one block at its natural 198 registers.
template <int N>
__global__ void __launch_bounds__(32 * ADJ_WARPS, 2) k_phase2_adj(const GP P, const double *__restrict__ U,
                                                              const double *__restrict__ Pr,
                                                              const double *__restrict__ T1,
                                                              const double *__restrict__ LF, double *__restrict__ LU,
                                                              double *__restrict__ LT1)
{
  using CF = AdjCfg<N>;
  constexpr int DoF = CF::DoF, LPW = CF::LPW, LC = CF::LC, RP = CF::RP;
  extern __shared__ double sm[];
  const int nz = P.nz, NumG = P.NumG;
  const int IF = blockIdx.y, L0 = blockIdx.x * LC;
  const size_t fs = (size_t)nz * NumG;
  double *pw = sm;
  double *ow = pw + (size_t)A_NQ * RP * DoF;
  double *scr = ow + (size_t)B_NQ * LC * DoF;
  double *rk = scr + (size_t)ADJ_WARPS * ADJ_NS * 32;   // [4][LC+1][DoF]
  // [5][RP][DoF]: the contributions of the CTA's nodes to the state adjoint
  // at levels L0-2 .. L0+LC+1, summed here (shared-memory atomics) and added
  // to LU once per (field, level, node) at the end
  double *sacc = rk + (size_t)4 * (LC + 1) * DoF;
  for (int s = threadIdx.x; s < 5 * RP * DoF; s += CF::THREADS) sacc[s] = 0.0;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int sub = lane / DoF, ID = lane - sub * DoF;
  const int lv = L0 + warp * LPW + sub;
  const bool act = sub < LPW && lv < nz;
  // lambda of this node and level, loaded while the planes are staged
  double lam_r = 0, lam_u = 0, lam_v = 0, lam_th = 0, lam_whi = 0, lam_wlo = 0;
  if (act) {
    const double *L = LF + (size_t)nz * P.glob[IF * DoF + ID] + lv;
    lam_r = L[0]; lam_u = L[fs]; lam_v = L[2 * fs]; lam_th = L[4 * fs];
    if (lv < nz - 1) lam_whi = L[3 * fs];
    if (lv > 0) lam_wlo = L[3 * fs - 1];
  }
  adj_stage<N>(P, U, Pr, T1, pw, ow, rk, IF, L0);
  __syncthreads();

  const int I = ID % N, Jn = ID / N;
  const int p0 = lv - (L0 - 2), li = lv - L0;
  double *sw = scr + (size_t)warp * ADJ_NS * 32 + sub * DoF;
#define SC(q, id) sw[(q) * 32 + (id)]
#define AW(q, p, id) pw[((q) * RP + (p)) * DoF + (id)]
#define BW(q, id) ow[((size_t)(q) * LC + li) * DoF + (id)]
  double DI[N], DJ[N], DTI[N], DTJ[N], WTI[N], WTJ[N];
#pragma unroll
  for (int k = 0; k < N; ++k) {
    DI[k] = P.D[I + N * k];
    DJ[k] = P.D[Jn + N * k];
    DTI[k] = P.D[k + N * I];
    DTJ[k] = P.D[k + N * Jn];
    WTI[k] = P.DW[k + N * I];
    WTJ[k] = P.DW[k + N * Jn];
  }
  const bool top = act && lv < nz - 1, bot = act && lv > 0;
  const int g = act ? P.glob[IF * DoF + ID] : 0;
#define ADDU(f, lev, val) atomicAdd(sacc + ((f) * RP + (lev) - (L0 - 2)) * DoF + ID, (val))
  // wl of any node of this plane (the surface value from no normal flow)
  auto wl_at = [&](int n) {
    return lv == 0 ? -(AW(A_D310, p0, n) * AW(A_U, p0, n) + AW(A_D320, p0, n) * AW(A_V, p0, n)) / AW(A_D330, p0, n)
                   : AW(A_W, p0 - 1, n);
  };
  // adjoint of theta at level lev of this node -> rho*theta and rho
  auto add_theta = [&](int lev, double ath) {
    const int pl = lev - (L0 - 2);
    const double q = ath * AW(A_IR, pl, ID);
    ADDU(4, lev, q);
    ADDU(0, lev, -q * AW(A_TH, pl, ID));
  };
  // adjoint of the pressure at level lev of this node -> rho*theta
  auto add_p = [&](int lev, double ap) {
    const int pl = lev - (L0 - 2);
    ADDU(4, lev, ap * AW(A_DPD, pl, ID));
  };

  // ---------------- forward quantities of this node ----------------
  double rho = 1, u = 0, v = 0, wh = 0, wl = 0, th = 0, MC = 1, Js = 1, J0 = 0, J1 = 0, fc = 0, M0 = 1, M1 = 0;
  double d110 = 0, d111 = 0, d120 = 0, d121 = 0, d210 = 0, d211 = 0, d220 = 0, d221 = 0;
  double d11 = 0, d12 = 0, d21 = 0, d22 = 0;
  double e310 = 0, e311 = 0, e320 = 0, e321 = 0, e330 = 1, e331 = 1;
  double GDx = 0, GDy = 0, U1 = 0, U2 = 0, V1 = 0, V2 = 0, W1 = 0, W2 = 0, Gradu = 0, Gradv = 0;
  double iMC = 1, iJs = 1, irho = 1, i33 = 0.5;   // reciprocals used throughout
  if (act) {
    rho = AW(A_RHO, p0, ID); u = AW(A_U, p0, ID); v = AW(A_V, p0, ID); wh = AW(A_W, p0, ID); th = AW(A_TH, p0, ID);
    e310 = AW(A_D310, p0, ID); e311 = AW(A_D311, p0, ID); e320 = AW(A_D320, p0, ID);
    e321 = AW(A_D321, p0, ID); e330 = AW(A_D330, p0, ID); e331 = AW(A_D331, p0, ID);
    J0 = AW(A_J0, p0, ID); J1 = BW(B_J1, ID); fc = BW(B_FC, ID);
    M0 = AW(A_M0, p0, ID); M1 = AW(A_M1, p0, ID);
    MC = M0 + M1;
    Js = J0 + J1;
    iMC = 1.0 / MC;
    iJs = 1.0 / Js;
    irho = 1.0 / rho;
    i33 = 1.0 / (e330 + e331);
    wl = wl_at(ID);
    d110 = BW(B_D110, ID); d111 = BW(B_D111, ID); d120 = BW(B_D120, ID); d121 = BW(B_D121, ID);
    d210 = BW(B_D210, ID); d211 = BW(B_D211, ID); d220 = BW(B_D220, ID); d221 = BW(B_D221, ID);
    d11 = d110 + d111; d12 = d120 + d121; d21 = d210 + d211; d22 = d220 + d221;
    // hyperviscosity: gradient of the cached theta Laplacian
    double Dxc = 0, Dyc = 0, DXp = 0, DYp = 0;
#pragma unroll
    for (int k = 0; k < N; ++k) {
      Dxc += DI[k] * BW(B_C1 + 4, k + N * Jn);
      Dyc += DJ[k] * BW(B_C1 + 4, I + N * k);
      DXp += DI[k] * AW(A_P, p0, k + N * Jn);
      DYp += DJ[k] * AW(A_P, p0, I + N * k);
    }
    GDx = (d11 * Dxc + d21 * Dyc) * iJs;
    GDy = (d12 * Dxc + d22 * Dyc) * iJs;
    const double GZg = -P.Grav * rho * Js * i33;
    Gradu = d11 * DXp + d21 * DYp + GZg * (e310 + e311);
    Gradv = d12 * DXp + d22 * DYp + GZg * (e320 + e321);
    // momentum: U1..W2
    const double tu0 = e330 * v - e320 * wl, tu1 = e331 * v - e321 * wh;
    const double tv0 = e330 * u - e310 * wl, tv1 = e331 * u - e311 * wh;
    const double tw0 = e320 * u - e310 * v, tw1 = e321 * u - e311 * v;
    U1 = U2 = 0.5 * (tu1 - tu0);
    V1 = V2 = 0.5 * (tv1 - tv0);
    W1 = W2 = 0.5 * (tw1 - tw0);
#pragma unroll
    for (int k = 0; k < N; ++k) {
      const int nx = k + N * Jn, ny = I + N * k;
      const double wlx = wl_at(nx), wly = wl_at(ny), whx = AW(A_W, p0, nx), why = AW(A_W, p0, ny);
      const double ux = AW(A_U, p0, nx), uy = AW(A_U, p0, ny), vx = AW(A_V, p0, nx), vy = AW(A_V, p0, ny);
      U1 += DI[k] * (-BW(B_D120, nx) * wlx) + DJ[k] * (-BW(B_D220, ny) * wly);
      U2 += DI[k] * (-BW(B_D121, nx) * whx) + DJ[k] * (-BW(B_D221, ny) * why);
      V1 += DI[k] * (-BW(B_D110, nx) * wlx) + DJ[k] * (-BW(B_D210, ny) * wly);
      V2 += DI[k] * (-BW(B_D111, nx) * whx) + DJ[k] * (-BW(B_D211, ny) * why);
      W1 += DI[k] * (BW(B_D120, nx) * ux - BW(B_D110, nx) * vx) + DJ[k] * (BW(B_D220, ny) * uy - BW(B_D210, ny) * vy);
      W2 += DI[k] * (BW(B_D121, nx) * ux - BW(B_D111, nx) * vx) + DJ[k] * (BW(B_D221, ny) * uy - BW(B_D211, ny) * vy);
    }
  }
  const double K1s = 0.5 * (u * u + v * v) + 0.5 * (wl * wl);
  const double K2s = 0.5 * (u * u + v * v) + 0.5 * (wh * wh);

  // ---------------- reverse ----------------
  double ar = 0, au = 0, av = 0, awh = 0, awl = 0, ath = 0, ap = 0;
  // mu, mv: (-v W1 - wl V1 - v W2 - wh V2 + FU)/MC, (u W1 - wl U1 + u W2 - wh U2 + FV)/MC
  const double amu = lam_u * iMC, amv = lam_v * iMC;
  double aU1 = -wl * amv, aU2 = -wh * amv, aV1 = -wl * amu, aV2 = -wh * amu;
  double aW1 = -v * amu + u * amv, aW2 = aW1;
  av += -(W1 + W2) * amu;
  au += (W1 + W2) * amv;
  awl += -V1 * amu - U1 * amv;
  awh += -V2 * amu - U2 * amv;
  double aFU = amu, aFV = amv, aFW1 = 0, aFW2 = 0;
  // Coriolis
  av += fc * Js * aFU;
  au += -fc * Js * aFV;
  // gradient part: gu = (GuF1 + GuF2 - Gradu/rho)/MC, gv likewise
  const double aG1u = amu, aG1v = amv;   // adjoints of GuF1 = GuF2, GvF1 = GvF2
  double aGradu = -amu * irho, aGradv = -amv * irho;
  ar += (Gradu * amu + Gradv * amv) * irho * irho;
  const double aDXK1 = -(d110 * aG1u + d120 * aG1v), aDYK1 = -(d210 * aG1u + d220 * aG1v);
  const double aDXK2 = -(d111 * aG1u + d121 * aG1v), aDYK2 = -(d211 * aG1u + d221 * aG1v);
  double aK1s = 0, aK2s = 0;
  double aGZs = -(e310 * aG1u + e320 * aG1v + e311 * aG1u + e321 * aG1v);   // GZ = 0.5 (K2s - K1s)
  double aGZb = -(e310 * aG1u + e320 * aG1v);                                // GZ = 0.5 (K1s - K2b), bot
  double aGZt = -(e311 * aG1u + e321 * aG1v);                                // GZ = 0.5 (K1a - K2s), top
  // w: upper node (interface lv) and lower node (interface lv-1)
  double aNh = 0, aNl = 0;
  if (top) {
    const int pa = p0 + 1;
    const double rho1 = AW(A_RHO, pa, ID), u1 = AW(A_U, pa, ID), v1 = AW(A_V, pa, ID);
    const double M0a = AW(A_M0, pa, ID), J0a = AW(A_J0, pa, ID), D330a = AW(A_D330, pa, ID);
    const double D320a = AW(A_D320, pa, ID), D310a = AW(A_D310, pa, ID), pa_ = AW(A_P, pa, ID);
    const double den = rho1 * M0a + rho * M1;
    const double tu1 = e331 * v - e321 * wh, tv1 = e331 * u - e311 * wh;
    const double tu0a = D330a * v1 - D320a * wh, tv0a = D330a * u1 - D310a * wh, tw0a = D320a * u1 - D310a * v1;
    const double tw1 = e321 * u - e311 * v;
    const double FluxUZt = 0.5 * (tu0a - tu1), FluxVZt = 0.5 * (tv0a - tv1), FluxWZt = 0.5 * (tw0a - tw1);
    const double FW2 = u * FluxVZt + v * FluxUZt;
    const double Nh = u * V2 + v * U2 + FW2;
    const double K1a = 0.5 * (u1 * u1 + v1 * v1) + 0.5 * (wh * wh);
    const double GZt = 0.5 * (K1a - K2s), GZs = 0.5 * (K2s - K1s);
    const double GwF2 = -rho * GZt * e331 - rho * GZs * e331;
    const double GZp = 0.5 * (pa_ - AW(A_P, p0, ID));
    const double Gradp = -(GZp * (e331 + D330a) + P.Grav * (rho * J1 + rho1 * J0a));
    const double iden = 1.0 / den;
    const double whi = (rho * Nh + GwF2 + Gradp) * iden;
    // whi = (rho Nh + GwF2 + Gradp) / den
    const double lw = lam_whi * iden;
    aNh = rho * lw;
    ar += Nh * lw;
    const double aGwF2 = lw, aGradp = lw, aden = -whi * lw;
    const double arho1 = M0a * aden - P.Grav * J0a * aGradp;
    ar += M1 * aden - P.Grav * J1 * aGradp;
    add_p(lv + 1, -0.5 * (e331 + D330a) * aGradp);
    ap += 0.5 * (e331 + D330a) * aGradp;
    // GwF2 = -rho e331 (GZt + GZs)
    ar += -(GZt + GZs) * e331 * aGwF2;
    aGZt += -rho * e331 * aGwF2;
    aGZs += -rho * e331 * aGwF2;
    // Nh = u V2 + v U2 + FW2
    aV2 += u * aNh;
    aU2 += v * aNh;
    au += V2 * aNh;
    av += U2 * aNh;
    aFW2 += aNh;
    // K1a (upper node's bottom K): GZt = 0.5 (K1a - K2s)
    const double aK1a = 0.5 * aGZt;
    aK2s += -0.5 * aGZt;
    double au1 = u1 * aK1a, av1 = v1 * aK1a;
    awh += wh * aK1a;
    // top vertical momentum fluxes: FU += -v FWZt - wh FVZt; FV += u FWZt - wh FUZt; FW2 += u FVZt + v FUZt
    av += -FluxWZt * aFU + FluxUZt * aFW2;
    awh += -FluxVZt * aFU - FluxUZt * aFV;
    au += FluxWZt * aFV + FluxVZt * aFW2;
    const double aFWZt = -v * aFU + u * aFV, aFVZt = -wh * aFU + u * aFW2, aFUZt = -wh * aFV + v * aFW2;
    // FluxXZt = 0.5 (tx0a - tx1)
    const double atu0a = 0.5 * aFUZt, atv0a = 0.5 * aFVZt, atw0a = 0.5 * aFWZt;
    const double atu1 = -0.5 * aFUZt, atv1 = -0.5 * aFVZt, atw1 = -0.5 * aFWZt;
    // tu0a = D330a v1 - D320a wh; tv0a = D330a u1 - D310a wh; tw0a = D320a u1 - D310a v1
    av1 += D330a * atu0a - D310a * atw0a;
    au1 += D330a * atv0a + D320a * atw0a;
    awh += -D320a * atu0a - D310a * atv0a;
    // tu1 = e331 v - e321 wh; tv1 = e331 u - e311 wh; tw1 = e321 u - e311 v
    av += e331 * atu1 - e311 * atw1;
    au += e331 * atv1 + e321 * atw1;
    awh += -e321 * atu1 - e311 * atv1;
    ADDU(0, lv + 1, arho1);
    ADDU(1, lv + 1, au1);
    ADDU(2, lv + 1, av1);
  }
  if (bot) {
    const int pb = p0 - 1;
    const double rhob = AW(A_RHO, pb, ID), ub = AW(A_U, pb, ID), vb = AW(A_V, pb, ID), wb = AW(A_W, pb, ID);
    const double M1b = AW(A_M1, pb, ID), D331b = AW(A_D331, pb, ID), D321b = AW(A_D321, pb, ID);
    const double D311b = AW(A_D311, pb, ID);
    const double den = rhob * M1b + rho * M0;
    const double tu0 = e330 * v - e320 * wl, tv0 = e330 * u - e310 * wl, tw0 = e320 * u - e310 * v;
    const double tu1b = D331b * vb - D321b * wb, tv1b = D331b * ub - D311b * wb, tw1b = D321b * ub - D311b * vb;
    const double FluxUZ = 0.5 * (tu0 - tu1b), FluxVZ = 0.5 * (tv0 - tv1b), FluxWZ = 0.5 * (tw0 - tw1b);
    const double FW1 = u * FluxVZ + v * FluxUZ;
    const double Nl = u * V1 + v * U1 + FW1;
    const double K2b = 0.5 * (ub * ub + vb * vb) + 0.5 * (wb * wb);
    const double GZ1 = 0.5 * (K1s - K2b), GZ2 = 0.5 * (K2s - K1s);
    const double GwF1 = -rho * GZ1 * e330 - rho * GZ2 * e330;
    const double iden = 1.0 / den;
    const double wlo = (rho * Nl + GwF1) * iden;
    const double lw = lam_wlo * iden;
    aNl = rho * lw;
    ar += Nl * lw;
    const double aGwF1 = lw, aden = -wlo * lw;
    double arhob = M1b * aden;
    ar += M0 * aden;
    ar += -(GZ1 + GZ2) * e330 * aGwF1;
    const double aGZ1 = -rho * e330 * aGwF1, aGZ2 = -rho * e330 * aGwF1;
    aK1s += 0.5 * aGZ1 - 0.5 * aGZ2;
    double aK2b = -0.5 * aGZ1;
    aK2s += 0.5 * aGZ2;
    // Nl = u V1 + v U1 + FW1
    aV1 += u * aNl;
    aU1 += v * aNl;
    au += V1 * aNl;
    av += U1 * aNl;
    aFW1 += aNl;
    // GZ = 0.5 (K1s - K2b) in GuF1, GvF1
    aK1s += 0.5 * aGZb;
    aK2b += -0.5 * aGZb;
    // bottom vertical momentum fluxes: FU += -v FWZ - wl FVZ; FV += u FWZ - wl FUZ; FW1 += u FVZ + v FUZ
    av += -FluxWZ * aFU + FluxUZ * aFW1;
    awl += -FluxVZ * aFU - FluxUZ * aFV;
    au += FluxWZ * aFV + FluxVZ * aFW1;
    const double aFWZ = -v * aFU + u * aFV, aFVZ = -wl * aFU + u * aFW1, aFUZ = -wl * aFV + v * aFW1;
    const double atu0 = 0.5 * aFUZ, atv0 = 0.5 * aFVZ, atw0 = 0.5 * aFWZ;
    const double atu1b = -0.5 * aFUZ, atv1b = -0.5 * aFVZ, atw1b = -0.5 * aFWZ;
    // tu0 = e330 v - e320 wl; tv0 = e330 u - e310 wl; tw0 = e320 u - e310 v
    av += e330 * atu0 - e310 * atw0;
    au += e330 * atv0 + e320 * atw0;
    awl += -e320 * atu0 - e310 * atv0;
    // tu1b = D331b vb - D321b wb; tv1b = D331b ub - D311b wb; tw1b = D321b ub - D311b vb
    double aub = D331b * atv1b + D321b * atw1b + ub * aK2b;
    double avb = D331b * atu1b - D311b * atw1b + vb * aK2b;
    double awb = -D321b * atu1b - D311b * atv1b + wb * aK2b;
    ADDU(0, lv - 1, arhob);
    ADDU(1, lv - 1, aub);
    ADDU(2, lv - 1, avb);
    ADDU(3, lv - 1, awb);
  }
  // U1.. init: 0.5 (t1 - t0) with t's from this node
  {
    const double aUi = aU1 + aU2, aVi = aV1 + aV2, aWi = aW1 + aW2;
    // tu0 = e330 v - e320 wl, tu1 = e331 v - e321 wh (and tv, tw)
    av += 0.5 * aUi * (e331 - e330);
    awh += -0.5 * aUi * e321;
    awl += 0.5 * aUi * e320;
    au += 0.5 * aVi * (e331 - e330);
    awh += -0.5 * aVi * e311;
    awl += 0.5 * aVi * e310;
    au += 0.5 * aWi * (e321 - e320);
    av += -0.5 * aWi * (e311 - e310);
  }
  // GZ = 0.5 (K2s - K1s)
  aK2s += 0.5 * aGZs;
  aK1s += -0.5 * aGZs;
  // Gradu = d11 DXp + d21 DYp + GZg (e310 + e311); GZg = -g rho Js / (e330 + e331)
  {
    const double aGZg = (e310 + e311) * aGradu + (e320 + e321) * aGradv;
    ar += -P.Grav * Js * i33 * aGZg;
  }
  const double aDXp = d11 * aGradu + d12 * aGradv, aDYp = d21 * aGradu + d22 * aGradv;

  // ---- transposed round 1: momentum sums (adjoints of U1..W2) ----
  if (act) {
    SC(0, ID) = aU1; SC(1, ID) = aU2; SC(2, ID) = aV1; SC(3, ID) = aV2; SC(4, ID) = aW1; SC(5, ID) = aW2;
  }
  __syncwarp();
  if (act) {
    double x[6] = {0, 0, 0, 0, 0, 0}, y[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int k = 0; k < N; ++k)
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        x[q] += DTI[k] * SC(q, k + N * Jn);
        y[q] += DTJ[k] * SC(q, I + N * k);
      }
    // U1: x -> tempuZ1 lo (-d120 wl), y -> tempuZ2 lo (-d220 wl); U2: -d121 wh, -d221 wh;
    // V1: -d110 wl, -d210 wl; V2: -d111 wh, -d211 wh; W1: d120 u - d110 v, d220 u - d210 v;
    // W2: d121 u - d111 v, d221 u - d211 v
    awl += -d120 * x[0] - d220 * y[0] - d110 * x[2] - d210 * y[2];
    awh += -d121 * x[1] - d221 * y[1] - d111 * x[3] - d211 * y[3];
    au += d120 * x[4] + d220 * y[4] + d121 * x[5] + d221 * y[5];
    av += -d110 * x[4] - d210 * y[4] - d111 * x[5] - d211 * y[5];
  }
  __syncwarp();
  // ---- transposed round 2: kinetic-energy and pressure sums ----
  if (act) {
    SC(0, ID) = aDXK1; SC(1, ID) = aDYK1; SC(2, ID) = aDXK2; SC(3, ID) = aDYK2; SC(4, ID) = aDXp; SC(5, ID) = aDYp;
  }
  __syncwarp();
  if (act) {
#pragma unroll
    for (int k = 0; k < N; ++k) {
      aK1s += DTI[k] * SC(0, k + N * Jn) + DTJ[k] * SC(1, I + N * k);
      aK2s += DTI[k] * SC(2, k + N * Jn) + DTJ[k] * SC(3, I + N * k);
      ap += DTI[k] * SC(4, k + N * Jn) + DTJ[k] * SC(5, I + N * k);
    }
    // K1s = 0.5 (u^2 + v^2) + 0.5 wl^2, K2s likewise with wh
    au += u * (aK1s + aK2s);
    av += v * (aK1s + aK2s);
    awl += wl * aK1s;
    awh += wh * aK2s;
  }
  __syncwarp();
  // ---- transposed round 3: flux divergences (HR, HTH) ----
  const double aDivRho = lam_r * iMC, aDivTr = lam_th * iMC;
  if (act) { SC(0, ID) = aDivRho; SC(1, ID) = aDivTr; }
  __syncwarp();
  if (act) {
    double xr = 0, yr = 0, xt = 0, yt = 0;
#pragma unroll
    for (int k = 0; k < N; ++k) {
      xr += DTI[k] * SC(0, k + N * Jn);
      yr += DTJ[k] * SC(0, I + N * k);
      xt += DTI[k] * SC(1, k + N * Jn);
      yt += DTJ[k] * SC(1, I + N * k);
    }
    const double uc = -rho * (d11 * u + d12 * v), vc = -rho * (d21 * u + d22 * v);
    const double auc = xr + th * xt, avc = yr + th * yt;
    ath += uc * xt + vc * yt;
    ar += -(d11 * u + d12 * v) * auc - (d21 * u + d22 * v) * avc;
    au += -rho * (d11 * auc + d21 * avc);
    av += -rho * (d12 * auc + d22 * avc);
  }
  __syncwarp();
  // ---- transposed round 4: weak derivatives of the hyperviscosity ----
  const double nuC = P.nuCurl, nuG = P.nuGrad, nuD = P.nuDiv;
  const double aFuC = nuC * amu, aFuD = -nuG * amu, aFvC = nuC * amv, aFvD = -nuG * amv;
  if (act) {
    SC(0, ID) = d12 * aFuC - d11 * aFvC;   // DxCurl
    SC(1, ID) = d22 * aFuC - d21 * aFvC;   // DyCurl
    SC(2, ID) = d11 * aFuD + d12 * aFvD;   // DxDiv
    SC(3, ID) = d21 * aFuD + d22 * aFvD;   // DyDiv
    SC(4, ID) = -nuD * aDivTr;             // DivTh
  }
  __syncwarp();
  double acu = 0, adv = 0, aDxc = 0, aDyc = 0;
  if (act) {
    double ab1 = 0, ab2 = 0, ab3 = 0, ab4 = 0;
#pragma unroll
    for (int k = 0; k < N; ++k) {
      ab1 += WTI[k] * SC(0, k + N * Jn) + WTJ[k] * SC(1, I + N * k);
      ab2 += WTI[k] * SC(2, k + N * Jn) + WTJ[k] * SC(3, I + N * k);
      ab3 += WTI[k] * SC(4, k + N * Jn);
      ab4 += WTJ[k] * SC(4, I + N * k);
    }
    acu = ab1 * iJs;
    adv = ab2 * iJs;
    // b3 = rho (d11 GDx + d12 GDy), b4 = rho (d21 GDx + d22 GDy)
    ar += (d11 * GDx + d12 * GDy) * ab3 + (d21 * GDx + d22 * GDy) * ab4;
    const double aGDx = rho * (d11 * ab3 + d21 * ab4), aGDy = rho * (d12 * ab3 + d22 * ab4);
    aDxc = (d11 * aGDx + d12 * aGDy) * iJs;
    aDyc = (d21 * aGDx + d22 * aGDy) * iJs;
  }
  __syncwarp();
  // ---- transposed round 5: first derivatives of the cache ----
  if (act) { SC(0, ID) = acu; SC(1, ID) = adv; SC(2, ID) = aDxc; SC(3, ID) = aDyc; }
  __syncwarp();
  if (act) {
    double aa1 = 0, aa2 = 0, aa3 = 0, aa4 = 0, ac5 = 0;
#pragma unroll
    for (int k = 0; k < N; ++k) {
      aa1 += DTI[k] * SC(0, k + N * Jn);
      aa2 += DTJ[k] * SC(0, I + N * k);
      aa3 += DTI[k] * SC(1, k + N * Jn);
      aa4 += DTJ[k] * SC(1, I + N * k);
      ac5 += DTI[k] * SC(2, k + N * Jn) + DTJ[k] * SC(3, I + N * k);
    }
    // a1 = d11 c2 - d12 c1; a2 = d21 c2 - d22 c1; a3 = d11 c3 + d12 c4; a4 = d21 c3 + d22 c4
    double *T = LT1 + (size_t)nz * g + lv;
    atomicAdd(T, -d12 * aa1 - d22 * aa2);
    atomicAdd(T + fs, d11 * aa1 + d21 * aa2);
    atomicAdd(T + 2 * fs, d11 * aa3 + d21 * aa4);
    atomicAdd(T + 3 * fs, d12 * aa3 + d22 * aa4);
    atomicAdd(T + 4 * fs, ac5);
  }
  if (act) {

  // ---- interface fluxes of rho and rho*theta (top: interface lv, bottom: lv-1) ----
  auto iface = [&](int il, double aWc, double aF) {
    const int pl = il - (L0 - 2);
    const double *rki = rk + (size_t)(il - (L0 - 1)) * DoF + ID;
    constexpr size_t rs = (size_t)(LC + 1) * DoF;
    const double kR1 = rki[0], kL1 = rki[rs], kL2 = rki[2 * rs], kR2 = rki[3 * rs];
    const int lm = il > 0 ? il - 1 : il, lp2 = il + 2 < nz ? il + 2 : il + 1;
    const double wI = AW(A_W, pl, ID);
    const double rL = AW(A_RHO, pl, ID), uL = AW(A_U, pl, ID), vL = AW(A_V, pl, ID);
    const double rR = AW(A_RHO, pl + 1, ID), uR = AW(A_U, pl + 1, ID), vR = AW(A_V, pl + 1, ID);
    const double a311 = AW(A_D311, pl, ID), a321 = AW(A_D321, pl, ID), a331 = AW(A_D331, pl, ID);
    const double b310 = AW(A_D310, pl + 1, ID), b320 = AW(A_D320, pl + 1, ID), b330 = AW(A_D330, pl + 1, ID);
    const double wCon = rL * (a311 * uL + a321 * vL + a331 * wI) + rR * (b310 * uR + b320 * vR + b330 * wI);
    // A mass flux within the rounding of its dot products (metric row times
    // velocity) has no direction: at a state with w = 0 over flat orography,
    // the horizontal metric entries of the row (analytically zero) leave
    // |wCon| ~ 1e-16 |row| |velocity| with a sign set by rounding.  There the
    // upwind flux sits on its kink and the adjoint takes the symmetric slope
    // (as for wCon == 0), which central differences see, instead of the side
    // the rounding picked.
    const double wMag =
        fabs(rL) * (fabs(a311) + fabs(a321) + fabs(a331)) * (fabs(uL) + fabs(vL) + fabs(wI)) +
        fabs(rR) * (fabs(b310) + fabs(b320) + fabs(b330)) * (fabs(uR) + fabs(vR) + fabs(wI));
    const double wEff = fabs(wCon) <= 1e-13 * wMag ? 0.0 : wCon;
    double aw, aLL, aL, aR, aRR;
    upwind_adj(AW(A_TH, lm - (L0 - 2), ID), AW(A_TH, pl, ID), AW(A_TH, pl + 1, ID), AW(A_TH, lp2 - (L0 - 2), ID), kR1,
               kL1, kL2, kR2, wEff, aF, aw, aLL, aL, aR, aRR);
    add_theta(lm, aLL);
    add_theta(il, aL);
    add_theta(il + 1, aR);
    add_theta(lp2, aRR);
    const double awc = aWc + aw;
    ADDU(0, il, (a311 * uL + a321 * vL + a331 * wI) * awc);
    ADDU(1, il, rL * a311 * awc);
    ADDU(2, il, rL * a321 * awc);
    ADDU(3, il, (rL * a331 + rR * b330) * awc);
    ADDU(0, il + 1, (b310 * uR + b320 * vR + b330 * wI) * awc);
    ADDU(1, il + 1, rR * b310 * awc);
    ADDU(2, il + 1, rR * b320 * awc);
  };
  if (top) iface(lv, -0.5 * aDivRho, -aDivTr);
  if (bot) iface(lv - 1, 0.5 * aDivRho, aDivTr);

  // ---- own node: pressure, theta, lower w ----
  add_p(lv, ap);
  add_theta(lv, ath);
  if (lv == 0) {
    au += -e310 / e330 * awl;
    av += -e320 / e330 * awl;
  } else {
    ADDU(3, lv - 1, awl);
  }
  ADDU(0, lv, ar);
  ADDU(1, lv, au);
  ADDU(2, lv, av);
  ADDU(3, lv, awh);
  }
  // the CTA's sums into the state adjoint, level fastest
  __syncthreads();
  for (int s = threadIdx.x; s < 5 * RP * DoF; s += CF::THREADS) {
    const int f = s / (RP * DoF), r = s - f * (RP * DoF);
    const int n = r / RP, p = r - n * RP;
    const int lev = L0 - 2 + p;
    const double x = sacc[(f * RP + p) * DoF + n];
    if (lev < 0 || lev >= nz || x == 0.0) continue;
    atomicAdd(LU + (size_t)nz * P.glob[IF * DoF + n] + lev + (size_t)f * fs, x);
  }
#undef ADDU
#undef SC
#undef AW
#undef BW
}

// Reverse of phase 1 (no tracers), given lambda_T1 (the adjoint of the DSS'd
// cache, broadcast to the element nodes).  Phase 1 is linear in u, v and
// theta = rho*theta / rho.  Laid out like the forward phase 1: one CTA per
// (element, tile of LT levels), one thread per (node, level), level fastest,
// so the metric, cache and state loads and the atomic adds into LU are runs
// of consecutive levels; the two derivative rounds meet at CTA barriers.
template <int N>
struct AdjHV1Tile {
  static constexpr int LT = N == 5 ? 16 : 256 / (N * N);
  static constexpr int THREADS = LT * N * N;
};

template <int N>
__global__ void __launch_bounds__(AdjHV1Tile<N>::THREADS, 3) k_hypervisc1_adj(const GP P, const double *__restrict__ U,
                                                                          const double *__restrict__ LT1,
                                                                          double *__restrict__ LU)
{
  constexpr int DoF = N * N, LT = AdjHV1Tile<N>::LT;
  __shared__ double s[5][LT * DoF];
  const int nz = P.nz, NumG = P.NumG;
  const int IF = blockIdx.y;
  const size_t cs = (size_t)DoF * nz, fs = (size_t)nz * NumG;
  const int t = threadIdx.x;
  const int lvl = t % LT, ID = t / LT;
  const int l = blockIdx.x * LT + lvl;
  const bool act = ID < DoF && l < nz;
  const int I = ID % N, Jn = ID / N;
  const int si = lvl * DoF + ID, row = lvl * DoF;
#define SC(q, id) s[q][row + (id)]
  double DTI[N], DTJ[N], WTI[N], WTJ[N];
#pragma unroll
  for (int k = 0; k < N; ++k) {
    DTI[k] = P.D[k + N * I];
    DTJ[k] = P.D[k + N * Jn];
    WTI[k] = P.DW[k + N * I];
    WTJ[k] = P.DW[k + N * Jn];
  }
  int g = 0;
  double d11 = 0, d12 = 0, d21 = 0, d22 = 0, Js = 1, MC = 1;
  if (act) {
    g = P.glob[IF * DoF + ID];
    const double *mt = P.met + ((size_t)IF * NCOMP * DoF + ID) * nz + l;
    d11 = mt[C_D11_0 * cs] + mt[C_D11_1 * cs];
    d12 = mt[C_D12_0 * cs] + mt[C_D12_1 * cs];
    d21 = mt[C_D21_0 * cs] + mt[C_D21_1 * cs];
    d22 = mt[C_D22_0 * cs] + mt[C_D22_1 * cs];
    Js = mt[C_J0 * cs] + mt[C_J1 * cs];
    MC = P.M[l + (size_t)nz * g] + P.M[l + (size_t)nz * (g + (size_t)NumG)];
    const double *L = LT1 + (size_t)nz * g + l;
    // out0 = -FuC/MC, out1 = -FvC/MC, out2 = FuD/MC, out3 = FvD/MC, out4 = DivTh/MC
    const double iMC = 1.0 / MC;
    const double aFuC = -L[0] * iMC, aFvC = -L[fs] * iMC, aFuD = L[2 * fs] * iMC, aFvD = L[3 * fs] * iMC;
    s[4][si] = L[4 * fs] * iMC;           // DivTh
    s[0][si] = d12 * aFuC - d11 * aFvC;   // DxCurl
    s[1][si] = d22 * aFuC - d21 * aFvC;   // DyCurl
    s[2][si] = d11 * aFuD + d12 * aFvD;   // DxDiv
    s[3][si] = d21 * aFuD + d22 * aFvD;   // DyDiv
  }
  __syncthreads();
  double as5 = 0, as6 = 0, as7 = 0, as8 = 0;
  if (act) {
#pragma unroll
    for (int k = 0; k < N; ++k) {
      as5 += WTI[k] * SC(0, k + N * Jn) + WTJ[k] * SC(1, I + N * k);
      as6 += WTI[k] * SC(2, k + N * Jn) + WTJ[k] * SC(3, I + N * k);
      as7 += WTI[k] * SC(4, k + N * Jn);
      as8 += WTJ[k] * SC(4, I + N * k);
    }
  }
  __syncthreads();
  // s5 = cu/Js, s6 = dv/Js, s7 = d11 GDx + d12 GDy, s8 = d21 GDx + d22 GDy,
  // GDx = (d11 Dxc + d21 Dyc)/Js, GDy = (d12 Dxc + d22 Dyc)/Js
  if (act) {
    const double aGDx = d11 * as7 + d21 * as8, aGDy = d12 * as7 + d22 * as8, iJs = 1.0 / Js;
    s[0][si] = as5 * iJs;
    s[1][si] = as6 * iJs;
    s[2][si] = (d11 * aGDx + d12 * aGDy) * iJs;
    s[3][si] = (d21 * aGDx + d22 * aGDy) * iJs;
  }
  __syncthreads();
  if (!act) return;
  double as0 = 0, as1 = 0, as2 = 0, as3 = 0, as4 = 0;
#pragma unroll
  for (int k = 0; k < N; ++k) {
    as0 += DTI[k] * SC(0, k + N * Jn);
    as1 += DTJ[k] * SC(0, I + N * k);
    as2 += DTI[k] * SC(1, k + N * Jn);
    as3 += DTJ[k] * SC(1, I + N * k);
    as4 += DTI[k] * SC(2, k + N * Jn) + DTJ[k] * SC(3, I + N * k);
  }
  // s0 = d11 v - d12 u; s1 = d21 v - d22 u; s2 = d11 u + d12 v; s3 = d21 u + d22 v; s4 = theta
  const double au = -d12 * as0 - d22 * as1 + d11 * as2 + d21 * as3;
  const double av = d11 * as0 + d21 * as1 + d12 * as2 + d22 * as3;
  const double *Ug = U + (size_t)nz * g + l;
  const double rho = Ug[0], rth = Ug[4 * fs];
  double *LUg = LU + (size_t)nz * g + l;
  atomicAdd(LUg + fs, au);
  atomicAdd(LUg + 2 * fs, av);
  const double q = as4 / rho;
  atomicAdd(LUg + 4 * fs, q);
  atomicAdd(LUg, -q * (rth / rho));
#undef SC
}


// One reverse sweep of the three stage quantities: Lk0, Lk1 (adjoints of k1,
// k2) and LV (adjoint of the step's initial state), from Lt = F'^T AR of the
// stage and AR (adjoint of its right-hand side r = F + cA k1 + cB k2):
//   stage 3 (L != null): Lk0 = m0 L + cA AR + a0 Lt, Lk1 = m1 L + cB AR + a1 Lt, LV += L + Lt
//   stage 2 (Lk0 != null): Lk0 += cA AR + a0 Lt, LV += Lt
//   stage 1: LV += Lt
__global__ void __launch_bounds__(256) k_adj_update(long long n, const double *__restrict__ L,
                                                    const double *__restrict__ AR, const double *__restrict__ Lt,
                                                    double *__restrict__ LV, double *__restrict__ Lk0,
                                                    double *__restrict__ Lk1, double m0, double m1, double cA,
                                                    double cB, double a0, double a1)
{
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double lt = Lt[i];
  if (L) {
    const double l = L[i], ar = AR[i];
    Lk0[i] = m0 * l + cA * ar + a0 * lt;
    Lk1[i] = m1 * l + cB * ar + a1 * lt;
    LV[i] = LV[i] + (l + lt);
  } else if (Lk0) {
    Lk0[i] = Lk0[i] + (cA * AR[i] + a0 * lt);
    LV[i] = LV[i] + lt;
  } else {
    LV[i] = LV[i] + lt;
  }
}

// Reverse of the column Schur solve of one stage, k = L(bands) r
// (TriDiagKernel!, SchurSolveFKernel!, triSolve!, SchurSolveBKernel!:
// src/Integration/SchurSolve.jl:1-114).  Given mu (times the scalar mus), the
// adjoint of k, writes AR, the adjoint of r, and adds the adjoint that flows
// through the Jacobian bands (JacSchur.jl:40-73) into LV (fields rho and
// rho*theta of the step's initial state).
//
// The stage's k (kx), kept by the forward stage, gives everything else the
// reverse needs: the tridiagonal solution x is its w field, and the
// right-hand side of rho and rho*theta follows from SchurSolveB,
// r0(l) = k0(l)/fac - JB(0,0,l) x(l) - JB(0,1,l-1) x(l-1) (r4 with JB(3,.)).
// The forward sweep solves M x = b with M(i,i) = t1(i), M(i+1,i) = t2(i),
// M(i,i+1) = t0(i+1) (the reference's triSolve!); here M^T y = ax is solved by
// the warp's lanes (warp_tri_solve on the transposed bands).  One warp per
// column throughout.
constexpr int CA_ARR = 18;   // per-warp arrays of nz entries

__global__ void __launch_bounds__(32 * COL_WARPS, 4) k_column_adj(const GP P, const double *__restrict__ mu, double mus,
                                                                 const double *__restrict__ kx,
                                                                 const double *__restrict__ jbg,
                                                                 const double *__restrict__ Vn, double fac,
                                                                 double *__restrict__ AR, double *__restrict__ LV)
{
  extern __shared__ double csm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g0 = blockIdx.x * COL_WARPS, g = g0 + warp;
  const int nz = P.nz, n = nz - 1, NV = P.NV, NumG = P.NumG;
  const bool valid = g < NumG;
  const int LS = nz;
  double *sw = csm + (size_t)warp * CA_ARR * LS;
  double *r0 = sw, *r4 = sw + LS, *av0 = sw + 2 * LS, *av4 = sw + 3 * LS;
  double *jb = sw + 4 * LS;          // [8][nz]
  double *tri = sw + 12 * LS;        // [3][nz]: t0, t1, t2
  double *x = sw + 15 * LS;
  double *ay = sw + 16 * LS;         // ax, then y
  double *accR0 = sw + 17 * LS;      // interface l-1's share of level l (rho)
  const size_t fs = (size_t)nz * NumG;
  const size_t js = (size_t)NumG * n;
#define JB(arr, r, i) jb[((arr) * 2 + (r)) * LS + (i)]
  // 1. x, the bands, the adjoints of the k of rho and rho*theta; fields
  //    outside the Schur system: AR = fac mu; then the right-hand side of rho
  //    and rho*theta
  if (valid) {
    for (int l = lane; l < nz; l += 32) {
      const size_t o0 = l + (size_t)nz * g;
#pragma unroll
      for (int f = 1; f < MAXNV; ++f) {
        if (f >= NV) break;
        if (f != 3 && f != 4) AR[o0 + f * fs] = fac * (mus * mu[o0 + f * fs]);
      }
      av0[l] = fac * (mus * mu[o0]);
      av4[l] = fac * (mus * mu[o0 + 4 * fs]);
      if (l < n) {
        x[l] = kx[o0 + 3 * fs];
        for (int rr = 0; rr < 8; ++rr) jb[rr * LS + l] = jbg[rr * js + (size_t)g * n + l];
      }
    }
    __syncwarp();
    const double invfac2 = 1.0 / fac / fac;
    for (int l = lane; l < nz; l += 32) {
      const size_t o0 = l + (size_t)nz * g;
      double s0 = kx[o0] / fac, s4 = kx[o0 + 4 * fs] / fac;
      if (l < n) { s0 -= JB(0, 0, l) * x[l]; s4 -= JB(3, 0, l) * x[l]; }
      if (l > 0) { s0 -= JB(0, 1, l - 1) * x[l - 1]; s4 -= JB(3, 1, l - 1) * x[l - 1]; }
      r0[l] = s0;
      r4[l] = s4;
    }
    for (int l = lane; l < n; l += 32) {
      tri[LS + l] = invfac2 - JB(1, 1, l) * JB(0, 0, l) - JB(1, 0, l) * JB(0, 1, l) - JB(2, 1, l) * JB(3, 0, l) -
                    JB(2, 0, l) * JB(3, 1, l);
      tri[l] = l == 0 ? 0.0 : -JB(1, 0, l - 1) * JB(0, 0, l) - JB(2, 0, l - 1) * JB(3, 0, l);
      tri[2 * LS + l] = l == n - 1 ? 0.0 : -JB(1, 1, l + 1) * JB(0, 1, l) - JB(2, 1, l + 1) * JB(3, 1, l);
      // reverse of SchurSolveB: v0'(l) = r0(l) + JB(0,0,l) x(l) + JB(0,1,l-1) x(l-1), v4' likewise; kw = x
      ay[l] = mus * mu[l + (size_t)nz * g + 3 * fs] + JB(0, 0, l) * av0[l] + JB(3, 0, l) * av4[l] +
              JB(0, 1, l) * av0[l + 1] + JB(3, 1, l) * av4[l + 1];
    }
  }
  __syncwarp();
  if (!valid) return;   // warp-uniform; nothing below synchronises the block
  // 2. M^T y = ax with the warp's lanes: M^T(i,i) = t1(i), M^T(i+1,i) = t0(i+1),
  //    M^T(i,i+1) = t2(i), i.e. warp_tri_solve with t0 and t2 exchanged and
  //    shifted by one level; y overwrites ax
  warp_tri_solve(tri + 2 * LS - 1, tri + LS, tri + 1, ay, ay, n, lane);
  __syncwarp();
  // 3. adjoint of r, and the band adjoints (TriDiag, SchurSolveF, SchurSolveB)
  //    of interface l, whose share of level l is added here and whose share
  //    of level l+1 is passed on through aR0 / aR4
  double *aR0 = accR0, *aR4 = tri + 1 * LS;   // t1 is dead after the solve
  for (int l = lane; l < nz; l += 32) {
    const size_t o0 = l + (size_t)nz * g;
    double ar0 = av0[l], ar4 = av4[l];
    if (l < n) { ar0 += JB(1, 1, l) * ay[l]; ar4 += JB(2, 1, l) * ay[l]; }
    if (l > 0) { ar0 += JB(1, 0, l - 1) * ay[l - 1]; ar4 += JB(2, 0, l - 1) * ay[l - 1]; }
    AR[o0] = ar0;
    AR[o0 + 3 * fs] = l < n ? ay[l] / fac : 0.0;
    AR[o0 + 4 * fs] = ar4;
  }
  // dp/d(rho*theta) of every level and its derivative factor kappa/(1-kappa) dp/(rho*theta)
  const double ex = P.kappa / (1.0 - P.kappa);
  double *dP = tri, *dPd = tri + 2 * LS;   // t0, t2 are dead after the sweep
  // dp/d(rho*theta) is recovered from the step's bands, JWRhoTh = +-dp / (RhoF h)
  // (h = (dzL + dzR) / 2): level l < n from interface l (its lower level), the
  // top level from interface n - 1 (its upper level); no pow per level
  const double *V0c = Vn + (size_t)nz * g;
  for (int l = lane; l < nz; l += 32) {
    const double Th = V0c[l + 4 * fs] + 0.0;
    const int li = l < n ? l : n - 1;
    const double dzL = P.dz[li + (size_t)nz * g], dzR = P.dz[li + 1 + (size_t)nz * g], dzs = dzL + dzR;
    const double RhoF = (V0c[li] * dzL + V0c[li + 1] * dzR) / dzs;
    const double d = (l < n ? JB(2, 1, li) : -JB(2, 0, li)) * RhoF * (0.5 * dzs);
    dP[l] = d;
    dPd[l] = ex * d / Th;
  }
  __syncwarp();
  double accL0[2] = {0.0, 0.0}, accL4[2] = {0.0, 0.0};
#pragma unroll
  for (int it = 0; it < 2; ++it) {
    const int l = lane + 32 * it;
    if (l >= n) continue;
    const double *y = ay;
    double a[4][2] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};   // a[arr][r] = adjoint of JB(arr, r, l)
    // adjoint of M(i,j) is -y(i) x(j)
    const double at1 = -y[l] * x[l];
    const double at0 = l > 0 ? -y[l - 1] * x[l] : 0.0;              // t0(l) = M(l-1,l)
    const double at0n = l + 1 < n ? -y[l] * x[l + 1] : 0.0;         // t0(l+1) = M(l,l+1)
    const double at2 = l + 1 < n ? -y[l + 1] * x[l] : 0.0;          // t2(l) = M(l+1,l)
    const double at2p = l > 0 ? -y[l] * x[l - 1] : 0.0;             // t2(l-1) = M(l,l-1)
    // t1(l)
    a[1][1] += -JB(0, 0, l) * at1; a[0][0] += -JB(1, 1, l) * at1;
    a[1][0] += -JB(0, 1, l) * at1; a[0][1] += -JB(1, 0, l) * at1;
    a[2][1] += -JB(3, 0, l) * at1; a[3][0] += -JB(2, 1, l) * at1;
    a[2][0] += -JB(3, 1, l) * at1; a[3][1] += -JB(2, 0, l) * at1;
    // t0(l) = -JB(1,0,l-1) JB(0,0,l) - JB(2,0,l-1) JB(3,0,l)
    if (l > 0) { a[0][0] += -JB(1, 0, l - 1) * at0; a[3][0] += -JB(2, 0, l - 1) * at0; }
    // t0(l+1) = -JB(1,0,l) JB(0,0,l+1) - JB(2,0,l) JB(3,0,l+1)
    if (l + 1 < n) { a[1][0] += -JB(0, 0, l + 1) * at0n; a[2][0] += -JB(3, 0, l + 1) * at0n; }
    // t2(l) = -JB(1,1,l+1) JB(0,1,l) - JB(2,1,l+1) JB(3,1,l)
    if (l + 1 < n) { a[0][1] += -JB(1, 1, l + 1) * at2; a[3][1] += -JB(2, 1, l + 1) * at2; }
    // t2(l-1) = -JB(1,1,l) JB(0,1,l-1) - JB(2,1,l) JB(3,1,l-1)
    if (l > 0) { a[1][1] += -JB(0, 1, l - 1) * at2p; a[2][1] += -JB(3, 1, l - 1) * at2p; }
    // SchurSolveF: v3new(l) = r3/fac + JB(1,1,l) r0(l) + JB(1,0,l) r0(l+1) + JB(2,1,l) r4(l) + JB(2,0,l) r4(l+1)
    a[1][1] += y[l] * r0[l]; a[1][0] += y[l] * r0[l + 1];
    a[2][1] += y[l] * r4[l]; a[2][0] += y[l] * r4[l + 1];
    // SchurSolveB: JB(0,0,l) x(l) in v0'(l), JB(0,1,l) x(l) in v0'(l+1), JB(3,.) in v4'
    a[0][0] += av0[l] * x[l]; a[0][1] += av0[l + 1] * x[l];
    a[3][0] += av4[l] * x[l]; a[3][1] += av4[l + 1] * x[l];
    // bands of interface l from rho, rho*theta at l, l+1 (JacSchurKernel!)
    const double *V0 = Vn + (size_t)nz * g;
    const double RhoL = V0[l], RhoR = V0[l + 1];
    const double dzL = P.dz[l + (size_t)nz * g], dzR = P.dz[l + 1 + (size_t)nz * g], dzs = dzL + dzR;
    const double idzL = 1.0 / dzL, idzR = 1.0 / dzR, idzs = 1.0 / dzs, ih = 2.0 * idzs;
    const double iR = 1.0 / ((RhoL * dzL + RhoR * dzR) * idzs);   // 1 / RhoF
    // jb0 = -RhoF/dzL, jb1 = RhoF/dzR, jb4 = -dPR/RhoF/h, jb5 = dPL/RhoF/h, h = dzs/2,
    // jb2 = -g dzR/RhoF/dzs, jb3 = -g dzL/RhoF/dzs, jb6 = -RhoThF/dzL, jb7 = RhoThF/dzR
    const double aRhoF = -a[0][0] * idzL + a[0][1] * idzR + (a[2][0] * dP[l + 1] - a[2][1] * dP[l]) * iR * iR * ih +
                         (a[1][0] * dzR + a[1][1] * dzL) * P.Grav * iR * iR * idzs;
    const double adPR = -a[2][0] * iR * ih, adPL = a[2][1] * iR * ih;
    const double aThF = -a[3][0] * idzL + a[3][1] * idzR;
    accL0[it] = aRhoF * dzL * idzs;
    accL4[it] = aThF * dzL * idzs + adPL * dPd[l];
    aR0[l + 1] = aRhoF * dzR * idzs;
    aR4[l + 1] = aThF * dzR * idzs + adPR * dPd[l + 1];
  }
  __syncwarp();
#pragma unroll
  for (int it = 0; it < 2; ++it) {
    const int l = lane + 32 * it;
    if (l >= nz) continue;
    const size_t o0 = l + (size_t)nz * g;
    const double r0s = l > 0 ? aR0[l] : 0.0, r4s = l > 0 ? aR4[l] : 0.0;
    LV[o0] += accL0[it] + r0s;
    LV[o0 + 4 * fs] += accL4[it] + r4s;
  }
#undef JB
}

}  // namespace cgd
