// cgd_batch.cuh - batched ensemble: the members of an ensemble (grids of any
// nPanel and nz that share the polynomial order and the tracer count) advance
// together, one launch per kernel of a Rosenbrock-W stage over a flat work
// list that spans every member.
//
// A work item is (member, block x, block y) of the member's own launch grid;
// the kernel bodies are the single-member ones, given the member's
// parameters from constant memory.  One ensemble step is one CUDA graph of
// 15 launches, whatever the number of members.
//
// The fused form (kb_stage, p = 4) runs a whole stage - pressure, phase 1,
// its DSS, phase 2, the column solve and update, the next stage's pressure -
// as one persistent cooperative launch whose CTAs walk the same work lists,
// with a grid barrier between the parts: one ensemble step is three
// launches.  Within one launch no array is read, rewritten and read again
// (phase 2 writes a second contribution buffer C2, the stage-3 state goes to
// a second stage buffer Vst2), so no CTA can read a line that an earlier part
// of the same launch left in its caches before another CTA rewrote it.
#pragma once
#include "cgd_phase2.cuh"

namespace cgd {

constexpr int BMAX = 64;   // members of one ensemble

struct BMember {
  double *U;                     // the member's state (device), updated in place
  double *Vst, *k1, *k2, *C, *T1, *jbg;
  double *P0, *Pst;              // pressure of the state and of the stage state
  double dt;
  double *C2, *Vst2;             // fused form only: phase-2 contributions, stage-3 state
};

struct WItem {
  int m, x, y;
};

__constant__ GP c_bgp[BMAX];
__constant__ BMember c_bm[BMAX];
__constant__ RK c_brk;

// Phase 1 of the split form, with the single-member kernel's level tile
// (HV1Tile) and its dynamic shared memory.
template <int N, int NT, typename R>
__global__ void __launch_bounds__(HV1Tile<N, R>::THREADS, HV1Tile<N, R>::MINB)
    kb_hypervisc1w(const WItem *__restrict__ w, const int stage)
{
  extern __shared__ __align__(16) unsigned char hvb_dyn[];
  const WItem it = w[blockIdx.x];
  const BMember &B = c_bm[it.m];
  hypervisc1_body<N, NT, R, HV1Tile<N, R>::LT>(c_bgp[it.m], stage == 0 ? B.U : B.Vst, B.C, it.x, it.y,
                                               reinterpret_cast<R *>(hvb_dyn));
}

__global__ void __launch_bounds__(256) kb_pressure(const WItem *__restrict__ w, const int stage_state)
{
  const WItem it = w[blockIdx.x];
  const BMember &B = c_bm[it.m];
  pressure_body(c_bgp[it.m], stage_state ? B.Vst : B.U, stage_state ? B.Pst : B.P0,
                (long long)it.x * blockDim.x + threadIdx.x);
}

template <bool C32>
__global__ void __launch_bounds__(256) kb_gather(const WItem *__restrict__ w)
{
  const WItem it = w[blockIdx.x];
  const BMember &B = c_bm[it.m];
  gather_body<false, true, C32>(c_bgp[it.m], B.C, B.T1, (long long)it.x * blockDim.x + threadIdx.x);
}

// W > 0: phase 2 in CTAs of W warps (levels, for p = 4) instead of the default
template <int N, int NT, typename R, int W = 0>
__global__ void __launch_bounds__(P2Cfg<N, NT, R, W>::THREADS, P2Cfg<N, NT, R, W>::MINB)
    kb_phase2(const WItem *__restrict__ w, const int stage)
{
  const WItem it = w[blockIdx.x];
  const BMember &B = c_bm[it.m];
  phase2_body<N, NT, R, W>(c_bgp[it.m], stage == 0 ? B.U : B.Vst, stage == 0 ? B.P0 : B.Pst, B.T1, B.C, it.x, it.y);
}

template <int MODE, bool C32>
__global__ void __launch_bounds__(32 * COL_WARPS, 4) kb_column(const WItem *__restrict__ w)
{
  const WItem it = w[blockIdx.x];
  const BMember &B = c_bm[it.m];
  ColArgs a;
  a.C = B.C;
  a.Vn = B.U;
  a.k1 = B.k1;
  a.k2 = B.k2;
  a.jbg = B.jbg;
  a.v = nullptr;
  a.jb4[0] = a.jb4[1] = a.jb4[2] = a.jb4[3] = nullptr;
  a.dt = B.dt;
  a.fac = B.dt * c_brk.gamma;
  a.rk = c_brk;
  a.Vs = MODE == 0 ? B.U : B.Vst;
  a.ps = MODE == 0 ? B.P0 : B.Pst;
  if (MODE == 0) { a.kout = B.k1; a.Vout = B.Vst; }
  else if (MODE == 1) { a.kout = B.k2; a.Vout = B.Vst; }
  else { a.kout = nullptr; a.Vout = B.U; }
  column_body<MODE, C32>(c_bgp[it.m], a, it.x);
}

// ---------------------------------------------------------------------------
// Fused stage kernel
// ---------------------------------------------------------------------------
// Grid barrier.  Every CTA is resident (cooperative launch).  Thread 0 of a
// CTA reads the generation, fences, and arrives on the counter; the last
// arrival resets the counter and publishes the next generation with a
// release store; the others poll it with acquire loads.  A wait longer than
// GBAR_NS (or GBAR_SPINS polls) records a timeout and the CTA leaves the
// kernel; the CTAs still waiting then time out in turn, so the launch ends
// and the host reports CGD_ERR_TIMEOUT.
struct GridBar {
  unsigned int count, gen;
  int timeout;
};
constexpr unsigned long long GBAR_NS = 5000000000ull;
constexpr unsigned int GBAR_SPINS = 1u << 26;

__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int *p)
{
  unsigned int v;
  asm volatile("ld.acquire.gpu.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u32(unsigned int *p, unsigned int v)
{
  asm volatile("st.release.gpu.u32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long globaltimer_ns()
{
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
  return t;
}

__device__ __forceinline__ bool grid_sync(GridBar *gb, unsigned long long limit_ns = GBAR_NS)
{
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    const unsigned int g0 = ld_acquire_u32(&gb->gen);
    __threadfence();
    if (atomicAdd(&gb->count, 1u) == gridDim.x - 1) {
      atomicExch(&gb->count, 0u);
      __threadfence();
      st_release_u32(&gb->gen, g0 + 1u);
    } else {
      const unsigned long long t0 = globaltimer_ns();
      for (unsigned int it = 0; ld_acquire_u32(&gb->gen) == g0; ++it) {
        if (it >= GBAR_SPINS || globaltimer_ns() - t0 > limit_ns) {
          atomicExch(&gb->timeout, 1);
          ok = 0;
          break;
        }
        __nanosleep(256);
      }
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// Check of the grid barrier: every CTA counts its arrival before each of
// `rounds` barriers; after barrier r, thread 0 of each CTA must see at least
// gridDim.x * (r + 1) arrivals, else it counts a violation.  A CTA whose wait
// timed out leaves (the barrier records the timeout).
__global__ void __launch_bounds__(256) k_barrier_probe(GridBar *gb, unsigned long long limit_ns, int rounds,
                                                       unsigned int *arrivals, int *violations)
{
  for (int r = 0; r < rounds; ++r) {
    if (threadIdx.x == 0) atomicAdd(arrivals, 1u);
    if (!grid_sync(gb, limit_ns)) return;
    if (threadIdx.x == 0 && ld_acquire_u32(arrivals) < gridDim.x * (unsigned)(r + 1)) atomicAdd(violations, 1);
  }
}

// work lists of the fused kernel: 0 phase-1 tiles, 1 blocks of 256
// column-levels (DSS gather, pressure), 2 phase-2 chunks (the default
// FUSED_P2_WARPS-warp CTAs), 3 blocks of COL_WARPS columns
constexpr int FUSED_P2_WARPS = 8;
// the split form's alternative phase-2 CTA for p = 4 (autotuner), work list 4
constexpr int P2_ALT_WARPS = 16;
struct FusedArgs {
  const WItem *w[5];
  int n[5];
  GridBar *bar;
};

__device__ __forceinline__ double *fused_stage_state(const BMember &B, int stage)
{
  return stage == 0 ? B.U : (stage == 1 ? B.Vst : B.Vst2);
}

// One Rosenbrock-W stage of every member in one launch of 256-thread CTAs,
// each walking the work lists with stride gridDim.x.
template <int N, int NT, typename R>
__global__ void __launch_bounds__(256, 2) kb_stage(const FusedArgs A, const int stage)
{
  constexpr bool C32 = sizeof(R) == sizeof(float);
  static_assert(P2Cfg<N, NT, R, FUSED_P2_WARPS>::THREADS == 256, "phase-2 chunks of 256 threads");
  static_assert(P2Cfg<N, NT, R, FUSED_P2_WARPS>::LC == P2Cfg<N, NT, R>::LC, "the default phase-2 work list");
  static_assert(32 * COL_WARPS == 256, "column blocks of 256 threads");
  extern __shared__ double fsm[];   // each part's shared arrays in turn (phase 1, phase 2, column)
  if (stage == 0) {   // pressure of the step's state
    for (int i = blockIdx.x; i < A.n[1]; i += gridDim.x) {
      const WItem it = A.w[1][i];
      const BMember &B = c_bm[it.m];
      pressure_body(c_bgp[it.m], B.U, B.P0, (long long)it.x * 256 + threadIdx.x);
    }
    if (!grid_sync(A.bar)) return;
  }
  // phase 1 of the hyperviscosity -> C
  for (int i = blockIdx.x; i < A.n[0]; i += gridDim.x) {
    const WItem it = A.w[0][i];
    const BMember &B = c_bm[it.m];
    hypervisc1_body<N, NT, R>(c_bgp[it.m], fused_stage_state(B, stage), B.C, it.x, it.y, reinterpret_cast<R *>(fsm));
    __syncthreads();   // the next item reuses the shared arrays
  }
  if (!grid_sync(A.bar)) return;
  // its DSS -> T1
  for (int i = blockIdx.x; i < A.n[1]; i += gridDim.x) {
    const WItem it = A.w[1][i];
    const BMember &B = c_bm[it.m];
    gather_body<false, true, C32>(c_bgp[it.m], B.C, B.T1, (long long)it.x * 256 + threadIdx.x);
  }
  if (!grid_sync(A.bar)) return;
  // phase 2 -> C2
  for (int i = blockIdx.x; i < A.n[2]; i += gridDim.x) {
    const WItem it = A.w[2][i];
    const BMember &B = c_bm[it.m];
    phase2_body<N, NT, R, FUSED_P2_WARPS>(c_bgp[it.m], fused_stage_state(B, stage), stage == 0 ? B.P0 : B.Pst,
                                          B.T1, B.C2, it.x, it.y);
    __syncthreads();
  }
  if (!grid_sync(A.bar)) return;
  // owner gather of phase 2, Jacobian, Schur solve, stage update
  for (int i = blockIdx.x; i < A.n[3]; i += gridDim.x) {
    const WItem it = A.w[3][i];
    const BMember &B = c_bm[it.m];
    ColArgs a;
    a.C = B.C2;
    a.Vn = B.U;
    a.k1 = B.k1;
    a.k2 = B.k2;
    a.jbg = B.jbg;
    a.v = nullptr;
    a.jb4[0] = a.jb4[1] = a.jb4[2] = a.jb4[3] = nullptr;
    a.dt = B.dt;
    a.fac = B.dt * c_brk.gamma;
    a.rk = c_brk;
    a.Vs = fused_stage_state(B, stage);
    a.ps = stage == 0 ? B.P0 : B.Pst;
    if (stage == 0) {
      a.kout = B.k1; a.Vout = B.Vst;
      column_body<0, C32>(c_bgp[it.m], a, it.x);
    } else if (stage == 1) {
      a.kout = B.k2; a.Vout = B.Vst2;
      column_body<1, C32>(c_bgp[it.m], a, it.x);
    } else {
      a.kout = nullptr; a.Vout = B.U;
      column_body<2, C32>(c_bgp[it.m], a, it.x);
    }
    __syncthreads();
  }
  if (stage == 2) return;
  if (!grid_sync(A.bar)) return;
  // pressure of the next stage state
  for (int i = blockIdx.x; i < A.n[1]; i += gridDim.x) {
    const WItem it = A.w[1][i];
    const BMember &B = c_bm[it.m];
    pressure_body(c_bgp[it.m], stage == 0 ? B.Vst : B.Vst2, B.Pst, (long long)it.x * 256 + threadIdx.x);
  }
}

}  // namespace cgd
