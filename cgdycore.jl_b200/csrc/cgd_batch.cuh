// cgd_batch.cuh - batched ensemble: the members of an ensemble (grids of any
// nPanel and nz that share the polynomial order and the tracer count) advance
// together, one launch per kernel of a Rosenbrock-W stage over a flat work
// list that spans every member.
//
// A work item is (member, block x, block y) of the member's own launch grid;
// the kernel bodies are the single-member ones, given the member's
// parameters from constant memory.  One ensemble step is one CUDA graph of
// 15 launches, whatever the number of members.
#pragma once
#include "cgd_phase2.cuh"

namespace cgd {

constexpr int BMAX = 64;   // members of one ensemble

struct BMember {
  double *U;                     // the member's state (device), updated in place
  double *Vst, *k1, *k2, *C, *T1, *jbg;
  double *P0, *Pst;              // pressure of the state and of the stage state
  double dt;
};

struct WItem {
  int m, x, y;
};

__constant__ GP c_bgp[BMAX];
__constant__ BMember c_bm[BMAX];
__constant__ RK c_brk;

template <int N, int NT, typename R>
__global__ void __launch_bounds__(256, 4) kb_hypervisc1(const WItem *__restrict__ w, const int stage)
{
  const WItem it = w[blockIdx.x];
  const BMember &B = c_bm[it.m];
  hypervisc1_body<N, NT, R>(c_bgp[it.m], stage == 0 ? B.U : B.Vst, B.C, it.x, it.y);
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

template <int N, int NT, typename R>
__global__ void __launch_bounds__(P2Cfg<N, NT, R>::THREADS, P2Cfg<N, NT, R>::MINB) kb_phase2(const WItem *__restrict__ w, const int stage)
{
  const WItem it = w[blockIdx.x];
  const BMember &B = c_bm[it.m];
  phase2_body<N, NT, R>(c_bgp[it.m], stage == 0 ? B.U : B.Vst, stage == 0 ? B.P0 : B.Pst, B.T1, B.C, it.x, it.y);
}

template <int MODE, bool C32>
__global__ void __launch_bounds__(32 * COL_WARPS, MODE == 2 ? 3 : 4) kb_column(const WItem *__restrict__ w)
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
  a.bands = nullptr;
  a.dt = B.dt;
  a.fac = B.dt * c_brk.gamma;
  a.rk = c_brk;
  if (MODE == 0) { a.kout = B.k1; a.Vout = B.Vst; }
  else if (MODE == 1) { a.kout = B.k2; a.Vout = B.Vst; }
  else { a.kout = nullptr; a.Vout = B.U; }
  column_body<MODE, C32>(c_bgp[it.m], a, it.x);
}

}  // namespace cgd
