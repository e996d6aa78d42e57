// cgd_b200.cu - C ABI of the B200 hot path (see include/cgd_b200.h).
//
// Host-side runtime: validates the caller's grid, builds the owner-gather
// maps and the compact element metric once, owns the device work buffers and
// the stream, and drives the kernels.  One Rosenbrock-W step (3 stages x
// {hyperviscosity + DSS, tendency + DSS, fused column stage}) is captured
// once into a CUDA graph and replayed per step.
#include "../../include/cgd_b200.h"
#include "cgd_kernels.cuh"
#include "cgd_phase2.cuh"
#include "cgd_batch.cuh"
#include "cgd_init.cuh"
#include "cgd_output.cuh"
#include "cgd_adjoint_launch.h"

#include <cuda_runtime.h>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <chrono>
#include <mutex>
#include <string>
#include <vector>

using namespace cgd;

namespace {

constexpr int NPROF = 15;   // kernels per step whose durations are recorded

struct Buf {
  void *p = nullptr;
  size_t bytes = 0;
};

}  // namespace

// What the reverse of one Rosenbrock-W step reads: the stage states, their
// DSS'd phase-1 caches and pressures, the stage k and the Jacobian bands of
// the step's initial state u0.
struct StepTape {
  double *U0 = nullptr, *V2 = nullptr, *V3 = nullptr, *T1[3] = {}, *P[3] = {};
  double *k[3] = {}, *jbg = nullptr;
  const double *u0 = nullptr;   // the initial state (U0, or the caller's array)
  double dt = 0.0;
  bool recorded = false;
  std::vector<void *> mem;      // owned device buffers
};

struct cgd_handle {
  cgd_config cfg{};
  int N = 0, DoF = 0, nz = 0, NF = 0, NumG = 0, NumTr = 0, NV = 0;
  int device = 0;
  cudaStream_t stream = nullptr;
  // Work the caller queued before a call is ordered before the call's own
  // work: every entry records order_ev on the caller's stream (the legacy
  // default stream unless cgd_set_caller_stream names another) and makes the
  // library's stream wait for it.
  cudaStream_t caller = cudaStreamLegacy;
  cudaEvent_t order_ev = nullptr;
  std::vector<Buf> bufs;
  double *met = nullptr, *M = nullptr, *dz = nullptr;
  int *glob = nullptr, *inv_ptr = nullptr;
  long long *inv_off = nullptr, *inv_tab = nullptr;
  double *C = nullptr, *T1 = nullptr, *Vst = nullptr, *k1 = nullptr, *k2 = nullptr;
  double *Ubuf = nullptr, *Fbuf = nullptr, *bands = nullptr, *part = nullptr, *scal = nullptr;
  double *jbg = nullptr;   // Jacobian bands of the current step, [8][NumG][nz-1]
  double *pres = nullptr, *pres_st = nullptr;   // pressure of the state and of the stage state
  double *aLF = nullptr, *aLU = nullptr, *aLT1 = nullptr;   // adjoint buffers (allocated on first use)
  // step adjoint workspace: stage states, stage tendencies, k adjoints, ...
  double *aLk[2] = {}, *aAR = nullptr, *aLV = nullptr, *aLt = nullptr;
  StepTape work_tape;              // cgd_ros_step_adjoint's own replay
  std::vector<StepTape> tapes;     // cgd_tape_record_step slots
  double *mmass = nullptr;
  int *flag = nullptr;
  GP gp{};
  RK rk{};
  bool have_bands = false;
  // step graph
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  double *graph_U = nullptr;
  double graph_dt = 0.0;
  // profiling events (recorded inside the graph when CGD_PROFILE is set)
  bool profile = false;
  bool capturing = false;
  cudaEvent_t ev[NPROF + 1] = {};
  // mixed form: FP32 horizontal derivative sums around an FP64 reference
  // profile (the horizontal mean of the first state the handle sees)
  bool mix = false, have_ref = false;
  double *pref = nullptr, *thref = nullptr;
  // column physics (cgd_set_physics)
  std::vector<int> glob_host;                   // 0-based Glob, kept for the per-column set-up
  double *coslat = nullptr, *sinlat = nullptr, *dampc = nullptr;
  // horizontal domain decomposition (cgd_create_part): this rank's halo
  bool decomposed = false;
  int nghost = 0, nsend = 0;
  std::vector<int32_t> nb_rank, send_ptr, recv_ptr;
  int *send_list = nullptr;                     // device copy
  // elements [0, nbnd) touch other ranks (all sent contributions are theirs);
  // the interior's phase 1 and phase 2 run on `side` while the boundary's
  // contributions are exchanged
  int nbnd = 0;
  cudaStream_t side = nullptr;
  cudaEvent_t xa = nullptr, xb = nullptr;
  // element range of the next phase-1 / phase-2 launch ([el0, el0 + neln), all when neln < 0)
  int el0 = 0, neln = -1;
  double *sbuf = nullptr, *rbuf = nullptr;      // packed contributions, NC*nz per item
  cgd_exchange_fn xfn = nullptr;
  void *xuser = nullptr;
  // output interpolation (allocated on first use): the weights, staged host
  // inputs and staged host output
  double *ointer = nullptr, *ostage = nullptr, *ocell = nullptr;
  size_t ocell_n = 0;
  std::string last_error;
};

namespace {

// Band scratch of the allocation-free Schur solve (cgd_jac_schur_solve_noalloc).
__device__ __align__(256) double g_noalloc_scratch[CGD_NOALLOC_SCRATCH_DOUBLES];
constexpr int NOALLOC_MAX_DEVICES = 64;
double *g_noalloc_ptr[NOALLOC_MAX_DEVICES] = {};
std::mutex g_noalloc_mu;

thread_local std::string g_last_error;

int cuda_fail(cgd_handle *h, cudaError_t e, const char *what)
{
  char buf[256];
  snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
  g_last_error = buf;
  if (h) h->last_error = buf;
  return CGD_ERR_CUDA;
}

#define CK(call)                                         \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return cuda_fail(h, e_, #call); \
  } while (0)

// True the first time a call site asks on the current device (the site's
// own mask); launch attributes such as the dynamic shared-memory limit are
// per device.
bool first_on_device(std::atomic<unsigned long long> &done)
{
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return true;
  const unsigned long long bit = 1ull << dev;
  return !(done.fetch_or(bit) & bit);
}

template <typename T>
int dalloc(cgd_handle *h, T **p, size_t count)
{
  size_t bytes = count * sizeof(T);
  if (bytes == 0) bytes = sizeof(T);
  void *q = nullptr;
  CK(cudaMalloc(&q, bytes));
  h->bufs.push_back(Buf{q, bytes});
  *p = static_cast<T *>(q);
  return CGD_OK;
}

bool is_device_ptr(const void *p)
{
  cudaPointerAttributes a;
  cudaError_t e = cudaPointerGetAttributes(&a, p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}


// The element range of a phase-1 or phase-2 launch: all elements, or the
// range the decomposed step set (cgd_handle::el0, neln).
GP ranged_gp(const cgd_handle *h, int &nIF)
{
  GP gp = h->gp;
  nIF = h->neln < 0 ? h->NF : h->neln;
  gp.IF0 = h->neln < 0 ? 0 : h->el0;
  return gp;
}

template <int N, int NT, typename R>
void launch_hv1r(cgd_handle *h, const double *U, double *C)
{
  using T = HV1Tile<N, R>;
  constexpr size_t smem = HV1Smem<N, NT, R, T::LT>::BYTES;
  static std::atomic<unsigned long long> attr{0};
  if (first_on_device(attr))
    cudaFuncSetAttribute(k_hypervisc1<N, NT, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int nIF;
  const GP gp = ranged_gp(h, nIF);
  if (nIF <= 0) return;
  dim3 grid((h->nz + T::LT - 1) / T::LT, nIF);   // the level tiles of one element run back to back
  k_hypervisc1<N, NT, R><<<grid, T::THREADS, smem, h->stream>>>(gp, U, C);
}

template <int N, int NT>
void launch_hv1t(cgd_handle *h, const double *U, double *C)
{
  if (h->mix) launch_hv1r<N, NT, float>(h, U, C);
  else launch_hv1r<N, NT, double>(h, U, C);
}

template <int N>
void launch_hv1(cgd_handle *h, const double *U, double *C)
{
  switch (h->NumTr) {
    case 0: launch_hv1t<N, 0>(h, U, C); break;
    case 1: launch_hv1t<N, 1>(h, U, C); break;
    case 2: launch_hv1t<N, 2>(h, U, C); break;
    case 3: launch_hv1t<N, 3>(h, U, C); break;
    default: launch_hv1t<N, 4>(h, U, C); break;
  }
}

template <int N, int NT, typename R>
void launch_p2r(cgd_handle *h, const double *U, const double *Pr, const double *T1, double *C)
{
  using CF = P2Cfg<N, NT, R>;
  static std::atomic<unsigned long long> attr{0};
  if (first_on_device(attr)) {
    cudaFuncSetAttribute(k_phase2<N, NT, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CF::SMEM);
  }
  int nIF;
  const GP gp = ranged_gp(h, nIF);
  if (nIF <= 0) return;
  dim3 grid((h->nz + CF::LC - 1) / CF::LC, nIF);
  k_phase2<N, NT, R><<<grid, CF::THREADS, CF::SMEM, h->stream>>>(gp, U, Pr, T1, C);
}

template <int N, int NT>
void launch_p2(cgd_handle *h, const double *U, const double *Pr, const double *T1, double *C)
{
  if (h->mix) launch_p2r<N, NT, float>(h, U, Pr, T1, C);
  else launch_p2r<N, NT, double>(h, U, Pr, T1, C);
}

template <int N>
void launch_p2(cgd_handle *h, const double *U, const double *Pr, const double *T1, double *C)
{
  switch (h->NumTr) {
    case 0: launch_p2<N, 0>(h, U, Pr, T1, C); break;
    case 1: launch_p2<N, 1>(h, U, Pr, T1, C); break;
    case 2: launch_p2<N, 2>(h, U, Pr, T1, C); break;
    case 3: launch_p2<N, 3>(h, U, Pr, T1, C); break;
    default: launch_p2<N, 4>(h, U, Pr, T1, C); break;
  }
}

void hv1(cgd_handle *h, const double *U, double *C)
{
  switch (h->N) {
    case 2: launch_hv1<2>(h, U, C); break;
    case 3: launch_hv1<3>(h, U, C); break;
    case 4: launch_hv1<4>(h, U, C); break;
    default: launch_hv1<5>(h, U, C); break;
  }
}

void phase2(cgd_handle *h, const double *U, const double *Pr, const double *T1, double *C)
{
  switch (h->N) {
    case 2: launch_p2<2>(h, U, Pr, T1, C); break;
    case 3: launch_p2<3>(h, U, Pr, T1, C); break;
    case 4: launch_p2<4>(h, U, Pr, T1, C); break;
    default: launch_p2<5>(h, U, Pr, T1, C); break;
  }
}

void pressure(cgd_handle *h, const double *U, double *p)
{
  const long long n = (long long)h->nz * h->NumG;
  k_pressure<<<(unsigned)((n + 255) / 256), 256, 0, h->stream>>>(h->gp, U, p);
}

// The column physics added to a tendency (no launch when none is set).
void physics(cgd_handle *h, const double *U, const double *p, double *F)
{
  if (!h->gp.held_suarez && !h->gp.damping) return;
  const long long n = (long long)h->nz * h->NumG;
  k_physics<<<(unsigned)((n + 255) / 256), 256, 0, h->stream>>>(h->gp, U, p, F);
}

// wsplit: the phase-2 tendency (w split into two contributions, FP64 output);
// otherwise phase 1, whose output is the cache (stored like the contributions)
// or, with tendency_out, an FP64 array for the caller.
void gather(cgd_handle *h, const double *C, double *out, bool wsplit, bool tendency_out = false)
{
  long long n = (long long)h->nz * h->NumG;
  const unsigned nb = (unsigned)((n + 255) / 256);
  if (h->mix) {
    if (wsplit) k_gather<true, false, true><<<nb, 256, 0, h->stream>>>(h->gp, C, out);
    else if (tendency_out) k_gather<false, false, true><<<nb, 256, 0, h->stream>>>(h->gp, C, out);
    else k_gather<false, true, true><<<nb, 256, 0, h->stream>>>(h->gp, C, out);
  } else {
    if (wsplit) k_gather<true, false, false><<<nb, 256, 0, h->stream>>>(h->gp, C, out);
    else if (tendency_out) k_gather<false, false, false><<<nb, 256, 0, h->stream>>>(h->gp, C, out);
    else k_gather<false, true, false><<<nb, 256, 0, h->stream>>>(h->gp, C, out);
  }
}

template <int MODE, bool C32>
void column_t(cgd_handle *h, const ColArgs &a)
{
  size_t smem = (size_t)COL_WARPS * COL_ARR * h->nz * sizeof(double);
  static std::atomic<unsigned long long> attr{0};
  if (first_on_device(attr)) {   // up to 8 warps x 15 arrays x 64 levels
    cudaFuncSetAttribute(k_column<MODE, C32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         COL_WARPS * COL_ARR * 64 * (int)sizeof(double));
  }
  k_column<MODE, C32><<<(h->NumG + COL_WARPS - 1) / COL_WARPS, 32 * COL_WARPS, smem, h->stream>>>(h->gp, a);
}

template <int MODE>
void column(cgd_handle *h, const ColArgs &a)
{
  if (h->mix) column_t<MODE, true>(h, a);
  else column_t<MODE, false>(h, a);
}

// Event between two kernels of a step launched without the graph (the
// profiled step, see cgd_ros_step).
void rec(cgd_handle *h, int i)
{
  if (h->profile && !h->capturing && i >= 0 && i <= NPROF) cudaEventRecord(h->ev[i], h->stream);
}

// Arguments of the column stages of one SSP-Knoth step of U.
ColArgs step_args(cgd_handle *h, double *U, double dt)
{
  ColArgs a{};
  a.Vn = U;
  a.k1 = h->k1;
  a.k2 = h->k2;
  a.dt = dt;
  a.fac = dt * h->rk.gamma;
  a.rk = h->rk;
  a.C = h->C;
  a.jbg = h->jbg;
  return a;
}

// The three pieces of a Rosenbrock-W stage, split at the two direct-stiffness
// summations (where a decomposed grid exchanges element contributions):
//   piece 0: (stage 1: the pressure of the step's state) phase 1 -> C
//   piece 1: DSS of phase 1 -> T1, phase 2 -> C
//   piece 2: column stage (DSS of phase 2, solve, update), then the pressure
//            of the next stage state
// e counts the profiling events of the single-process step.
void stage_piece(cgd_handle *h, double *U, const ColArgs &a0, int stage, int piece, int &e)
{
  const double *Vsrc = stage == 0 ? U : h->Vst;
  if (piece == 0) {
    if (stage == 0) {
      pressure(h, U, h->pres);
      rec(h, e++);
    }
    hv1(h, Vsrc, h->C);
    rec(h, e++);
  } else if (piece == 1) {
    gather(h, h->C, h->T1, false);
    rec(h, e++);
    phase2(h, Vsrc, stage == 0 ? h->pres : h->pres_st, h->T1, h->C);
    rec(h, e++);
  } else {
    ColArgs a = a0;
    a.Vs = Vsrc;
    a.ps = stage == 0 ? h->pres : h->pres_st;
    if (stage == 0) {
      a.kout = h->k1; a.Vout = h->Vst;
      column<0>(h, a);
      rec(h, e++);
      pressure(h, h->Vst, h->pres_st);
    } else if (stage == 1) {
      a.kout = h->k2; a.Vout = h->Vst;
      column<1>(h, a);
      rec(h, e++);
      pressure(h, h->Vst, h->pres_st);
    } else {
      a.kout = nullptr; a.Vout = U;
      column<2>(h, a);
    }
    rec(h, e++);
  }
}

// One SSP-Knoth step on device state U (in place).
void enqueue_step(cgd_handle *h, double *U, double dt)
{
  const ColArgs a = step_args(h, U, dt);
  int e = 0;
  rec(h, e++);
  for (int stage = 0; stage < 3; ++stage)
    for (int piece = 0; piece < 3; ++piece) stage_piece(h, U, a, stage, piece, e);
}

// ---- decomposed grids: packing, unpacking and the exchange of contributions
// Pack the first nf contribution slots of the element nodes in send_list
// (item j at j*nf*nz, field f at +f*nz).
__global__ void __launch_bounds__(256) k_halo_pack(const double *__restrict__ C, double *__restrict__ sbuf,
                                                   const int *__restrict__ list, int n, int nf, int DoF, int NC,
                                                   int nz)
{
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * nf * nz) return;
  const int item = (int)(t / ((long long)nf * nz));
  const int r = (int)(t - (long long)item * nf * nz);
  const int f = r / nz, l = r - f * nz;
  const int c = list[item], IF = c / DoF, ID = c - IF * DoF;
  sbuf[t] = C[(((size_t)IF * NC + f) * DoF + ID) * nz + l];
}
// Unpack received contributions into the ghost slots of C: slot j is node
// j % DoF of the pseudo-element NF + j / DoF.
__global__ void __launch_bounds__(256) k_halo_unpack(const double *__restrict__ rbuf, double *__restrict__ C, int n,
                                                     int NF, int nf, int DoF, int NC, int nz)
{
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * nf * nz) return;
  const int j = (int)(t / ((long long)nf * nz));
  const int r = (int)(t - (long long)j * nf * nz);
  const int f = r / nz, l = r - f * nz;
  const int pe = NF + j / DoF, node = j % DoF;
  C[(((size_t)pe * NC + f) * DoF + node) * nz + l] = rbuf[t];
}

void halo_pack(cgd_handle *h, int nf)
{
  const long long n = (long long)h->nsend * nf * h->nz;
  if (n) k_halo_pack<<<(unsigned)((n + 255) / 256), 256, 0, h->stream>>>(h->C, h->sbuf, h->send_list, h->nsend, nf,
                                                                         h->DoF, h->NV + 1, h->nz);
}
void halo_unpack(cgd_handle *h, int nf)
{
  const long long n = (long long)h->nghost * nf * h->nz;
  if (n) k_halo_unpack<<<(unsigned)((n + 255) / 256), 256, 0, h->stream>>>(h->rbuf, h->C, h->nghost, h->NF, nf,
                                                                           h->DoF, h->NV + 1, h->nz);
}

// The exchange of one DSS point among the ranks of an in-process group (all
// on one stream): rank r's ghost slots from neighbour s are s's packed
// segment for r, copied device to device.
int group_exchange(cgd_handle *const *parts, int n, int nf, cudaStream_t st)
{
  for (int r = 0; r < n; ++r) {
    cgd_handle *h = parts[r];
    for (size_t i = 0; i < h->nb_rank.size(); ++i) {
      const int sr = h->nb_rank[i];
      const cgd_handle *q = parts[sr];
      size_t j = 0;
      while (j < q->nb_rank.size() && q->nb_rank[j] != r) ++j;
      const size_t per = (size_t)nf * h->nz;
      const size_t cnt = (size_t)(h->recv_ptr[i + 1] - h->recv_ptr[i]) * per;
      if (!cnt) continue;
      cudaError_t e = cudaMemcpyAsync(h->rbuf + (size_t)h->recv_ptr[i] * per, q->sbuf + (size_t)q->send_ptr[j] * per,
                                      cnt * sizeof(double), cudaMemcpyDeviceToDevice, st);
      if (e != cudaSuccess) return cuda_fail(h, e, "group exchange");
    }
  }
  return CGD_OK;
}

// The exchange of one DSS point through the caller's transport (one process
// per rank).
int callback_exchange(cgd_handle *h, int nf)
{
  if (h->nb_rank.empty()) return CGD_OK;
  if (!h->xfn) {
    g_last_error = "decomposed grid without an exchange function (cgd_set_exchange)";
    return CGD_ERR_INVALID_ARG;
  }
  const int rc = h->xfn(h->xuser, (void *)h->stream, nf, h->sbuf, h->rbuf);
  if (rc) {
    g_last_error = "the exchange function failed";
    return CGD_ERR_CUDA;
  }
  return CGD_OK;
}

// One step (or, with rhs_only, one tendency into F) of every part of a
// decomposed grid, the parts' pieces interleaved with the exchanges.  n > 1:
// an in-process group on parts[0]'s stream; n == 1: one rank of a
// multi-process run, exchanging through its callback.  At both DSS points
// the boundary elements' kernel runs first on the main stream, whose packing
// and exchange then follow, while the interior elements' kernel runs on the
// side stream; the main stream waits for it before the gather.
int part_pieces(cgd_handle *const *parts, int n, double *const *U, double dt, bool rhs_only, double *const *F)
{
  cgd_handle *h0 = parts[0];
  cgd_handle *h = h0;   // for CK()
  const int nf1 = 5 + h0->NumTr, nf2 = h0->NV + 1;
  bool interior = false;
  for (int r = 0; r < n; ++r) interior = interior || parts[r]->nbnd < parts[r]->NF;
  if (interior && !h0->side) {
    CK(cudaStreamCreateWithFlags(&h0->side, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&h0->xa, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&h0->xb, cudaEventDisableTiming));
  }
  auto xchg = [&](int nf) -> int {
    for (int r = 0; r < n; ++r) halo_pack(parts[r], nf);
    int rc = n > 1 ? group_exchange(parts, n, nf, h0->stream) : callback_exchange(h0, nf);
    if (rc) return rc;
    for (int r = 0; r < n; ++r) halo_unpack(parts[r], nf);
    return CGD_OK;
  };
  // kern(r) launches part r's phase-1 or phase-2 kernel on its stream over
  // its current element range
  auto split = [&](int nf, auto &&kern) -> int {
    if (!interior) {
      for (int r = 0; r < n; ++r) kern(r);
      return xchg(nf);
    }
    const cudaStream_t main = h0->stream;
    CK(cudaEventRecord(h0->xa, main));
    CK(cudaStreamWaitEvent(h0->side, h0->xa, 0));
    for (int r = 0; r < n; ++r) {   // boundary elements, main stream
      parts[r]->el0 = 0;
      parts[r]->neln = parts[r]->nbnd;
      kern(r);
    }
    for (int r = 0; r < n; ++r) {   // interior elements, side stream
      cgd_handle *q = parts[r];
      q->el0 = q->nbnd;
      q->neln = q->NF - q->nbnd;
      q->stream = h0->side;
      kern(r);
      q->stream = main;
      q->neln = -1;
    }
    CK(cudaEventRecord(h0->xb, h0->side));
    if (int rc = xchg(nf)) return rc;
    CK(cudaStreamWaitEvent(main, h0->xb, 0));
    return CGD_OK;
  };
  if (rhs_only) {
    if (int rc = split(nf1, [&](int r) { hv1(parts[r], U[r], parts[r]->C); })) return rc;
    for (int r = 0; r < n; ++r) {
      cgd_handle *q = parts[r];
      gather(q, q->C, q->T1, false);
      pressure(q, U[r], q->pres);
    }
    if (int rc = split(nf2, [&](int r) { phase2(parts[r], U[r], parts[r]->pres, parts[r]->T1, parts[r]->C); }))
      return rc;
    for (int r = 0; r < n; ++r) {
      gather(parts[r], parts[r]->C, F[r], true);
      physics(parts[r], U[r], parts[r]->pres, F[r]);
    }
    return CGD_OK;
  }
  std::vector<ColArgs> a(n);
  for (int r = 0; r < n; ++r) a[r] = step_args(parts[r], U[r], dt);
  int e = 0;
  for (int stage = 0; stage < 3; ++stage) {
    auto vsrc = [&](int r) -> const double * { return stage == 0 ? U[r] : parts[r]->Vst; };
    if (stage == 0)
      for (int r = 0; r < n; ++r) pressure(parts[r], U[r], parts[r]->pres);
    if (int rc = split(nf1, [&](int r) { hv1(parts[r], vsrc(r), parts[r]->C); })) return rc;
    for (int r = 0; r < n; ++r) gather(parts[r], parts[r]->C, parts[r]->T1, false);
    auto p2 = [&](int r) {
      cgd_handle *q = parts[r];
      phase2(q, vsrc(r), stage == 0 ? q->pres : q->pres_st, q->T1, q->C);
    };
    if (int rc = split(nf2, p2)) return rc;
    for (int r = 0; r < n; ++r) stage_piece(parts[r], U[r], a[r], stage, 2, e);
  }
  return CGD_OK;
}

// Mixed form: the reference profile from the first state (before any capture).
void ensure_ref(cgd_handle *h, const double *Ud)
{
  if (!h->mix || h->have_ref) return;
  k_refprof<<<h->nz, 256, 0, h->stream>>>(h->gp, Ud, h->pref, h->thref);
  h->have_ref = true;
}

void free_graph(cgd_handle *h)
{
  if (h->gexec) cudaGraphExecDestroy(h->gexec);
  if (h->graph) cudaGraphDestroy(h->graph);
  h->gexec = nullptr;
  h->graph = nullptr;
  h->graph_U = nullptr;
}

int check_cfg(const cgd_config *c)
{
  if (!c) return CGD_ERR_INVALID_ARG;
  if (c->OrdPoly < 1 || c->OrdPoly > 4) return CGD_ERR_UNSUPPORTED;
  if (c->nz < 2 || c->nz > 64) return CGD_ERR_UNSUPPORTED;
  if (c->NumTr < 0 || c->NumTr > MAXTR) return CGD_ERR_UNSUPPORTED;
  if (c->NF <= 0 || c->NumG <= 0) return CGD_ERR_SHAPE;
  if (c->precision != CGD_PREC_FP64 && c->precision != CGD_PREC_MIXED) return CGD_ERR_INVALID_ARG;
  if (!(c->Rd > 0) || !(c->Cpd > c->Rd) || !(c->p0 > 0) || !(c->Grav > 0)) return CGD_ERR_INVALID_ARG;
  return CGD_OK;
}

}  // namespace

extern "C" {

const char *cgd_version(void)
{
#ifdef CGD_FAST
  return "cgd_b200 1.0 fast (sm_100a, FP64 owner-gather DSS, -fmad=false, reciprocal mass/Jacobian/density)";
#else
  return "cgd_b200 1.0 exact (sm_100a, FP64 owner-gather DSS, -fmad=false, bit-identical to the CPU restatement)";
#endif
}

const char *cgd_strerror(int code)
{
  switch (code) {
    case CGD_OK: return "ok";
    case CGD_ERR_INVALID_ARG: return "invalid argument";
    case CGD_ERR_SHAPE: return "extents inconsistent with the grid";
    case CGD_ERR_CUDA: return g_last_error.empty() ? "CUDA runtime error" : g_last_error.c_str();
    case CGD_ERR_NONFINITE: return "non-finite value in the state";
    case CGD_ERR_TIMEOUT: return "bounded device wait timed out";
    case CGD_ERR_INDEX: return "Glob index out of range or global DOF without element";
    case CGD_ERR_UNSUPPORTED: return "option not supported by this build";
    case CGD_ERR_NO_DEVICE: return "no usable CUDA device";
    default: return "unknown error";
  }
}

static int create_impl(const cgd_config *cfg, const int64_t *glob, const double *DS, const double *DW,
                       const double *dXdxI, const double *J, const double *X, const double *M, const double *dz,
                       const cgd_halo *halo, cgd_handle **out);

int cgd_create(const cgd_config *cfg, const int64_t *glob, const double *DS, const double *DW,
               const double *dXdxI, const double *J, const double *X, const double *M,
               const double *dz, cgd_handle **out)
{
  return create_impl(cfg, glob, DS, DW, dXdxI, J, X, M, dz, nullptr, out);
}

int cgd_create_part(const cgd_config *cfg, const int64_t *glob, const double *DS, const double *DW,
                    const double *dXdxI, const double *J, const double *X, const double *M, const double *dz,
                    const cgd_halo *halo, cgd_handle **out)
{
  if (!halo) return CGD_ERR_INVALID_ARG;
  return create_impl(cfg, glob, DS, DW, dXdxI, J, X, M, dz, halo, out);
}

static int create_impl(const cgd_config *cfg, const int64_t *glob, const double *DS, const double *DW,
                       const double *dXdxI, const double *J, const double *X, const double *M, const double *dz,
                       const cgd_halo *halo, cgd_handle **out)
{
  if (!out) return CGD_ERR_INVALID_ARG;
  *out = nullptr;
  int rc = check_cfg(cfg);
  if (rc) return rc;
  if (!glob || !DS || !DW || !dXdxI || !J || !X || !M || !dz) return CGD_ERR_INVALID_ARG;
  if (halo) {
    // the decomposed grid exchanges FP64 contributions
    if (cfg->precision != CGD_PREC_FP64) return CGD_ERR_UNSUPPORTED;
    if (halo->nnb < 0 || (halo->nnb > 0 && (!halo->nb_rank || !halo->send_ptr || !halo->send_list ||
                                            !halo->recv_ptr)) ||
        !halo->contrib_ptr || !halo->contrib)
      return CGD_ERR_INVALID_ARG;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return CGD_ERR_NO_DEVICE;
  }
  cgd_handle *h = new cgd_handle();
  h->cfg = *cfg;
  h->N = cfg->OrdPoly + 1;
  h->DoF = h->N * h->N;
  h->nz = cfg->nz;
  h->NF = cfg->NF;
  h->NumG = cfg->NumG;
  h->NumTr = cfg->NumTr;
  h->NV = 5 + cfg->NumTr;
  const int DoF = h->DoF, nz = h->nz, NF = h->NF, NumG = h->NumG, NV = h->NV, N = h->N;
  cudaGetDevice(&h->device);

  // ---- owner-gather map: contributors of each global DOF, ascending (IF, ID)
  std::vector<int> cnt(NumG + 1, 0);
  for (size_t i = 0; i < (size_t)DoF * NF; ++i) {
    int64_t g = glob[i];
    if (g < 1 || g > NumG) { delete h; return CGD_ERR_INDEX; }
    cnt[g] += 1;
  }
  std::vector<int> ptr(NumG + 1, 0);
  for (int g = 0; g < NumG; ++g) {
    if (cnt[g + 1] == 0) { delete h; return CGD_ERR_INDEX; }
    ptr[g + 1] = ptr[g] + cnt[g + 1];
  }
  std::vector<long long> off(ptr[NumG]);
  std::vector<int> fill(ptr.begin(), ptr.end() - 1);
  std::vector<int> glob0((size_t)DoF * NF);
  for (int IF = 0; IF < NF; ++IF)
    for (int ID = 0; ID < DoF; ++ID) {
      int g = (int)glob[ID + (size_t)DoF * IF] - 1;
      glob0[ID + (size_t)DoF * IF] = g;
      off[fill[g]++] = ((long long)IF * (NV + 1) * DoF + ID) * nz;
    }
  // a decomposed grid: the contributor lists come from the halo plan, in
  // ascending global (element, node) order, local element nodes and ghost
  // slots (the contributions received from the neighbours) interleaved
  int nghost = 0, nsend = 0;
  if (halo) {
    const int nnb = halo->nnb;
    nghost = nnb ? halo->recv_ptr[nnb] : 0;
    nsend = nnb ? halo->send_ptr[nnb] : 0;
    if (nghost < 0 || nsend < 0) { delete h; return CGD_ERR_INVALID_ARG; }
    for (int i = 0; i < nnb; ++i)
      if (halo->recv_ptr[i + 1] < halo->recv_ptr[i] || halo->send_ptr[i + 1] < halo->send_ptr[i]) {
        delete h;
        return CGD_ERR_INVALID_ARG;
      }
    for (int i = 0; i < nsend; ++i)
      if (halo->send_list[i] < 0 || halo->send_list[i] >= DoF * NF) { delete h; return CGD_ERR_INDEX; }
    if (halo->contrib_ptr[0] != 0) { delete h; return CGD_ERR_INVALID_ARG; }
    std::vector<int> p2(NumG + 1);
    for (int g = 0; g <= NumG; ++g) {
      p2[g] = halo->contrib_ptr[g];
      if (g && (p2[g] <= p2[g - 1])) { delete h; return CGD_ERR_INDEX; }   // every DOF has a contributor
    }
    std::vector<long long> o2(p2[NumG]);
    for (int q = 0; q < p2[NumG]; ++q) {
      const int c = halo->contrib[q];
      if (c >= 0) {
        if (c >= DoF * NF) { delete h; return CGD_ERR_INDEX; }
        o2[q] = ((long long)(c / DoF) * (NV + 1) * DoF + c % DoF) * nz;
      } else {
        const int j = -1 - c;
        if (j >= nghost) { delete h; return CGD_ERR_INDEX; }
        o2[q] = ((long long)(NF + j / DoF) * (NV + 1) * DoF + j % DoF) * nz;
      }
    }
    ptr.swap(p2);
    off.swap(o2);
    h->decomposed = true;
    h->nghost = nghost;
    h->nsend = nsend;
    // the interior overlaps the exchanges only when every sent contribution
    // is a boundary element's
    h->nbnd = NF;
    if (halo->nb_boundary >= 0 && halo->nb_boundary <= NF) {
      bool ok = true;
      for (int i = 0; i < nsend; ++i) ok = ok && halo->send_list[i] / DoF < halo->nb_boundary;
      if (ok) h->nbnd = halo->nb_boundary;
    }
    h->nb_rank.assign(halo->nb_rank, halo->nb_rank + nnb);
    h->send_ptr.assign(halo->send_ptr, halo->send_ptr + nnb + 1);
    h->recv_ptr.assign(halo->recv_ptr, halo->recv_ptr + nnb + 1);
    if (!nnb) {
      h->send_ptr.assign(1, 0);
      h->recv_ptr.assign(1, 0);
    }
  }

  // ---- compact metric [IF][comp][ID][nz]: on the host, or on the device
  // (k_compact_metric, the same expressions) when the reference-layout
  // metric is device memory
  const size_t ENL = (size_t)DoF * nz * NF;
  const bool dev_metric = is_device_ptr(dXdxI) && is_device_ptr(J) && is_device_ptr(X);
  std::vector<double> met(dev_metric ? 0 : ENL * NCOMP);
  const double Omega2 = 2.0 * cfg->Omega;
  for (int IF = 0; IF < (dev_metric ? 0 : NF); ++IF)
    for (int ID = 0; ID < DoF; ++ID)
      for (int Iz = 0; Iz < nz; ++Iz) {
        auto dx = [&](int a, int b, int K) {
          return dXdxI[(size_t)(a - 1) + 3 * ((b - 1) + 3 * (K + 2 * (ID + (size_t)DoF * (Iz + (size_t)nz * IF))))];
        };
        auto jj = [&](int K) { return J[ID + (size_t)DoF * (K + 2 * (Iz + (size_t)nz * IF))]; };
        auto xx = [&](int K, int c) { return X[ID + (size_t)DoF * (K + 2 * (c + 3 * (Iz + (size_t)nz * IF)))]; };
        double v[NCOMP];
        v[C_D11_0] = dx(1, 1, 0); v[C_D11_1] = dx(1, 1, 1);
        v[C_D12_0] = dx(1, 2, 0); v[C_D12_1] = dx(1, 2, 1);
        v[C_D21_0] = dx(2, 1, 0); v[C_D21_1] = dx(2, 1, 1);
        v[C_D22_0] = dx(2, 2, 0); v[C_D22_1] = dx(2, 2, 1);
        v[C_D31_0] = dx(3, 1, 0); v[C_D31_1] = dx(3, 1, 1);
        v[C_D32_0] = dx(3, 2, 0); v[C_D32_1] = dx(3, 2, 1);
        v[C_D33_0] = dx(3, 3, 0); v[C_D33_1] = dx(3, 3, 1);
        v[C_J0] = jj(0); v[C_J1] = jj(1);
        // CoriolisShallow at the layer midpoint (src/GPU/Coriolis.jl:18-28,
        // src/GPU/MomentumKernel.jl:156-159)
        double x = 0.5 * (xx(0, 0) + xx(1, 0));
        double y = 0.5 * (xx(0, 1) + xx(1, 1));
        double z = 0.5 * (xx(0, 2) + xx(1, 2));
        double sinlat = z / std::sqrt(x * x + y * y + z * z);
        v[C_FCOR] = Omega2 * sinlat;
        // RecU4 (src/GPU/OperatorKernel.jl:1044-1059): the J-only factors of the
        // interface between Iz and Iz+1, with the column-end clamping of
        // DivRhoTrUpwind3New2Kernel! (OperatorKernel.jl:667-683)
        v[C_RK0] = v[C_RK1] = v[C_RK2] = v[C_RK3] = 0.0;
        if (Iz < nz - 1) {
          auto js = [&](int lev) {
            return J[ID + (size_t)DoF * (0 + 2 * (lev + (size_t)nz * IF))] +
                   J[ID + (size_t)DoF * (1 + 2 * (lev + (size_t)nz * IF))];
          };
          double JLL = js(Iz > 0 ? Iz - 1 : 0), JL = js(Iz), JR = js(Iz + 1), JRR = js(Iz + 2 < nz ? Iz + 2 : nz - 1);
          v[C_RK0] = (JL / (JL + JR)) * ((JLL + JL) / (JLL + JL + JR));
          v[C_RK1] = (JL / (JLL + JL)) * (JR / (JLL + JL + JR));
          v[C_RK2] = (JR / (JR + JL)) * ((JRR + JR) / (JL + JR + JRR));
          v[C_RK3] = (JR / (JRR + JR)) * (JL / (JL + JR + JRR));
        }
        for (int c = 0; c < NCOMP; ++c) met[(((size_t)IF * NCOMP + c) * DoF + ID) * nz + Iz] = v[c];
      }

  // ---- device resources
  if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->order_ev, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return CGD_ERR_CUDA;
  }
  const size_t S = (size_t)nz * NumG;
#define TRY(x) do { int r_ = (x); if (r_) { cgd_destroy(h); return r_; } } while (0)
  TRY(dalloc(h, &h->met, ENL * NCOMP));
  TRY(dalloc(h, &h->M, 2 * S));
  TRY(dalloc(h, &h->dz, S));
  TRY(dalloc(h, &h->glob, glob0.size()));
  TRY(dalloc(h, &h->inv_ptr, ptr.size()));
  TRY(dalloc(h, &h->inv_off, off.size()));
  // the first four contributors of every DOF in one 32-byte row (-1 past the
  // count; a DOF with more than four is marked -1 in its first entry)
  std::vector<long long> tab((size_t)4 * NumG, -1);
  for (int g = 0; g < NumG; ++g)
    if (ptr[g + 1] - ptr[g] <= 4)
      for (int q = ptr[g]; q < ptr[g + 1]; ++q) tab[(size_t)4 * g + (q - ptr[g])] = off[q];
  TRY(dalloc(h, &h->inv_tab, tab.size()));
  // contribution buffer: the local elements, then the ghost pseudo-elements
  const size_t ghost_elems = ((size_t)nghost + DoF - 1) / DoF;
  TRY(dalloc(h, &h->C, ENL * (NV + 1) + ghost_elems * DoF * nz * (NV + 1)));
  if (halo) {
    TRY(dalloc(h, &h->send_list, (size_t)std::max(nsend, 1)));
    TRY(dalloc(h, &h->sbuf, (size_t)std::max(nsend, 1) * (NV + 1) * nz));
    TRY(dalloc(h, &h->rbuf, (size_t)std::max(nghost, 1) * (NV + 1) * nz));
  }
  TRY(dalloc(h, &h->T1, S * NV));
  TRY(dalloc(h, &h->Vst, S * NV));
  TRY(dalloc(h, &h->k1, S * NV));
  TRY(dalloc(h, &h->k2, S * NV));
  TRY(dalloc(h, &h->Ubuf, S * NV));
  TRY(dalloc(h, &h->Fbuf, S * NV));
  TRY(dalloc(h, &h->bands, 8 * (size_t)(nz - 1) * NumG));
  TRY(dalloc(h, &h->jbg, 8 * (size_t)(nz - 1) * NumG));
  TRY(dalloc(h, &h->pres, S));
  TRY(dalloc(h, &h->pres_st, S));
  h->mix = cfg->precision == CGD_PREC_MIXED;
  TRY(dalloc(h, &h->pref, nz));
  TRY(dalloc(h, &h->thref, nz));
  TRY(dalloc(h, &h->part, 1024));
  TRY(dalloc(h, &h->scal, 4));
  TRY(dalloc(h, &h->mmass, S));
  TRY(dalloc(h, &h->flag, 4));
  // host or device sources (unified addressing tells them apart)
  auto up = [&](void *dst, const void *src, size_t bytes) {
    return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, h->stream);
  };
  if (dev_metric) {
    const long long n = (long long)ENL;
    k_compact_metric<<<(unsigned)((n + 255) / 256), 256, 0, h->stream>>>(DoF, nz, NF, Omega2, dXdxI, J, X, h->met);
  }
  if ((!dev_metric && up(h->met, met.data(), met.size() * 8)) || cudaGetLastError() != cudaSuccess || up(h->M, M, 2 * S * 8) || up(h->dz, dz, S * 8) ||
      up(h->glob, glob0.data(), glob0.size() * 4) || up(h->inv_ptr, ptr.data(), ptr.size() * 4) ||
      up(h->inv_off, off.data(), off.size() * 8) || up(h->inv_tab, tab.data(), tab.size() * 8) ||
      (halo && nsend && up(h->send_list, halo->send_list, (size_t)nsend * 4))) {
    cudaError_t e = cudaGetLastError();
    cuda_fail(h, e, "cgd_create upload");
    cgd_destroy(h);
    return CGD_ERR_CUDA;
  }
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) {
    cuda_fail(h, cudaGetLastError(), "cgd_create sync");
    cgd_destroy(h);
    return CGD_ERR_CUDA;
  }

  h->glob_host = glob0;
  GP &P = h->gp;
  P.N = N; P.DoF = DoF; P.nz = nz; P.NF = NF; P.NumG = NumG; P.NumTr = h->NumTr; P.NV = NV; P.NC = NV + 1;
  P.met = h->met; P.M = h->M; P.dz = h->dz; P.glob = h->glob; P.inv_ptr = h->inv_ptr; P.inv_off = h->inv_off;
  P.inv_tab = h->inv_tab;
  P.pref = h->pref; P.thref = h->thref;
  for (int i = 0; i < 25; ++i) { P.D[i] = 0.0; P.DW[i] = 0.0; }
  for (int i = 0; i < N * N; ++i) { P.D[i] = DS[i]; P.DW[i] = DW[i]; }
  P.Grav = cfg->Grav; P.Rd = cfg->Rd; P.p0 = cfg->p0; P.kappa = cfg->Rd / cfg->Cpd;
  P.nuCurl = cfg->HyperDCurl; P.nuGrad = cfg->HyperDGrad; P.nuDiv = cfg->HyperDDiv;

  // SSP-Knoth: a = alpha/Gamma, c = -inv(Gamma), m = Gamma'\b (RosenbrockMethod.jl:26-47)
  RK &r = h->rk;
  memset(&r, 0, sizeof r);
  r.a[1][0] = 1.0; r.a[2][0] = 0.25; r.a[2][1] = 0.25;
  r.c[1][0] = 0.0; r.c[2][0] = -0.75; r.c[2][1] = -0.75;
  double b1 = 1.0 / 6.0, b2 = 1.0 / 6.0, b3 = 2.0 / 3.0;
  r.m[2] = b3 / 1.0;
  r.m[1] = (b2 - (-0.75) * r.m[2]) / 1.0;
  r.m[0] = (b1 - (-0.75) * r.m[2]) / 1.0;
  r.gamma = 1.0;

  const char *pe = getenv("CGD_PROFILE");
  h->profile = pe && pe[0] == '1';
  if (h->profile)
    for (int i = 0; i <= NPROF; ++i) cudaEventCreate(&h->ev[i]);

#undef TRY
  *out = h;
  return CGD_OK;
}

void cgd_destroy(cgd_handle *h)
{
  if (!h) return;
  if (h->stream) cudaStreamSynchronize(h->stream);
  free_graph(h);
  for (auto &b : h->bufs) cudaFree(b.p);
  for (void *q : h->work_tape.mem) cudaFree(q);
  for (auto &t : h->tapes)
    for (void *q : t.mem) cudaFree(q);
  for (int i = 0; i <= NPROF; ++i)
    if (h->ev[i]) cudaEventDestroy(h->ev[i]);
  if (h->order_ev) cudaEventDestroy(h->order_ev);
  if (h->xa) cudaEventDestroy(h->xa);
  if (h->xb) cudaEventDestroy(h->xb);
  if (h->side) cudaStreamDestroy(h->side);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

// Order the call after the caller's queued work (see cgd_handle::caller).
static int enter(cgd_handle *h)
{
  CK(cudaEventRecord(h->order_ev, h->caller));
  CK(cudaStreamWaitEvent(h->stream, h->order_ev, 0));
  return CGD_OK;
}

// Stage a state/tendency pointer: device pointers are used in place, host
// pointers are copied into the handle's buffer (in == true) first.
static int stage_in(cgd_handle *h, const double *p, double *buf, bool copy, double **dev)
{
  if (is_device_ptr(p)) {
    *dev = const_cast<double *>(p);
    return CGD_OK;
  }
  if (copy) CK(cudaMemcpyAsync(buf, p, (size_t)h->nz * h->NumG * h->NV * 8, cudaMemcpyHostToDevice, h->stream));
  *dev = buf;
  return CGD_OK;
}

static int finish(cgd_handle *h)
{
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(h->stream));
  return CGD_OK;
}

int cgd_prepare(cgd_handle *h, const double *U, double *p)
{
  if (!h || !U || !p) return CGD_ERR_INVALID_ARG;
  if (int erc = enter(h)) return erc;
  double *Ud;
  int rc = stage_in(h, U, h->Ubuf, true, &Ud);
  if (rc) return rc;
  bool pdev = is_device_ptr(p);
  double *pd = pdev ? p : h->Fbuf;
  long long n = (long long)h->nz * h->NumG;
  k_pressure<<<(unsigned)((n + 255) / 256), 256, 0, h->stream>>>(h->gp, Ud, pd);
  if (!pdev) CK(cudaMemcpyAsync(p, pd, n * 8, cudaMemcpyDeviceToHost, h->stream));
  return finish(h);
}

int cgd_hypervisc_phase1(cgd_handle *h, const double *U, double *Temp1)
{
  if (!h || !U || !Temp1) return CGD_ERR_INVALID_ARG;
  if (int erc = enter(h)) return erc;
  double *Ud;
  int rc = stage_in(h, U, h->Ubuf, true, &Ud);
  if (rc) return rc;
  bool tdev = is_device_ptr(Temp1);
  double *td = tdev ? Temp1 : h->Fbuf;
  ensure_ref(h, Ud);
  hv1(h, Ud, h->C);
  gather(h, h->C, td, false, true);
  if (!tdev)
    CK(cudaMemcpyAsync(Temp1, td, (size_t)h->nz * h->NumG * h->NV * 8, cudaMemcpyDeviceToHost, h->stream));
  return finish(h);
}

int cgd_rhs(cgd_handle *h, const double *U, double *F)
{
  if (!h || !U || !F) return CGD_ERR_INVALID_ARG;
  if (int erc = enter(h)) return erc;
  double *Ud;
  int rc = stage_in(h, U, h->Ubuf, true, &Ud);
  if (rc) return rc;
  ensure_ref(h, Ud);
  bool fdev = is_device_ptr(F);
  double *fd = fdev ? F : h->Fbuf;
  if (h->decomposed) {   // one rank of a decomposed grid: exchange through the callback
    if ((rc = part_pieces(&h, 1, &Ud, 0.0, true, &fd))) return rc;
    if (!fdev) CK(cudaMemcpyAsync(F, fd, (size_t)h->nz * h->NumG * h->NV * 8, cudaMemcpyDeviceToHost, h->stream));
    return finish(h);
  }
  hv1(h, Ud, h->C);
  gather(h, h->C, h->T1, false);
  pressure(h, Ud, h->pres);
  phase2(h, Ud, h->pres, h->T1, h->C);
  gather(h, h->C, fd, true);
  physics(h, Ud, h->pres, fd);
  if (!fdev) CK(cudaMemcpyAsync(F, fd, (size_t)h->nz * h->NumG * h->NV * 8, cudaMemcpyDeviceToHost, h->stream));
  return finish(h);
}

// The four band arrays inside the handle's contiguous (4, 2, nz-1, NumG) buffer.
static Bands4 handle_bands(cgd_handle *h)
{
  const size_t bs = (size_t)2 * (h->nz - 1) * h->NumG;
  return Bands4{{h->bands, h->bands + bs, h->bands + 2 * bs, h->bands + 3 * bs}};
}

static void launch_jac(cgd_handle *h, const double *Ud, const Bands4 &out)
{
  const long long n = (long long)(h->nz - 1) * h->NumG;
  k_jac<<<(unsigned)((n + 255) / 256), 256, 0, h->stream>>>(h->gp, Ud, out);
}

int cgd_jac(cgd_handle *h, const double *U, double *bands)
{
  if (!h || !U) return CGD_ERR_INVALID_ARG;
  if (int erc = enter(h)) return erc;
  double *Ud;
  int rc = stage_in(h, U, h->Ubuf, true, &Ud);
  if (rc) return rc;
  launch_jac(h, Ud, handle_bands(h));
  if (bands) {
    size_t bytes = (size_t)8 * (h->nz - 1) * h->NumG * 8;
    CK(cudaMemcpyAsync(bands, h->bands, bytes, is_device_ptr(bands) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                       h->stream));
  }
  rc = finish(h);
  if (!rc) h->have_bands = true;
  return rc;
}

int cgd_jac_bands(cgd_handle *h, const double *U, double *JRhoW, double *JWRho, double *JWRhoTh, double *JRhoThW)
{
  if (!h || !U || !JRhoW || !JWRho || !JWRhoTh || !JRhoThW) return CGD_ERR_INVALID_ARG;
  if (int erc = enter(h)) return erc;
  double *Ud;
  int rc = stage_in(h, U, h->Ubuf, true, &Ud);
  if (rc) return rc;
  double *user[4] = {JRhoW, JWRho, JWRhoTh, JRhoThW};
  bool dev[4];
  for (int i = 0; i < 4; ++i) dev[i] = is_device_ptr(user[i]);
  // the handle's own bands (for cgd_schur_solve) and the caller's arrays
  const Bands4 hb = handle_bands(h);
  launch_jac(h, Ud, hb);
  const size_t bytes = (size_t)2 * (h->nz - 1) * h->NumG * 8;
  for (int i = 0; i < 4; ++i)
    CK(cudaMemcpyAsync(user[i], hb.b[i], bytes, dev[i] ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                       h->stream));
  rc = finish(h);
  if (!rc) h->have_bands = true;
  return rc;
}

// The column Schur solve (MODE 3) with the given band arrays.
static int schur_solve_with(cgd_handle *h, double *k, double *v, const Bands4 &b, double fac)
{
  double *vd, *kd;
  int rc = stage_in(h, v, h->Ubuf, true, &vd);
  if (rc) return rc;
  bool kdev = is_device_ptr(k);
  kd = kdev ? k : h->Fbuf;
  ColArgs a{};
  a.v = vd;
  a.kout = kd;
  for (int i = 0; i < 4; ++i) a.jb4[i] = b.b[i];
  a.fac = fac;
  a.dt = fac;
  column<3>(h, a);
  size_t bytes = (size_t)h->nz * h->NumG * h->NV * 8;
  if (!kdev) CK(cudaMemcpyAsync(k, kd, bytes, cudaMemcpyDeviceToHost, h->stream));
  if (vd != v) CK(cudaMemcpyAsync(v, vd, bytes, cudaMemcpyDeviceToHost, h->stream));
  return finish(h);
}

int cgd_schur_solve(cgd_handle *h, double *k, double *v, double fac)
{
  if (!h || !k || !v || !(fac > 0)) return CGD_ERR_INVALID_ARG;
  if (!h->have_bands) return CGD_ERR_INVALID_ARG;
  if (int erc = enter(h)) return erc;
  return schur_solve_with(h, k, v, handle_bands(h), fac);
}

int cgd_schur_solve_bands(cgd_handle *h, double *k, double *v, const double *JRhoW, const double *JWRho,
                          const double *JWRhoTh, const double *JRhoThW, double fac)
{
  if (!h || !k || !v || !JRhoW || !JWRho || !JWRhoTh || !JRhoThW || !(fac > 0)) return CGD_ERR_INVALID_ARG;
  if (int erc = enter(h)) return erc;
  const double *user[4] = {JRhoW, JWRho, JWRhoTh, JRhoThW};
  Bands4 b = handle_bands(h);
  const size_t bytes = (size_t)2 * (h->nz - 1) * h->NumG * 8;
  for (int i = 0; i < 4; ++i) {
    if (is_device_ptr(user[i])) {
      b.b[i] = const_cast<double *>(user[i]);   // read only
    } else {
      // host bands are staged into the handle's band buffer, which then no
      // longer holds the last cgd_jac's bands
      CK(cudaMemcpyAsync(b.b[i], user[i], bytes, cudaMemcpyHostToDevice, h->stream));
      h->have_bands = false;
    }
  }
  return schur_solve_with(h, k, v, b, fac);
}

int cgd_ros_step(cgd_handle *h, double *U, double dt, int32_t nsteps)
{
  if (!h || !U || !(dt > 0) || nsteps < 0) return CGD_ERR_INVALID_ARG;
  if (int erc = enter(h)) return erc;
  double *Ud;
  int rc = stage_in(h, U, h->Ubuf, true, &Ud);
  if (rc) return rc;
  ensure_ref(h, Ud);
  if (h->decomposed) {   // one rank of a decomposed grid: steps with the callback's exchanges, not captured
    for (int s = 0; s < nsteps; ++s)
      if ((rc = part_pieces(&h, 1, &Ud, dt, false, nullptr))) return rc;
    if (Ud != U)
      CK(cudaMemcpyAsync(U, Ud, (size_t)h->nz * h->NumG * h->NV * 8, cudaMemcpyDeviceToHost, h->stream));
    return finish(h);
  }
  if (!h->gexec || h->graph_U != Ud || h->graph_dt != dt) {
    free_graph(h);
    CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    h->capturing = true;
    enqueue_step(h, Ud, dt);
    h->capturing = false;
    cudaError_t e = cudaStreamEndCapture(h->stream, &h->graph);
    if (e != cudaSuccess) return cuda_fail(h, e, "cudaStreamEndCapture");
    CK(cudaGraphInstantiate(&h->gexec, h->graph, 0));
    h->graph_U = Ud;
    h->graph_dt = dt;
  }
  // With CGD_PROFILE=1 the last step of the call is launched kernel by kernel
  // with events in between (same kernels, same stream), so the per-kernel
  // durations of that step can be read with cgd_kernel_times.
  const int ngraph = h->profile && nsteps > 0 ? nsteps - 1 : nsteps;
  for (int s = 0; s < ngraph; ++s) CK(cudaGraphLaunch(h->gexec, h->stream));
  if (ngraph < nsteps) enqueue_step(h, Ud, dt);
  if (h->cfg.flags & CGD_FLAG_CHECK_FINITE) {
    CK(cudaMemsetAsync(h->flag, 0, sizeof(int), h->stream));
    long long n = (long long)h->nz * h->NumG * h->NV;
    k_nonfinite<<<1184, 256, 0, h->stream>>>(Ud, n, h->flag);
  }
  if (Ud != U)
    CK(cudaMemcpyAsync(U, Ud, (size_t)h->nz * h->NumG * h->NV * 8, cudaMemcpyDeviceToHost, h->stream));
  rc = finish(h);
  if (rc) return rc;
  if (h->cfg.flags & CGD_FLAG_CHECK_FINITE) {
    int f = 0;
    CK(cudaMemcpy(&f, h->flag, sizeof(int), cudaMemcpyDeviceToHost));
    if (f) return CGD_ERR_NONFINITE;
  }
  return CGD_OK;
}

int cgd_set_physics(cgd_handle *h, const cgd_physics *ph, const double *X)
{
  if (!h || !ph) return CGD_ERR_INVALID_ARG;
  if (h->mix && (ph->held_suarez || ph->damping)) return CGD_ERR_UNSUPPORTED;
  if (ph->damping && !(ph->damp_stride > 0)) return CGD_ERR_INVALID_ARG;
  const int nz = h->nz, NumG = h->NumG, DoF = h->DoF, NF = h->NF;
  if ((ph->held_suarez || ph->damping) && !X) return CGD_ERR_INVALID_ARG;
  GP &P = h->gp;
  if (ph->held_suarez || ph->damping) {
    // positions (reference layout (N*N, 2, 3, nz, NF)), from the device if need be
    const size_t nx = (size_t)DoF * 6 * nz * NF;
    std::vector<double> xh;
    const double *Xh = X;
    if (is_device_ptr(X)) {
      xh.resize(nx);
      CK(cudaMemcpy(xh.data(), X, nx * 8, cudaMemcpyDeviceToHost));
      Xh = xh.data();
    }
    auto xx = [&](int ID, int K, int c, int Iz, int IF) {
      return Xh[ID + (size_t)DoF * (K + 2 * (c + 3 * (Iz + (size_t)nz * IF)))];
    };
    // per column, from its highest-numbered element node (the last to write
    // it): the surface latitude (MetricLowerBoundaryKernel!,
    // src/DyCore/DiscretizationCG.jl:159-178, cart2sphere
    // src/Grids/Geometry.jl:65-73) and the damping rate at the layer-midpoint
    // height zP (GridSizeSphereKernel!, DiscretizationCG.jl:119-144; DampingW,
    // src/GPU/dampingGPU.jl:1-19)
    std::vector<double> cl(NumG), sl(NumG), dc((size_t)nz * NumG, 0.0);
    const double pi = 3.141592653589793, Rad = ph->Rad;
    for (int IF = 0; IF < NF; ++IF)
      for (int ID = 0; ID < DoF; ++ID) {
        const int g = h->glob_host[ID + (size_t)DoF * IF];
        const double x = xx(ID, 0, 0, 0, IF), y = xx(ID, 0, 1, 0, IF), z = xx(ID, 0, 2, 0, IF);
        const double r = std::sqrt(x * x + y * y + z * z);
        const double lat = std::asin(z / r);
        cl[g] = std::cos(lat);
        sl[g] = std::sin(lat);
        for (int Iz = 0; Iz < nz; ++Iz) {
          const double xm = 0.5 * (xx(ID, 0, 0, Iz, IF) + xx(ID, 1, 0, Iz, IF));
          const double ym = 0.5 * (xx(ID, 0, 1, Iz, IF) + xx(ID, 1, 1, Iz, IF));
          const double zm = 0.5 * (xx(ID, 0, 2, Iz, IF) + xx(ID, 1, 2, Iz, IF));
          const double rm = std::sqrt(xm * xm + ym * ym + zm * zm);
          const double zP = std::max(rm - Rad, 0.0);
          double c = 0.0;
          if (ph->damping && zP >= ph->damp_H - ph->damp_stride) {
            const double sn = std::sin(0.5 * pi * (1.0 - (ph->damp_H - zP) / ph->damp_stride));
            c = ph->damp_relax * (sn * sn);
          }
          dc[Iz + (size_t)nz * g] = c;
        }
      }
    if (!h->coslat) {
      if (int rc = dalloc(h, &h->coslat, NumG)) return rc;
      if (int rc = dalloc(h, &h->sinlat, NumG)) return rc;
      if (int rc = dalloc(h, &h->dampc, (size_t)nz * NumG)) return rc;
    }
    CK(cudaMemcpy(h->coslat, cl.data(), NumG * 8, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(h->sinlat, sl.data(), NumG * 8, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(h->dampc, dc.data(), dc.size() * 8, cudaMemcpyHostToDevice));
  }
  P.held_suarez = ph->held_suarez ? 1 : 0;
  P.damping = ph->damping ? 1 : 0;
  const double hs[8] = {ph->k_a, ph->k_f, ph->k_s, ph->DeltaT_y, ph->DeltaTh_z, ph->T_equator, ph->T_min,
                        ph->sigma_b};
  for (int i = 0; i < 8; ++i) P.hs[i] = hs[i];
  P.coslat = h->coslat;
  P.sinlat = h->sinlat;
  P.dampc = h->dampc;
  free_graph(h);   // the captured step holds the old parameters
  return CGD_OK;
}

int cgd_metric_sphere(int32_t OrdPoly, int32_t nz, int32_t NF, const double *FP, const double *xw, const double *DS,
                      const double *z, double H, double Rad, double *X, double *dXdxI, double *J)
{
  cgd_handle *h = nullptr;   // for CK(): errors are reported through g_last_error
  if (OrdPoly < 1 || OrdPoly > 4 || nz < 1 || NF < 1) return CGD_ERR_UNSUPPORTED;
  if (!FP || !xw || !DS || !z || !X || !dXdxI || !J || !(H > 0) || !(Rad > 0)) return CGD_ERR_INVALID_ARG;
  if (!is_device_ptr(X) || !is_device_ptr(dXdxI) || !is_device_ptr(J)) return CGD_ERR_INVALID_ARG;
  const int N = OrdPoly + 1;
  const size_t nfp = (size_t)NF * 12, nin = nfp + N + N * N + nz + 1;
  double *buf = nullptr;
  CK(cudaMalloc(&buf, nin * sizeof(double)));
  double *dFP = buf, *dxw = dFP + nfp, *dDS = dxw + N, *dz = dDS + N * N;
  cudaError_t e = cudaMemcpy(dFP, FP, nfp * 8, cudaMemcpyDefault);
  if (e == cudaSuccess) e = cudaMemcpy(dxw, xw, (size_t)N * 8, cudaMemcpyDefault);
  if (e == cudaSuccess) e = cudaMemcpy(dDS, DS, (size_t)N * N * 8, cudaMemcpyDefault);
  if (e == cudaSuccess) e = cudaMemcpy(dz, z, (size_t)(nz + 1) * 8, cudaMemcpyDefault);
  if (e == cudaSuccess) {
    const long long n = (long long)NF * N * N;
    const unsigned nb = (unsigned)((n + 255) / 256);
    switch (N) {
      case 2: k_metric_sphere<2><<<nb, 256>>>(nz, NF, dFP, dxw, dDS, dz, H, Rad, X, dXdxI, J); break;
      case 3: k_metric_sphere<3><<<nb, 256>>>(nz, NF, dFP, dxw, dDS, dz, H, Rad, X, dXdxI, J); break;
      case 4: k_metric_sphere<4><<<nb, 256>>>(nz, NF, dFP, dxw, dDS, dz, H, Rad, X, dXdxI, J); break;
      default: k_metric_sphere<5><<<nb, 256>>>(nz, NF, dFP, dxw, dDS, dz, H, Rad, X, dXdxI, J); break;
    }
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
  }
  cudaFree(buf);
  if (e != cudaSuccess) return cuda_fail(h, e, "cgd_metric_sphere");
  return CGD_OK;
}

int cgd_mass_dz(int32_t OrdPoly, int32_t nz, int32_t NF, int32_t NumG, const int64_t *glob, const double *w,
                const double *J, const double *X, double *M, double *MMass, double *dz)
{
  cgd_handle *h = nullptr;
  if (OrdPoly < 1 || OrdPoly > 4 || nz < 1 || NF < 1 || NumG < 1) return CGD_ERR_UNSUPPORTED;
  if (!glob || !w || !J || !X || !M || !MMass || !dz) return CGD_ERR_INVALID_ARG;
  if (!is_device_ptr(J) || !is_device_ptr(X) || !is_device_ptr(M) || !is_device_ptr(MMass) || !is_device_ptr(dz))
    return CGD_ERR_INVALID_ARG;
  const int N = OrdPoly + 1, DoF = N * N;
  // contributors of each DOF in ascending (element, node) order
  std::vector<int> ptr(NumG + 1, 0), idx((size_t)DoF * NF);
  for (size_t i = 0; i < (size_t)DoF * NF; ++i) {
    const int64_t g = glob[i];
    if (g < 1 || g > NumG) return CGD_ERR_INDEX;
    ptr[g] += 1;
  }
  for (int g = 0; g < NumG; ++g) {
    if (ptr[g + 1] == 0) return CGD_ERR_INDEX;
    ptr[g + 1] += ptr[g];
  }
  std::vector<int> fill(ptr.begin(), ptr.end() - 1);
  for (size_t i = 0; i < (size_t)DoF * NF; ++i) idx[fill[glob[i] - 1]++] = (int)i;   // i = IF*DoF + ID, ascending
  int *dptr = nullptr;
  CK(cudaMalloc(&dptr, (ptr.size() + idx.size() + 1) * sizeof(int) + (size_t)N * sizeof(double)));
  int *didx = dptr + ptr.size();
  double *dw = reinterpret_cast<double *>(didx + idx.size() + (idx.size() + ptr.size()) % 2);
  cudaError_t e = cudaMemcpy(dptr, ptr.data(), ptr.size() * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(didx, idx.data(), idx.size() * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dw, w, (size_t)N * 8, cudaMemcpyDefault);
  if (e == cudaSuccess) {
    const long long n = (long long)nz * NumG;
    k_mass_dz<<<(unsigned)((n + 255) / 256), 256>>>(N, nz, NumG, dptr, didx, dw, J, X, M, MMass, dz);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
  }
  cudaFree(dptr);
  if (e != cudaSuccess) return cuda_fail(h, e, "cgd_mass_dz");
  return CGD_OK;
}

int cgd_set_exchange(cgd_handle *h, cgd_exchange_fn fn, void *user)
{
  if (!h || !h->decomposed) return CGD_ERR_INVALID_ARG;
  h->xfn = fn;
  h->xuser = user;
  return CGD_OK;
}

int cgd_halo_buffers(cgd_handle *h, double **send, int64_t *send_doubles, double **recv, int64_t *recv_doubles)
{
  if (!h || !h->decomposed || !send || !send_doubles || !recv || !recv_doubles) return CGD_ERR_INVALID_ARG;
  *send = h->sbuf;
  *recv = h->rbuf;
  *send_doubles = (int64_t)h->nsend * (h->NV + 1) * h->nz;
  *recv_doubles = (int64_t)h->nghost * (h->NV + 1) * h->nz;
  return CGD_OK;
}

// Checks of an in-process group: parts[r] is rank r, one device, ranks and
// exchange sizes consistent.  The parts then run on parts[0]'s stream.
static int group_enter(cgd_handle *const *parts, int32_t n, std::vector<cudaStream_t> &saved)
{
  if (!parts || n < 1) return CGD_ERR_INVALID_ARG;
  for (int r = 0; r < n; ++r) {
    cgd_handle *h = parts[r];
    if (!h || !h->decomposed || h->device != parts[0]->device || h->NV != parts[0]->NV || h->nz != parts[0]->nz)
      return CGD_ERR_INVALID_ARG;
    for (size_t i = 0; i < h->nb_rank.size(); ++i) {
      const int sr = h->nb_rank[i];
      if (sr < 0 || sr >= n || sr == r) return CGD_ERR_INVALID_ARG;
      const cgd_handle *q = parts[sr];
      size_t j = 0;
      while (j < q->nb_rank.size() && q->nb_rank[j] != r) ++j;
      if (j == q->nb_rank.size()) return CGD_ERR_INVALID_ARG;
      if (h->recv_ptr[i + 1] - h->recv_ptr[i] != q->send_ptr[j + 1] - q->send_ptr[j]) return CGD_ERR_SHAPE;
    }
  }
  for (int r = 0; r < n; ++r)
    if (int rc = enter(parts[r])) return rc;
  saved.resize(n);
  for (int r = 0; r < n; ++r) {
    saved[r] = parts[r]->stream;
    parts[r]->stream = parts[0]->stream;
  }
  // work queued on a part's own stream before the call comes first
  for (int r = 1; r < n; ++r) {
    cgd_handle *h = parts[r];
    cudaEventRecord(h->order_ev, saved[r]);
    cudaStreamWaitEvent(parts[0]->stream, h->order_ev, 0);
  }
  return CGD_OK;
}

static int group_leave(cgd_handle *const *parts, int32_t n, const std::vector<cudaStream_t> &saved, int rc)
{
  for (int r = 0; r < n && r < (int)saved.size(); ++r) parts[r]->stream = saved[r];
  if (rc) return rc;
  return finish(parts[0]);
}

int cgd_group_rhs(cgd_handle *const *parts, int32_t n, const double *const *U, double *const *F)
{
  if (!U || !F) return CGD_ERR_INVALID_ARG;
  for (int r = 0; r < n; ++r)
    if (!U[r] || !F[r] || !is_device_ptr(U[r]) || !is_device_ptr(F[r])) return CGD_ERR_INVALID_ARG;
  std::vector<cudaStream_t> saved;
  if (int rc = group_enter(parts, n, saved)) return rc;
  std::vector<double *> Ud(n);
  for (int r = 0; r < n; ++r) Ud[r] = const_cast<double *>(U[r]);
  const int rc = part_pieces(parts, n, Ud.data(), 0.0, true, F);
  return group_leave(parts, n, saved, rc);
}

int cgd_group_ros_step(cgd_handle *const *parts, int32_t n, double *const *U, double dt, int32_t nsteps)
{
  if (!U || !(dt > 0) || nsteps < 0) return CGD_ERR_INVALID_ARG;
  for (int r = 0; r < n; ++r)
    if (!U[r] || !is_device_ptr(U[r])) return CGD_ERR_INVALID_ARG;
  std::vector<cudaStream_t> saved;
  if (int rc = group_enter(parts, n, saved)) return rc;
  int rc = CGD_OK;
  for (int s = 0; s < nsteps && !rc; ++s) rc = part_pieces(parts, n, U, dt, false, nullptr);
  return group_leave(parts, n, saved, rc);
}

int cgd_mass_integral(cgd_handle *h, const double *U, const double *MMass, double *out)
{
  if (!h || !U || !MMass || !out) return CGD_ERR_INVALID_ARG;
  if (int erc = enter(h)) return erc;
  double *Ud;
  int rc = stage_in(h, U, h->Ubuf, true, &Ud);
  if (rc) return rc;
  const size_t S = (size_t)h->nz * h->NumG;
  const double *mm = MMass;
  if (!is_device_ptr(MMass)) {
    CK(cudaMemcpyAsync(h->mmass, MMass, S * 8, cudaMemcpyHostToDevice, h->stream));
    mm = h->mmass;
  }
  const int nb = 592;
  k_mass_partial<<<nb, 256, 0, h->stream>>>(Ud, mm, (long long)S, h->part);
  k_mass_final<<<1, 32, 0, h->stream>>>(h->part, nb, h->scal);
  CK(cudaMemcpyAsync(out, h->scal, 8, cudaMemcpyDeviceToHost, h->stream));
  return finish(h);
}

// ---- output interpolation (the reference's VTK output path)
int cgd_vtk_inter(int32_t OrdPoly, int32_t OrdPrint, const double *xw, double *inter)
{
  if (!xw || !inter || OrdPoly < 1 || OrdPoly > 4 || OrdPrint < 1 || OrdPrint > OUT_MAX_PRINT)
    return CGD_ERR_INVALID_ARG;
  const int N = OrdPoly + 1, OP = OrdPrint;
  // DG.Lagrange (src/DG/Lagrange.jl:1-9)
  auto lagrange = [&](double x, int iP) {
    double f = 1.0;
    for (int i = 0; i < N; ++i)
      if (i != iP) f = f * (x - xw[i]) / (xw[iP] - xw[i]);
    return f;
  };
  for (int i = 0; i < OP * OP * N * N; ++i) inter[i] = 0.0;
  // the sub-cell corners as vtkStruct steps them (src/Outputs/vtkSphere.jl:199-219)
  const double dd = 2.0 / OP;
  double eta0 = -1.0;
  for (int jRef = 0; jRef < OP; ++jRef) {
    double ksi0 = -1.0;
    const double eta1 = eta0 + dd;
    for (int iRef = 0; iRef < OP; ++iRef) {
      const double ksi1 = ksi0 + dd;
      for (int j = 0; j < N; ++j)
        for (int i = 0; i < N; ++i) {
          double &v = inter[iRef + OP * (jRef + OP * (i + N * j))];
          v = v + lagrange(0.5 * (ksi0 + ksi1), i) * lagrange(0.5 * (eta0 + eta1), j);
        }
      ksi0 = ksi1;
    }
    eta0 = eta1;
  }
  return CGD_OK;
}

namespace {

// Device copies for one interpolation call: the weights always (host or
// device), an (nz, NumG) input into staging slot `slot` when it is host
// memory.
int out_prepare(cgd_handle *h, const double *inter, int OP)
{
  if (OP < 1 || OP > OUT_MAX_PRINT) return CGD_ERR_INVALID_ARG;
  if (!h->ointer) {
    if (int rc = dalloc(h, &h->ointer, (size_t)OUT_MAX_PRINT * OUT_MAX_PRINT * 25)) return rc;
  }
  CK(cudaMemcpyAsync(h->ointer, inter, (size_t)OP * OP * h->DoF * 8, cudaMemcpyDefault, h->stream));
  return CGD_OK;
}

int out_input(cgd_handle *h, const double *a, int slot, const double **dev)
{
  if (!a || is_device_ptr(a)) {
    *dev = a;
    return CGD_OK;
  }
  const size_t S = (size_t)h->nz * h->NumG;
  if (!h->ostage) {
    if (int rc = dalloc(h, &h->ostage, 3 * S)) return rc;
  }
  CK(cudaMemcpyAsync(h->ostage + slot * S, a, S * 8, cudaMemcpyHostToDevice, h->stream));
  *dev = h->ostage + slot * S;
  return CGD_OK;
}

// Device destination for `count` doubles of cell values: the caller's
// pointer, or the handle's staging buffer for host memory.
int out_cells(cgd_handle *h, double *cell, size_t count, double **dev)
{
  if (is_device_ptr(cell)) {
    *dev = cell;
    return CGD_OK;
  }
  if (h->ocell_n < count) {
    if (h->ocell) {
      CK(cudaStreamSynchronize(h->stream));
      for (size_t i = 0; i < h->bufs.size(); ++i)
        if (h->bufs[i].p == h->ocell) {
          cudaFree(h->ocell);
          h->bufs.erase(h->bufs.begin() + i);
          break;
        }
      h->ocell = nullptr;
      h->ocell_n = 0;
    }
    if (int rc = dalloc(h, &h->ocell, count)) return rc;
    h->ocell_n = count;
  }
  *dev = h->ocell;
  return CGD_OK;
}

size_t out_count(const cgd_handle *h, int OP) { return (size_t)OP * OP * h->nz * h->NF; }

unsigned out_blocks(const cgd_handle *h, int OP) { return (unsigned)((out_count(h, OP) + 255) / 256); }

void launch_vort(cgd_handle *h, const double *U, int OP, double *cell)
{
  const int N = h->N, LT = 256 / (N * N);
  const dim3 grid((h->nz + LT - 1) / LT, h->NF);
  switch (N) {
    case 2: k_interp_vort<2><<<grid, 256, 0, h->stream>>>(h->gp, U, h->ointer, OP, cell); break;
    case 3: k_interp_vort<3><<<grid, 256, 0, h->stream>>>(h->gp, U, h->ointer, OP, cell); break;
    case 4: k_interp_vort<4><<<grid, 256, 0, h->stream>>>(h->gp, U, h->ointer, OP, cell); break;
    default: k_interp_vort<5><<<grid, 256, 0, h->stream>>>(h->gp, U, h->ointer, OP, cell); break;
  }
}

}  // namespace

int cgd_interpolate(cgd_handle *h, const double *c, const double *rhoc, const double *inter, int32_t OrdPrint,
                    double *cCell)
{
  if (!h || !c || !inter || !cCell) return CGD_ERR_INVALID_ARG;
  if (int erc = enter(h)) return erc;
  if (int rc = out_prepare(h, inter, OrdPrint)) return rc;
  const double *cd, *rd;
  double *od;
  if (int rc = out_input(h, c, 0, &cd)) return rc;
  if (int rc = out_input(h, rhoc, 1, &rd)) return rc;
  const size_t n = out_count(h, OrdPrint);
  if (int rc = out_cells(h, cCell, n, &od)) return rc;
  k_interp<<<out_blocks(h, OrdPrint), 256, 0, h->stream>>>(h->gp, cd, rd, INTERP_C, h->ointer, OrdPrint, od);
  if (od != cCell) CK(cudaMemcpyAsync(cCell, od, n * 8, cudaMemcpyDeviceToHost, h->stream));
  return finish(h);
}

int cgd_interpolate_wb(cgd_handle *h, const double *u, const double *v, const double *w, const double *inter,
                       int32_t OrdPrint, double *cCell)
{
  if (!h || !u || !v || !w || !inter || !cCell) return CGD_ERR_INVALID_ARG;
  if (int erc = enter(h)) return erc;
  if (int rc = out_prepare(h, inter, OrdPrint)) return rc;
  const double *ud, *vd, *wd;
  double *od;
  if (int rc = out_input(h, u, 0, &ud)) return rc;
  if (int rc = out_input(h, v, 1, &vd)) return rc;
  if (int rc = out_input(h, w, 2, &wd)) return rc;
  const size_t n = out_count(h, OrdPrint);
  if (int rc = out_cells(h, cCell, n, &od)) return rc;
  k_interp_wb<<<out_blocks(h, OrdPrint), 256, 0, h->stream>>>(h->gp, ud, vd, wd, h->ointer, OrdPrint, od);
  if (od != cCell) CK(cudaMemcpyAsync(cCell, od, n * 8, cudaMemcpyDeviceToHost, h->stream));
  return finish(h);
}

int cgd_interpolate_vort(cgd_handle *h, const double *U, const double *inter, int32_t OrdPrint, double *cCell)
{
  if (!h || !U || !inter || !cCell) return CGD_ERR_INVALID_ARG;
  if (int erc = enter(h)) return erc;
  if (int rc = out_prepare(h, inter, OrdPrint)) return rc;
  double *Ud, *od;
  if (int rc = stage_in(h, U, h->Ubuf, true, &Ud)) return rc;
  const size_t n = out_count(h, OrdPrint);
  if (int rc = out_cells(h, cCell, n, &od)) return rc;
  launch_vort(h, Ud, OrdPrint, od);
  if (od != cCell) CK(cudaMemcpyAsync(cCell, od, n * 8, cudaMemcpyDeviceToHost, h->stream));
  return finish(h);
}

int cgd_output_fields(cgd_handle *h, const double *U, const int32_t *fields, int32_t nfields, const double *inter,
                      int32_t OrdPrint, double *out)
{
  if (!h || !U || !fields || nfields < 1 || !inter || !out) return CGD_ERR_INVALID_ARG;
  for (int k = 0; k < nfields; ++k) {
    const int f = fields[k];
    const bool ok = (f >= CGD_OUT_RHO && f <= CGD_OUT_WB_UV) || (f >= CGD_OUT_TR && f < CGD_OUT_TR + h->NumTr);
    if (!ok) return CGD_ERR_INVALID_ARG;
  }
  if (int erc = enter(h)) return erc;
  if (int rc = out_prepare(h, inter, OrdPrint)) return rc;
  double *Ud, *od;
  if (int rc = stage_in(h, U, h->Ubuf, true, &Ud)) return rc;
  const size_t n = out_count(h, OrdPrint);
  if (int rc = out_cells(h, out, n * nfields, &od)) return rc;
  const size_t fs = (size_t)h->nz * h->NumG;
  const double *rho = Ud, *u = Ud + fs, *v = Ud + 2 * fs, *w = Ud + 3 * fs, *rth = Ud + 4 * fs;
  const unsigned nb = out_blocks(h, OrdPrint);
  const double *W = h->ointer;
  for (int k = 0; k < nfields; ++k) {
    double *cell = od + (size_t)k * n;
    const int f = fields[k];
    switch (f) {
      case CGD_OUT_RHO: k_interp<<<nb, 256, 0, h->stream>>>(h->gp, rho, nullptr, INTERP_C, W, OrdPrint, cell); break;
      case CGD_OUT_U: k_interp<<<nb, 256, 0, h->stream>>>(h->gp, u, nullptr, INTERP_C, W, OrdPrint, cell); break;
      case CGD_OUT_V: k_interp<<<nb, 256, 0, h->stream>>>(h->gp, v, nullptr, INTERP_C, W, OrdPrint, cell); break;
      case CGD_OUT_WB: k_interp_wb<<<nb, 256, 0, h->stream>>>(h->gp, u, u, w, W, OrdPrint, cell); break;
      case CGD_OUT_WB_UV: k_interp_wb<<<nb, 256, 0, h->stream>>>(h->gp, u, v, w, W, OrdPrint, cell); break;
      case CGD_OUT_TH: k_interp<<<nb, 256, 0, h->stream>>>(h->gp, rth, rho, INTERP_POTT, W, OrdPrint, cell); break;
      case CGD_OUT_PRES: k_interp<<<nb, 256, 0, h->stream>>>(h->gp, rth, nullptr, INTERP_PRES, W, OrdPrint, cell); break;
      case CGD_OUT_VORT: launch_vort(h, Ud, OrdPrint, cell); break;
      default:   // tracer ratio rho*q / rho
        k_interp<<<nb, 256, 0, h->stream>>>(h->gp, Ud + (size_t)(5 + f - CGD_OUT_TR) * fs, rho, INTERP_C, W, OrdPrint,
                                            cell);
        break;
    }
  }
  if (od != out) CK(cudaMemcpyAsync(out, od, n * nfields * 8, cudaMemcpyDeviceToHost, h->stream));
  return finish(h);
}

int cgd_jac_schur_solve_noalloc(const cgd_config *cfg, const double *U, const double *dz,
                                double *k, double *v, double fac, void *stream)
{
  cgd_handle *h = nullptr;   // for CK(): errors are reported through g_last_error
  if (!cfg || !U || !dz || !k || !v || !(fac > 0)) return CGD_ERR_INVALID_ARG;
  if (cfg->nz < 2 || cfg->nz > 64 || cfg->NumTr < 0 || cfg->NumTr > MAXTR) return CGD_ERR_UNSUPPORTED;
  if (cfg->NumG <= 0) return CGD_ERR_SHAPE;
  if (!(cfg->Rd > 0) || !(cfg->Cpd > cfg->Rd) || !(cfg->p0 > 0) || !(cfg->Grav > 0)) return CGD_ERR_INVALID_ARG;
  const size_t need = (size_t)8 * (cfg->nz - 1) * cfg->NumG;
  if (need > CGD_NOALLOC_SCRATCH_DOUBLES) {
    char buf[200];
    snprintf(buf, sizeof buf, "8*(nz-1)*NumG = %zu doubles exceeds the static scratch of %u doubles", need,
             CGD_NOALLOC_SCRATCH_DOUBLES);
    g_last_error = buf;
    return CGD_ERR_SHAPE;
  }
  if (!is_device_ptr(U) || !is_device_ptr(dz) || !is_device_ptr(k) || !is_device_ptr(v)) return CGD_ERR_INVALID_ARG;
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return CGD_ERR_UNSUPPORTED;
  double *bands = nullptr;
  {
    // once per device, with that device current: the device address of the
    // static array (its host-side name is only a stand-in)
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
      void *p = nullptr;
      CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
      CK(cudaFuncSetAttribute(k_column<3, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              COL_WARPS * COL_ARR * 64 * (int)sizeof(double)));
      g_noalloc_ptr[dev] = static_cast<double *>(p);
    }
    bands = g_noalloc_ptr[dev];
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  GP P{};
  P.nz = cfg->nz; P.NumG = cfg->NumG; P.NumTr = cfg->NumTr; P.NV = 5 + cfg->NumTr; P.NC = P.NV + 1;
  P.dz = dz; P.Grav = cfg->Grav; P.Rd = cfg->Rd; P.p0 = cfg->p0; P.kappa = cfg->Rd / cfg->Cpd;
  const long long n = (long long)(P.nz - 1) * P.NumG;
  const size_t bs = (size_t)2 * (P.nz - 1) * P.NumG;
  const Bands4 b4{{bands, bands + bs, bands + 2 * bs, bands + 3 * bs}};
  k_jac<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(P, U, b4);
  ColArgs a{};
  a.v = v;
  a.kout = k;
  for (int i = 0; i < 4; ++i) a.jb4[i] = b4.b[i];
  a.fac = fac;
  a.dt = fac;
  const size_t smem = (size_t)COL_WARPS * COL_ARR * P.nz * sizeof(double);
  k_column<3, false><<<(P.NumG + COL_WARPS - 1) / COL_WARPS, 32 * COL_WARPS, smem, st>>>(P, a);
  // launch errors only: the work stays ordered on the caller's stream, which
  // the caller synchronises (or orders further work on) itself
  CK(cudaGetLastError());
  return CGD_OK;
}

}  // extern "C"

namespace {

int adjoint_alloc(cgd_handle *h, bool step)
{
  const size_t S = (size_t)h->nz * h->NumG, SV = S * h->NV;
  int rc = CGD_OK;
  if (!h->aLF) {
    rc = dalloc(h, &h->aLF, SV);
    if (!rc) rc = dalloc(h, &h->aLU, SV);
    if (!rc) rc = dalloc(h, &h->aLT1, S * 5);
  }
  if (!rc && step && !h->aAR) {
    for (int i = 0; i < 2 && !rc; ++i) rc = dalloc(h, &h->aLk[i], SV);
    if (!rc) rc = dalloc(h, &h->aAR, SV);
    if (!rc) rc = dalloc(h, &h->aLV, SV);
    if (!rc) rc = dalloc(h, &h->aLt, SV);
  }
  return rc;
}

// LU = (dF/dU)^T LF at the device state Ud (LU zeroed here).  T1 and pres
// are the state's DSS'd phase-1 cache and pressure when the caller has them,
// else null (computed here).
int rhs_adjoint_core(cgd_handle *h, const double *Ud, const double *LFd, double *LUd, const double *T1 = nullptr,
                     const double *pres = nullptr)
{
  const size_t S = (size_t)h->nz * h->NumG;
  if (!T1) {
    hv1(h, Ud, h->C);
    gather(h, h->C, h->T1, false);
    pressure(h, Ud, h->pres);
    T1 = h->T1;
    pres = h->pres;
  }
  CK(cudaMemsetAsync(LUd, 0, S * h->NV * 8, h->stream));
  CK(cudaMemsetAsync(h->aLT1, 0, S * 5 * 8, h->stream));
  CK(launch_rhs_adjoint(h->gp, Ud, T1, pres, LFd, LUd, h->aLT1, h->stream));
  return CGD_OK;
}

int column_adj(cgd_handle *h, const double *mu, double mus, const double *kx, const double *jbg, const double *Vn,
               double fac, double *AR, double *LV)
{
  CK(launch_column_adjoint(h->gp, mu, mus, kx, jbg, Vn, fac, AR, LV, h->stream));
  return CGD_OK;
}

// Device buffers of a step tape (own_u0: the tape keeps a copy of the step's
// initial state; otherwise it points at the caller's array during the call).
int tape_alloc(cgd_handle *h, StepTape &t, bool own_u0)
{
  if (!t.mem.empty()) return CGD_OK;
  const size_t S = (size_t)h->nz * h->NumG, SV = S * h->NV, SJ = (size_t)8 * (h->nz - 1) * h->NumG;
  auto get = [&](double **p, size_t n) -> int {
    void *q = nullptr;
    CK(cudaMalloc(&q, n * sizeof(double)));
    t.mem.push_back(q);
    *p = static_cast<double *>(q);
    return CGD_OK;
  };
  int rc = own_u0 ? get(&t.U0, SV) : CGD_OK;
  if (!rc) rc = get(&t.V2, SV);
  if (!rc) rc = get(&t.V3, SV);
  for (int i = 0; i < 3 && !rc; ++i) rc = get(&t.T1[i], S * 5);
  for (int i = 0; i < 3 && !rc; ++i) rc = get(&t.P[i], S);
  for (int i = 0; i < 3 && !rc; ++i) rc = get(&t.k[i], SV);
  if (!rc) rc = get(&t.jbg, SJ);
  return rc;
}

// One forward step from the device state u0 (kept in the tape when it owns a
// copy), recording what its reverse reads; U1 goes to Uout (may be u0's
// array when the tape owns its copy).  Not captured: the tape's buffers
// differ from the graph's.
int record_step(cgd_handle *h, StepTape &t, const double *u0, double dt, double *Uout)
{
  const size_t SV = (size_t)h->nz * h->NumG * h->NV;
  if (t.U0) {
    if (t.U0 != u0) CK(cudaMemcpyAsync(t.U0, u0, SV * 8, cudaMemcpyDeviceToDevice, h->stream));
    t.u0 = t.U0;
  } else {
    t.u0 = u0;
  }
  t.dt = dt;
  ColArgs a{};
  a.Vn = t.u0;
  a.k1 = t.k[0];
  a.k2 = t.k[1];
  a.dt = dt;
  a.fac = dt * h->rk.gamma;
  a.rk = h->rk;
  a.C = h->C;
  a.jbg = t.jbg;
  const double *Vs[3] = {t.u0, t.V2, t.V3};
  for (int st = 0; st < 3; ++st) {
    hv1(h, Vs[st], h->C);
    gather(h, h->C, t.T1[st], false);
    pressure(h, Vs[st], t.P[st]);
    phase2(h, Vs[st], t.P[st], t.T1[st], h->C);
    a.kout = t.k[st];
    if (st == 0) { a.Vout = t.V2; column<0>(h, a); }
    else if (st == 1) { a.Vout = t.V3; column<1>(h, a); }
    else { a.Vout = Uout ? Uout : h->Vst; column<2>(h, a); }
  }
  CK(cudaGetLastError());
  t.recorded = true;
  return CGD_OK;
}

// Lin (device, h->aLV) = (dU1/dU0)^T L for the recorded step:
// U1 = U0 + sum m_i k_i; k_i = L (F(V_i) + sum_j c_ij/dt k_j); V_i = U0 + sum_j a_ij k_j
int reverse_step(cgd_handle *h, const StepTape &t, const double *L)
{
  const size_t SV = (size_t)h->nz * h->NumG * h->NV;
  const RK &rk = h->rk;
  const double dt = t.dt, fac = dt * rk.gamma;
  const double *Vs[3] = {t.u0, t.V2, t.V3};
  CK(cudaMemsetAsync(h->aLV, 0, SV * 8, h->stream));
  const long long n = (long long)SV;
  for (int st = 2; st >= 0; --st) {
    const double cA = st >= 1 ? rk.c[st][0] / dt : 0.0, cB = st == 2 ? rk.c[st][1] / dt : 0.0;
    const double *mu = st == 2 ? L : h->aLk[st];
    int rc = column_adj(h, mu, st == 2 ? rk.m[2] : 1.0, t.k[st], t.jbg, t.u0, fac, h->aAR, h->aLV);
    if (rc) return rc;
    rc = rhs_adjoint_core(h, Vs[st], h->aAR, h->aLt, t.T1[st], t.P[st]);
    if (rc) return rc;
    // r_st = F(V_st) + c_st0/dt k1 + c_st1/dt k2; V_st = U0 + a_st0 k1 + a_st1 k2
    if (st == 2)
      CK(launch_adjoint_update(n, L, h->aAR, h->aLt, h->aLV, h->aLk[0], h->aLk[1], rk.m[0], rk.m[1], cA, cB,
                               rk.a[2][0], rk.a[2][1], h->stream));
    else if (st == 1)
      CK(launch_adjoint_update(n, nullptr, h->aAR, h->aLt, h->aLV, h->aLk[0], nullptr, 0.0, 0.0, cA, 0.0,
                               rk.a[1][0], 0.0, h->stream));
    else
      CK(launch_adjoint_update(n, nullptr, nullptr, h->aLt, h->aLV, nullptr, nullptr, 0.0, 0.0, 0.0, 0.0, 0.0,
                               0.0, h->stream));
  }
  return CGD_OK;
}

int adjoint_out(cgd_handle *h, double *Lin)
{
  const size_t SV = (size_t)h->nz * h->NumG * h->NV;
  if (is_device_ptr(Lin)) CK(cudaMemcpyAsync(Lin, h->aLV, SV * 8, cudaMemcpyDeviceToDevice, h->stream));
  else CK(cudaMemcpyAsync(Lin, h->aLV, SV * 8, cudaMemcpyDeviceToHost, h->stream));
  return finish(h);
}

const double *adjoint_in(cgd_handle *h, const double *Lout)
{
  if (is_device_ptr(Lout)) return Lout;
  const size_t SV = (size_t)h->nz * h->NumG * h->NV;
  if (cudaMemcpyAsync(h->aLF, Lout, SV * 8, cudaMemcpyHostToDevice, h->stream) != cudaSuccess) return nullptr;
  return h->aLF;
}

}  // namespace

extern "C" {

int cgd_ros_step_adjoint(cgd_handle *h, const double *U0, const double *Lout, double *Lin, double dt)
{
  if (!h || !U0 || !Lout || !Lin || !(dt > 0)) return CGD_ERR_INVALID_ARG;
  if (h->mix || h->NumTr != 0 || h->gp.held_suarez || h->gp.damping) return CGD_ERR_UNSUPPORTED;
  int rc = adjoint_alloc(h, true);
  if (!rc) rc = tape_alloc(h, h->work_tape, false);
  if (!rc) rc = enter(h);
  if (rc) return rc;
  double *Ud;
  rc = stage_in(h, U0, h->Ubuf, true, &Ud);
  if (rc) return rc;
  const double *L = adjoint_in(h, Lout);
  if (!L) return cuda_fail(h, cudaGetLastError(), "cgd_ros_step_adjoint");
  rc = record_step(h, h->work_tape, Ud, dt, nullptr);   // U1 itself is not needed
  if (!rc) rc = reverse_step(h, h->work_tape, L);
  if (rc) return rc;
  return adjoint_out(h, Lin);
}

int cgd_tape_record_step(cgd_handle *h, int32_t slot, double *U, double dt)
{
  if (!h || !U || !(dt > 0) || slot < 0 || slot >= CGD_TAPE_MAX_SLOTS) return CGD_ERR_INVALID_ARG;
  if (h->mix || h->NumTr != 0 || h->gp.held_suarez || h->gp.damping) return CGD_ERR_UNSUPPORTED;
  if ((size_t)slot >= h->tapes.size()) h->tapes.resize(slot + 1);
  int rc = adjoint_alloc(h, true);
  if (!rc) rc = tape_alloc(h, h->tapes[slot], true);
  if (!rc) rc = enter(h);
  if (rc) return rc;
  double *Ud;
  rc = stage_in(h, U, h->Ubuf, true, &Ud);
  if (rc) return rc;
  rc = record_step(h, h->tapes[slot], Ud, dt, Ud);
  if (rc) return rc;
  if (Ud != U)
    CK(cudaMemcpyAsync(U, Ud, (size_t)h->nz * h->NumG * h->NV * 8, cudaMemcpyDeviceToHost, h->stream));
  return finish(h);
}

int cgd_tape_step_adjoint(cgd_handle *h, int32_t slot, const double *Lout, double *Lin)
{
  if (!h || !Lout || !Lin || slot < 0 || (size_t)slot >= h->tapes.size()) return CGD_ERR_INVALID_ARG;
  if (!h->tapes[slot].recorded) return CGD_ERR_INVALID_ARG;
  int rc = enter(h);
  if (rc) return rc;
  const double *L = adjoint_in(h, Lout);
  if (!L) return cuda_fail(h, cudaGetLastError(), "cgd_tape_step_adjoint");
  rc = reverse_step(h, h->tapes[slot], L);
  if (rc) return rc;
  return adjoint_out(h, Lin);
}

int cgd_tape_release(cgd_handle *h)
{
  if (!h) return CGD_ERR_INVALID_ARG;
  CK(cudaStreamSynchronize(h->stream));
  for (auto &t : h->tapes)
    for (void *q : t.mem) cudaFree(q);
  h->tapes.clear();
  return CGD_OK;
}

int64_t cgd_tape_bytes_per_step(const cgd_handle *h)
{
  if (!h) return CGD_ERR_INVALID_ARG;
  const int64_t S = (int64_t)h->nz * h->NumG, SV = S * h->NV, SJ = (int64_t)8 * (h->nz - 1) * h->NumG;
  return 8 * (6 * SV + 15 * S + 3 * S + SJ);
}

}  // extern "C"

namespace {

int cgd_rhs_adjoint_impl(cgd_handle *h, const double *U, const double *LF, double *LU)
{
  if (!h || !U || !LF || !LU) return CGD_ERR_INVALID_ARG;
  if (h->mix || h->NumTr != 0 || h->gp.held_suarez || h->gp.damping) return CGD_ERR_UNSUPPORTED;
  const size_t S = (size_t)h->nz * h->NumG;
  int arc = adjoint_alloc(h, false);
  if (!arc) arc = enter(h);
  if (arc) return arc;
  double *Ud;
  int rc = stage_in(h, U, h->Ubuf, true, &Ud);
  if (rc) return rc;
  const double *LFd = LF;
  if (!is_device_ptr(LF)) {
    CK(cudaMemcpyAsync(h->aLF, LF, S * h->NV * 8, cudaMemcpyHostToDevice, h->stream));
    LFd = h->aLF;
  }
  const bool udev = is_device_ptr(LU);
  double *LUd = udev ? LU : h->aLU;
  rc = rhs_adjoint_core(h, Ud, LFd, LUd);
  if (rc) return rc;
  if (!udev) CK(cudaMemcpyAsync(LU, LUd, S * h->NV * 8, cudaMemcpyDeviceToHost, h->stream));
  return finish(h);
}

}  // namespace

extern "C" {
int cgd_rhs_adjoint(cgd_handle *h, const double *U, const double *LF, double *LU)
{
  return cgd_rhs_adjoint_impl(h, U, LF, LU);
}

int cgd_set_caller_stream(cgd_handle *h, void *stream)
{
  if (!h) return CGD_ERR_INVALID_ARG;
  h->caller = stream ? static_cast<cudaStream_t>(stream) : cudaStreamLegacy;
  return CGD_OK;
}

int cgd_get_stream(cgd_handle *h, void **stream)
{
  if (!h || !stream) return CGD_ERR_INVALID_ARG;
  *stream = (void *)h->stream;
  return CGD_OK;
}

int cgd_kernel_times(cgd_handle *h, char *names, int32_t names_len, double *ms, int32_t nmax)
{
  if (!h || !ms) return CGD_ERR_INVALID_ARG;
  if (!h->profile) return CGD_ERR_UNSUPPORTED;
  static const char *nm[NPROF] = {"pressure", "hypervisc1", "gather", "phase2", "column", "pressure",
                                  "hypervisc1", "gather", "phase2", "column", "pressure",
                                  "hypervisc1", "gather", "phase2", "column"};
  std::string all;
  int n = nmax < NPROF ? nmax : NPROF;
  for (int i = 0; i < n; ++i) {
    float t = 0.f;
    if (cudaEventElapsedTime(&t, h->ev[i], h->ev[i + 1]) != cudaSuccess) {
      cudaGetLastError();
      t = -1.f;
    }
    ms[i] = t;
    all += nm[i];
    if (i + 1 < n) all += ";";
  }
  if (names && names_len > 0) {
    strncpy(names, all.c_str(), names_len - 1);
    names[names_len - 1] = 0;
  }
  return n;
}

}  // extern "C"

// ===========================================================================
// Batched ensemble (cgd_batch_*): the members' steps as one graph of 15
// launches over flat work lists.
// ===========================================================================
// Work lists of an ensemble: 0 phase-1 tiles of 256/N^2 levels, 1 column-level
// blocks of 256 (pressure, gather), 2 phase-2 chunks, 3 column blocks, 4 phase-2
// chunks of the 16-warp form, 5 phase-1 tiles of the split form (HV1Tile: 16
// levels at p = 4 in FP64, else as list 0)
constexpr int BATCH_LISTS = 6;

struct cgd_batch {
  std::vector<cgd_handle *> mem;
  int N = 0, NT = 0, nzmax = 0;
  bool mix = false;
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t order_ev = nullptr;   // orders a step after the first member's caller stream
  // work lists, one set per candidate order; a candidate is (order, form):
  // candidate c runs order c % NORD in form c / NORD: split into 15 launches
  // (FORM_SPLIT), split with phase 2 in 16-level CTAs (FORM_SPLIT16, p = 4),
  // as three fused stage launches (FORM_FUSED), or every member's own
  // single-member step on its own stream inside the graph (FORM_MEMBERS;
  // orders 0 and 1: one member after the other, as given or the largest
  // first; order 2: all members as concurrent branches)
  static constexpr int NORD = 3;
  static constexpr int FORM_SPLIT = 0, FORM_SPLIT16 = 1, FORM_FUSED = 2, FORM_MEMBERS = 3, NFORM = 4;
  static constexpr int NCAND = NFORM * NORD;
  WItem *w[NORD][BATCH_LISTS] = {};
  int n[BATCH_LISTS] = {};
  cudaGraph_t graph[NCAND] = {};
  cudaGraphExec_t gexec[NCAND] = {};
  bool use[NCAND] = {};
  int chosen = 0;
  bool tuned = false, autotune = false;
  double tune_ms[NCAND] = {};
  // fused form: grid (CTAs resident on the device), dynamic shared memory,
  // barrier state, second contribution and stage buffers per member
  int fgrid = 0;
  size_t fsmem = 0;
  GridBar *bar = nullptr;
  std::vector<double *> C2, Vst2;
  std::vector<GP> gps;
  std::vector<BMember> bms;
  std::vector<void *> scratch;
  // the members form: fork and join events, and the states and time steps
  // its graphs were captured with (their kernels take the state pointers)
  cudaEvent_t fork_ev = nullptr;
  std::vector<cudaEvent_t> join_ev;
  std::vector<double *> gU[NCAND];
  std::vector<double> gdt[NCAND];
  std::string last_error;
};

namespace {

const char *const ORDER_NAME[cgd_batch::NORD] = {"member-major", "largest-member-first", "members-interleaved"};
const char *const FORM_NAME[cgd_batch::NFORM] = {"split", "split16", "fused", "members"};
int form_of(int cand) { return cand / cgd_batch::NORD; }
// the order's name; in the members form order 2 forks the members at once
const char *order_name(int cand)
{
  return form_of(cand) == cgd_batch::FORM_MEMBERS && cand % cgd_batch::NORD == 2
             ? "members-concurrent"
             : ORDER_NAME[cand % cgd_batch::NORD];
}
// levels per phase-2 CTA of a form
int phase2_levels(int N, int form)
{
  if (form == cgd_batch::FORM_SPLIT16) return P2Cfg<5, 0, double, P2_ALT_WARPS>::LC;
  switch (N) {
    case 2: return P2Cfg<2, 0, double>::LC;
    case 3: return P2Cfg<3, 0, double>::LC;
    case 4: return P2Cfg<4, 0, double>::LC;
    default: return P2Cfg<5, 0, double>::LC;
  }
}

int batch_fail(cgd_batch *b, cudaError_t e, const char *what)
{
  char buf[256];
  snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
  g_last_error = buf;
  if (b) b->last_error = buf;
  return CGD_ERR_CUDA;
}
#define BCK(call)                                          \
  do {                                                     \
    cudaError_t e_ = (call);                               \
    if (e_ != cudaSuccess) return batch_fail(b, e_, #call); \
  } while (0)

// Work items of every kernel of a stage for every member, in one of three
// orders: members one after the other, the largest member first, or the
// members' items interleaved one by one.
void batch_lists(const cgd_batch *b, int order, std::vector<WItem> out[BATCH_LISTS])
{
  const int nm = (int)b->mem.size();
  std::vector<std::vector<WItem>> per[BATCH_LISTS];
  for (int k = 0; k < BATCH_LISTS; ++k) per[k].resize(nm);
  const int DoF = b->N * b->N;
  const int LT = 256 / DoF;
  const int LTW = b->mix ? LT : (b->N == 5 ? HV1Tile<5, double>::LT : LT);   // list 5
  int LC = 0, LCA = 0;   // phase-2 levels per CTA: default, alternative (p = 4 only)
  switch (b->N) {
    case 2: LC = LCA = P2Cfg<2, 0, double>::LC; break;
    case 3: LC = LCA = P2Cfg<3, 0, double>::LC; break;
    case 4: LC = LCA = P2Cfg<4, 0, double>::LC; break;
    default: LC = P2Cfg<5, 0, double>::LC; LCA = P2Cfg<5, 0, double, P2_ALT_WARPS>::LC; break;
  }
  for (int m = 0; m < nm; ++m) {
    const cgd_handle *h = b->mem[m];
    for (int IF = 0; IF < h->NF; ++IF)
      for (int t = 0; t < (h->nz + LT - 1) / LT; ++t) per[0][m].push_back({m, t, IF});
    const long long ncl = (long long)h->nz * h->NumG;
    for (long long t = 0; t < (ncl + 255) / 256; ++t) per[1][m].push_back({m, (int)t, 0});
    for (int IF = 0; IF < h->NF; ++IF)
      for (int c = 0; c < (h->nz + LC - 1) / LC; ++c) per[2][m].push_back({m, c, IF});
    for (int c = 0; c < (h->NumG + COL_WARPS - 1) / COL_WARPS; ++c) per[3][m].push_back({m, c, 0});
    for (int IF = 0; IF < h->NF; ++IF)
      for (int c = 0; c < (h->nz + LCA - 1) / LCA; ++c) per[4][m].push_back({m, c, IF});
    for (int IF = 0; IF < h->NF; ++IF)
      for (int t = 0; t < (h->nz + LTW - 1) / LTW; ++t) per[5][m].push_back({m, t, IF});
  }
  std::vector<int> ord(nm);
  for (int m = 0; m < nm; ++m) ord[m] = m;
  if (order == 1)
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int c) {
      return (long long)b->mem[a]->NF * b->mem[a]->nz > (long long)b->mem[c]->NF * b->mem[c]->nz;
    });
  for (int k = 0; k < BATCH_LISTS; ++k) {
    out[k].clear();
    if (order == 2) {
      size_t mx = 0;
      for (int m = 0; m < nm; ++m) mx = std::max(mx, per[k][m].size());
      for (size_t i = 0; i < mx; ++i)
        for (int m = 0; m < nm; ++m)
          if (i < per[k][m].size()) out[k].push_back(per[k][m][i]);
    } else {
      for (int m : ord) out[k].insert(out[k].end(), per[k][m].begin(), per[k][m].end());
    }
  }
}

template <int N, int NT, typename R>
void batch_enqueue_t(cgd_batch *b, WItem *const *w, bool p2alt)
{
  using CF = P2Cfg<N, NT, R>;
  using CFA = P2Cfg<N, NT, R, P2_ALT_WARPS>;
  static std::atomic<unsigned long long> attr{0};
  const size_t csmem = (size_t)COL_WARPS * COL_ARR * b->nzmax * sizeof(double);
  if (first_on_device(attr)) {
    cudaFuncSetAttribute(kb_phase2<N, NT, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CF::SMEM);
    cudaFuncSetAttribute(kb_hypervisc1w<N, NT, R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)HV1Smem<N, NT, R, HV1Tile<N, R>::LT>::BYTES);
    if constexpr (N == 5)
      cudaFuncSetAttribute(kb_phase2<N, NT, R, P2_ALT_WARPS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)CFA::SMEM);
    constexpr bool C32 = sizeof(R) == sizeof(float);
    for (auto f : {kb_column<0, C32>, kb_column<1, C32>, kb_column<2, C32>})
      cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, COL_WARPS * COL_ARR * 64 * (int)sizeof(double));
  }
  kb_pressure<<<b->n[1], 256, 0, b->stream>>>(w[1], 0);
  for (int stage = 0; stage < 3; ++stage) {
    using HT = HV1Tile<N, R>;
    kb_hypervisc1w<N, NT, R><<<b->n[5], HT::THREADS, HV1Smem<N, NT, R, HT::LT>::BYTES, b->stream>>>(w[5], stage);
    kb_gather<sizeof(R) == sizeof(float)><<<b->n[1], 256, 0, b->stream>>>(w[1]);
    if constexpr (N == 5) {
      if (p2alt) kb_phase2<N, NT, R, P2_ALT_WARPS><<<b->n[4], CFA::THREADS, CFA::SMEM, b->stream>>>(w[4], stage);
      else kb_phase2<N, NT, R><<<b->n[2], CF::THREADS, CF::SMEM, b->stream>>>(w[2], stage);
    } else {
      kb_phase2<N, NT, R><<<b->n[2], CF::THREADS, CF::SMEM, b->stream>>>(w[2], stage);
    }
    constexpr bool C32 = sizeof(R) == sizeof(float);
    if (stage == 0) kb_column<0, C32><<<b->n[3], 32 * COL_WARPS, csmem, b->stream>>>(w[3]);
    else if (stage == 1) kb_column<1, C32><<<b->n[3], 32 * COL_WARPS, csmem, b->stream>>>(w[3]);
    else kb_column<2, C32><<<b->n[3], 32 * COL_WARPS, csmem, b->stream>>>(w[3]);
    if (stage < 2) kb_pressure<<<b->n[1], 256, 0, b->stream>>>(w[1], 1);
  }
}

template <int N, typename R>
void batch_enqueue_n(cgd_batch *b, WItem *const *w, bool p2alt)
{
  switch (b->NT) {
    case 0: batch_enqueue_t<N, 0, R>(b, w, p2alt); break;
    case 1: batch_enqueue_t<N, 1, R>(b, w, p2alt); break;
    case 2: batch_enqueue_t<N, 2, R>(b, w, p2alt); break;
    case 3: batch_enqueue_t<N, 3, R>(b, w, p2alt); break;
    default: batch_enqueue_t<N, 4, R>(b, w, p2alt); break;
  }
}

template <typename R>
void batch_enqueue_r(cgd_batch *b, WItem *const *w, bool p2alt)
{
  switch (b->N) {
    case 2: batch_enqueue_n<2, R>(b, w, p2alt); break;
    case 3: batch_enqueue_n<3, R>(b, w, p2alt); break;
    case 4: batch_enqueue_n<4, R>(b, w, p2alt); break;
    default: batch_enqueue_n<5, R>(b, w, p2alt); break;
  }
}

// The fused form (p = 4): three cooperative launches of kb_stage per step.
// The barrier counter is cleared before each (a launch that timed out may
// have left it non-zero).
template <int NT, typename R>
cudaError_t batch_enqueue_fused_t(cgd_batch *b, WItem *const *w)
{
  FusedArgs fa{};
  for (int k = 0; k < 5; ++k) {
    fa.w[k] = w[k];
    fa.n[k] = b->n[k];
  }
  fa.bar = b->bar;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  for (int stage = 0; stage < 3; ++stage) {
    cudaError_t e = cudaMemsetAsync(&b->bar->count, 0, sizeof(unsigned int), b->stream);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)b->fgrid);
    cfg.blockDim = dim3(256);
    cfg.dynamicSmemBytes = b->fsmem;
    cfg.stream = b->stream;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    e = cudaLaunchKernelEx(&cfg, kb_stage<5, NT, R>, fa, stage);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

template <typename R>
cudaError_t batch_enqueue_fused_r(cgd_batch *b, WItem *const *w)
{
  switch (b->NT) {
    case 0: return batch_enqueue_fused_t<0, R>(b, w);
    case 1: return batch_enqueue_fused_t<1, R>(b, w);
    case 2: return batch_enqueue_fused_t<2, R>(b, w);
    case 3: return batch_enqueue_fused_t<3, R>(b, w);
    default: return batch_enqueue_fused_t<4, R>(b, w);
  }
}

// Launch limits of the fused kernel on this device: dynamic shared memory
// (the larger of phase 2's and the column's) and the CTAs that fit at once.
template <int NT, typename R>
cudaError_t fused_setup_t(cgd_batch *b)
{
  using CF = P2Cfg<5, NT, R, FUSED_P2_WARPS>;
  const size_t csm = (size_t)COL_WARPS * COL_ARR * b->nzmax * sizeof(double);
  b->fsmem = std::max(std::max(CF::SMEM, csm), HV1Smem<5, NT, R>::BYTES);
  cudaError_t e = cudaFuncSetAttribute(kb_stage<5, NT, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->fsmem);
  if (e != cudaSuccess) return e;
  int per_sm = 0, sms = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kb_stage<5, NT, R>, 256, b->fsmem);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
  b->fgrid = per_sm * sms;
  return e;
}

template <typename R>
cudaError_t fused_setup_r(cgd_batch *b)
{
  switch (b->NT) {
    case 0: return fused_setup_t<0, R>(b);
    case 1: return fused_setup_t<1, R>(b);
    case 2: return fused_setup_t<2, R>(b);
    case 3: return fused_setup_t<3, R>(b);
    default: return fused_setup_t<4, R>(b);
  }
}

// The members form: every member's step (the single-member kernels, its own
// buffers) on the member's stream, forked from the batch stream and joined
// back.  Orders 0 and 1 chain the members one after the other (as given, or
// the largest first): each member then runs alone on the device, as in
// cgd_ros_step.  Order 2 forks all members at once, one independent branch
// each.
cudaError_t batch_enqueue_members(cgd_batch *b, int order, double *const *U, const double *dt)
{
  const int nm = (int)b->mem.size();
  const bool serial = order < 2;
  std::vector<int> ord(nm);
  for (int m = 0; m < nm; ++m) ord[m] = m;
  if (order == 1)
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int c) {
      return (long long)b->mem[a]->NF * b->mem[a]->nz > (long long)b->mem[c]->NF * b->mem[c]->nz;
    });
  cudaError_t e = serial ? cudaSuccess : cudaEventRecord(b->fork_ev, b->stream);
  for (int m : ord) {
    if (e != cudaSuccess) break;
    cgd_handle *h = b->mem[m];
    if (serial) e = cudaEventRecord(b->fork_ev, b->stream);   // after the previous member's join
    if (e == cudaSuccess) e = cudaStreamWaitEvent(h->stream, b->fork_ev, 0);
    if (e != cudaSuccess) break;
    h->capturing = true;   // no profiling events inside the graph
    enqueue_step(h, U[m], dt[m]);
    h->capturing = false;
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaEventRecord(b->join_ev[m], h->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(b->stream, b->join_ev[m], 0);
  }
  return e;
}

cudaError_t batch_enqueue(cgd_batch *b, int cand)
{
  WItem *const *w = b->w[cand % cgd_batch::NORD];
  const int form = form_of(cand);
  if (form == cgd_batch::FORM_FUSED)
    return b->mix ? batch_enqueue_fused_r<float>(b, w) : batch_enqueue_fused_r<double>(b, w);
  if (b->mix) batch_enqueue_r<float>(b, w, form == cgd_batch::FORM_SPLIT16);
  else batch_enqueue_r<double>(b, w, form == cgd_batch::FORM_SPLIT16);
  return cudaSuccess;
}

// 1 if a fused launch timed out at a grid barrier (the flag is cleared)
int fused_timed_out(cgd_batch *b)
{
  if (!b->bar) return 0;
  int t = 0;
  if (cudaMemcpy(&t, &b->bar->timeout, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return 1;
  if (t) cudaMemset(&b->bar->timeout, 0, sizeof(int));
  return t != 0;
}

int batch_upload(cgd_batch *b)
{
  const size_t nm = b->mem.size();
  BCK(cudaMemcpyToSymbolAsync(c_bgp, b->gps.data(), nm * sizeof(GP), 0, cudaMemcpyHostToDevice, b->stream));
  BCK(cudaMemcpyToSymbolAsync(c_bm, b->bms.data(), nm * sizeof(BMember), 0, cudaMemcpyHostToDevice, b->stream));
  BCK(cudaMemcpyToSymbolAsync(c_brk, &b->mem[0]->rk, sizeof(RK), 0, cudaMemcpyHostToDevice, b->stream));
  return CGD_OK;
}

}  // namespace

extern "C" {

int cgd_batch_create(cgd_handle *const *members, int32_t nmembers, int32_t flags, cgd_batch **out)
{
  cgd_batch *b = nullptr;
  if (!members || !out || nmembers < 1) return CGD_ERR_INVALID_ARG;
  if (nmembers > BMAX) return CGD_ERR_UNSUPPORTED;
  for (int m = 0; m < nmembers; ++m) {
    const cgd_handle *h = members[m];
    if (!h) return CGD_ERR_INVALID_ARG;
    if (h->N != members[0]->N || h->NumTr != members[0]->NumTr || h->mix != members[0]->mix ||
        h->device != members[0]->device)
      return CGD_ERR_SHAPE;
  }
  b = new cgd_batch;
  b->mem.assign(members, members + nmembers);
  b->N = members[0]->N;
  b->NT = members[0]->NumTr;
  b->mix = members[0]->mix;
  b->device = members[0]->device;
  b->autotune = (flags & CGD_BATCH_AUTOTUNE) != 0;
  const bool want_fused = (flags & CGD_BATCH_FUSED) != 0;
  if (want_fused && b->N != 5) {
    delete b;
    return CGD_ERR_UNSUPPORTED;
  }
  for (auto h : b->mem) b->nzmax = std::max(b->nzmax, h->nz);
  int rc = CGD_OK;
  do {
    cudaError_t e = cudaSetDevice(b->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->order_ev, cudaEventDisableTiming);
    if (e != cudaSuccess) { rc = batch_fail(b, e, "cgd_batch_create stream"); break; }
    // candidates: the autotuner times every order, split and (p = 4, when
    // the device launches cooperative kernels) fused; otherwise the first
    // order, split or fused as asked
    bool fused_ok = false;
    if (b->N == 5 && (b->autotune || want_fused)) {
      int coop = 0;
      e = cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, b->device);
      if (e == cudaSuccess && coop) e = b->mix ? fused_setup_r<float>(b) : fused_setup_r<double>(b);
      if (e != cudaSuccess) { rc = batch_fail(b, e, "cgd_batch_create fused setup"); break; }
      fused_ok = coop && b->fgrid > 0;
    }
    if (want_fused && !fused_ok) { rc = CGD_ERR_UNSUPPORTED; break; }
    const bool want_members = (flags & CGD_BATCH_MEMBERS) != 0;
    const int first = want_fused ? cgd_batch::FORM_FUSED * cgd_batch::NORD
                                 : want_members ? cgd_batch::FORM_MEMBERS * cgd_batch::NORD : 0;
    for (int c = 0; c < cgd_batch::NCAND; ++c) {
      const int form = form_of(c);
      const bool avail = form == cgd_batch::FORM_SPLIT || (form == cgd_batch::FORM_SPLIT16 && b->N == 5) ||
                         (form == cgd_batch::FORM_FUSED && fused_ok) ||
                         form == cgd_batch::FORM_MEMBERS;
      b->use[c] = b->autotune ? avail : c == first;
    }
    e = cudaEventCreateWithFlags(&b->fork_ev, cudaEventDisableTiming);
    b->join_ev.assign(nmembers, nullptr);
    for (int m = 0; m < nmembers && e == cudaSuccess; ++m)
      e = cudaEventCreateWithFlags(&b->join_ev[m], cudaEventDisableTiming);
    if (e != cudaSuccess) { rc = batch_fail(b, e, "cgd_batch_create events"); break; }
    if (!b->autotune) b->chosen = first;
    if (fused_ok) {
      void *p = nullptr;
      e = cudaMalloc(&p, sizeof(GridBar));
      if (e == cudaSuccess) e = cudaMemset(p, 0, sizeof(GridBar));
      b->bar = static_cast<GridBar *>(p);
      for (int m = 0; m < nmembers && e == cudaSuccess; ++m) {
        const cgd_handle *h = members[m];
        const size_t S = (size_t)h->nz * h->NumG;
        const size_t ENL = (size_t)h->N * h->N * h->nz * h->NF;
        void *c2 = nullptr, *v2 = nullptr;
        e = cudaMalloc(&c2, ENL * (h->NV + 1) * sizeof(double));
        b->C2.push_back(static_cast<double *>(c2));
        if (e == cudaSuccess) e = cudaMalloc(&v2, S * h->NV * sizeof(double));
        b->Vst2.push_back(static_cast<double *>(v2));
      }
      if (e != cudaSuccess) { rc = batch_fail(b, e, "cgd_batch_create fused buffers"); break; }
    }
    const int nord = b->autotune ? cgd_batch::NORD : 1;
    for (int o = 0; o < nord && !rc; ++o) {
      std::vector<WItem> lists[BATCH_LISTS];
      batch_lists(b, o, lists);
      for (int k = 0; k < BATCH_LISTS; ++k) {
        b->n[k] = (int)lists[k].size();
        void *p = nullptr;
        e = cudaMalloc(&p, lists[k].size() * sizeof(WItem));
        if (e == cudaSuccess)
          e = cudaMemcpy(p, lists[k].data(), lists[k].size() * sizeof(WItem), cudaMemcpyHostToDevice);
        b->w[o][k] = static_cast<WItem *>(p);
        if (e != cudaSuccess) { rc = batch_fail(b, e, "cgd_batch_create work lists"); break; }
      }
    }
  } while (false);
  if (rc) { cgd_batch_destroy(b); return rc; }
  b->gps.resize(nmembers);
  b->bms.resize(nmembers);
  for (int m = 0; m < nmembers; ++m) b->gps[m] = members[m]->gp;
  *out = b;
  return CGD_OK;
}

void cgd_batch_destroy(cgd_batch *b)
{
  if (!b) return;
  if (b->stream) cudaStreamSynchronize(b->stream);
  for (int c = 0; c < cgd_batch::NCAND; ++c) {
    if (b->gexec[c]) cudaGraphExecDestroy(b->gexec[c]);
    if (b->graph[c]) cudaGraphDestroy(b->graph[c]);
  }
  for (int o = 0; o < cgd_batch::NORD; ++o)
    for (int k = 0; k < BATCH_LISTS; ++k)
      if (b->w[o][k]) cudaFree(b->w[o][k]);
  for (void *p : b->scratch) cudaFree(p);
  for (double *p : b->C2) if (p) cudaFree(p);
  for (double *p : b->Vst2) if (p) cudaFree(p);
  if (b->bar) cudaFree(b->bar);
  if (b->order_ev) cudaEventDestroy(b->order_ev);
  if (b->fork_ev) cudaEventDestroy(b->fork_ev);
  for (cudaEvent_t ev : b->join_ev)
    if (ev) cudaEventDestroy(ev);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

int cgd_batch_step(cgd_batch *b, double *const *U, const double *dt, int32_t nsteps)
{
  if (!b || !U || !dt || nsteps < 0) return CGD_ERR_INVALID_ARG;
  const int nm = (int)b->mem.size();
  for (int m = 0; m < nm; ++m) {
    if (!U[m] || !(dt[m] > 0)) return CGD_ERR_INVALID_ARG;
    if (!is_device_ptr(U[m])) return CGD_ERR_INVALID_ARG;
  }
  BCK(cudaSetDevice(b->device));
  BCK(cudaEventRecord(b->order_ev, b->mem[0]->caller));
  BCK(cudaStreamWaitEvent(b->stream, b->order_ev, 0));
  // mixed members: the reference profile from their first state
  for (int m = 0; m < nm; ++m) {
    cgd_handle *h = b->mem[m];
    if (h->mix && !h->have_ref) {
      if (int erc = enter(h)) return erc;
      ensure_ref(h, U[m]);
      BCK(cudaStreamSynchronize(h->stream));
    }
  }
  auto set_members = [&](double *const *state) {
    for (int m = 0; m < nm; ++m) {
      const cgd_handle *h = b->mem[m];
      b->bms[m] = BMember{state[m], h->Vst, h->k1, h->k2, h->C, h->T1, h->jbg, h->pres, h->pres_st, dt[m],
                          b->C2.empty() ? nullptr : b->C2[m], b->Vst2.empty() ? nullptr : b->Vst2[m]};
    }
  };
  // the members form's graph for the given states and time steps (captured
  // again when they change)
  auto capture_members = [&](int c, double *const *state) -> int {
    const std::vector<double *> su(state, state + nm);
    const std::vector<double> sd(dt, dt + nm);
    if (b->gexec[c] && b->gU[c] == su && b->gdt[c] == sd) return CGD_OK;
    if (b->gexec[c]) { cudaGraphExecDestroy(b->gexec[c]); b->gexec[c] = nullptr; }
    if (b->graph[c]) { cudaGraphDestroy(b->graph[c]); b->graph[c] = nullptr; }
    BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    const cudaError_t le = batch_enqueue_members(b, c % cgd_batch::NORD, state, dt);
    cudaError_t e = cudaStreamEndCapture(b->stream, &b->graph[c]);
    if (le != cudaSuccess) return batch_fail(b, le, "cgd_batch_step members capture");
    if (e != cudaSuccess) return batch_fail(b, e, "cgd_batch_step capture");
    BCK(cudaGraphInstantiate(&b->gexec[c], b->graph[c], 0));
    b->gU[c] = su;
    b->gdt[c] = sd;
    return CGD_OK;
  };
  for (int c = 0; c < cgd_batch::NCAND; ++c) {
    if (!b->use[c] || b->gexec[c] || form_of(c) == cgd_batch::FORM_MEMBERS) continue;
    BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    const cudaError_t le = batch_enqueue(b, c);
    cudaError_t e = cudaStreamEndCapture(b->stream, &b->graph[c]);
    if (le != cudaSuccess) return batch_fail(b, le, "cgd_batch_step fused launch");
    if (e != cudaSuccess) return batch_fail(b, e, "cgd_batch_step capture");
    BCK(cudaGraphInstantiate(&b->gexec[c], b->graph[c], 0));
  }
  if (b->autotune && !b->tuned) {
    // each candidate order advances copies of the states by one step after one
    // warm-up step; the fastest is kept
    std::vector<double *> copies(nm);
    if (b->scratch.empty()) {
      for (int m = 0; m < nm; ++m) {
        void *p = nullptr;
        BCK(cudaMalloc(&p, (size_t)b->mem[m]->nz * b->mem[m]->NumG * b->mem[m]->NV * sizeof(double)));
        b->scratch.push_back(p);
      }
    }
    for (int m = 0; m < nm; ++m) copies[m] = static_cast<double *>(b->scratch[m]);
    // the timing events are destroyed on every way out of this block
    struct EventPair {
      cudaEvent_t a = nullptr, b = nullptr;
      ~EventPair()
      {
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
      }
    } ev;
    BCK(cudaEventCreate(&ev.a));
    BCK(cudaEventCreate(&ev.b));
    cudaEvent_t e0 = ev.a, e1 = ev.b;
    for (int c = 0; c < cgd_batch::NCAND; ++c) {
      if (!b->use[c]) continue;
      for (int m = 0; m < nm; ++m) {
        const cgd_handle *h = b->mem[m];
        BCK(cudaMemcpyAsync(copies[m], U[m], (size_t)h->nz * h->NumG * h->NV * sizeof(double),
                            cudaMemcpyDeviceToDevice, b->stream));
      }
      set_members(copies.data());
      int rc = batch_upload(b);
      if (rc) return rc;
      if (form_of(c) == cgd_batch::FORM_MEMBERS && (rc = capture_members(c, copies.data()))) return rc;
      BCK(cudaGraphLaunch(b->gexec[c], b->stream));
      BCK(cudaEventRecord(e0, b->stream));
      BCK(cudaGraphLaunch(b->gexec[c], b->stream));
      BCK(cudaEventRecord(e1, b->stream));
      BCK(cudaEventSynchronize(e1));
      float ms = 0.f;
      BCK(cudaEventElapsedTime(&ms, e0, e1));
      b->tune_ms[c] = ms;
      if (form_of(c) == cgd_batch::FORM_FUSED && fused_timed_out(b)) {
        g_last_error = "cgd_batch_step: a fused stage launch timed out at a grid barrier";
        return CGD_ERR_TIMEOUT;
      }
    }
    b->chosen = 0;
    for (int c = 1; c < cgd_batch::NCAND; ++c)
      if (b->use[c] && b->tune_ms[c] < b->tune_ms[b->chosen]) b->chosen = c;
    b->tuned = true;
  }
  set_members(U);
  int rc = batch_upload(b);
  if (rc) return rc;
  if (form_of(b->chosen) == cgd_batch::FORM_MEMBERS && (rc = capture_members(b->chosen, U))) return rc;
  for (int s = 0; s < nsteps; ++s) BCK(cudaGraphLaunch(b->gexec[b->chosen], b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  BCK(cudaGetLastError());
  if (form_of(b->chosen) == cgd_batch::FORM_FUSED && fused_timed_out(b)) {
    g_last_error = "cgd_batch_step: a fused stage launch timed out at a grid barrier";
    return CGD_ERR_TIMEOUT;
  }
  return CGD_OK;
}

int cgd_grid_barrier_check(int32_t rounds, int32_t absent, double limit_s, int32_t *violations)
{
  if (rounds < 1 || !(limit_s > 0) || limit_s > 10.0 || !violations) return CGD_ERR_INVALID_ARG;
  int dev = 0, sms = 0, per_sm = 0, coop = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_barrier_probe, 256, 0);
  if (e != cudaSuccess) return batch_fail(nullptr, e, "cgd_grid_barrier_check setup");
  if (!coop || per_sm < 1) return CGD_ERR_UNSUPPORTED;
  // one allocation: the barrier, the arrival counter, the violation count
  struct Probe {
    GridBar bar;
    unsigned int arrivals;
    int violations;
  };
  Probe *pd = nullptr;
  e = cudaMalloc(&pd, sizeof(Probe));
  if (e != cudaSuccess) return batch_fail(nullptr, e, "cgd_grid_barrier_check alloc");
  Probe init{};
  // a participant that never arrives: the counter starts one ahead, so the
  // last real arrival is never the last one
  if (absent) init.bar.count = 1u;
  e = cudaMemcpy(pd, &init, sizeof(Probe), cudaMemcpyHostToDevice);
  const unsigned grid = (unsigned)(absent ? 1 : std::min(per_sm, 2) * sms);
  const unsigned long long limit_ns = (unsigned long long)(limit_s * 1e9);
  if (e == cudaSuccess) {
    GridBar *gb = &pd->bar;
    unsigned int *arr = &pd->arrivals;
    int *vio = &pd->violations;
    void *args[] = {&gb, const_cast<unsigned long long *>(&limit_ns), &rounds, &arr, &vio};
    e = cudaLaunchCooperativeKernel((const void *)k_barrier_probe, dim3(grid), dim3(256), args, 0, nullptr);
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  Probe out{};
  if (e == cudaSuccess) e = cudaMemcpy(&out, pd, sizeof(Probe), cudaMemcpyDeviceToHost);
  cudaFree(pd);
  if (e != cudaSuccess) return batch_fail(nullptr, e, "cgd_grid_barrier_check");
  *violations = out.violations;
  return out.bar.timeout ? CGD_ERR_TIMEOUT : CGD_OK;
}

int cgd_batch_tuning(cgd_batch *b, char *desc, int32_t len)
{
  if (!b || !desc || len < 1) return CGD_ERR_INVALID_ARG;
  const int form = form_of(b->chosen);
  std::string s = std::string("order=") + order_name(b->chosen) + ";stage=" +
                  (form == cgd_batch::FORM_FUSED ? "fused" : form == cgd_batch::FORM_MEMBERS ? "members" : "split") +
                  ";phase2_levels=" +
                  std::to_string(phase2_levels(b->N, form));
  if (b->tuned) {
    char buf[96];
    for (int c = 0; c < cgd_batch::NCAND; ++c) {
      if (!b->use[c]) continue;
      snprintf(buf, sizeof buf, ";%s/%s=%.3fms", order_name(c), FORM_NAME[form_of(c)],
               b->tune_ms[c]);
      s += buf;
    }
  }
  snprintf(desc, (size_t)len, "%s", s.c_str());
  return CGD_OK;
}

int cgd_batch_get_stream(cgd_batch *b, void **stream)
{
  if (!b || !stream) return CGD_ERR_INVALID_ARG;
  *stream = b->stream;
  return CGD_OK;
}

}  // extern "C"
