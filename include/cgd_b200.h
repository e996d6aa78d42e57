/*
 * cgd_b200.h - C ABI of the B200 (sm_100a) implementation of CGDycore.jl's
 * nonhydrostatic spectral-element hot path: the tendency (RHS) with its two
 * direct-stiffness summations, the vertical acoustic Jacobian, the column
 * Schur/tridiagonal solve and the SSP-Knoth Rosenbrock-W step.
 *
 * Plain pointers and sizes only.  Arrays use the reference's column-major
 * (Julia) layouts, so a caller holding the reference's arrays passes them
 * unchanged:
 *   Glob   int64 (N*N, NF), 1-based                 CG.Glob
 *   DS, DW (N, N)                                   CG.DS, CG.DW
 *   dXdxI  (3, 3, 2, N*N, nz, NF)                   Metric.dXdxI
 *   J      (N*N, 2, nz, NF)                         Metric.J
 *   X      (N*N, 2, 3, nz, NF)                      Metric.X
 *   M      (nz, NumG, 2)                            CG.M
 *   dz     (nz, NumG)                               Metric.dz
 *   U,F,k,v (nz, NumG, NV), NV = 5 + NumTr          state / tendency
 *           fields: rho, u, v, w (at the top interface of each layer),
 *           rho*theta, rho*q_1 ... rho*q_NumTr
 *
 * State/tendency pointers may be device memory (zero copy, e.g. a CuArray
 * or a torch tensor) or host memory (staged through device buffers owned by
 * the handle); the library tells them apart with cudaPointerGetAttributes.
 * Every call waits for the work the caller has queued on its stream (see
 * cgd_set_caller_stream), runs on the handle's CUDA stream and returns when
 * the result is complete.  A handle is not thread safe.
 *
 * Every function returns CGD_OK (0) or a negative error code; no exception
 * crosses the ABI and no device trap is used.  cgd_strerror() names a code.
 */
#ifndef CGD_B200_H
#define CGD_B200_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

#define CGD_OK 0
#define CGD_ERR_INVALID_ARG -1      /* null pointer, bad size or option */
#define CGD_ERR_SHAPE -2            /* extents inconsistent with the grid */
#define CGD_ERR_CUDA -3             /* a CUDA runtime call failed */
#define CGD_ERR_NONFINITE -4        /* NaN/Inf detected in the state */
#define CGD_ERR_TIMEOUT -5          /* a bounded device wait gave up */
#define CGD_ERR_INDEX -6            /* Glob entry out of range / unused id */
#define CGD_ERR_UNSUPPORTED -7      /* option not built into this library */
#define CGD_ERR_NO_DEVICE -8        /* no usable CUDA device */

#define CGD_PREC_FP64 0             /* everything in FP64 */
#define CGD_PREC_MIXED 1            /* FP32 perturbations, FP64 reference/column */
/* The mixed form evaluates the horizontal derivative sums of the tendency in
 * FP32, on pressure and theta minus an FP64 per-level reference profile (the
 * horizontal mean of each level of the first state the handle is given);
 * the vertical terms, the column Jacobian and Schur solve, the stage
 * updates and the reductions stay FP64.  No counterpart in the reference. */

#define CGD_FLAG_CHECK_FINITE 1     /* cgd_ros_step scans the state for NaN/Inf */

typedef struct cgd_config {
  int32_t OrdPoly;     /* p; N = p + 1 GLL nodes per direction (1 <= p <= 4) */
  int32_t nz;          /* layers (2 <= nz <= 64) */
  int32_t NumTr;       /* passive tracers (0 <= NumTr <= 4) */
  int32_t NF;          /* elements */
  int32_t NumG;        /* horizontal global DOFs */
  int32_t precision;   /* CGD_PREC_* */
  int32_t flags;       /* CGD_FLAG_* */
  int32_t reserved;
  /* PhysParameters (src/DyCore/GlobalVariables.jl:188-230) */
  double Grav, Rd, Cpd, p0, Omega;
  /* hyperdiffusion coefficients (Model.HyperDCurl/HyperDGrad/HyperDDiv) */
  double HyperDCurl, HyperDGrad, HyperDDiv;
} cgd_config;

typedef struct cgd_handle cgd_handle;

/* Builds the device-side grid: owner-gather maps from Glob, the compact
 * element metric, lumped mass, dz and the Coriolis parameter at layer
 * midpoints.  Host pointers, or device pointers for dXdxI, J, X, M and dz
 * (e.g. from cgd_metric_sphere / cgd_mass_dz); nothing is kept after the
 * call.
 * Replaces DyCore.InitSphere's device arrays (src/DyCore/InitDriver.jl:1-55,
 * src/DyCore/DiscretizationCG.jl:1-78) as consumed by the hot path. */
int cgd_create(const cgd_config *cfg, const int64_t *glob, const double *DS,
               const double *DW, const double *dXdxI, const double *J,
               const double *X, const double *M, const double *dz,
               cgd_handle **out);
void cgd_destroy(cgd_handle *h);

/* Horizontal domain decomposition.  One rank's part of the grid is a grid of
 * its own (its elements, the DOFs they touch, numbered locally) plus its
 * halo: the reference partitions the faces over MPI ranks
 * (src/Grids/InitGrid.jl:34-43, src/Grids/SubGridGhost.jl:1-239) and sums
 * each rank's boundary values with its neighbours' after both DSS points of
 * a tendency (ExchangeData3DSendGPU / ExchangeData3DRecvGPU!,
 * src/Parallels/Exchange.jl:938-1071; src/GPU/FcnGPU.jl:777-913).  Here the
 * ranks exchange element-node contributions and every rank sums all
 * contributors of a DOF in ascending global (element, node) order, so every
 * rank's DSS'd values, and the column solves that follow, equal the
 * single-process ones bit for bit.  Element-node indices are IF*DoF + ID of
 * the local numbering, 0-based. */
typedef struct cgd_halo {
  int32_t nnb;                 /* neighbour ranks */
  int32_t nb_boundary;         /* the first nb_boundary local elements touch another rank */
  const int32_t *nb_rank;      /* [nnb] ascending */
  const int32_t *send_ptr;     /* [nnb+1] offsets into send_list */
  const int32_t *send_list;    /* element nodes whose contributions go to nb_rank[i], in its slot order */
  const int32_t *recv_ptr;     /* [nnb+1]: ghost slots recv_ptr[i] .. recv_ptr[i+1]-1 come from nb_rank[i] */
  const int32_t *contrib_ptr;  /* [NumG+1] */
  const int32_t *contrib;      /* contributors of each local DOF, ascending global (element, node) order:
                                  c >= 0 a local element node, c < 0 the ghost slot -1-c */
} cgd_halo;

/* A rank's part of a decomposed grid (arguments as cgd_create, over the
 * rank's own elements and DOFs; M and dz are the single-process values at
 * its DOFs).  FP64 only (CGD_ERR_UNSUPPORTED for the mixed form).
 * cgd_rhs and cgd_ros_step on such a handle exchange contributions through
 * the function set with cgd_set_exchange; cgd_group_rhs and
 * cgd_group_ros_step run the parts of one process together instead.
 * The element partition and the plan come from cgd_b200.parallel (host). */
int cgd_create_part(const cgd_config *cfg, const int64_t *glob, const double *DS, const double *DW,
                    const double *dXdxI, const double *J, const double *X, const double *M, const double *dz,
                    const cgd_halo *halo, cgd_handle **out);

/* The exchange of one DSS point, supplied by the caller (e.g. NCCL peer
 * sends/receives between processes): nf contribution fields of nz levels per
 * element node are packed in `send` (neighbour i's items from
 * send_ptr[i]*nf*nz on) and must be received into `recv` (neighbour i's
 * items from recv_ptr[i]*nf*nz on) before the function returns, or be
 * ordered before later work on `stream` (the handle's cudaStream_t, on which
 * the packing was enqueued).  Returns 0 on success. */
typedef int (*cgd_exchange_fn)(void *user, void *stream, int32_t nf, const double *send, double *recv);
int cgd_set_exchange(cgd_handle *h, cgd_exchange_fn fn, void *user);
/* The device buffers the exchange reads and fills (sizes in doubles, for
 * nf = NV + 1). */
int cgd_halo_buffers(cgd_handle *h, double **send, int64_t *send_doubles, double **recv, int64_t *recv_doubles);

/* All parts of a decomposed grid in one process on one device (parts[r] is
 * rank r): the tendency F[r] = Fcn(U[r]) or nsteps Rosenbrock-W steps of
 * every U[r] in place, each DSS point exchanging the parts' contributions by
 * device copies.  Device pointers.  Ordered after the work queued on every
 * part's caller stream; returns with the work complete. */
int cgd_group_rhs(cgd_handle *const *parts, int32_t n, const double *const *U, double *const *F);
int cgd_group_ros_step(cgd_handle *const *parts, int32_t n, double *const *U, double dt, int32_t nsteps);

/* The grid's floating-point arrays formed on the device (the host keeps the
 * integer topology and Glob numbering).  Replaces the set-up kernels
 * JacobiSphere3Kernel! (src/Grids/JacobiSphere3GPU.jl:102-215, shallow
 * atmosphere, Sleve height at zero orography, src/Grids/Adapt.jl:19-31),
 * MassCGKernel! (src/DyCore/MassCG.jl:61-75) and GridSizeSphereKernel!
 * (src/DyCore/DiscretizationCG.jl:119-144).
 * cgd_metric_sphere: X, dXdxI, J (layouts above; device memory) from the
 * element corner points FP (NF, 4, 3; row-major), the GLL nodes xw (N),
 * DS (N, N) and the level heights z (nz + 1), top height H, radius Rad.  The
 * device's sin/cos/asin/atan2 may differ from a host libm in the last bit.
 * cgd_mass_dz: M (nz, NumG, 2), MMass (nz, NumG), dz (nz, NumG) (device
 * memory) from Glob (host), the GLL weights w (N) and the device X and J;
 * contributors summed in ascending (element, node) order.
 * cgd_create accepts these device arrays directly and then forms its
 * element metric on the device too.  Both calls synchronise the device. */
int cgd_metric_sphere(int32_t OrdPoly, int32_t nz, int32_t NF, const double *FP, const double *xw, const double *DS,
                      const double *z, double H, double Rad, double *X, double *dXdxI, double *J);
int cgd_mass_dz(int32_t OrdPoly, int32_t nz, int32_t NF, int32_t NumG, const int64_t *glob, const double *w,
                const double *J, const double *X, double *M, double *MMass, double *dz);

/* Column physics in the tendency tail, after the DSS (src/GPU/FcnGPU.jl:953-966):
 *   held_suarez  the dry Held-Suarez forcing, ForceKernel! with
 *                HeldSuarezDryExample's Force (src/GPU/OperatorKernel.jl:1073-1080,
 *                src/Examples/initial.jl:513-531; default parameters
 *                ParamHeldSuarezDrySphere, src/Examples/parameters.jl:122-131):
 *                Rayleigh friction of u, v below sigma_b and Newtonian
 *                relaxation of the temperature to Teq(lat, sigma);
 *   damping      DampKernel! with DampingW (OperatorKernel.jl:1061-1071,
 *                src/GPU/dampingGPU.jl:1-19): w relaxed at the rate
 *                damp_relax sin^2(pi/2 (1 - (damp_H - zP)/damp_stride)) in the top
 *                damp_stride metres below damp_H (zP the layer-midpoint height).
 * X is the node positions (N*N, 2, 3, nz, NF) (host or device) and Rad the
 * radius: each column's latitude (of its surface node) and zP are formed
 * once here, on the host.  Every later tendency (cgd_rhs) and step includes
 * the terms.  FP64 handles (CGD_ERR_UNSUPPORTED for the mixed form); the
 * adjoints do not differentiate them (CGD_ERR_UNSUPPORTED while set). */
typedef struct cgd_physics {
  int32_t held_suarez, damping;
  double k_a, k_f, k_s, DeltaT_y, DeltaTh_z, T_equator, T_min, sigma_b;
  double damp_H, damp_stride, damp_relax;
  double Rad;
} cgd_physics;
int cgd_set_physics(cgd_handle *h, const cgd_physics *phys, const double *X);

/* Pressure p (nz, NumG) from the state.
 * Replaces GPU.FcnPrepareGPU! / PressureKernel! (src/GPU/DiagnosticKernel.jl:96-115,180-218). */
int cgd_prepare(cgd_handle *h, const double *U, double *p);

/* Phase-1 hyperviscosity with its DSS: Temp1 (nz, NumG, 5 + NumTr).
 * Replaces HyperViscKernel!/HyperViscTracerKernel! + the first
 * ExchangeData3D (src/GPU/ViscKernel.jl:1-84,169-218; src/GPU/FcnGPU.jl:744-802). */
int cgd_hypervisc_phase1(cgd_handle *h, const double *U, double *Temp1);

/* Tendency F = Fcn(U) including FcnPrepare (pressure in register).
 * Replaces GPU.FcnGPU!(F,U,...,::CompressibleShallow) (src/GPU/FcnGPU.jl:552-968). */
int cgd_rhs(cgd_handle *h, const double *U, double *F);

/* Adjoint of the tendency: LU = (dF/dU)^T LF at the state U (all three
 * (nz, NumG, NV)), FP64, no tracers (CGD_ERR_UNSUPPORTED otherwise).
 * Hand-written reverse of the two phases and their direct-stiffness
 * summations (the adjoint of the owner gather is a broadcast).  Sums are
 * accumulated with atomics, so repeated calls agree to rounding, not bit for
 * bit.  No counterpart in the reference (it has no adjoint). */
int cgd_rhs_adjoint(cgd_handle *h, const double *U, const double *LF, double *LU);

/* Vertical acoustic Jacobian bands from U, kept in the handle; optionally
 * copied to bands (4, 2, nz-1, NumG) = JRhoW, JWRho, JWRhoTh, JRhoThW.
 * Replaces DyCore.JacSchurGPU! (src/DyCore/JacSchur.jl:3-75). */
int cgd_jac(cgd_handle *h, const double *U, double *bands);

/* The same bands written into the four caller-owned arrays of the
 * reference's JCache (src/Integration/JacCache.jl:1-20,62-70), each
 * (2, nz-1, NumG), device or host memory; the handle keeps a copy too.
 * Replaces JacSchurGPU!(J, U, ...) (src/DyCore/JacSchur.jl:3-27), which
 * fills J.JRhoW, J.JWRho, J.JWRhoTh and J.JRhoThW. */
int cgd_jac_bands(cgd_handle *h, const double *U, double *JRhoW, double *JWRho, double *JWRhoTh,
                  double *JRhoThW);

/* Column Schur solve with the bands of the last cgd_jac/cgd_jac_bands: k
 * from v (v is overwritten as in the reference), fac = dt*gamma.
 * Replaces Integration.SchurSolveGPU! (src/Integration/SchurSolve.jl:149-177)
 * when the bands stay inside the library. */
int cgd_schur_solve(cgd_handle *h, double *k, double *v, double fac);

/* Column Schur solve with the bands passed explicitly, as the reference's
 * SchurSolveGPU!(k, v, J, fac, Cache, Global) reads them from J
 * (src/Integration/SchurSolve.jl:149-177): JRhoW, JWRho, JWRhoTh, JRhoThW
 * each (2, nz-1, NumG), device memory (read in place) or host memory
 * (staged through the handle's band buffer, which then no longer holds the
 * bands of the last cgd_jac).  The tridiagonal matrix (J.tri) is formed
 * from the bands on every call.  k from v, v overwritten, fac = dt*gamma. */
int cgd_schur_solve_bands(cgd_handle *h, double *k, double *v, const double *JRhoW, const double *JWRho,
                          const double *JWRhoTh, const double *JRhoThW, double fac);

/* nsteps SSP-Knoth Rosenbrock-W steps of size dt, in place.  One step is a
 * captured CUDA graph (3 stages x {hyperviscosity+DSS, tendency+DSS,
 * fused column Schur solve}).
 * Replaces Integration.RosenbrockSchur! (src/Integration/RosenbrockSchur.jl:1-33)
 * inside TimeStepper! (src/Integration/TimeStepper.jl:103-124). */
int cgd_ros_step(cgd_handle *h, double *U, double dt, int32_t nsteps);

/* Adjoint of one Rosenbrock-W step U1 = step(U0, dt): Lin = (dU1/dU0)^T Lout
 * (all three (nz, NumG, NV)), FP64, no tracers (CGD_ERR_UNSUPPORTED
 * otherwise).  Replays the forward step from U0 (keeping the stage states,
 * phase-1 caches, pressures and k, and the bands), then runs the stages in
 * reverse: the transposed
 * column Schur solve (including the derivative of the Jacobian bands with
 * respect to U0), the tendency adjoint at the stage state, and the stage
 * combinations.  Multi-step gradients chain this call over checkpointed
 * states.  No counterpart in the reference (it has no adjoint). */
int cgd_ros_step_adjoint(cgd_handle *h, const double *U0, const double *Lout, double *Lin, double dt);

/* Recorded steps for multi-step gradients.  cgd_tape_record_step advances U
 * by one step in place (as cgd_ros_step, but not as a captured graph) and
 * keeps in tape slot `slot` what the step's reverse reads: a copy of the
 * initial state, the stage states, their phase-1 caches and pressures, the
 * stage k and the Jacobian bands (cgd_tape_bytes_per_step bytes of device
 * memory per slot, allocated on first use of the slot).
 * cgd_tape_step_adjoint then gives Lin = (dU1/dU0)^T Lout for the step in
 * that slot without replaying it.  A checkpointed gradient records each
 * segment's steps into slots 0..k-1 and runs their adjoints backwards.
 * cgd_tape_release frees every slot.  FP64 handles without tracers
 * (CGD_ERR_UNSUPPORTED otherwise).  No counterpart in the reference. */
#define CGD_TAPE_MAX_SLOTS 4096
int cgd_tape_record_step(cgd_handle *h, int32_t slot, double *U, double dt);
int cgd_tape_step_adjoint(cgd_handle *h, int32_t slot, const double *Lout, double *Lin);
int cgd_tape_release(cgd_handle *h);
int64_t cgd_tape_bytes_per_step(const cgd_handle *h);

/* sum(rho * MMass) over all DOFs, reduced in FP64 on the device (MMass is
 * the caller's lumped quadrature mass (nz, NumG)).
 * Replaces Parallels.GlobalIntegral (src/Parallels/Exchange.jl:1163-1166). */
int cgd_mass_integral(cgd_handle *h, const double *U, const double *MMass, double *out);

/* ---- Output: the state interpolated to OrdPrint x OrdPrint sub-cells per
 * element and layer, the cell data of the reference's VTK files.
 * inter (OrdPrint, OrdPrint, N, N): inter[I,J,i,j] = L_i(xi_I) L_j(eta_J),
 * L the GLL Lagrange basis, (xi_I, eta_J) the sub-cell centres.
 * cCell (OrdPrint, OrdPrint, nz, NF).  1 <= OrdPrint <= 8.  Inputs and
 * outputs may be host or device memory (as the state pointers above). */

/* The weights from the N = OrdPoly + 1 GLL points xw (host memory, no device
 * work).  Replaces the vtkInter of Outputs.vtkStruct
 * (src/Outputs/vtkSphere.jl:199-219). */
int cgd_vtk_inter(int32_t OrdPoly, int32_t OrdPrint, const double *xw, double *inter);

/* cCell from c (nz, NumG), each nodal value divided by rhoc (nz, NumG)
 * first when rhoc is not NULL.  Replaces Outputs.InterpolateGPU! and
 * InterpolateRhoGPU! (src/Outputs/vtkOutputKernel.jl:49-74,97-121,215-233,254-272). */
int cgd_interpolate(cgd_handle *h, const double *c, const double *rhoc, const double *inter, int32_t OrdPrint,
                    double *cCell);

/* Layer-mean w (0.5 (w(l) + w(l-1)); in the lowest layer the surface value
 * w0 = -(u dXdxI[3,1] + v dXdxI[3,2]) / dXdxI[3,3] of the lower node) from u,
 * v, w (nz, NumG).  Replaces Outputs.InterpolateWBGPU!
 * (src/Outputs/vtkOutputKernel.jl:123-159,274-291). */
int cgd_interpolate_wb(cgd_handle *h, const double *u, const double *v, const double *w, const double *inter,
                       int32_t OrdPrint, double *cCell);

/* Element-local vertical vorticity of the state's u, v (no direct-stiffness
 * summation), divided by J.  Replaces Outputs.InterpolateVortGPU!
 * (src/Outputs/vtkOutputKernel.jl:1-47,186-212), whose atomic sums have no
 * fixed order; here every sum runs in ascending node order. */
int cgd_interpolate_vort(cgd_handle *h, const double *U, const double *inter, int32_t OrdPrint, double *cCell);

/* Output quantities of cgd_output_fields, by the reference's cNames
 * (unstructured_vtkSphere, src/Outputs/vtkSphere.jl:337-510). */
#define CGD_OUT_RHO 0     /* "Rho" */
#define CGD_OUT_U 1       /* "u" */
#define CGD_OUT_V 2       /* "v" */
#define CGD_OUT_WB 3      /* "wB": as the reference calls it, with u passed for v (vtkSphere.jl:401-407) */
#define CGD_OUT_TH 4      /* "Th": (p0/p)^(Rd/Cpd) T of the dry model (Cache.AuxG[:,:,3]) */
#define CGD_OUT_PRES 5    /* "Pres": the dry model's pressure (Cache.AuxG[:,:,1]) */
#define CGD_OUT_VORT 6    /* "Vort" */
#define CGD_OUT_WB_UV 7   /* layer-mean w with the surface value from u and v */
#define CGD_OUT_TR 16     /* "Tr1" = CGD_OUT_TR, "Tr2" = CGD_OUT_TR + 1, ...: rho*q / rho */

/* The listed quantities of the state U (nz, NumG, NV) in one call, each
 * launched on the handle's stream as soon as the previous one is queued:
 * out holds nfields cCell arrays back to back (one copy to the host at the
 * end when out is host memory).  Replaces the interpolation and copy loop of
 * Outputs.unstructured_vtkSphere (src/Outputs/vtkSphere.jl:356-510); the
 * file itself is written by the caller. */
int cgd_output_fields(cgd_handle *h, const double *U, const int32_t *fields, int32_t nfields, const double *inter,
                      int32_t OrdPrint, double *out);

/* Allocation-free Jacobian + column Schur solve.  Some callers cannot let a
 * library allocate device memory: a host runtime whose device memory belongs
 * to its own pool allocator (CUDA.jl, PyTorch), where a cudaMalloc or
 * cudaFree behind the pool's back synchronises the device, fragments it or
 * is forbidden by the embedding application.  This entry point allocates
 * nothing.  No counterpart in the reference (its solve always uses the
 * JCache arrays allocated with the model).
 * Computes the vertical acoustic Jacobian bands of U and solves k from v
 * (v is updated as by cgd_schur_solve), with fac = dt*gamma.  Uses only
 * cfg->nz, NumG, NumTr, Grav, Rd, Cpd, p0.  U, dz, k, v must be device
 * memory.  The work is enqueued on `stream` (a cudaStream_t, NULL = the
 * legacy default stream) and the call returns without waiting for it: the
 * caller synchronises that stream, or orders later work after it, before
 * reading k or v.  Launch errors are returned; errors of the running
 * kernels surface at the caller's next synchronisation.
 * Scratch: the bands live in one file-scope device array of
 * CGD_NOALLOC_SCRATCH_DOUBLES doubles (32 MiB).  Each library file
 * (libcgd_b200.so and libcgd_b200_exact.so) holds its own array on every
 * GPU where that file is used, until the process exits.  8*(nz-1)*NumG must
 * not exceed it, otherwise CGD_ERR_SHAPE.  The first call on a device looks
 * up the array's device address (cudaGetSymbolAddress, with that device
 * current) and keeps it for the life of the process, so make that first
 * call before any stream capture, and do not reset the device
 * (cudaDeviceReset) between calls.  Every call overwrites the whole band
 * region it uses, so nothing needs clearing between calls; calls through
 * the same library file whose work overlaps on one GPU share the array and
 * race, so order them on one stream. */
#define CGD_NOALLOC_SCRATCH_DOUBLES (4u * 1024u * 1024u)
int cgd_jac_schur_solve_noalloc(const cgd_config *cfg, const double *U, const double *dz,
                                double *k, double *v, double fac, void *stream);

/* Batched ensemble.  Members are handles that share OrdPoly, NumTr, the
 * precision and the device; their grids (nPanel, nz) may differ.  One
 * ensemble step advances every member by one Rosenbrock-W step of its own
 * dt, as one CUDA graph over flat work lists spanning all members (the
 * kernels of one stage read each member's parameters from constant memory):
 * either 15 launches (split form) or, with CGD_BATCH_FUSED (OrdPoly 4 only,
 * CGD_ERR_UNSUPPORTED otherwise), three persistent cooperative launches, one
 * per stage, each running pressure, both tendency phases with their DSS and
 * the column solve and update with a grid barrier between them (fused form;
 * it allocates a second contribution buffer and a second stage state per
 * member; a barrier wait that exceeds a few seconds ends the launch and the
 * step returns CGD_ERR_TIMEOUT).  Calls on different batches must not run
 * concurrently: they share those constant tables.  The member handles must
 * stay alive and must not be stepped on their own while their batch steps.
 * With CGD_BATCH_MEMBERS the graph instead holds every member's own step
 * (the single-member kernels and buffers, bit-identical to cgd_ros_step of
 * that member) on the member's stream, forked from the batch stream and
 * joined back, the members one after the other (members form); its kernels
 * take the state pointers, so its graph is captured again when the states
 * or time steps passed to cgd_batch_step change.
 * With CGD_BATCH_AUTOTUNE the first cgd_batch_step times the candidates -
 * each work-list order (member-major, largest member first, interleaved) in
 * the split form and, for OrdPoly 4, in the split form with phase 2 in
 * 8-level instead of 16-level CTAs and in the fused form, and the members
 * form with the members in the given order, the largest first, or all at
 * once as concurrent branches - on copies of the states and keeps the
 * fastest; cgd_batch_tuning reports it.
 * No counterpart in the reference, which runs one configuration per job. */
#define CGD_BATCH_AUTOTUNE 1
#define CGD_BATCH_FUSED 2
#define CGD_BATCH_MEMBERS 4
typedef struct cgd_batch cgd_batch;
int cgd_batch_create(cgd_handle *const *members, int32_t nmembers, int32_t flags, cgd_batch **out);
/* U[m] device pointers, dt[m] step sizes; nsteps ensemble steps, in place. */
int cgd_batch_step(cgd_batch *b, double *const *U, const double *dt, int32_t nsteps);
/* Check of the grid barrier that the fused stage kernel uses (a bounded spin
 * on a generation word).  absent = 0: a cooperative launch of two CTAs per
 * SM passes `rounds` barriers, and *violations counts the CTAs that got past
 * a barrier before every CTA had arrived (0 expected).  absent != 0: one CTA
 * waits for a participant that never arrives; its wait ends after limit_s
 * seconds (at most 10) and the call returns CGD_ERR_TIMEOUT, leaving the
 * context usable.  Runs on the current device and synchronises it.  No
 * counterpart in the reference. */
int cgd_grid_barrier_check(int32_t rounds, int32_t absent, double limit_s, int32_t *violations);
/* The chosen candidate and the timed ones ("order=...;stage=split|fused;
 * phase2_levels=<levels per phase-2 CTA>;<order>/<split|split8|fused>=..ms;..."). */
int cgd_batch_tuning(cgd_batch *b, char *desc, int32_t len);
int cgd_batch_get_stream(cgd_batch *b, void **stream);
void cgd_batch_destroy(cgd_batch *b);

/* The handle's CUDA stream (cudaStream_t) so a caller can order its own
 * work or timing events with the library's.  No counterpart in the
 * reference (KernelAbstractions owns its queue). */
int cgd_get_stream(cgd_handle *h, void **stream);

/* Device arrays the caller passes may still be being written by work it
 * queued on its own stream.  Every call first makes the handle's stream wait
 * for that work (an event recorded on the caller's stream), so no explicit
 * synchronisation is needed before a call; every call returns with its own
 * work complete.  The caller's stream is the legacy default stream (the one
 * PyTorch uses by default) unless set here: a cudaStream_t, or NULL for the
 * legacy default stream again.  A CUDA.jl caller passes its task's stream.
 * Batches follow the caller stream of their first member.  No counterpart
 * in the reference (its kernels and arrays share one KernelAbstractions
 * queue). */
int cgd_set_caller_stream(cgd_handle *h, void *stream);

/* Average duration (ms) of the last timed launches of each kernel family
 * recorded when CGD_PROFILE=1; names separated by ';'.  Diagnostics only. */
int cgd_kernel_times(cgd_handle *h, char *names, int32_t names_len, double *ms, int32_t nmax);

const char *cgd_strerror(int code);
/* Library build string (arch, options). */
const char *cgd_version(void);

#ifdef __cplusplus
}
#endif
#endif /* CGD_B200_H */
