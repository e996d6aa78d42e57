# CGDB200.jl - Julia binding of libcgd_b200.so for CGDycore.jl.
#
# Drop-in replacements for the functions that CGDycore.jl passes into
# Integration.TimeStepper! (src/Integration/TimeStepper.jl:1,103-124):
#
#   Fcn!             = GPU.FcnGPU!          (src/GPU/FcnGPU.jl:552)
#   FcnPrepare!      = GPU.FcnPrepareGPU!   (src/GPU/DiagnosticKernel.jl:180)
#   Jac!             = DyCore.JacSchurGPU!  (src/DyCore/JacSchur.jl:3)
#   RosenbrockSchur! = Integration.RosenbrockSchur! (src/Integration/RosenbrockSchur.jl:1)
#
# and for the VTK output, the interpolation kernels of
# Outputs.unstructured_vtkSphere (src/Outputs/vtkOutputKernel.jl).
#
# The arguments are the reference's own (CG, Metric, Phys, Cache, Exchange,
# Global, Param, DiscType); the library keeps its device copies of the grid
# in a handle created once from them.  State arrays (CuArray or Array,
# Float64, layout (nz, NumG, NV)) are passed by pointer without copies when
# they live on the device.
module CGDB200

const libcgd = get(ENV, "CGD_B200_LIB", joinpath(@__DIR__, "..", "libcgd_b200.so"))

# struct cgd_config (include/cgd_b200.h)
struct CgdConfig
  OrdPoly::Int32
  nz::Int32
  NumTr::Int32
  NF::Int32
  NumG::Int32
  precision::Int32
  flags::Int32
  reserved::Int32
  Grav::Float64
  Rd::Float64
  Cpd::Float64
  p0::Float64
  Omega::Float64
  HyperDCurl::Float64
  HyperDGrad::Float64
  HyperDDiv::Float64
end

mutable struct Handle
  ptr::Ptr{Cvoid}
end

check(rc, what) = rc == 0 || error("$what: " * unsafe_string(ccall((:cgd_strerror, libcgd), Cstring, (Cint,), rc)))

hostcopy(a) = Array{eltype(a)}(a)

# One handle per (Global, precision): Global is the reference's per-model
# struct that every injected function receives (SchurSolveGPU! gets no CG or
# Metric), so the handle created from (CG, Metric, Phys, Global) on first use
# is found again from Global alone.  A mixed-form handle and an FP64 handle of
# the same model are different handles.
const HANDLES = IdDict{Any,Dict{Bool,Handle}}()

function config(CG, Global, Phys; mixed = false, check_finite = false)
  CgdConfig(CG.OrdPoly, Global.Grid.nz, Global.Model.NumTr, Global.Grid.NumFaces, CG.NumG,
            mixed ? 1 : 0, check_finite ? 1 : 0, 0,
            Phys.Grav, Phys.Rd, Phys.Cpd, Phys.p0, Phys.Omega,
            Global.Model.HyperDCurl, Global.Model.HyperDGrad, Global.Model.HyperDDiv)
end

# mixed = true selects the mixed form (FP32 horizontal derivative sums and DSS
# around an FP64 per-level reference; FP64 column solve).
function handle(CG, Metric, Phys, Global; mixed = false)
  byprec = get!(HANDLES, Global) do
    Dict{Bool,Handle}()
  end
  get!(byprec, mixed) do
    cfg = Ref(config(CG, Global, Phys; mixed = mixed))
    glob = Int64.(hostcopy(CG.Glob))
    DS, DW = hostcopy(CG.DS), hostcopy(CG.DW)
    dXdxI, J, X = hostcopy(Metric.dXdxI), hostcopy(Metric.J), hostcopy(Metric.X)
    M, dz = hostcopy(CG.M), hostcopy(Metric.dz)
    out = Ref{Ptr{Cvoid}}(C_NULL)
    rc = ccall((:cgd_create, libcgd), Cint,
               (Ref{CgdConfig}, Ptr{Int64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64},
                Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ref{Ptr{Cvoid}}),
               cfg, glob, DS, DW, dXdxI, J, X, M, dz, out)
    check(rc, "cgd_create")
    h = Handle(out[])
    finalizer(x -> ccall((:cgd_destroy, libcgd), Cvoid, (Ptr{Cvoid},), x.ptr), h)
    h
  end
end

# The handle of a model whose handle exists already (the injected functions
# that receive no CG or Metric).
function handle(Global; mixed = false)
  byprec = get(HANDLES, Global, nothing)
  (byprec === nothing || !haskey(byprec, mixed)) &&
    error("CGDB200: no handle for this Global; call FcnB200!, FcnPrepareB200! or JacB200! first")
  byprec[mixed]
end

# Pointer of a host Array or a CuArray (CUDA.jl converts CuArray to CuPtr;
# the library accepts either kind of address).
dptr(a::Array{Float64}) = pointer(a)
dptr(a) = reinterpret(Ptr{Float64}, UInt(pointer(a)))

# FcnPrepare!(U, CG, Metric, Phys, Cache, Exchange, Global, Param, DiscType):
# the pressure is recomputed in registers by every kernel that needs it, so
# this only refreshes Cache.AuxG[:,:,1] when the caller wants p on the host side.
function FcnPrepareB200!(U, CG, Metric, Phys, Cache, Exchange, Global, Param, DiscType)
  h = handle(CG, Metric, Phys, Global)
  p = Cache.AuxG
  GC.@preserve U p begin
    check(ccall((:cgd_prepare, libcgd), Cint, (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}),
                h.ptr, dptr(U), dptr(p)), "cgd_prepare")
  end
end

# Fcn!(F, U, CG, Metric, Phys, Cache, Exchange, Global, Param, DiscType)
function FcnB200!(F, U, CG, Metric, Phys, Cache, Exchange, Global, Param, DiscType)
  h = handle(CG, Metric, Phys, Global)
  GC.@preserve F U begin
    check(ccall((:cgd_rhs, libcgd), Cint, (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}),
                h.ptr, dptr(U), dptr(F)), "cgd_rhs")
  end
end

# Jac!(JCache, U, CG, Metric, Phys, Cache, Global, Param, DiscType) =
# DyCore.JacSchurGPU! (src/DyCore/JacSchur.jl:3-27): fills the four band
# arrays of the JStruct (src/Integration/JacCache.jl:62-66), each
# (2, nz-1, NumG), so the reference's own SchurSolveGPU! or SchurSolveB200!
# can read them.  JCache.CompTri is set as the reference's RosenbrockSchur!
# expects (the library forms the tridiagonal matrix from the bands itself).
function JacB200!(JCache, U, CG, Metric, Phys, Cache, Global, Param, DiscType)
  h = handle(CG, Metric, Phys, Global)
  GC.@preserve U JCache begin
    check(ccall((:cgd_jac_bands, libcgd), Cint,
                (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}),
                h.ptr, dptr(U), dptr(JCache.JRhoW), dptr(JCache.JWRho), dptr(JCache.JWRhoTh),
                dptr(JCache.JRhoThW)), "cgd_jac_bands")
  end
  JCache.CompTri = true
end

# SchurSolve!(k, v, J, fac, Cache, Global) = Integration.SchurSolveGPU!
# (src/Integration/SchurSolve.jl:149-177) with the reference's signature: the
# bands come from J (filled by JacB200! or by the reference's JacSchurGPU!).
function SchurSolveB200!(k, v, J, fac, Cache, Global)
  h = handle(Global)
  GC.@preserve k v J begin
    check(ccall((:cgd_schur_solve_bands, libcgd), Cint,
                (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64},
                 Ptr{Float64}, Cdouble),
                h.ptr, dptr(k), dptr(v), dptr(J.JRhoW), dptr(J.JWRho), dptr(J.JWRhoTh), dptr(J.JRhoThW),
                fac), "cgd_schur_solve_bands")
  end
  J.CompTri = false
end

# RosenbrockSchur!(V, dt, Fcn!, FcnPrepare!, Jac, CG, Metric, Phys, Cache,
# JCache, Exchange, Global, Param, DiscType): one SSP-Knoth step in place, as
# one CUDA graph.  Fcn!/FcnPrepare!/Jac are ignored (the library fuses them).
function RosenbrockSchurB200!(V, dt, Fcn!, FcnPrepare!, Jac, CG, Metric, Phys, Cache, JCache,
                              Exchange, Global, Param, DiscType)
  h = handle(CG, Metric, Phys, Global)
  GC.@preserve V begin
    check(ccall((:cgd_ros_step, libcgd), Cint, (Ptr{Cvoid}, Ptr{Float64}, Cdouble, Int32),
                h.ptr, dptr(V), dt, Int32(1)), "cgd_ros_step")
  end
end

# Allocation-free Jacobian + Schur solve (no counterpart in the reference),
# for a caller whose device memory belongs to CUDA.jl's pool allocator:
# bands in a static 32 MiB device array per library file;
# 8*(nz-1)*NumG <= 4_194_304.  The work is enqueued on `stream` and not
# waited for: synchronise that stream before reading k or v.
function JacSchurSolveNoAlloc!(k, v, U, dz, CG, Global, Phys, fac; stream = C_NULL)
  cfg = Ref(config(CG, Global, Phys))
  GC.@preserve k v U dz begin
    check(ccall((:cgd_jac_schur_solve_noalloc, libcgd), Cint,
                (Ref{CgdConfig}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Cdouble, Ptr{Cvoid}),
                cfg, dptr(U), dptr(dz), dptr(k), dptr(v), fac, stream), "cgd_jac_schur_solve_noalloc")
  end
end

# Batched ensemble: member handles (same OrdPoly, NumTr, precision) advance
# together, one CUDA graph per ensemble step (cgd_batch_step); states must be
# CuArrays.
mutable struct Batch
  ptr::Ptr{Cvoid}
  members::Vector{Handle}
end

function Batch(members::Vector{Handle}; autotune = true, fused = false, members_form = false)
  out = Ref{Ptr{Cvoid}}(C_NULL)
  ptrs = [m.ptr for m in members]
  flags = (autotune ? 1 : 0) | (fused ? 2 : 0) | (members_form ? 4 : 0)
  check(ccall((:cgd_batch_create, libcgd), Cint, (Ptr{Ptr{Cvoid}}, Int32, Int32, Ref{Ptr{Cvoid}}),
              ptrs, Int32(length(ptrs)), Int32(flags), out), "cgd_batch_create")
  b = Batch(out[], members)
  finalizer(x -> ccall((:cgd_batch_destroy, libcgd), Cvoid, (Ptr{Cvoid},), x.ptr), b)
  b
end

function step!(b::Batch, states, dts::Vector{Float64}; nsteps = 1)
  ptrs = [dptr(u) for u in states]
  GC.@preserve states begin
    check(ccall((:cgd_batch_step, libcgd), Cint, (Ptr{Cvoid}, Ptr{Ptr{Float64}}, Ptr{Float64}, Int32),
                b.ptr, ptrs, dts, Int32(nsteps)), "cgd_batch_step")
  end
end

# Column physics in the tendency tail (struct cgd_physics): the dry
# Held-Suarez forcing with the reference's ParamHeldSuarezDrySphere values
# (Param) and the Rayleigh damping of w in the top StrideDamp metres below H.
struct CgdPhysics
  held_suarez::Int32
  damping::Int32
  k_a::Float64
  k_f::Float64
  k_s::Float64
  DeltaT_y::Float64
  DeltaTh_z::Float64
  T_equator::Float64
  T_min::Float64
  sigma_b::Float64
  damp_H::Float64
  damp_stride::Float64
  damp_relax::Float64
  Rad::Float64
end

function set_physics!(h::Handle, Param, Metric, Phys; held_suarez = true, damping = nothing)
  dH, dS, dR = damping === nothing ? (0.0, 1.0, 0.0) : damping
  ph = Ref(CgdPhysics(Int32(held_suarez), Int32(damping !== nothing), Param.k_a, Param.k_f, Param.k_s,
                      Param.DeltaT_y, Param.DeltaTh_z, Param.T_equator, Param.T_min, Param.sigma_b,
                      dH, dS, dR, Phys.RadEarth))
  X = hostcopy(Metric.X)
  GC.@preserve X begin
    check(ccall((:cgd_set_physics, libcgd), Cint, (Ptr{Cvoid}, Ref{CgdPhysics}, Ptr{Float64}), h.ptr, ph,
                pointer(X)), "cgd_set_physics")
  end
end

# The stream whose queued work every call waits for (a cudaStream_t; a
# CUDA.jl caller passes CUDA.stream().handle); C_NULL = the legacy default stream.
function set_caller_stream!(h::Handle, stream)
  check(ccall((:cgd_set_caller_stream, libcgd), Cint, (Ptr{Cvoid}, Ptr{Cvoid}),
              h.ptr, reinterpret(Ptr{Cvoid}, stream)), "cgd_set_caller_stream")
end

# Non-mutating forms of the step and the tendency (the functions the
# ChainRulesCore rules in CGDB200Rules.jl differentiate).
function RosenbrockStep(U, dt, CG, Metric, Phys, Global)
  h = handle(CG, Metric, Phys, Global)
  U1 = copy(U)
  GC.@preserve U1 begin
    check(ccall((:cgd_ros_step, libcgd), Cint, (Ptr{Cvoid}, Ptr{Float64}, Cdouble, Int32),
                h.ptr, dptr(U1), dt, Int32(1)), "cgd_ros_step")
  end
  U1
end

function Fcn(U, CG, Metric, Phys, Global)
  h = handle(CG, Metric, Phys, Global)
  F = similar(U)
  GC.@preserve F U begin
    check(ccall((:cgd_rhs, libcgd), Cint, (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}),
                h.ptr, dptr(U), dptr(F)), "cgd_rhs")
  end
  F
end

# Adjoints (no counterpart in the reference; FP64 handles without tracers).
# FcnAdjointB200!: LU = (dF/dU)^T LF at U, F being FcnB200!'s tendency.
function FcnAdjointB200!(LU, U, LF, CG, Metric, Phys, Global)
  h = handle(CG, Metric, Phys, Global)
  GC.@preserve LU U LF begin
    check(ccall((:cgd_rhs_adjoint, libcgd), Cint, (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}),
                h.ptr, dptr(U), dptr(LF), dptr(LU)), "cgd_rhs_adjoint")
  end
end

# RosenbrockStepAdjointB200!: Lin = (dU1/dU0)^T Lout for one step
# U1 = RosenbrockSchurB200!(U0, dt); U0 is not modified.  A gradient over
# many steps chains this call backwards over stored (checkpointed) states.
function RosenbrockStepAdjointB200!(Lin, U0, Lout, dt, CG, Metric, Phys, Global)
  h = handle(CG, Metric, Phys, Global)
  GC.@preserve Lin U0 Lout begin
    check(ccall((:cgd_ros_step_adjoint, libcgd), Cint,
                (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Cdouble),
                h.ptr, dptr(U0), dptr(Lout), dptr(Lin), dt), "cgd_ros_step_adjoint")
  end
end

# ---- Output interpolation (src/Outputs/vtkOutputKernel.jl).  The reference's
# kernels take (cCell, c, Inter, Glob); these take the model's Global instead
# of Glob (the handle holds Glob and the metric).  Inter and the arrays may be
# host Arrays or CuArrays; column slices such as U[:,:,RhoPos] are contiguous.

# vtkStruct's vtkInter (src/Outputs/vtkSphere.jl:199-219) from CG.xwCPU.
function VtkInterB200(OrdPoly, OrdPrint, xw)
  inter = zeros(Float64, OrdPrint, OrdPrint, OrdPoly + 1, OrdPoly + 1)
  x = Vector{Float64}(xw)
  check(ccall((:cgd_vtk_inter, libcgd), Cint, (Int32, Int32, Ptr{Float64}, Ptr{Float64}),
              OrdPoly, OrdPrint, x, inter), "cgd_vtk_inter")
  inter
end

# InterpolateGPU!(cCell, c, Inter, Glob) (vtkOutputKernel.jl:215)
function InterpolateB200!(cCell, c, Inter, Global)
  h = handle(Global)
  GC.@preserve cCell c Inter begin
    check(ccall((:cgd_interpolate, libcgd), Cint,
                (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Int32, Ptr{Float64}),
                h.ptr, dptr(c), C_NULL, dptr(Inter), size(Inter, 1), dptr(cCell)), "cgd_interpolate")
  end
end

# InterpolateRhoGPU!(cCell, c, Rho, Inter, Glob) (vtkOutputKernel.jl:254)
function InterpolateRhoB200!(cCell, c, Rho, Inter, Global)
  h = handle(Global)
  GC.@preserve cCell c Rho Inter begin
    check(ccall((:cgd_interpolate, libcgd), Cint,
                (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Int32, Ptr{Float64}),
                h.ptr, dptr(c), dptr(Rho), dptr(Inter), size(Inter, 1), dptr(cCell)), "cgd_interpolate")
  end
end

# InterpolateWBGPU!(cCell, u, v, w, Inter, dXdxI, Glob) (vtkOutputKernel.jl:274)
function InterpolateWBB200!(cCell, u, v, w, Inter, Global)
  h = handle(Global)
  GC.@preserve cCell u v w Inter begin
    check(ccall((:cgd_interpolate_wb, libcgd), Cint,
                (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Int32, Ptr{Float64}),
                h.ptr, dptr(u), dptr(v), dptr(w), dptr(Inter), size(Inter, 1), dptr(cCell)), "cgd_interpolate_wb")
  end
end

# InterpolateVortGPU!(Vort, U, Inter, FE, Metric) (vtkOutputKernel.jl:186)
function InterpolateVortB200!(Vort, U, Inter, Global)
  h = handle(Global)
  GC.@preserve Vort U Inter begin
    check(ccall((:cgd_interpolate_vort, libcgd), Cint,
                (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Int32, Ptr{Float64}),
                h.ptr, dptr(U), dptr(Inter), size(Inter, 1), dptr(Vort)), "cgd_interpolate_vort")
  end
end

# CGD_OUT_* codes of cgd_output_fields by the reference's cNames
const OUTPUT_CODES = Dict("Rho" => 0, "u" => 1, "v" => 2, "wB" => 3, "Th" => 4, "Pres" => 5, "Vort" => 6,
                          "Tr1" => 16, "Tr2" => 17, "Tr3" => 18, "Tr4" => 19)

# All of Global.Output.cNames in one call: out (OrdPrint, OrdPrint, nz, NF, nfields).
function OutputFieldsB200!(out, U, cNames, Inter, Global)
  h = handle(Global)
  codes = Int32[OUTPUT_CODES[n] for n in cNames]
  GC.@preserve out U Inter codes begin
    check(ccall((:cgd_output_fields, libcgd), Cint,
                (Ptr{Cvoid}, Ptr{Float64}, Ptr{Int32}, Int32, Ptr{Float64}, Int32, Ptr{Float64}),
                h.ptr, dptr(U), codes, length(codes), dptr(Inter), size(Inter, 1), dptr(out)), "cgd_output_fields")
  end
end

end # module
