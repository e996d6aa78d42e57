# ChainRulesCore rules for the B200 library's step and tendency, so Zygote or
# any ChainRules-based reverse mode differentiates a Julia loop over
# CGDB200.RosenbrockStep / CGDB200.Fcn through the hand-written adjoints
# (cgd_ros_step_adjoint, cgd_rhs_adjoint).  FP64 handles without tracers.
#
#   include("CGDB200.jl"); include("CGDB200Rules.jl")
#   using .CGDB200, .CGDB200Rules
#   g = Zygote.gradient(U0 -> J(foldl((U, _) -> CGDB200.RosenbrockStep(U, dt, CG, Metric, Phys, Global),
#                                     1:n; init = U0)), U0)
#
# Reverse mode through a loop keeps every intermediate state; for long runs
# use checkpointing (ChainRulesCore's or a manual one, as
# Dycore.steps_adjoint does in the Python binding).
module CGDB200Rules

using ChainRulesCore
import ..CGDB200

function ChainRulesCore.rrule(::typeof(CGDB200.RosenbrockStep), U, dt, CG, Metric, Phys, Global)
  U1 = CGDB200.RosenbrockStep(U, dt, CG, Metric, Phys, Global)
  function RosenbrockStep_pullback(dU1)
    Lin = similar(U)
    CGDB200.RosenbrockStepAdjointB200!(Lin, U, unthunk(dU1), dt, CG, Metric, Phys, Global)
    return (NoTangent(), Lin, NoTangent(), NoTangent(), NoTangent(), NoTangent(), NoTangent())
  end
  return U1, RosenbrockStep_pullback
end

function ChainRulesCore.rrule(::typeof(CGDB200.Fcn), U, CG, Metric, Phys, Global)
  F = CGDB200.Fcn(U, CG, Metric, Phys, Global)
  function Fcn_pullback(dF)
    LU = similar(U)
    CGDB200.FcnAdjointB200!(LU, U, unthunk(dF), CG, Metric, Phys, Global)
    return (NoTangent(), LU, NoTangent(), NoTangent(), NoTangent(), NoTangent())
  end
  return F, Fcn_pullback
end

end # module
