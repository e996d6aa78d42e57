"""cgd_b200 - B200 (sm_100a) implementation of CGDycore.jl's nonhydrostatic
spectral-element hot path (tendency + direct-stiffness summation +
Rosenbrock-W column Schur solve) behind a C ABI (include/cgd_b200.h).

Host-side modules:
  grid     cubed-sphere topology, Glob numbering, GLL element, metric, mass
  physics  physical parameters, baroclinic-wave initial state, run configs
  model    Dycore: fcn / fcn_prepare / jac / schur_solve / rosenbrock_schur /
           time_stepper over libcgd_b200.so, and their adjoints
           (fcn_adjoint / ros_step_adjoint / steps_adjoint); Ensemble:
           batched members
  adjoint  gradients of scalar functionals of a run (BoxPressureFunctional)
  parallel horizontal domain decomposition: element partition, halo plans,
           the DSS exchange over torch.distributed
  build    compiles libcgd_b200.so for sm_100a
"""
from . import grid, physics  # noqa: F401
from ._lib import CgdError, lib  # noqa: F401
from .model import Dycore, Ensemble, PartGroup, setup  # noqa: F401
