"""ctypes binding of libcgd_b200.so (the sm_100a hot-path library).

The library is built in tree (``__graft_entry__.build()`` or
``python -m cgd_b200.build``); importing this module never falls back to a
CPU implementation: if the shared library is missing, loading fails loudly.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.dirname(_HERE)
LIB_PATH = os.path.join(PKG_DIR, "libcgd_b200.so")               # fast build
LIB_PATH_EXACT = os.path.join(PKG_DIR, "libcgd_b200_exact.so")   # bit-exact build

CGD_OK = 0
ERRORS = {
    -1: "CGD_ERR_INVALID_ARG", -2: "CGD_ERR_SHAPE", -3: "CGD_ERR_CUDA", -4: "CGD_ERR_NONFINITE",
    -5: "CGD_ERR_TIMEOUT", -6: "CGD_ERR_INDEX", -7: "CGD_ERR_UNSUPPORTED", -8: "CGD_ERR_NO_DEVICE",
}
PREC_FP64, PREC_MIXED = 0, 1
NOALLOC_SCRATCH_DOUBLES = 4 * 1024 * 1024
FLAG_CHECK_FINITE = 1
BATCH_AUTOTUNE = 1
BATCH_FUSED = 2
BATCH_MEMBERS = 4

# every symbol declared in include/cgd_b200.h
EXPORTS = [
    "cgd_create", "cgd_destroy", "cgd_prepare", "cgd_hypervisc_phase1", "cgd_rhs", "cgd_jac",
    "cgd_jac_bands", "cgd_schur_solve", "cgd_schur_solve_bands", "cgd_ros_step", "cgd_mass_integral", "cgd_jac_schur_solve_noalloc", "cgd_get_stream",
    "cgd_kernel_times", "cgd_strerror", "cgd_version",
    "cgd_rhs_adjoint", "cgd_ros_step_adjoint", "cgd_set_caller_stream",
    "cgd_tape_record_step", "cgd_tape_step_adjoint", "cgd_tape_release", "cgd_tape_bytes_per_step",
    "cgd_batch_create", "cgd_batch_step", "cgd_batch_tuning", "cgd_batch_get_stream", "cgd_batch_destroy",
    "cgd_grid_barrier_check",
    "cgd_create_part", "cgd_set_exchange", "cgd_halo_buffers", "cgd_group_rhs", "cgd_group_ros_step",
    "cgd_metric_sphere", "cgd_mass_dz", "cgd_set_physics",
    "cgd_vtk_inter", "cgd_interpolate", "cgd_interpolate_wb", "cgd_interpolate_vort", "cgd_output_fields",
]

# output quantities of cgd_output_fields (CGD_OUT_* in include/cgd_b200.h)
OUT_RHO, OUT_U, OUT_V, OUT_WB, OUT_TH, OUT_PRES, OUT_VORT, OUT_WB_UV, OUT_TR = 0, 1, 2, 3, 4, 5, 6, 7, 16


class CgdConfig(ctypes.Structure):
    _fields_ = [("OrdPoly", ctypes.c_int32), ("nz", ctypes.c_int32), ("NumTr", ctypes.c_int32),
                ("NF", ctypes.c_int32), ("NumG", ctypes.c_int32), ("precision", ctypes.c_int32),
                ("flags", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("Grav", ctypes.c_double), ("Rd", ctypes.c_double), ("Cpd", ctypes.c_double),
                ("p0", ctypes.c_double), ("Omega", ctypes.c_double),
                ("HyperDCurl", ctypes.c_double), ("HyperDGrad", ctypes.c_double),
                ("HyperDDiv", ctypes.c_double)]


class CgdHalo(ctypes.Structure):
    _fields_ = [("nnb", ctypes.c_int32), ("nb_boundary", ctypes.c_int32), ("nb_rank", ctypes.c_void_p),
                ("send_ptr", ctypes.c_void_p), ("send_list", ctypes.c_void_p), ("recv_ptr", ctypes.c_void_p),
                ("contrib_ptr", ctypes.c_void_p), ("contrib", ctypes.c_void_p)]


# int (*cgd_exchange_fn)(void *user, void *stream, int32_t nf, const double *send, double *recv)
EXCHANGE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p,
                               ctypes.c_void_p)


class CgdPhysics(ctypes.Structure):
    _fields_ = [("held_suarez", ctypes.c_int32), ("damping", ctypes.c_int32)] + [
        (n, ctypes.c_double) for n in ("k_a", "k_f", "k_s", "DeltaT_y", "DeltaTh_z", "T_equator", "T_min",
                                      "sigma_b", "damp_H", "damp_stride", "damp_relax", "Rad")]


class CgdError(RuntimeError):
    def __init__(self, code, what=""):
        self.code = code
        msg = lib().cgd_strerror(code).decode() if _libs else ERRORS.get(code, "error")
        super().__init__(f"{what}: {ERRORS.get(code, code)} ({msg})")


_libs = {}


def lib(exact=False):
    """Load the fast (default) or the exact build (raises OSError if it has
    not been built; there is no fallback)."""
    path = LIB_PATH_EXACT if exact else LIB_PATH
    if path not in _libs:
        if not os.path.exists(path):
            raise OSError(f"{path} not found: build it with __graft_entry__.build()")
        L = ctypes.CDLL(path)
        vp, i32, dbl = ctypes.c_void_p, ctypes.c_int32, ctypes.c_double
        L.cgd_create.argtypes = [ctypes.POINTER(CgdConfig)] + [vp] * 8 + [ctypes.POINTER(vp)]
        L.cgd_create.restype = ctypes.c_int
        L.cgd_destroy.argtypes = [vp]
        L.cgd_destroy.restype = None
        L.cgd_rhs_adjoint.argtypes = [vp, vp, vp, vp]
        L.cgd_rhs_adjoint.restype = ctypes.c_int
        L.cgd_ros_step_adjoint.argtypes = [vp, vp, vp, vp, ctypes.c_double]
        L.cgd_ros_step_adjoint.restype = ctypes.c_int
        L.cgd_set_caller_stream.argtypes = [vp, vp]
        L.cgd_set_caller_stream.restype = ctypes.c_int
        L.cgd_tape_record_step.argtypes = [vp, i32, vp, ctypes.c_double]
        L.cgd_tape_record_step.restype = ctypes.c_int
        L.cgd_tape_step_adjoint.argtypes = [vp, i32, vp, vp]
        L.cgd_tape_step_adjoint.restype = ctypes.c_int
        L.cgd_tape_release.argtypes = [vp]
        L.cgd_tape_release.restype = ctypes.c_int
        L.cgd_tape_bytes_per_step.argtypes = [vp]
        L.cgd_tape_bytes_per_step.restype = ctypes.c_int64
        L.cgd_create_part.argtypes = [ctypes.POINTER(CgdConfig)] + [vp] * 8 + [ctypes.POINTER(CgdHalo),
                                                                              ctypes.POINTER(vp)]
        L.cgd_create_part.restype = ctypes.c_int
        L.cgd_set_exchange.argtypes = [vp, EXCHANGE_FN, vp]
        L.cgd_set_exchange.restype = ctypes.c_int
        L.cgd_halo_buffers.argtypes = [vp, ctypes.POINTER(vp), ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(vp),
                                       ctypes.POINTER(ctypes.c_int64)]
        L.cgd_halo_buffers.restype = ctypes.c_int
        L.cgd_group_rhs.argtypes = [vp, i32, vp, vp]
        L.cgd_group_rhs.restype = ctypes.c_int
        L.cgd_group_ros_step.argtypes = [vp, i32, vp, ctypes.c_double, i32]
        L.cgd_group_ros_step.restype = ctypes.c_int
        L.cgd_set_physics.argtypes = [vp, ctypes.POINTER(CgdPhysics), vp]
        L.cgd_set_physics.restype = ctypes.c_int
        L.cgd_metric_sphere.argtypes = [i32, i32, i32, vp, vp, vp, vp, dbl, dbl, vp, vp, vp]
        L.cgd_metric_sphere.restype = ctypes.c_int
        L.cgd_mass_dz.argtypes = [i32, i32, i32, i32, vp, vp, vp, vp, vp, vp, vp]
        L.cgd_mass_dz.restype = ctypes.c_int
        L.cgd_grid_barrier_check.argtypes = [i32, i32, ctypes.c_double, ctypes.POINTER(i32)]
        L.cgd_vtk_inter.argtypes = [i32, i32, vp, vp]
        L.cgd_interpolate.argtypes = [vp, vp, vp, vp, i32, vp]
        L.cgd_interpolate_wb.argtypes = [vp, vp, vp, vp, vp, i32, vp]
        L.cgd_interpolate_vort.argtypes = [vp, vp, vp, i32, vp]
        L.cgd_output_fields.argtypes = [vp, vp, vp, i32, vp, i32, vp]
        L.cgd_grid_barrier_check.restype = ctypes.c_int
        for f in ("cgd_prepare", "cgd_hypervisc_phase1", "cgd_rhs", "cgd_jac"):
            getattr(L, f).argtypes = [vp, vp, vp]
            getattr(L, f).restype = ctypes.c_int
        L.cgd_schur_solve.argtypes = [vp, vp, vp, dbl]
        L.cgd_schur_solve.restype = ctypes.c_int
        L.cgd_jac_bands.argtypes = [vp] * 6
        L.cgd_jac_bands.restype = ctypes.c_int
        L.cgd_schur_solve_bands.argtypes = [vp] * 7 + [dbl]
        L.cgd_schur_solve_bands.restype = ctypes.c_int
        L.cgd_ros_step.argtypes = [vp, vp, dbl, i32]
        L.cgd_ros_step.restype = ctypes.c_int
        L.cgd_mass_integral.argtypes = [vp, vp, vp, vp]
        L.cgd_mass_integral.restype = ctypes.c_int
        L.cgd_jac_schur_solve_noalloc.argtypes = [ctypes.POINTER(CgdConfig), vp, vp, vp, vp, dbl, vp]
        L.cgd_jac_schur_solve_noalloc.restype = ctypes.c_int
        L.cgd_batch_create.argtypes = [vp, i32, i32, ctypes.POINTER(vp)]
        L.cgd_batch_create.restype = ctypes.c_int
        L.cgd_batch_step.argtypes = [vp, vp, vp, i32]
        L.cgd_batch_step.restype = ctypes.c_int
        L.cgd_batch_tuning.argtypes = [vp, ctypes.c_char_p, i32]
        L.cgd_batch_tuning.restype = ctypes.c_int
        L.cgd_batch_get_stream.argtypes = [vp, ctypes.POINTER(vp)]
        L.cgd_batch_get_stream.restype = ctypes.c_int
        L.cgd_batch_destroy.argtypes = [vp]
        L.cgd_batch_destroy.restype = None
        L.cgd_get_stream.argtypes = [vp, ctypes.POINTER(vp)]
        L.cgd_get_stream.restype = ctypes.c_int
        L.cgd_kernel_times.argtypes = [vp, ctypes.c_char_p, i32, vp, i32]
        L.cgd_kernel_times.restype = ctypes.c_int
        L.cgd_strerror.argtypes = [ctypes.c_int]
        L.cgd_strerror.restype = ctypes.c_char_p
        L.cgd_version.argtypes = []
        L.cgd_version.restype = ctypes.c_char_p
        _libs[path] = L
    return _libs[path]


def check(rc, what):
    if rc != CGD_OK:
        raise CgdError(rc, what)
    return rc
