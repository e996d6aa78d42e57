"""Host-side mirror of the reference's hot-path interface.

The reference injects its GPU functions into the time loop as arguments
(``TimeStepper!(U, GPU.FcnGPU!, GPU.FcnPrepareGPU!, DyCore.JacSchurGPU!, ...)``,
Examples/testNHSphere.jl:508-509, src/Integration/TimeStepper.jl:1).  The
``Dycore`` object exposes the same operations, each a single call into
libcgd_b200.so:

  ==========================  ==============================================
  Dycore method               reference
  ==========================  ==============================================
  fcn_prepare(U)              GPU.FcnPrepareGPU! (DiagnosticKernel.jl:180)
  fcn(U)                      GPU.FcnGPU!(::CompressibleShallow) (FcnGPU.jl:552)
  hypervisc_phase1(U)         first phase of FcnGPU! (FcnGPU.jl:744-802)
  jac(U)                      DyCore.JacSchurGPU! (JacSchur.jl:3)
  jac_bands(J, U)             JacSchurGPU!(J, U, ...) filling the JCache bands
  schur_solve(v, fac)         Integration.SchurSolveGPU! (SchurSolve.jl:149)
  schur_solve_bands(k,v,J,f)  SchurSolveGPU!(k, v, J, fac, ...) with J's bands
  rosenbrock_schur(U, dt)     Integration.RosenbrockSchur! (RosenbrockSchur.jl:1)
  time_stepper(U, dt, n)      the Rosenbrock branch of TimeStepper! (TimeStepper.jl:103-124)
  mass_integral(U)            Parallels.GlobalIntegral (Exchange.jl:1163)
  interpolate(c, inter, rhoc) Outputs.InterpolateGPU! / InterpolateRhoGPU! (vtkOutputKernel.jl:215,254)
  interpolate_wb(u,v,w,inter) Outputs.InterpolateWBGPU! (vtkOutputKernel.jl:274)
  interpolate_vort(U, inter)  Outputs.InterpolateVortGPU! (vtkOutputKernel.jl:186)
  output_fields(U, codes, i)  the interpolation loop of unstructured_vtkSphere (vtkSphere.jl:337)
  fcn_adjoint(U, LF)          (no counterpart) (dF/dU)^T LF
  ros_step_adjoint(U0, L, dt) (no counterpart) adjoint of one step
  steps_adjoint(U0, L, dt, n) (no counterpart) checkpointed n-step gradient
  tape_record_step(...)       (no counterpart) recorded steps for it
  ==========================  ==============================================

State arrays are (nz, NumG, NV) in column-major order: a Fortran-ordered
float64 numpy array (host memory; copied through the library's buffers) or a
contiguous float64 CUDA torch tensor of shape (NV, NumG, nz) (device memory;
zero copy).  Errors raise ``CgdError`` with the library's error code.
"""
import ctypes

import numpy as np

from . import _lib
from .physics import PhysParameters


def _ptr(a, shape=None, writable=False):
    """Raw pointer of a numpy array (Fortran float64) or a torch tensor."""
    if isinstance(a, np.ndarray):
        if a.dtype != np.float64 or not a.flags.f_contiguous:
            raise ValueError("state arrays must be Fortran-ordered float64")
        if shape is not None and a.shape != tuple(shape):
            raise ValueError(f"expected shape {tuple(shape)}, got {a.shape}")
        if writable and not a.flags.writeable:
            raise ValueError("array is read-only")
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        import torch
        if a.dtype != torch.float64 or not a.is_contiguous():
            raise ValueError("tensors must be contiguous float64")
        if shape is not None and a.numel() != int(np.prod(shape)):
            raise ValueError("tensor has the wrong number of elements")
        return a.data_ptr()
    raise TypeError("expected a numpy array or a torch tensor")


class JacBands(tuple):
    """The four Jacobian band arrays of the reference's JStruct, in its field
    order for the solve: JRhoW, JWRho, JWRhoTh, JRhoThW."""

    def __new__(cls, JRhoW, JWRho, JWRhoTh, JRhoThW):
        return super().__new__(cls, (JRhoW, JWRho, JWRhoTh, JRhoThW))

    JRhoW = property(lambda self: self[0])
    JWRho = property(lambda self: self[1])
    JWRhoTh = property(lambda self: self[2])
    JRhoThW = property(lambda self: self[3])


def _copy(a):
    """A copy of a state array: Fortran-ordered for numpy, a clone for torch."""
    if isinstance(a, np.ndarray):
        return np.array(a, order="F", copy=True)
    return a.clone()


def _assign(dst, src):
    if isinstance(dst, np.ndarray):
        dst[...] = src
    else:
        dst.copy_(src)


def _empty_like(a):
    if isinstance(a, np.ndarray):
        return np.empty_like(a, order="F")
    return a.new_empty(a.shape)


class Dycore:
    """One model instance on the current CUDA device."""

    def __init__(self, grid, NumTr=0, nu=(0.0, 0.0, 0.0), phys=None, precision="fp64",
                 check_finite=False, exact=False, halo=None):
        """grid: the whole grid, or with halo (a parallel.HaloPlan) one
        rank's part of a decomposed grid (HaloPlan.local_grid)."""
        self.grid = grid
        self.phys = phys or PhysParameters(RadEarth=grid.Rad)
        self.nz, self.NumG, self.NF = grid.nz, grid.NumG, grid.NF
        self.NumTr, self.NV = NumTr, 5 + NumTr
        self.shape = (self.nz, self.NumG, self.NV)
        self.exact = exact
        self._L = L = _lib.lib(exact)
        cfg = _lib.CgdConfig()
        cfg.OrdPoly, cfg.nz, cfg.NumTr = grid.OrdPoly, grid.nz, NumTr
        cfg.NF, cfg.NumG = grid.NF, grid.NumG
        cfg.precision = _lib.PREC_MIXED if precision == "mixed" else _lib.PREC_FP64
        cfg.flags = _lib.FLAG_CHECK_FINITE if check_finite else 0
        ph = self.phys
        cfg.Grav, cfg.Rd, cfg.Cpd, cfg.p0, cfg.Omega = ph.Grav, ph.Rd, ph.Cpd, ph.p0, ph.Omega
        cfg.HyperDCurl, cfg.HyperDGrad, cfg.HyperDDiv = nu
        # host arrays, or the device tensors of grid.init_grid_sphere_device
        self._keep = [x if hasattr(x, "data_ptr") else np.asfortranarray(x, dtype=t) for x, t in (
            (grid.glob, np.int64), (grid.DS, np.float64), (grid.DW, np.float64),
            (grid.dXdxI, np.float64), (grid.J, np.float64), (grid.X, np.float64),
            (grid.M, np.float64), (grid.dz, np.float64))]
        ptrs = [k.data_ptr() if hasattr(k, "data_ptr") else k.ctypes.data for k in self._keep]
        h = ctypes.c_void_p()
        self.halo = halo
        if halo is None:
            rc = L.cgd_create(ctypes.byref(cfg), *ptrs, ctypes.byref(h))
        else:
            arrs = [np.ascontiguousarray(a, np.int32) for a in (halo.neighbours, halo.send_ptr, halo.send_list,
                                                               halo.recv_ptr, halo.contrib_ptr, halo.contrib)]
            hs = _lib.CgdHalo(int(halo.neighbours.size), int(halo.nb_boundary), *[a.ctypes.data for a in arrs])
            rc = L.cgd_create_part(ctypes.byref(cfg), *ptrs, ctypes.byref(hs), ctypes.byref(h))
        self._keep = None
        _lib.check(rc, "cgd_create")
        self._xfn = None
        self.h = h
        self._mmass = grid.MMass if hasattr(grid.MMass, "data_ptr") else np.asfortranarray(grid.MMass)

    def set_physics(self, held_suarez=None, damping=None):
        """Column physics in the tendency tail: held_suarez = True (the
        reference's ParamHeldSuarezDrySphere values) or a dict of them;
        damping = (H, StrideDamp, Relax) for the Rayleigh damping of w in the
        top StrideDamp metres below H.  None switches a term off."""
        from .physics import HELD_SUAREZ
        ph = _lib.CgdPhysics()
        hs = dict(HELD_SUAREZ, **(held_suarez if isinstance(held_suarez, dict) else {}))
        ph.held_suarez = int(bool(held_suarez))
        for k, v in hs.items():
            setattr(ph, k, float(v))
        ph.damping = int(damping is not None)
        ph.damp_H, ph.damp_stride, ph.damp_relax = damping if damping is not None else (0.0, 1.0, 0.0)
        ph.Rad = float(self.grid.Rad)
        X = self.grid.X
        xp = X.data_ptr() if hasattr(X, "data_ptr") else np.asfortranarray(X).ctypes.data
        _lib.check(self._L.cgd_set_physics(self.h, ctypes.byref(ph), xp), "cgd_set_physics")

    def set_transport(self, transport):
        """The exchange of a decomposed grid's rank between processes:
        transport.exchange(send_views, recv_views) (parallel.TorchTransport)
        is called at every DSS point with device views of the library's
        packed buffers, on the library's stream."""
        import torch
        P = self.halo
        sp, sn, rp, rn = ctypes.c_void_p(), ctypes.c_int64(), ctypes.c_void_p(), ctypes.c_int64()
        _lib.check(self._L.cgd_halo_buffers(self.h, ctypes.byref(sp), ctypes.byref(sn), ctypes.byref(rp),
                                            ctypes.byref(rn)), "cgd_halo_buffers")
        sbuf = torch.as_tensor(_DevArray(sp.value, max(1, sn.value)), device="cuda")
        rbuf = torch.as_tensor(_DevArray(rp.value, max(1, rn.value)), device="cuda")
        nz, nnb = self.nz, P.neighbours.size

        def exchange(user, stream, nf, send, recv):
            try:
                per = int(nf) * nz
                with torch.cuda.stream(torch.cuda.ExternalStream(stream)):
                    sv = [sbuf[P.send_ptr[i] * per:P.send_ptr[i + 1] * per] for i in range(nnb)]
                    rv = [rbuf[P.recv_ptr[i] * per:P.recv_ptr[i + 1] * per] for i in range(nnb)]
                    transport.exchange(sv, rv)
                return 0
            except Exception:   # noqa: BLE001 - reported to the library as a failed exchange
                return -1

        self._xfn = _lib.EXCHANGE_FN(exchange)   # kept alive with the handle
        self._xbufs = (sbuf, rbuf)
        _lib.check(self._L.cgd_set_exchange(self.h, self._xfn, None), "cgd_set_exchange")

    def close(self):
        if getattr(self, "h", None):
            try:
                self._L.cgd_destroy(self.h)
            except (TypeError, AttributeError):   # interpreter shutdown
                pass
            self.h = None

    def __del__(self):
        self.close()

    def new_state(self):
        return np.zeros(self.shape, order="F")

    def fcn_prepare(self, U, p=None):
        p = np.zeros((self.nz, self.NumG), order="F") if p is None else p
        _lib.check(self._L.cgd_prepare(self.h, _ptr(U, self.shape), _ptr(p, (self.nz, self.NumG), True)),
                   "cgd_prepare")
        return p

    def fcn(self, U, F=None):
        F = self.new_state() if F is None else F
        _lib.check(self._L.cgd_rhs(self.h, _ptr(U, self.shape), _ptr(F, self.shape, True)), "cgd_rhs")
        return F

    def fcn_adjoint(self, U, LF, LU=None):
        """(dF/dU)^T LF at U: the hand-written adjoint of the tendency (FP64, no
        tracers)."""
        LU = self.new_state() if LU is None else LU
        _lib.check(self._L.cgd_rhs_adjoint(self.h, _ptr(U, self.shape), _ptr(LF, self.shape),
                                           _ptr(LU, self.shape, True)), "cgd_rhs_adjoint")
        return LU

    def ros_step_adjoint(self, U0, Lout, dt, Lin=None):
        """(dU1/dU0)^T Lout for one Rosenbrock-W step U1 = step(U0, dt): the
        hand-written adjoint of the step (FP64, no tracers).  U0 is left
        unchanged."""
        Lin = self.new_state() if Lin is None else Lin
        _lib.check(self._L.cgd_ros_step_adjoint(self.h, _ptr(U0, self.shape), _ptr(Lout, self.shape),
                                                _ptr(Lin, self.shape, True), float(dt)),
                   "cgd_ros_step_adjoint")
        return Lin

    def tape_record_step(self, slot, U, dt):
        """One step of U in place, recording what its reverse reads in tape
        slot `slot` (tape_bytes_per_step() bytes of device memory)."""
        _lib.check(self._L.cgd_tape_record_step(self.h, int(slot), _ptr(U, self.shape, True), float(dt)),
                   "cgd_tape_record_step")
        return U

    def tape_step_adjoint(self, slot, Lout, Lin=None):
        """(dU1/dU0)^T Lout for the step recorded in `slot`."""
        Lin = self.new_state() if Lin is None else Lin
        _lib.check(self._L.cgd_tape_step_adjoint(self.h, int(slot), _ptr(Lout, self.shape),
                                                 _ptr(Lin, self.shape, True)), "cgd_tape_step_adjoint")
        return Lin

    def tape_release(self):
        _lib.check(self._L.cgd_tape_release(self.h), "cgd_tape_release")

    def tape_bytes_per_step(self):
        return int(self._L.cgd_tape_bytes_per_step(self.h))

    def checkpoint_every(self, nsteps, mem_budget=16 << 30):
        """Checkpoint spacing of steps_adjoint: every state when the n states
        fit in mem_budget bytes, else about sqrt(n) (at most n/every + every
        states held)."""
        state_bytes = int(np.prod(self.shape)) * 8
        if int(nsteps) * state_bytes <= mem_budget:
            return 1
        return max(1, int(round(int(nsteps) ** 0.5)))

    def steps_adjoint(self, U0, Lout, dt, nsteps, every=None, mem_budget=16 << 30, tape=None):
        """(dU_n/dU0)^T Lout for n = nsteps Rosenbrock-W steps from U0, by
        chaining step adjoints backwards over checkpoints: the forward run
        keeps the state every `every` steps (default: checkpoint_every), and
        the reverse sweep takes the segments from the last to the first.
        With tape (default: when a segment's recorded steps fit in
        mem_budget), each segment is re-run from its checkpoint recording
        every step (tape_record_step) and the step adjoints read the
        records; otherwise the segment's states are kept and each step
        adjoint replays its step (ros_step_adjoint).  At most nsteps/every
        checkpoints plus one segment are held.  The arrays may be host
        (numpy) or device (torch) arrays; checkpoints stay where U0 is.
        Lout may be a function of the final state U_n that returns the
        adjoint seed (U_n comes from the same forward run)."""
        nsteps = int(nsteps)
        every = self.checkpoint_every(nsteps, mem_budget) if every is None else max(1, int(every))
        if tape is None:
            tape = every * self.tape_bytes_per_step() <= mem_budget
        # one working state for every forward step, so the library's captured
        # step (bound to the state's address) is reused
        checkpoints = {0: _copy(U0)}
        work = _copy(U0)
        for s in range(1, nsteps):
            self.time_stepper(work, dt, 1)
            if s % every == 0:
                checkpoints[s] = _copy(work)
        if callable(Lout):
            Un = _copy(work)
            if nsteps > 0:
                self.time_stepper(Un, dt, 1)
            L = Lout(Un)
        else:
            L = _copy(Lout)
        top = nsteps
        try:
            for start in sorted(checkpoints, reverse=True):
                _assign(work, checkpoints[start])
                if tape:
                    for j in range(top - start):
                        self.tape_record_step(j, work, dt)
                    for j in reversed(range(top - start)):
                        L = self.tape_step_adjoint(j, L, _empty_like(L))
                else:
                    seg = [checkpoints[start]]
                    for _ in range(start + 1, top):
                        self.time_stepper(work, dt, 1)
                        seg.append(_copy(work))
                    for W in reversed(seg):
                        L = self.ros_step_adjoint(W, L, dt, _empty_like(L))
                top = start
        finally:
            if tape:
                self.tape_release()
        return L

    def hypervisc_phase1(self, U, Temp1=None):
        T = self.new_state() if Temp1 is None else Temp1
        _lib.check(self._L.cgd_hypervisc_phase1(self.h, _ptr(U, self.shape), _ptr(T, self.shape, True)),
                   "cgd_hypervisc_phase1")
        return T

    def jac(self, U):
        """Bands JRhoW, JWRho, JWRhoTh, JRhoThW as an array (4, 2, nz-1, NumG);
        each band is the reference's (2, nz-1, NumG) JCache array."""
        b = np.zeros(4 * 2 * (self.nz - 1) * self.NumG)
        _lib.check(self._L.cgd_jac(self.h, _ptr(U, self.shape), b.ctypes.data), "cgd_jac")
        return b.reshape((4, self.NumG, self.nz - 1, 2)).transpose(0, 3, 2, 1)

    def new_bands(self):
        """The reference's JCache band arrays JRhoW, JWRho, JWRhoTh, JRhoThW,
        each (2, nz-1, NumG) in column-major order (src/Integration/JacCache.jl:62-70)."""
        return JacBands(*[np.zeros((2, self.nz - 1, self.NumG), order="F") for _ in range(4)])

    def jac_bands(self, J, U):
        """Fill the four band arrays of J (JacBands of Fortran-ordered numpy
        arrays or of contiguous CUDA torch tensors of shape (NumG, nz-1, 2))
        from U, as JacSchurGPU!(J, U, ...) does."""
        shp = (2, self.nz - 1, self.NumG)
        _lib.check(self._L.cgd_jac_bands(self.h, _ptr(U, self.shape), *[_ptr(b, shp, True) for b in J]),
                   "cgd_jac_bands")
        return J

    def schur_solve_bands(self, k, v, J, fac):
        """k = (I/fac - J)^-1 v with the bands of J (SchurSolveGPU!(k, v, J, fac,
        Cache, Global)); v is updated in place as by the reference."""
        shp = (2, self.nz - 1, self.NumG)
        _lib.check(self._L.cgd_schur_solve_bands(self.h, _ptr(k, self.shape, True), _ptr(v, self.shape, True),
                                                 *[_ptr(b, shp) for b in J], float(fac)), "cgd_schur_solve_bands")
        return k

    def schur_solve(self, v, fac, k=None):
        """k = (I/fac - J)^-1 v with the bands of the last jac(); v is updated
        in place as by the reference."""
        k = self.new_state() if k is None else k
        _lib.check(self._L.cgd_schur_solve(self.h, _ptr(k, self.shape, True), _ptr(v, self.shape, True),
                                              float(fac)), "cgd_schur_solve")
        return k

    def rosenbrock_schur(self, U, dt):
        _lib.check(self._L.cgd_ros_step(self.h, _ptr(U, self.shape, True), float(dt), 1), "cgd_ros_step")
        return U

    def time_stepper(self, U, dt, nsteps):
        _lib.check(self._L.cgd_ros_step(self.h, _ptr(U, self.shape, True), float(dt), int(nsteps)),
                   "cgd_ros_step")
        return U

    def mass_integral(self, U):
        out = ctypes.c_double()
        mm = self._mmass.data_ptr() if hasattr(self._mmass, "data_ptr") else self._mmass.ctypes.data
        _lib.check(self._L.cgd_mass_integral(self.h, _ptr(U, self.shape), mm, ctypes.byref(out)),
                   "cgd_mass_integral")
        return out.value

    # ---- output interpolation (the reference's VTK output kernels)
    def _cells(self, like, OP):
        """Zeroed cell array (OrdPrint, OrdPrint, nz, NF) in Fortran order: a
        numpy array, or for a tensor `like` a tensor of shape (NF, nz, OP, OP)
        on its device (the same memory layout)."""
        if isinstance(like, np.ndarray):
            return np.zeros((OP, OP, self.nz, self.NF), order="F")
        import torch
        return torch.zeros((self.NF, self.nz, OP, OP), dtype=torch.float64, device=like.device)

    @staticmethod
    def _inter(inter):
        """The weights (OrdPrint, OrdPrint, N, N) of output.vtk_inter (host)."""
        inter = np.asfortranarray(inter, dtype=np.float64)
        if inter.ndim != 4 or inter.shape[0] != inter.shape[1]:
            raise ValueError("inter: (OrdPrint, OrdPrint, N, N)")
        return inter, inter.shape[0], inter.ctypes.data

    def interpolate(self, c, inter, rhoc=None, out=None):
        """InterpolateGPU! / InterpolateRhoGPU!: c (nz, NumG) at the
        OrdPrint x OrdPrint sub-cell centres, (OrdPrint, OrdPrint, nz, NF);
        each nodal value divided by rhoc first when given."""
        inter, OP, ip = self._inter(inter)
        out = self._cells(c, OP) if out is None else out
        two = (self.nz, self.NumG)
        _lib.check(self._L.cgd_interpolate(self.h, _ptr(c, two), _ptr(rhoc, two) if rhoc is not None else None, ip,
                                           OP, _ptr(out, (OP, OP, self.nz, self.NF), True)), "cgd_interpolate")
        return out

    def interpolate_wb(self, u, v, w, inter, out=None):
        """InterpolateWBGPU!: layer-mean w with the surface value from u, v."""
        inter, OP, ip = self._inter(inter)
        out = self._cells(w, OP) if out is None else out
        two = (self.nz, self.NumG)
        _lib.check(self._L.cgd_interpolate_wb(self.h, _ptr(u, two), _ptr(v, two), _ptr(w, two), ip, OP,
                                              _ptr(out, (OP, OP, self.nz, self.NF), True)), "cgd_interpolate_wb")
        return out

    def interpolate_vort(self, U, inter, out=None):
        """InterpolateVortGPU!: element-local vertical vorticity of the state."""
        inter, OP, ip = self._inter(inter)
        out = self._cells(U, OP) if out is None else out
        _lib.check(self._L.cgd_interpolate_vort(self.h, _ptr(U, self.shape), ip, OP,
                                                _ptr(out, (OP, OP, self.nz, self.NF), True)), "cgd_interpolate_vort")
        return out

    def output_fields(self, U, fields, inter, out=None):
        """The listed quantities (_lib.OUT_* codes) of the state in one call:
        out holds len(fields) cell arrays (OrdPrint, OrdPrint, nz, NF) back
        to back (numpy: shape (nfields, NF, nz, OP, OP); torch: flat)."""
        inter, OP, ip = self._inter(inter)
        codes = np.ascontiguousarray(fields, dtype=np.int32)
        n = OP * OP * self.nz * self.NF * codes.size
        if out is None:
            if isinstance(U, np.ndarray):
                out = np.zeros((codes.size, self.NF, self.nz, OP, OP))
            else:
                import torch
                out = torch.empty(n, dtype=torch.float64, device=U.device)
        if isinstance(out, np.ndarray):
            if out.size != n or not out.flags.c_contiguous or out.dtype != np.float64:
                raise ValueError("output array: C-contiguous float64 of nfields * OP^2 * nz * NF values")
            op = out.ctypes.data
        else:
            if out.numel() != n or out.dtype.itemsize != 8 or not out.is_contiguous():
                raise ValueError("output tensor: contiguous float64 of nfields * OP^2 * nz * NF values")
            op = out.data_ptr()
        _lib.check(self._L.cgd_output_fields(self.h, _ptr(U, self.shape), codes.ctypes.data, int(codes.size), ip, OP,
                                             op), "cgd_output_fields")
        return out

    def set_caller_stream(self, stream=None):
        """The stream whose queued work every call waits for before it reads
        its arguments: a cudaStream_t as an integer (e.g.
        torch.cuda.current_stream().cuda_stream), or None for the legacy
        default stream, PyTorch's default."""
        _lib.check(self._L.cgd_set_caller_stream(self.h, ctypes.c_void_p(stream) if stream else None),
                   "cgd_set_caller_stream")

    def stream(self):
        """The library's cudaStream_t as an integer handle."""
        s = ctypes.c_void_p()
        _lib.check(self._L.cgd_get_stream(self.h, ctypes.byref(s)), "cgd_get_stream")
        return s.value or 0

    def kernel_times(self, nmax=15):
        names = ctypes.create_string_buffer(512)
        ms = (ctypes.c_double * nmax)()
        n = self._L.cgd_kernel_times(self.h, names, 512, ms, nmax)
        if n < 0:
            raise _lib.CgdError(n, "cgd_kernel_times")
        return list(zip(names.value.decode().split(";"), list(ms)[:n]))


class _DevArray:
    """A device buffer of the library seen by torch (zero copy)."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": "<f8", "data": (int(ptr), False),
                                         "version": 3, "strides": None}


class PartGroup:
    """The parts of a decomposed grid run together in one process on one GPU
    (parts[r] is rank r's Dycore): each DSS point exchanges the parts'
    contributions by device copies.  The multi-process form runs the same
    kernels and exchanges with one Dycore per process (set_transport)."""

    def __init__(self, parts):
        self.parts = list(parts)
        self._L = self.parts[0]._L
        self._h = (ctypes.c_void_p * len(self.parts))(*[p.h for p in self.parts])

    def _ptrs(self, arrs, writable=False):
        return (ctypes.c_void_p * len(arrs))(*[_ptr(a, p.shape, writable) for a, p in zip(arrs, self.parts)])

    def fcn(self, U, F):
        _lib.check(self._L.cgd_group_rhs(self._h, len(self.parts), self._ptrs(U), self._ptrs(F, True)),
                   "cgd_group_rhs")
        return F

    def time_stepper(self, U, dt, nsteps):
        _lib.check(self._L.cgd_group_ros_step(self._h, len(self.parts), self._ptrs(U, True), float(dt),
                                              int(nsteps)), "cgd_group_ros_step")
        return U


class Ensemble:
    """Batched ensemble of Dycore members (same OrdPoly, NumTr and precision;
    any nPanel and nz): one ensemble step is one CUDA graph over flat work
    lists spanning every member (cgd_batch_step), either 15 launches or, with
    fused=True (OrdPoly 4), one persistent cooperative launch per stage; or,
    with members=True, one graph branch per member running that member's own
    step.  autotune=True times every work-list order in every form and keeps
    the fastest.  States are CUDA torch tensors, one per member, stepped in
    place."""

    def __init__(self, members, autotune=False, fused=False, members_form=False):
        self.members = list(members)
        self._L = self.members[0]._L
        arr = (ctypes.c_void_p * len(self.members))(*[m.h for m in self.members])
        b = ctypes.c_void_p()
        flags = ((_lib.BATCH_AUTOTUNE if autotune else 0) | (_lib.BATCH_FUSED if fused else 0) |
                 (_lib.BATCH_MEMBERS if members_form else 0))
        _lib.check(self._L.cgd_batch_create(arr, len(self.members), flags, ctypes.byref(b)), "cgd_batch_create")
        self.b = b

    def step(self, states, dts, nsteps=1):
        n = len(self.members)
        if len(states) != n or len(dts) != n:
            raise ValueError("one state and one dt per member")
        ptrs = (ctypes.c_void_p * n)(*[_ptr(u, m.shape, True) for u, m in zip(states, self.members)])
        dt = (ctypes.c_double * n)(*[float(x) for x in dts])
        _lib.check(self._L.cgd_batch_step(self.b, ptrs, dt, int(nsteps)), "cgd_batch_step")

    def tuning(self):
        buf = ctypes.create_string_buffer(1024)
        _lib.check(self._L.cgd_batch_tuning(self.b, buf, 1024), "cgd_batch_tuning")
        return buf.value.decode()

    def stream(self):
        s = ctypes.c_void_p()
        _lib.check(self._L.cgd_batch_get_stream(self.b, ctypes.byref(s)), "cgd_batch_get_stream")
        return s.value

    def close(self):
        if getattr(self, "b", None):
            try:
                self._L.cgd_batch_destroy(self.b)
            except (TypeError, AttributeError):   # interpreter shutdown
                pass
            self.b = None

    def __del__(self):
        self.close()


_SETUP_CACHE = {}


def _grid_and_state(cfg, where="host"):
    """Grid and seeded initial state of a configuration, built once per
    process (the arrays are read-only inputs of the library).  where="device"
    forms the grid's floating-point arrays on the GPU
    (grid.init_grid_sphere_device)."""
    from . import grid as G
    from . import physics as Ph
    key = (cfg.nPanel, cfg.OrdPoly, cfg.nz, cfg.stretch, cfg.H, cfg.NumTr, cfg.Up, cfg.theta_noise,
           cfg.seed_theta, cfg.seed_tracer, where)
    if key not in _SETUP_CACHE:
        phys = Ph.PhysParameters()
        init = G.init_grid_sphere_device if where == "device" else G.init_grid_sphere
        grid = init(cfg.nPanel, cfg.OrdPoly, cfg.levels(), cfg.H, phys.RadEarth)
        tl = Ph.tracer_centres(cfg.NumTr, cfg.seed_tracer) if cfg.NumTr else None
        U = Ph.initial_state(grid, phys, cfg.NumTr, tl, cfg.Up)
        Ph.theta_noise(U, cfg.theta_noise, cfg.seed_theta)
        _SETUP_CACHE.clear()
        _SETUP_CACHE[key] = (grid, U)
    return _SETUP_CACHE[key]


def setup(cfg_name_or_cfg, precision="fp64", check_finite=False, nz=None, nPanel=None, exact=False, where="host"):
    """Grid + initial state + Dycore for a named configuration
    (physics.CONFIGS).  Returns (dycore, U0, config); U0 is a fresh copy.
    where="device": the grid's floating-point arrays formed on the GPU."""
    from . import physics as Ph
    cfg = Ph.CONFIGS[cfg_name_or_cfg] if isinstance(cfg_name_or_cfg, str) else cfg_name_or_cfg
    if nz is not None or nPanel is not None:
        import dataclasses
        cfg = dataclasses.replace(cfg, nz=nz or cfg.nz, nPanel=nPanel or cfg.nPanel)
    phys = Ph.PhysParameters()
    grid, U = _grid_and_state(cfg, where)
    nu = Ph.hyperdiffusion(cfg.nPanel, cfg.OrdPoly)
    dyc = Dycore(grid, cfg.NumTr, nu, phys, precision=precision, check_finite=check_finite, exact=exact)
    return dyc, U.copy(order="F"), cfg
