"""Python mirror of the reference's solver interface over the C ABI.

``PressureSolver`` wraps one ``hfps_solver`` handle (include/hf_pressure_solver.h):
``set_coefficients`` plays NativeCartesianMgPlan::compile/update_coefficients,
``solve`` plays solve_pcg(op, MG, invocation) -> (x, LinearSolveResult),
``apply_operator``/``apply_preconditioner`` play LinearOperator::apply and
LinearPreconditioner::apply, and ``adjoint`` is the gradient path the
reference does not have.  Arguments may be numpy arrays (host memory) or
CUDA torch tensors (device memory, zero-copy).  There is no CPU fallback:
without the built library or a GPU every call raises.
"""
from __future__ import annotations

import ctypes
import dataclasses
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PACKAGE = os.path.dirname(HERE)
LIBRARY = os.path.join(PACKAGE, "libhfps.so")

HOST, DEVICE = 0, 1
FP64, MIXED = 0, 1
PCG, FGMRES, BICGSTAB = 0, 1, 2
NORM_PLAIN, NORM_SCALED = 0, 1
MG, IC0 = 0, 1
RECYCLE = {"none": 0, "capture": 1, "project": 2, "guard": 3}

STATUS = ["ok", "invalid_case", "invalid_plan", "allocation_failure", "mpi_failure",
          "numerical_failure", "rejected_step", "io_failure"]
TERMINATION = ["converged", "zero_rhs", "maximum_iterations", "breakdown", "non_finite",
               "operator_failure", "preconditioner_failure", "collective_failure",
               "invalid_plan"]


class SolverError(RuntimeError):
    def __init__(self, status: int, message: str, result=None):
        name = STATUS[status] if 0 <= status < len(STATUS) else str(status)
        super().__init__(f"{name}: {message}")
        self.status = status
        self.result = result


class Policy(ctypes.Structure):
    """hfps_policy = MgHierarchyPolicy + correction scaling."""

    _fields_ = [("point_smoother", ctypes.c_int), ("cycle", ctypes.c_int),
                ("pre_sweeps", ctypes.c_int), ("post_sweeps", ctypes.c_int),
                ("coarse_sweeps", ctypes.c_int), ("maximum_levels", ctypes.c_int),
                ("minimum_coarse_extent", ctypes.c_int), ("unit_linear", ctypes.c_int),
                ("chebyshev_lower_spectrum_fraction", ctypes.c_double),
                ("anisotropy_threshold", ctypes.c_double),
                ("diagonal_shortcut_maximum_ratio", ctypes.c_double),
                ("preconditioner", ctypes.c_int), ("null_space", ctypes.c_int)]

    @staticmethod
    def default() -> "Policy":
        p = Policy()
        _lib().hfps_default_policy(ctypes.byref(p))
        return p

    @staticmethod
    def production() -> "Policy":
        """production_pressure_mg_policy with unit (fixed) correction scaling."""
        p = Policy()
        _lib().hfps_production_policy(ctypes.byref(p))
        return p

    def replace(self, **kw) -> "Policy":
        p = Policy()
        ctypes.pointer(p)[0] = self
        for k, v in kw.items():
            setattr(p, k, v)
        return p


class Geometry(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("x_faces", ctypes.POINTER(ctypes.c_double)),
                ("y_faces", ctypes.POINTER(ctypes.c_double)),
                ("z_faces", ctypes.POINTER(ctypes.c_double)),
                ("boundary", ctypes.c_int * 6),
                ("cell_active", ctypes.c_void_p)]


class Control(ctypes.Structure):
    _fields_ = [("relative_tolerance", ctypes.c_double),
                ("absolute_tolerance", ctypes.c_double),
                ("maximum_iterations", ctypes.c_uint32),
                ("true_residual_interval", ctypes.c_uint32),
                ("restart", ctypes.c_uint32), ("algorithm", ctypes.c_int),
                ("precision", ctypes.c_int), ("recycle", ctypes.c_int),
                ("norm", ctypes.c_int)]


class Result(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("detail", ctypes.c_uint32),
                ("termination", ctypes.c_int), ("iterations", ctypes.c_uint32),
                ("initial_true_residual", ctypes.c_double),
                ("final_true_residual", ctypes.c_double),
                ("recursive_residual", ctypes.c_double), ("rhs_norm", ctypes.c_double),
                ("true_residual_limit", ctypes.c_double),
                ("operator_applies", ctypes.c_uint64),
                ("preconditioner_applies", ctypes.c_uint64),
                ("history_length", ctypes.c_uint32), ("levels", ctypes.c_uint32),
                ("seconds", ctypes.c_double), ("kernel_launches", ctypes.c_uint64),
                ("recycle_offered", ctypes.c_uint32), ("recycle_retained", ctypes.c_uint32),
                ("recycle_accepted", ctypes.c_uint32), ("recycle_captured", ctypes.c_uint32),
                ("recycle_projected_residual", ctypes.c_double)]

    def as_dict(self):
        d = {name: getattr(self, name) for name, _ in self._fields_}
        t = d["termination"]
        d["termination"] = TERMINATION[t] if 0 <= t < len(TERMINATION) else t
        return d


class Assembly(ctypes.Structure):
    """hfps_assembly (PressureCorrectionInput)."""
    _fields_ = [("bdf_order", ctypes.c_int), ("a0", ctypes.c_double), ("a1", ctypes.c_double),
                ("a2", ctypes.c_double), ("beta", ctypes.c_void_p),
                ("density_trial", ctypes.c_void_p), ("density_accepted", ctypes.c_void_p),
                ("density_previous", ctypes.c_void_p), ("drho_dp", ctypes.c_void_p),
                ("mass_source", ctypes.c_void_p), ("flux_x", ctypes.c_void_p),
                ("flux_y", ctypes.c_void_p), ("flux_z", ctypes.c_void_p)]


class OperatorView(ctypes.Structure):
    """hfps_operator_view: device coefficient arrays of the finest level."""
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("boundary", ctypes.c_int * 6),
                ("diagonal", ctypes.c_void_p), ("face_x", ctypes.c_void_p),
                ("face_y", ctypes.c_void_p), ("face_z", ctypes.c_void_p)]


_LIB = None

EXPORTS = ["hfps_default_policy", "hfps_production_policy", "hfps_default_control",
           "hfps_create", "hfps_set_coefficients", "hfps_set_beta", "hfps_assemble",
           "hfps_correct_flux", "hfps_solve",
           "hfps_apply_operator", "hfps_apply_preconditioner", "hfps_adjoint",
           "hfps_levels", "hfps_level_coefficients", "hfps_profile_kernel",
           "hfps_operator_dot_noalloc", "hfps_last_error", "hfps_destroy"]

KERNELS = {"operator": 0, "smooth_fp64": 1, "smooth_fp32": 2, "restrict_fp64": 3,
           "prolong_fp64": 4, "pcg_update": 5, "mg_fp64": 6, "mg_mixed": 7, "residual": 8}


def _lib():
    """Loads the in-tree library; raises if it was not built."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIBRARY):
            raise RuntimeError(f"{LIBRARY} is missing: run hundun-flow_b200/build.py")
        lib = ctypes.CDLL(LIBRARY)
        vp = ctypes.c_void_p
        lib.hfps_default_policy.argtypes = [ctypes.POINTER(Policy)]
        lib.hfps_production_policy.argtypes = [ctypes.POINTER(Policy)]
        lib.hfps_default_control.argtypes = [ctypes.POINTER(Control)]
        lib.hfps_create.argtypes = [ctypes.POINTER(Geometry), ctypes.POINTER(Policy), vp,
                                    ctypes.POINTER(vp)]
        lib.hfps_set_coefficients.argtypes = [vp, vp, vp, vp, vp, ctypes.c_int]
        lib.hfps_set_beta.argtypes = [vp, vp, vp, ctypes.c_int]
        lib.hfps_assemble.argtypes = [vp, ctypes.POINTER(Assembly), vp, ctypes.c_int]
        lib.hfps_correct_flux.argtypes = [vp, vp, vp, vp, vp, ctypes.c_double, vp, vp, vp,
                                          ctypes.c_int]
        lib.hfps_solve.argtypes = [vp, vp, vp, ctypes.c_int, ctypes.POINTER(Control),
                                   ctypes.POINTER(Result), vp, ctypes.c_uint32]
        lib.hfps_apply_operator.argtypes = [vp, vp, vp, ctypes.c_int]
        lib.hfps_apply_preconditioner.argtypes = [vp, vp, vp, ctypes.c_int, ctypes.c_int]
        lib.hfps_adjoint.argtypes = [vp, vp, vp, vp, vp, vp, vp, ctypes.c_int,
                                     ctypes.POINTER(Control), ctypes.POINTER(Result)]
        lib.hfps_levels.argtypes = [vp, ctypes.POINTER(ctypes.c_int), ctypes.c_int]
        lib.hfps_level_coefficients.argtypes = [vp, ctypes.c_int, vp, vp, vp, vp, vp]
        lib.hfps_profile_kernel.argtypes = [vp, ctypes.c_int, ctypes.c_int,
                                            ctypes.POINTER(ctypes.c_double),
                                            ctypes.POINTER(ctypes.c_double)]
        lib.hfps_operator_dot_noalloc.argtypes = [ctypes.POINTER(OperatorView), vp, vp, vp, vp]
        lib.hfps_last_error.argtypes = [vp]
        lib.hfps_last_error.restype = ctypes.c_char_p
        lib.hfps_destroy.argtypes = [vp]
        _LIB = lib
    return _LIB


def library_path() -> str:
    return LIBRARY


def _is_torch(a) -> bool:
    return type(a).__module__.startswith("torch")


def _ptr(a, cells: Optional[int] = None):
    """(pointer, memory) of a float64 numpy array or CUDA torch tensor."""
    if a is None:
        return None, HOST
    if _is_torch(a):
        import torch
        if a.dtype != torch.float64 or not a.is_contiguous():
            raise TypeError("torch arrays must be contiguous float64")
        if cells is not None and a.numel() != cells:
            raise ValueError(f"expected {cells} values, got {a.numel()}")
        return ctypes.c_void_p(a.data_ptr()), DEVICE if a.is_cuda else HOST
    if not isinstance(a, np.ndarray) or a.dtype != np.float64 or not a.flags.c_contiguous:
        raise TypeError("numpy arrays must be C-contiguous float64")
    if cells is not None and a.size != cells:
        raise ValueError(f"expected {cells} values, got {a.size}")
    return ctypes.c_void_p(a.ctypes.data), HOST


def _same_memory(*memories):
    kinds = {m for m in memories if m is not None}
    if len(kinds) > 1:
        raise ValueError("mix of host and device arrays in one call")
    return kinds.pop() if kinds else HOST


@dataclasses.dataclass
class SolveOptions:
    """LinearSolveControl fields (include/hundun/v04_linear.hpp:453-465)."""

    rtol: float = 1e-13
    atol: float = 0.0
    maxit: int = 400
    true_residual_interval: int = 4
    precision: int = FP64
    algorithm: int = PCG   # PCG (solve_pcg) or FGMRES (solve_fgmres)
    restart: int = 0       # FGMRES restart length (the reference's default is 12)
    recycle: str = "none"  # FGMRES: "none", "capture", "project", "guard"
    norm: int = 0          # NORM_PLAIN, or NORM_SCALED (the reference's max-scaled global_norm)


class PressureSolver:
    """One pressure system on one GPU (see module docstring)."""

    def __init__(self, shape, faces, boundary, active=None, policy: Optional[Policy] = None,
                 stream=None):
        lib = _lib()
        nx, ny, nz = (int(v) for v in shape)
        self.shape = (nx, ny, nz)
        self.cells = nx * ny * nz
        self.face_counts = ((nx + 1) * ny * nz, nx * (ny + 1) * nz, nx * ny * (nz + 1))
        self._faces = [np.ascontiguousarray(f, dtype=np.float64) for f in faces]
        g = Geometry()
        g.nx, g.ny, g.nz = nx, ny, nz
        g.x_faces = self._faces[0].ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        g.y_faces = self._faces[1].ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        g.z_faces = self._faces[2].ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        for f in range(6):
            g.boundary[f] = int(boundary[f])
        self.active = None
        if active is not None:
            self._active = np.ascontiguousarray(active, dtype=np.uint8).reshape(-1)
            self.active = self._active
            g.cell_active = self._active.ctypes.data
        self.policy = policy if policy is not None else Policy.default()
        handle = ctypes.c_void_p()
        stream_ptr = None
        if stream is not None:
            stream_ptr = ctypes.c_void_p(stream if isinstance(stream, int) else stream.cuda_stream)
        rc = lib.hfps_create(ctypes.byref(g), ctypes.byref(self.policy), stream_ptr,
                             ctypes.byref(handle))
        if rc != 0:
            msg = lib.hfps_last_error(None)
            raise SolverError(rc, f"hfps_create: {msg.decode() if msg else ''}")
        self._handle = handle
        self._lib = lib

    @classmethod
    def from_system(cls, system, policy: Optional[Policy] = None, stream=None,
                    set_coefficients: bool = True) -> "PressureSolver":
        """Builds the solver for a workloads.PressureSystem."""
        s = cls(system.shape, system.faces, system.boundary, system.active, policy, stream)
        if set_coefficients:
            s.set_coefficients(system.diagonal, system.face_x, system.face_y, system.face_z)
        return s

    def active_tensor(self, device):
        """Fluid mask as a float64 tensor (1 fluid, 0 solid) on `device`."""
        import torch
        return torch.as_tensor(self._active, device=device).to(torch.float64)

    # -- lifecycle ---------------------------------------------------------
    def close(self):
        if getattr(self, "_handle", None):
            self._lib.hfps_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, what, result=None):
        if rc != 0:
            msg = self._lib.hfps_last_error(self._handle)
            raise SolverError(rc, f"{what}: {msg.decode() if msg else ''}", result)

    # -- operator ------------------------------------------------------------
    def set_coefficients(self, diagonal, face_x, face_y, face_z):
        ps = [_ptr(a, n) for a, n in zip((diagonal, face_x, face_y, face_z),
                                         (self.cells,) + self.face_counts)]
        memory = _same_memory(*(m for _, m in ps))
        self._check(self._lib.hfps_set_coefficients(self._handle, *(p for p, _ in ps), memory),
                    "set_coefficients")

    def set_beta(self, beta, storage=None):
        pb, mb = _ptr(beta, self.cells)
        ps, ms = _ptr(storage, self.cells)
        memory = _same_memory(mb, ms if storage is not None else None)
        self._check(self._lib.hfps_set_beta(self._handle, pb, ps, memory), "set_beta")

    def assemble(self, beta, density_trial, density_accepted, drho_dp, fluxes, a0, a1=0.0,
                 a2=0.0, density_previous=None, mass_source=None, rhs=None):
        """Assembles the pressure-correction system on the device (hfps_assemble),
        makes it the solver's operator and returns rhs.  ``fluxes`` are the three
        predicted face-flux arrays; BDF2 when ``density_previous`` is given."""
        cells = [beta, density_trial, density_accepted, drho_dp]
        ptrs = [_ptr(a, self.cells) for a in cells]
        prev = _ptr(density_previous, self.cells)
        src = _ptr(mass_source, self.cells)
        flux = [_ptr(f, n) for f, n in zip(fluxes, self.face_counts)]
        out = rhs if rhs is not None else self._like(beta)
        po = _ptr(out, self.cells)
        memory = _same_memory(*(m for _, m in ptrs), *(m for _, m in flux), po[1],
                              prev[1] if density_previous is not None else None,
                              src[1] if mass_source is not None else None)
        a = Assembly()
        a.bdf_order = 2 if density_previous is not None else 1
        a.a0, a.a1, a.a2 = a0, a1, a2
        a.beta, a.density_trial, a.density_accepted, a.drho_dp = (p for p, _ in ptrs)
        a.density_previous = prev[0]
        a.mass_source = src[0]
        a.flux_x, a.flux_y, a.flux_z = (p for p, _ in flux)
        self._check(self._lib.hfps_assemble(self._handle, ctypes.byref(a), po[0], memory),
                    "assemble")
        return out

    def correct_flux(self, correction, coefficients, fluxes, scale=1.0):
        """fluxes[axis] += mass-flux response of ``correction`` (in place)."""
        pc = _ptr(correction, self.cells)
        cs = [_ptr(c, n) for c, n in zip(coefficients, self.face_counts)]
        qs = [_ptr(q, n) for q, n in zip(fluxes, self.face_counts)]
        memory = _same_memory(pc[1], *(m for _, m in cs), *(m for _, m in qs))
        self._check(self._lib.hfps_correct_flux(self._handle, pc[0], *(p for p, _ in cs),
                                                scale, *(p for p, _ in qs), memory),
                    "correct_flux")
        return fluxes

    def levels(self):
        shapes = (ctypes.c_int * 128)()
        count = self._lib.hfps_levels(self._handle, shapes, 32)
        return [tuple(shapes[4 * i:4 * i + 4]) for i in range(count)]

    def level_coefficients(self, level: int):
        nx, ny, nz, _ = self.levels()[level]
        d = np.empty((nz, ny, nx))
        fx = np.empty((nz, ny, nx + 1))
        fy = np.empty((nz, ny + 1, nx))
        fz = np.empty((nz + 1, ny, nx))
        v = np.empty((nz, ny, nx))
        self._check(self._lib.hfps_level_coefficients(
            self._handle, level, d.ctypes.data, fx.ctypes.data, fy.ctypes.data,
            fz.ctypes.data, v.ctypes.data), "level_coefficients")
        return d, fx, fy, fz, v

    def _like(self, a):
        if _is_torch(a):
            import torch
            return torch.empty_like(a)
        return np.empty_like(a)

    def apply_operator(self, x, out=None):
        y = out if out is not None else self._like(x)
        px, mx = _ptr(x, self.cells)
        py, my = _ptr(y, self.cells)
        self._check(self._lib.hfps_apply_operator(self._handle, px, py, _same_memory(mx, my)),
                    "apply_operator")
        return y

    def apply_preconditioner(self, r, out=None, precision: int = FP64):
        z = out if out is not None else self._like(r)
        pr, mr = _ptr(r, self.cells)
        pz, mz = _ptr(z, self.cells)
        self._check(self._lib.hfps_apply_preconditioner(self._handle, pr, pz,
                                                         _same_memory(mr, mz), precision),
                    "apply_preconditioner")
        return z

    def profile_kernel(self, kernel: str, repetitions: int = 20):
        """(mean ms per launch, algorithmic bytes per launch) of one kernel
        class timed with CUDA events on the solver's stream."""
        ms = ctypes.c_double()
        nbytes = ctypes.c_double()
        self._check(self._lib.hfps_profile_kernel(self._handle, KERNELS[kernel], repetitions,
                                                  ctypes.byref(ms), ctypes.byref(nbytes)),
                    "profile_kernel")
        return ms.value, nbytes.value

    # -- solve ---------------------------------------------------------------
    def _control(self, options: SolveOptions) -> Control:
        c = Control()
        self._lib.hfps_default_control(ctypes.byref(c))
        c.relative_tolerance = options.rtol
        c.absolute_tolerance = options.atol
        c.maximum_iterations = options.maxit
        c.true_residual_interval = options.true_residual_interval
        c.precision = options.precision
        c.algorithm = options.algorithm
        c.restart = options.restart if options.algorithm == FGMRES else 0
        if options.algorithm == FGMRES and c.restart == 0:
            c.restart = 12
        c.recycle = RECYCLE[options.recycle]
        c.norm = options.norm
        return c

    def solve(self, rhs, x0=None, options: Optional[SolveOptions] = None, out=None,
              history: bool = True, check: bool = True, **kw):
        """Returns (x, info).  ``x0`` defaults to zero; ``out`` receives x."""
        options = options or SolveOptions(**kw)
        x = out if out is not None else self._like(rhs)
        if x0 is None:
            x[...] = 0 if not _is_torch(x) else 0.0
        elif x0 is not x:
            x[...] = x0
        pb, mb = _ptr(rhs, self.cells)
        px, mx = _ptr(x, self.cells)
        memory = _same_memory(mb, mx)
        hist = np.zeros(options.maxit) if history else None
        result = Result()
        control = self._control(options)
        rc = self._lib.hfps_solve(self._handle, pb, px, memory, ctypes.byref(control),
                                  ctypes.byref(result),
                                  hist.ctypes.data if hist is not None else None,
                                  options.maxit if hist is not None else 0)
        info = result.as_dict()
        if hist is not None:
            info["history"] = hist[:result.history_length].copy()
        if check:
            self._check(rc, "solve", info)
        info["status_code"] = rc
        return x, info

    def adjoint(self, solution, dl_dp, options: Optional[SolveOptions] = None, **kw):
        """Returns (lambda, (grad_x, grad_y, grad_z), info)."""
        options = options or SolveOptions(**kw)
        lam = self._like(solution)
        if _is_torch(solution):
            import torch
            gx = torch.empty(self.face_counts[0], dtype=torch.float64, device=solution.device)
            gy = torch.empty(self.face_counts[1], dtype=torch.float64, device=solution.device)
            gz = torch.empty(self.face_counts[2], dtype=torch.float64, device=solution.device)
        else:
            gx, gy, gz = (np.empty(n) for n in self.face_counts)
        ptrs = [_ptr(a) for a in (solution, dl_dp, lam, gx, gy, gz)]
        memory = _same_memory(*(m for _, m in ptrs))
        result = Result()
        control = self._control(options)
        rc = self._lib.hfps_adjoint(self._handle, *(p for p, _ in ptrs), memory,
                                    ctypes.byref(control), ctypes.byref(result))
        info = result.as_dict()
        self._check(rc, "adjoint", info)
        return lam, (gx, gy, gz), info
