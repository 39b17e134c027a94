"""ctypes driver for the compiled reference solver (oracle/_ref/libhfps_ref.so).

Test infrastructure only (tests/, smoke() and bench.py's CPU legs): it runs
the reference's own NativeCartesianMgPlan, solve_pcg and solve_fgmres on a
PressureSystem.  Build it with ``make -C oracle ref`` in a tree where the
reference sources exist; the built library then travels with the checkout.
"""
from __future__ import annotations

import ctypes
import dataclasses
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY = os.path.join(HERE, "_ref", "libhfps_ref.so")

_lib = None


def available() -> bool:
    return os.path.exists(LIBRARY)


def _load():
    global _lib
    if _lib is None:
        lib = ctypes.CDLL(LIBRARY)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        lib.hfref_create.argtypes = [ctypes.c_int] * 3 + [dp] * 3 + [ip] + [dp] * 4 + [
            ctypes.c_void_p, ip, dp, ctypes.POINTER(ctypes.c_void_p)]
        lib.hfref_create.restype = ctypes.c_int
        lib.hfref_destroy.argtypes = [ctypes.c_void_p]
        lib.hfref_levels.argtypes = [ctypes.c_void_p, ip, ctypes.c_int]
        lib.hfref_levels.restype = ctypes.c_int
        lib.hfref_apply_operator.argtypes = [ctypes.c_void_p, dp, dp]
        lib.hfref_apply_mg.argtypes = [ctypes.c_void_p, dp, dp]
        lib.hfref_apply_cold.argtypes = [ctypes.c_void_p, dp, dp]
        lib.hfref_solve.argtypes = [ctypes.c_void_p, dp, dp, ctypes.c_double, ctypes.c_double,
                                    ctypes.c_int, ctypes.c_int, ctypes.c_int, dp]
        _lib = lib
    return _lib


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


@dataclasses.dataclass
class MgPolicy:
    """MgHierarchyPolicy fields (include/hundun/v04_linear.hpp:115-131).

    Defaults are the struct defaults: red-black V(2,2), 24 coarse sweeps.
    ``production()`` is production_pressure_mg_policy
    (src/solver_piso_detail.hpp:10-19).
    """

    smoother: int = 0  # 0 red-black, 1 Chebyshev-Jacobi
    cycle: int = 0  # 0 V, 1 F
    pre: int = 2
    post: int = 2
    coarse_sweeps: int = 24
    max_levels: int = 32
    min_coarse_extent: int = 3
    chebyshev_fraction: float = 0.3
    anisotropy_threshold: float = 4.0
    diagonal_shortcut: float = 0.0

    @staticmethod
    def production() -> "MgPolicy":
        return MgPolicy(smoother=1, cycle=1, pre=1, post=2, diagonal_shortcut=0.1)


class RefSession:
    """One compiled reference plan (geometry + coefficients + MG hierarchy)."""

    TERMINATION = ["converged", "zero_rhs", "maximum_iterations", "breakdown", "non_finite",
                   "operator_failure", "preconditioner_failure", "collective_failure",
                   "invalid_plan", "convergence_audit_failure"]

    PRECONDITIONERS = {"mg": 0, "iccg": 1, "dilu": 2}
    ALGORITHMS = {"pcg": 0, "fgmres": 1, "bicgstab": 2}

    def __init__(self, system, policy: Optional[MgPolicy] = None, algorithm: str = "pcg",
                 restart: int = 12, unit_linear: Optional[bool] = None,
                 preconditioner: str = "mg", null_space: str = "none"):
        """``algorithm`` "pcg" / "fgmres" / "bicgstab"; ``preconditioner`` "mg"
        (the plan), "iccg" (ColdPressureIccg, with PCG) or "dilu"
        (ColdPressureDilu, with BiCGSTAB); ``null_space`` "none" or "constant"
        (MgNullSpace of the plan)."""
        lib = _load()
        self.system = system
        policy = policy or MgPolicy()
        if unit_linear is None:
            unit_linear = algorithm == "pcg"
        nx, ny, nz = system.shape
        self._faces = [np.ascontiguousarray(f, dtype=np.float64) for f in system.faces]
        self._bc = (ctypes.c_int * 6)(*system.boundary)
        options = (ctypes.c_int * 12)(self.ALGORITHMS[algorithm], restart, policy.smoother,
                                      policy.cycle, policy.pre, policy.post, policy.coarse_sweeps,
                                      1 if unit_linear else 0, policy.max_levels,
                                      policy.min_coarse_extent,
                                      self.PRECONDITIONERS[preconditioner],
                                      {"none": 0, "constant": 1}[null_space])
        reals = (ctypes.c_double * 3)(policy.chebyshev_fraction, policy.anisotropy_threshold,
                                      policy.diagonal_shortcut)
        active = None
        if system.active is not None:
            self._active = np.ascontiguousarray(system.active, dtype=np.uint8)
            active = self._active.ctypes.data_as(ctypes.c_void_p)
        handle = ctypes.c_void_p()
        rc = lib.hfref_create(nx, ny, nz, _dp(self._faces[0]), _dp(self._faces[1]),
                              _dp(self._faces[2]), self._bc, _dp(system.diagonal),
                              _dp(system.face_x), _dp(system.face_y), _dp(system.face_z), active,
                              options, reals, ctypes.byref(handle))
        if rc != 0:
            raise RuntimeError(f"reference plan compile failed: status {rc}")
        self._handle = handle
        self._lib = lib

    def close(self):
        if getattr(self, "_handle", None):
            self._lib.hfref_destroy(self._handle)
            self._handle = None

    __del__ = close

    def levels(self):
        shapes = (ctypes.c_int * 128)()
        count = self._lib.hfref_levels(self._handle, shapes, 32)
        return [tuple(shapes[4 * i:4 * i + 4]) for i in range(count)]

    def apply_operator(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty_like(x)
        rc = self._lib.hfref_apply_operator(self._handle, _dp(x), _dp(y))
        if rc != 0:
            raise RuntimeError(f"reference operator failed: {rc}")
        return y

    def apply_cold(self, r: np.ndarray) -> np.ndarray:
        """One application of the cold-path preconditioner (ICCG or DILU)."""
        r = np.ascontiguousarray(r, dtype=np.float64)
        z = np.empty_like(r)
        rc = self._lib.hfref_apply_cold(self._handle, _dp(r), _dp(z))
        if rc != 0:
            raise RuntimeError(f"reference cold preconditioner failed: {rc}")
        return z

    def apply_mg(self, r: np.ndarray) -> np.ndarray:
        r = np.ascontiguousarray(r, dtype=np.float64)
        z = np.empty_like(r)
        rc = self._lib.hfref_apply_mg(self._handle, _dp(r), _dp(z))
        if rc != 0:
            raise RuntimeError(f"reference MG apply failed: {rc}")
        return z

    RECYCLE = {"none": 0, "capture": 1, "project": 2, "guard": 3}

    def solve(self, rhs: np.ndarray, x0: Optional[np.ndarray] = None, rtol: float = 1e-10,
              atol: float = 0.0, maxit: int = 400, true_residual_interval: int = 4,
              recycle: str = "none"):
        """``recycle`` (FGMRES): "capture" opens a capture session (PISO corrector 1),
        "project" projects its corrections (corrector 2), "guard" applies only the
        zero-seed initial-guess guard, "none" clears any session."""
        rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        x = np.zeros_like(rhs) if x0 is None else np.array(x0, dtype=np.float64, order="C")
        out = np.zeros(15)
        rc = self._lib.hfref_solve(self._handle, _dp(rhs), _dp(x), rtol, atol, maxit,
                                   true_residual_interval, self.RECYCLE[recycle], _dp(out))
        info = {
            "status": rc,
            "iterations": int(out[0]),
            "initial_true_residual": out[1],
            "final_true_residual": out[2],
            "termination": self.TERMINATION[int(out[3])] if 0 <= out[3] < 10 else int(out[3]),
            "rhs_norm": out[4],
            "limit": out[5],
            "operator_applies": int(out[6]),
            "preconditioner_applies": int(out[7]),
            "seconds": out[8],
            "setup_seconds": out[9],
            "recycle_offered": int(out[10]),
            "recycle_retained": int(out[11]),
            "recycle_accepted": bool(out[12]),
            "recycle_projected_residual": out[13],
            "recycle_cycle_corrections": int(out[14]),
        }
        return x, info


# ---------------------------------------------------------------------------
# The steps either side of the solve, from the reference's own sources
# (oracle/_ref/libhfps_ref_steps.so, built from ref_pressure_steps.cpp by
# ``make -C oracle ref``): face_pressure_coefficient, the pressure-system
# assembly and the flux correction.  The reference's runtime-axes geometry
# rounds every face coordinate to binary32 (copy_runtime_faces,
# src/mesh_cartesian.cpp:344-352); ``binary32_faces`` gives coordinates that
# survive that rounding unchanged, so both sides see the same mesh.

STEPS_LIBRARY = os.path.join(HERE, "_ref", "libhfps_ref_steps.so")
_steps = None


def steps_available() -> bool:
    return os.path.exists(STEPS_LIBRARY)


def binary32_faces(faces):
    return tuple(np.ascontiguousarray(np.asarray(f, dtype=np.float32).astype(np.float64))
                 for f in faces)


def _steps_lib():
    global _steps
    if _steps is None:
        lib = ctypes.CDLL(STEPS_LIBRARY)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        vp = ctypes.c_void_p
        geo = [ctypes.c_int] * 3 + [dp] * 3 + [ip]
        lib.hfref_face_coefficients.argtypes = geo + [dp] * 4
        lib.hfref_axis_metrics.argtypes = geo + [ctypes.c_int] + [dp] * 3
        lib.hfref_assemble.argtypes = geo + [dp] * 6 + [ctypes.c_int] + [ctypes.c_double] * 3 + [
            dp, dp, vp, dp, vp, dp, dp]
        lib.hfref_correct_flux.argtypes = geo + [dp] * 4 + [ctypes.c_double] + [dp] * 3
        _steps = lib
    return _steps


class RefSteps:
    """Face coefficients, assembly and flux correction of one grid, computed
    by the reference's code.  ``faces`` must be binary32-representable."""

    def __init__(self, shape, faces, boundary):
        self.shape = tuple(int(n) for n in shape)
        self.faces = tuple(np.ascontiguousarray(f, dtype=np.float64) for f in faces)
        for f in self.faces:
            if not np.array_equal(f, f.astype(np.float32).astype(np.float64)):
                raise ValueError("face coordinates must be binary32-representable")
        self._bc = (ctypes.c_int * 6)(*boundary)
        self._lib = _steps_lib()

    def _geo(self):
        nx, ny, nz = self.shape
        return (nx, ny, nz, _dp(self.faces[0]), _dp(self.faces[1]), _dp(self.faces[2]), self._bc)

    def _face_arrays(self):
        nx, ny, nz = self.shape
        return (np.zeros((nz, ny, nx + 1)), np.zeros((nz, ny + 1, nx)), np.zeros((nz + 1, ny, nx)))

    def face_coefficients(self, beta):
        beta = np.ascontiguousarray(beta, dtype=np.float64)
        out = self._face_arrays()
        rc = self._lib.hfref_face_coefficients(*self._geo(), _dp(beta), *(_dp(a) for a in out))
        if rc != 0:
            raise RuntimeError(f"reference face coefficients failed: {rc}")
        return out

    def axis_metrics(self, axis):
        n = self.shape[axis]
        faces, centres, widths = np.zeros(n + 1), np.zeros(n), np.zeros(n)
        rc = self._lib.hfref_axis_metrics(*self._geo(), axis, _dp(faces), _dp(centres),
                                          _dp(widths))
        if rc != 0:
            raise RuntimeError(f"reference metrics failed: {rc}")
        return faces, centres, widths

    def assemble(self, coefficients, fluxes, a0, a1, a2, rho, rho_n, drho_dp, rho_nm1=None,
                 mass_source=None):
        c = [np.ascontiguousarray(a, dtype=np.float64) for a in coefficients]
        q = [np.ascontiguousarray(a, dtype=np.float64) for a in fluxes]
        cells = [np.ascontiguousarray(a, dtype=np.float64) for a in (rho, rho_n, drho_dp)]
        prev = None if rho_nm1 is None else np.ascontiguousarray(rho_nm1, dtype=np.float64)
        src = None if mass_source is None else np.ascontiguousarray(mass_source, dtype=np.float64)
        diag = np.zeros_like(cells[0])
        rhs = np.zeros_like(cells[0])
        rc = self._lib.hfref_assemble(
            *self._geo(), *(_dp(a) for a in c), *(_dp(a) for a in q), 2 if prev is not None else 1,
            a0, a1, a2, _dp(cells[0]), _dp(cells[1]),
            None if prev is None else prev.ctypes.data_as(ctypes.c_void_p), _dp(cells[2]),
            None if src is None else src.ctypes.data_as(ctypes.c_void_p), _dp(diag), _dp(rhs))
        if rc != 0:
            raise RuntimeError(f"reference assembly failed: {rc}")
        return diag, rhs

    def correct_flux(self, correction, coefficients, fluxes, scale=1.0):
        p = np.ascontiguousarray(correction, dtype=np.float64)
        c = [np.ascontiguousarray(a, dtype=np.float64) for a in coefficients]
        q = [np.array(a, dtype=np.float64, order="C") for a in fluxes]
        rc = self._lib.hfref_correct_flux(*self._geo(), _dp(p), *(_dp(a) for a in c), scale,
                                          *(_dp(a) for a in q))
        if rc != 0:
            raise RuntimeError(f"reference flux correction failed: {rc}")
        return q
