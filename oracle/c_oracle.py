"""ctypes driver for the C restatement (oracle/libhfps_oracle.so).

Test infrastructure only: tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg use it as the checker.  ``make -C oracle`` builds the library.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY = os.path.join(HERE, "libhfps_oracle.so")

_lib = None


def build() -> str:
    subprocess.run(["make", "-C", HERE, "libhfps_oracle.so"], check=True,
                   stdout=subprocess.DEVNULL)
    return LIBRARY


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIBRARY):
            build()
        lib = ctypes.CDLL(LIBRARY)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        lib.hfo_create.argtypes = [ctypes.c_int] * 3 + [dp] * 3 + [ip] + [dp] * 4 + [
            ctypes.c_void_p, ip, dp, ip]
        lib.hfo_create.restype = ctypes.c_void_p
        lib.hfo_destroy.argtypes = [ctypes.c_void_p]
        lib.hfo_levels.argtypes = [ctypes.c_void_p, ip, ctypes.c_int]
        lib.hfo_levels.restype = ctypes.c_int
        lib.hfo_level_coefficients.argtypes = [ctypes.c_void_p, ctypes.c_int] + [ctypes.c_void_p] * 5
        lib.hfo_apply_operator.argtypes = [ctypes.c_void_p, dp, dp]
        lib.hfo_apply_level.argtypes = [ctypes.c_void_p, ctypes.c_int, dp, dp]
        lib.hfo_apply_mg.argtypes = [ctypes.c_void_p, dp, dp]
        lib.hfo_solve.argtypes = [ctypes.c_void_p, dp, dp, ctypes.c_double, ctypes.c_double,
                                  ctypes.c_int, ctypes.c_int, dp, dp, ctypes.c_int]
        lib.hfo_apply_preconditioner.argtypes = [ctypes.c_void_p, dp, dp]
        lib.hfo_solve_bicgstab.argtypes = [ctypes.c_void_p, dp, dp, ctypes.c_double,
                                           ctypes.c_double, ctypes.c_int, ctypes.c_int, dp, dp,
                                           ctypes.c_int]
        lib.hfo_solve_fgmres.argtypes = [ctypes.c_void_p, dp, dp, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_int, dp, dp, ctypes.c_int]
        _lib = lib
    return _lib


def _dp(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


TERMINATION = ["converged", "zero_rhs", "maximum_iterations", "breakdown", "non_finite"]


class OracleSession:
    """The C restatement for one system and one MG policy.

    ``line_order`` 0 reproduces the reference's lexicographic line
    Gauss-Seidel, 1 the zebra order of the CUDA path.
    """

    PRECONDITIONERS = {"mg": 0, "dic": 1}

    def __init__(self, system, policy=None, unit_linear: bool = True, line_order: int = 0,
                 preconditioner: str = "mg"):
        from ref_oracle import MgPolicy  # same policy record as the reference driver
        policy = policy or MgPolicy()
        lib = _load()
        nx, ny, nz = system.shape
        self.system = system
        self._faces = [np.ascontiguousarray(f, dtype=np.float64) for f in system.faces]
        bc = (ctypes.c_int * 6)(*system.boundary)
        options = (ctypes.c_int * 12)(0, 0, policy.smoother, policy.cycle, policy.pre, policy.post,
                                      policy.coarse_sweeps, 1 if unit_linear else 0,
                                      policy.max_levels, policy.min_coarse_extent, line_order,
                                      self.PRECONDITIONERS[preconditioner])
        reals = (ctypes.c_double * 3)(policy.chebyshev_fraction, policy.anisotropy_threshold,
                                      policy.diagonal_shortcut)
        active = None
        if system.active is not None:
            self._active = np.ascontiguousarray(system.active, dtype=np.uint8)
            active = self._active.ctypes.data_as(ctypes.c_void_p)
        status = ctypes.c_int()
        handle = lib.hfo_create(nx, ny, nz, _dp(self._faces[0]), _dp(self._faces[1]),
                                _dp(self._faces[2]), bc, _dp(system.diagonal), _dp(system.face_x),
                                _dp(system.face_y), _dp(system.face_z), active, options, reals,
                                ctypes.byref(status))
        if not handle:
            raise RuntimeError(f"oracle create failed: {status.value}")
        self._handle = ctypes.c_void_p(handle)
        self._lib = lib

    def close(self):
        if getattr(self, "_handle", None):
            self._lib.hfo_destroy(self._handle)
            self._handle = None

    __del__ = close

    def levels(self):
        shapes = (ctypes.c_int * 128)()
        count = self._lib.hfo_levels(self._handle, shapes, 32)
        return [tuple(shapes[4 * i:4 * i + 4]) for i in range(count)]

    def level_coefficients(self, level: int):
        nx, ny, nz, _ = self.levels()[level]
        d = np.empty((nz, ny, nx))
        fx = np.empty((nz, ny, nx + 1))
        fy = np.empty((nz, ny + 1, nx))
        fz = np.empty((nz + 1, ny, nx))
        v = np.empty((nz, ny, nx))
        self._lib.hfo_level_coefficients(self._handle, level, d.ctypes.data, fx.ctypes.data,
                                         fy.ctypes.data, fz.ctypes.data, v.ctypes.data)
        return d, fx, fy, fz, v

    def apply_operator(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty_like(x)
        self._lib.hfo_apply_operator(self._handle, _dp(x), _dp(y))
        return y

    def apply_level(self, level, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty_like(x)
        self._lib.hfo_apply_level(self._handle, level, _dp(x), _dp(y))
        return y

    def apply_preconditioner(self, r):
        r = np.ascontiguousarray(r, dtype=np.float64)
        z = np.empty_like(r)
        rc = self._lib.hfo_apply_preconditioner(self._handle, _dp(r), _dp(z))
        if rc != 0:
            raise RuntimeError(f"oracle preconditioner failed: {rc}")
        return z

    def apply_mg(self, r):
        r = np.ascontiguousarray(r, dtype=np.float64)
        z = np.empty_like(r)
        rc = self._lib.hfo_apply_mg(self._handle, _dp(r), _dp(z))
        if rc != 0:
            raise RuntimeError(f"oracle MG failed: {rc}")
        return z

    def solve(self, rhs, x0: Optional[np.ndarray] = None, rtol=1e-10, atol=0.0, maxit=400,
              true_residual_interval=4, algorithm: str = "pcg", restart: int = 12,
              recycle: str = "none"):
        """solve_pcg, or solve_fgmres(restart) when ``algorithm == "fgmres"``
        (build the session with unit_linear=False for the reference's
        residual-minimising MG scaling).  ``recycle`` as RefSession.solve.
        A solve that does not return ok publishes nothing: the returned x is
        the initial guess, as the reference leaves the caller's solution
        untouched for an unpublished candidate."""
        rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        x = np.zeros_like(rhs) if x0 is None else np.array(x0, dtype=np.float64, order="C")
        initial = x.copy()
        out = np.zeros(13)
        hist = np.zeros(maxit)
        if algorithm == "bicgstab":
            rc = self._lib.hfo_solve_bicgstab(self._handle, _dp(rhs), _dp(x), rtol, atol, maxit,
                                              true_residual_interval, _dp(out), _dp(hist), maxit)
        elif algorithm == "fgmres":
            modes = {"none": 0, "capture": 1, "project": 2, "guard": 3}
            rc = self._lib.hfo_solve_fgmres(self._handle, _dp(rhs), _dp(x), rtol, atol, maxit,
                                            true_residual_interval, restart, modes[recycle],
                                            _dp(out), _dp(hist), maxit)
        else:
            rc = self._lib.hfo_solve(self._handle, _dp(rhs), _dp(x), rtol, atol, maxit,
                                     true_residual_interval, _dp(out), _dp(hist), maxit)
        it = int(out[0])
        info = {
            "status": rc,
            "iterations": it,
            "initial_true_residual": out[1],
            "final_true_residual": out[2],
            "termination": TERMINATION[int(out[3])],
            "rhs_norm": out[4],
            "limit": out[5],
            "operator_applies": int(out[6]),
            "preconditioner_applies": int(out[7]),
            "history": hist[:it].copy(),
            "recycle_offered": int(out[8]),
            "recycle_retained": int(out[9]),
            "recycle_accepted": bool(out[10]),
            "recycle_projected_residual": out[11],
            "recycle_cycle_corrections": int(out[12]),
        }
        if rc != 0:
            x = initial
        return x, info
