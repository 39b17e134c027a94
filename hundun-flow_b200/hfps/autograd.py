"""torch.autograd wrapper around the adjoint path (used for gradient checks).

``pressure_solve(solver, rhs, face_x, face_y, face_z, storage)`` returns p
with p = A(c)^-1 rhs, where the diagonal is assembled as storage + sum of the
cell's six face coefficients (src/solver_pressure.cpp:223-226).  Backward
calls hfps_adjoint: one more solve with the same operator (A is symmetric)
gives lambda = dL/drhs, and the per-face gradients
dL/dc_f = -(lambda_i - lambda_j)(p_i - p_j) come from one fused kernel;
dL/dstorage_i = -lambda_i p_i.  No residual history is kept between the two
solves: the backward solve recomputes its own.
"""
from __future__ import annotations

import torch

from .solver import FP64, SolveOptions


def _diagonal(fx, fy, fz, storage, shape):
    nx, ny, nz = shape
    fx = fx.reshape(nz, ny, nx + 1)
    fy = fy.reshape(nz, ny + 1, nx)
    fz = fz.reshape(nz + 1, ny, nx)
    d = (fx[:, :, :-1] + fx[:, :, 1:] + fy[:, :-1, :] + fy[:, 1:, :] + fz[:-1, :, :]
         + fz[1:, :, :])
    if storage is not None:
        d = storage.reshape(nz, ny, nx) + d
    return d.reshape(-1).contiguous()


class PressureSolveFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, solver, options, rhs, face_x, face_y, face_z, storage):
        diag = _diagonal(face_x, face_y, face_z, storage, solver.shape)
        solver.set_coefficients(diag, face_x.contiguous(), face_y.contiguous(),
                                face_z.contiguous())
        p, info = solver.solve(rhs.contiguous(), options=options, history=False)
        ctx.solver = solver
        ctx.options = options
        ctx.has_storage = storage is not None
        ctx.save_for_backward(p)
        ctx.info = info
        return p

    @staticmethod
    def backward(ctx, grad_p):
        (p,) = ctx.saved_tensors
        lam, (gx, gy, gz), _ = ctx.solver.adjoint(p, grad_p.contiguous(), options=ctx.options)
        g_storage = None
        if ctx.has_storage:
            g_storage = -lam * p
            if ctx.solver.active is not None:
                g_storage = g_storage * ctx.solver.active_tensor(p.device)
        return None, None, lam, gx, gy, gz, g_storage


def pressure_solve(solver, rhs, face_x, face_y, face_z, storage=None,
                   options: SolveOptions | None = None):
    options = options or SolveOptions(rtol=1e-13, precision=FP64)
    return PressureSolveFunction.apply(solver, options, rhs, face_x, face_y, face_z, storage)
