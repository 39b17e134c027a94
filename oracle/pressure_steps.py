"""CPU restatement of the steps either side of the pressure solve -- TEST
INFRASTRUCTURE (used only by tests/ as the checker).

* assemble(): the pressure-correction system of assemble_pressure_system_impl
  (src/solver_pressure.cpp:110-332) with cell_volume
  (src/solver_cartesian.cpp:333-337), face_sum and outward_flux
  (src/solver_pressure.cpp:80-93), evaluated element-wise in the reference's
  operation order so that float64 results can be compared bit for bit;
* correct_flux(): the mass-flux response of a pressure correction
  (PressureCorrectionBoundaryPlan::jump_unchecked / mass_flux_response_unchecked,
  src/solver_piso.cpp:1605-1653) applied over all faces as the PISO
  publication loop does (src/solver_piso.cpp:7400-7420).

Paths are relative to versions/v0.4 of the reference.  The reference
functions need a compiled PISO coupler (bindings, certificates, boundary
plans) to be called, so parity for these two steps rests on this
restatement of the cited lines rather than on a compiled run.

Arrays are numpy float64 in the library's layout: cells (nz, ny, nx), faces
(nz, ny, nx+1), (nz, ny+1, nx), (nz+1, ny, nx).
"""
from __future__ import annotations

import numpy as np

NEUMANN = 1


def cell_volume(faces):
    """w_x * w_y * w_z per cell, widths as face-coordinate differences."""
    wx = np.diff(faces[0])
    wy = np.diff(faces[1])
    wz = np.diff(faces[2])
    return (wx[None, None, :] * wy[None, :, None]) * wz[:, None, None]


def face_sum(fx, fy, fz):
    """x-, x+, y-, y+, z-, z+ added left to right (face_sum, :80-85)."""
    return (((((fx[:, :, :-1] + fx[:, :, 1:]) + fy[:, :-1, :]) + fy[:, 1:, :]) + fz[:-1]) +
            fz[1:])


def outward_flux(qx, qy, qz):
    """x+ - x- + y+ - y- + z+ - z- left to right (outward_flux, :87-93)."""
    return (((((qx[:, :, 1:] - qx[:, :, :-1]) + qy[:, 1:, :]) - qy[:, :-1, :]) + qz[1:]) -
            qz[:-1])


def assemble(faces, fx, fy, fz, a0, a1, a2, rho, rho_n, drho_dp, qx, qy, qz,
             rho_nm1=None, mass_source=None):
    """(diag, rhs) of the pressure-correction system (:281-296)."""
    volume = cell_volume(faces)
    prev = rho_nm1 if rho_nm1 is not None else np.zeros_like(rho)
    source = mass_source if mass_source is not None else np.zeros_like(rho)
    defect = volume * ((((a0 * rho) + (a1 * rho_n)) + (a2 * prev)) - source)
    diag = ((a0 * volume) * drho_dp) + face_sum(fx, fy, fz)
    rhs = -(defect + outward_flux(qx, qy, qz))
    return diag, rhs


def _jump(p, axis, boundary):
    """Face jumps of cell field p along axis (jump_unchecked, :1605-1628)."""
    ax = {0: 2, 1: 1, 2: 0}[axis]  # numpy axis of the mesh axis
    n = p.shape[ax]
    shape = list(p.shape)
    shape[ax] = n + 1
    jump = np.empty(shape)
    lo = [slice(None)] * 3
    hi = [slice(None)] * 3
    inner = [slice(None)] * 3
    inner[ax] = slice(1, n)
    lo[ax] = slice(0, n - 1)
    hi[ax] = slice(1, n)
    jump[tuple(inner)] = p[tuple(hi)] - p[tuple(lo)]
    first = [slice(None)] * 3
    last = [slice(None)] * 3
    first[ax] = slice(0, 1)
    last[ax] = slice(n, n + 1)
    cell_first = [slice(None)] * 3
    cell_last = [slice(None)] * 3
    cell_first[ax] = slice(0, 1)
    cell_last[ax] = slice(n - 1, n)
    jump[tuple(first)] = 0.0 if boundary[2 * axis] == NEUMANN else p[tuple(cell_first)]
    jump[tuple(last)] = 0.0 if boundary[2 * axis + 1] == NEUMANN else -p[tuple(cell_last)]
    return jump


def correct_flux(p, coefficients, fluxes, boundary, scale=1.0):
    """New face fluxes q + (-c) * (scale * jump) (:1642-1653)."""
    out = []
    for axis in range(3):
        jump = _jump(p, axis, boundary)
        applied = jump if scale == 1.0 else scale * jump
        out.append(fluxes[axis] + (-coefficients[axis]) * applied)
    return out
