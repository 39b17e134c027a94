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


def axis_metrics(faces):
    """(centres, widths) of one axis as the reference's geometry compiler
    derives them (finish_axis_metrics, src/mesh_focus.cpp:584-600):
    width = right - left, centre = left + 0.5 * width."""
    f = np.asarray(faces, dtype=np.float64)
    widths = f[1:] - f[:-1]
    return f[:-1] + 0.5 * widths, widths


def face_coefficients(beta, faces, boundary):
    """Face coefficients of face_pressure_coefficient (src/solver_piso.cpp:
    1060-1136) for a cell mobility beta (the reference's density * r_au):
    interior faces A / (d_L / beta_L + d_R / beta_R) with d the centre-to-
    face distances; a Dirichlet boundary face 2 A / (d / beta_o + d /
    beta_g) with the ghost state equal to the owner's; Neumann 0.  A is the
    product of the two transverse widths in the reference's order (face_area,
    src/solver_cartesian.cpp:319-331).  Returns the x-, y-, z-face arrays."""
    metrics = [axis_metrics(f) for f in faces]
    (_, wx), (_, wy), (_, wz) = metrics
    out = []
    for axis in range(3):
        f = np.asarray(faces[axis], dtype=np.float64)
        centres, widths = metrics[axis]
        if axis == 0:
            area = (wy[:, None] * wz[None, :]).T[:, :, None]      # (nz, ny, 1)
        elif axis == 1:
            area = (wx[None, :] * wz[:, None])[:, None, :]        # (nz, 1, nx)
        else:
            area = (wx[None, :] * wy[:, None])[None, :, :]        # (1, ny, nx)
        b = np.moveaxis(beta, 2 - axis, -1)                       # axis last
        a = np.moveaxis(area, 2 - axis, -1)
        dl = f[1:-1] - centres[:-1]
        dr = centres[1:] - f[1:-1]
        interior = a / (dl / b[..., :-1] + dr / b[..., 1:])
        lo_d = centres[0] - f[0]
        hi_d = f[-1] - centres[-1]
        lo = 2.0 * a / (lo_d / b[..., :1] + lo_d / b[..., :1])
        hi = 2.0 * a / (hi_d / b[..., -1:] + hi_d / b[..., -1:])
        if boundary[2 * axis] == NEUMANN:
            lo = np.zeros_like(lo)
        if boundary[2 * axis + 1] == NEUMANN:
            hi = np.zeros_like(hi)
        coef = np.concatenate([lo, interior, hi], axis=-1)
        out.append(np.ascontiguousarray(np.moveaxis(coef, -1, 2 - axis)))
    return out


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
