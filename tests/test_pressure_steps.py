"""CPU tests of the restated steps either side of the solve (oracle/
pressure_steps.py): the assembly and the flux correction are consistent
with the operator the solve uses.

After a correction p' solves A p' = rhs, the corrected fluxes close the
continuity residual: outward_flux(dphi) equals the face part of A p'
(mass_flux_response, src/solver_piso.cpp:1642-1653, against the 7-point
row of PressureLinearOperator, src/solver_pressure.cpp:746-811), and the
assembled diagonal is the storage term plus that face part
(src/solver_pressure.cpp:281-296).
"""
import numpy as np

from hfps import workloads


def _faces_from(system):
    return system.face_x, system.face_y, system.face_z


def test_flux_response_divergence_is_the_face_operator():
    import pressure_steps
    s = workloads.make("sphere64", n=(9, 7, 6), seed=2)
    fx, fy, fz = _faces_from(s)
    rng = np.random.default_rng(5)
    p = rng.standard_normal(s.rhs.shape)
    zero = [np.zeros_like(f) for f in (fx, fy, fz)]
    dq = pressure_steps.correct_flux(p, (fx, fy, fz), zero, s.boundary)
    div = pressure_steps.outward_flux(*dq)
    # Face part of the operator: sum_f c_f (p_c - p_nb), Dirichlet nb = 0,
    # Neumann nb = p_c (a zero face coefficient contributes nothing).
    face_part = pressure_steps.face_sum(fx, fy, fz) * p
    pad = np.pad(p, 1)
    nb = [(fx[:, :, :-1], pad[1:-1, 1:-1, :-2]), (fx[:, :, 1:], pad[1:-1, 1:-1, 2:]),
          (fy[:, :-1, :], pad[1:-1, :-2, 1:-1]), (fy[:, 1:, :], pad[1:-1, 2:, 1:-1]),
          (fz[:-1], pad[:-2, 1:-1, 1:-1]), (fz[1:], pad[2:, 1:-1, 1:-1])]
    for (c, q), (axis, side) in zip(nb, [(0, 0), (0, 1), (1, 0), (1, 1), (2, 0), (2, 1)]):
        q = q.copy()
        if s.boundary[2 * axis + side] == pressure_steps.NEUMANN:
            edge = [slice(None)] * 3
            ax = 2 - axis
            edge[ax] = slice(0, 1) if side == 0 else slice(-1, None)
            q[tuple(edge)] = p[tuple(edge)]
        face_part = face_part - c * q
    assert np.allclose(div, face_part, rtol=1e-12, atol=1e-12 * np.abs(face_part).max())


def test_assembly_diagonal_is_storage_plus_faces():
    import pressure_steps
    s = workloads.make("wrinkled256", n=(10, 12, 8), stretch_y=1.05, seed=3)
    fx, fy, fz = _faces_from(s)
    rng = np.random.default_rng(6)
    rho = 1.0 + rng.random(s.rhs.shape)
    psi = 0.5 + rng.random(s.rhs.shape)
    q = [rng.standard_normal(f.shape) for f in (fx, fy, fz)]
    diag, rhs = pressure_steps.assemble(s.faces, fx, fy, fz, 1.5, -2.0, 0.5, rho, rho, psi, *q,
                                        rho_nm1=rho)
    volume = pressure_steps.cell_volume(s.faces)
    assert np.allclose(diag - pressure_steps.face_sum(fx, fy, fz), 1.5 * volume * psi,
                       rtol=1e-12)
    # a0 + a1 + a2 = 0 with equal densities: only the flux divergence remains.
    assert np.allclose(rhs, -pressure_steps.outward_flux(*q), atol=1e-12)


def test_boundary_jumps_and_flux_response_known_answers():
    """The reference's boundary semantics for the correction jump and the
    mass-flux response (tests/unit/solver_pressure_boundary_plan_test.cpp:
    203-223): a Neumann face has zero jump, a Dirichlet face on the high side
    has jump -p_owner (on the low side +p_owner: the boundary value is 0),
    interior faces p_hi - p_lo, and the response with coefficient 3 is
    -3 times the jump."""
    import pressure_steps
    N, D = pressure_steps.NEUMANN, workloads.DIRICHLET
    rng = np.random.default_rng(9)
    p = rng.standard_normal((3, 4, 5))  # (nz, ny, nx)
    boundary = (N, D, D, N, N, D)
    jx = pressure_steps._jump(p, 0, boundary)
    jy = pressure_steps._jump(p, 1, boundary)
    jz = pressure_steps._jump(p, 2, boundary)
    assert np.array_equal(jx[:, :, 0], np.zeros((3, 4)))           # x-min Neumann
    assert np.array_equal(jx[:, :, -1], -p[:, :, -1])               # x-max Dirichlet
    assert np.array_equal(jx[:, :, 1:-1], p[:, :, 1:] - p[:, :, :-1])
    assert np.array_equal(jy[:, 0, :], p[:, 0, :])                  # y-min Dirichlet
    assert np.array_equal(jy[:, -1, :], np.zeros((3, 5)))           # y-max Neumann
    assert np.array_equal(jz[0], np.zeros((4, 5)))                  # z-min Neumann
    assert np.array_equal(jz[-1], -p[-1])                           # z-max Dirichlet
    coefficients = [np.full(j.shape, 3.0) for j in (jx, jy, jz)]
    zero = [np.zeros(j.shape) for j in (jx, jy, jz)]
    dq = pressure_steps.correct_flux(p, coefficients, zero, boundary)
    for d, j in zip(dq, (jx, jy, jz)):
        assert np.array_equal(d, -3.0 * j)
