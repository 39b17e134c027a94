"""CPU tests of the oracle: the C restatement against the reference itself.

The C restatement (oracle/hfps_oracle.c) is pinned three ways:
* against golden fixtures recorded from the compiled reference sources
  (tests/golden/make_golden.py): operator action, MG correction (unit and
  residual-minimising scaling), the solve_pcg solution and the
  solve_fgmres(12) solution must match bit for bit;
* against the compiled reference live, when oracle/_ref is present;
* against the reference's own known-answer and property tests, ported:
  Chebyshev degrees 1-4 (tests/unit/solver_mg_chebyshev_test.cpp:797-841),
  IBM operator equivalence (tests/unit/solver_ibm_pressure_operator_test.cpp:
  131-233), monotone MG contraction (tests/numerical/
  solver_mg_convergence_test.cpp:630-800), the diagonal shortcut
  (tests/unit/solver_mg_chebyshev_test.cpp:1250-1300), line relaxation against point
  smoothing (tests/numerical/solver_mg_line_relaxation_test.cpp:316-335) and
  PCG against an independent direct solve (tests/mpi/
  solver_krylov_mpi_test.cpp:1141-1193).
"""
import dataclasses
import os

import numpy as np
import pytest

import golden_cases
from hfps import workloads

pytestmark = pytest.mark.usefixtures("oracle_built")


def _oracle(system, policy, unit_linear=True, line_order=0):
    import c_oracle
    return c_oracle.OracleSession(system, policy, unit_linear=unit_linear, line_order=line_order)


@pytest.mark.parametrize("name", sorted(golden_cases.index()))
def test_generator_matches_recorded_inputs(name):
    s = golden_cases.system(name)
    assert golden_cases.digest(s) == golden_cases.index()[name]["digest"]


@pytest.mark.parametrize("name", sorted(golden_cases.index()))
def test_restatement_reproduces_reference_golden(name):
    s = golden_cases.system(name)
    g = golden_cases.arrays(name)
    meta = golden_cases.index()[name]
    o = _oracle(s, golden_cases.policy(name))
    assert [list(l) for l in o.levels()] == meta["levels"]
    v = golden_cases.probe(s)
    assert np.array_equal(o.apply_operator(v), g["op"])
    assert np.array_equal(o.apply_mg(v), g["mg"])
    x, info = o.solve(s.rhs, rtol=1e-13, maxit=400)
    assert info["termination"] == "converged"
    assert info["iterations"] == meta["iterations_1e13"]
    assert np.array_equal(x, g["x"])


@pytest.mark.parametrize("name", sorted(golden_cases.index()))
def test_fgmres_restatement_reproduces_reference_golden(name):
    """solve_fgmres(12) with the residual-minimising MG plan
    (src/solver_krylov.cpp:1557-2650): same iterations, operator applies and
    solution bits as the reference."""
    s = golden_cases.system(name)
    g = golden_cases.arrays(name)
    meta = golden_cases.index()[name]
    o = _oracle(s, golden_cases.policy(name), unit_linear=False)
    assert np.array_equal(o.apply_mg(golden_cases.probe(s)), g["mg_residual_minimising"])
    x, info = o.solve(s.rhs, rtol=1e-13, maxit=400, algorithm="fgmres", restart=12)
    assert info["termination"] == "converged"
    assert info["iterations"] == meta["fgmres_iterations_1e13"]
    assert info["operator_applies"] == meta["fgmres_operator_applies"]
    assert info["final_true_residual"] == meta["fgmres_final_true_residual_1e13"]
    assert np.array_equal(x, g["x_fgmres"])


def test_fgmres_short_restart_matches_live_reference():
    """Restart lengths below the iteration count exercise the cycle-end
    restart and the interior true-residual audits."""
    import ref_oracle
    if not ref_oracle.available():
        pytest.skip("compiled reference not built (make -C oracle ref)")
    s = workloads.make("sphere64", n=(18, 14, 12), seed=8)
    for restart, tri in ((3, 4), (5, 2), (12, 4)):
        pol = ref_oracle.MgPolicy.production()
        r = ref_oracle.RefSession(s, pol, algorithm="fgmres", restart=restart)
        o = _oracle(s, pol, unit_linear=False)
        x1, i1 = r.solve(s.rhs, rtol=1e-12, true_residual_interval=tri)
        x2, i2 = o.solve(s.rhs, rtol=1e-12, true_residual_interval=tri, algorithm="fgmres",
                         restart=restart)
        assert (i1["iterations"], i1["operator_applies"]) == (i2["iterations"], i2["operator_applies"])
        assert np.array_equal(x1, x2)


@pytest.mark.parametrize("restart", [12, 4])
def test_recycling_restatement_reproduces_reference_golden(restart):
    """Two PISO correctors: corrector 1 captures its Arnoldi-cycle
    corrections, corrector 2 projects them before iterating
    (src/solver_linear_state.cpp:735-1037; src/solver_krylov.cpp:1745-2019)."""
    name = "sphere_24x20x16_prodF"
    s = golden_cases.system(name)
    meta = golden_cases.index()[name]["recycle"][str(restart)]
    gold = np.load(os.path.join(golden_cases.GOLDEN, "recycle_sphere_24x20x16_prodF.npz"))
    o = _oracle(s, golden_cases.policy(name), unit_linear=False)
    x1, i1 = o.solve(s.rhs, rtol=1e-10, algorithm="fgmres", restart=restart, recycle="capture")
    x2, i2 = o.solve(workloads.warm_start_rhs(s, 1), x0=x1, rtol=1e-10, algorithm="fgmres",
                     restart=restart, recycle="project")
    assert (i1["iterations"], i1["recycle_cycle_corrections"]) == (meta["capture_iterations"],
                                                                   meta["captured"])
    assert (i2["iterations"], i2["recycle_offered"], i2["recycle_retained"],
            i2["recycle_accepted"]) == (meta["project_iterations"], meta["offered"],
                                        meta["retained"], meta["accepted"])
    assert i2["recycle_projected_residual"] == meta["projected_residual"]
    assert np.array_equal(x1, gold[f"x1_r{restart}"])
    assert np.array_equal(x2, gold[f"x2_r{restart}"])


def test_recycling_short_restarts_and_guard_match_live_reference():
    import ref_oracle
    if not ref_oracle.available():
        pytest.skip("compiled reference not built (make -C oracle ref)")
    s = workloads.make("sphere64", n=(18, 14, 12), seed=8)
    pol = ref_oracle.MgPolicy.production()
    rhs2 = workloads.warm_start_rhs(s, 2)
    for restart in (3, 2):
        r = ref_oracle.RefSession(s, pol, algorithm="fgmres", restart=restart)
        o = _oracle(s, pol, unit_linear=False)
        kw = dict(algorithm="fgmres", restart=restart)
        y1, _ = r.solve(s.rhs, rtol=1e-10, recycle="capture")
        x1, _ = o.solve(s.rhs, rtol=1e-10, recycle="capture", **kw)
        y2, j2 = r.solve(rhs2, x0=y1, rtol=1e-10, recycle="project")
        x2, i2 = o.solve(rhs2, x0=x1, rtol=1e-10, recycle="project", **kw)
        assert np.array_equal(x2, y2)
        assert (i2["iterations"], i2["recycle_retained"]) == (j2["iterations"], j2["recycle_retained"])
        # zero-seed guard: a wild initial guess is replaced by x0 = 0
        y3, j3 = r.solve(rhs2, x0=50 * y1, rtol=1e-10, recycle="guard")
        x3, i3 = o.solve(rhs2, x0=50 * x1, rtol=1e-10, recycle="guard", **kw)
        assert j3["initial_true_residual"] == i3["initial_true_residual"] == j3["rhs_norm"]
        assert np.array_equal(x3, y3)


def test_restatement_matches_live_reference():
    import ref_oracle
    if not ref_oracle.available():
        pytest.skip("compiled reference not built (make -C oracle ref)")
    s = workloads.make("sphere64", n=(20, 13, 11), spheres=((0.4, 0.45, 0.5, 0.2),), seed=5)
    for pol in (ref_oracle.MgPolicy(), ref_oracle.MgPolicy.production(),
                ref_oracle.MgPolicy(cycle=1, pre=3, post=1, coarse_sweeps=7)):
        r = ref_oracle.RefSession(s, pol, algorithm="pcg")
        o = _oracle(s, pol)
        v = golden_cases.probe(s)
        assert np.array_equal(r.apply_mg(v), o.apply_mg(v))
        x1, i1 = r.solve(s.rhs, rtol=1e-11)
        x2, i2 = o.solve(s.rhs, rtol=1e-11)
        assert i1["iterations"] == i2["iterations"]
        assert np.array_equal(x1, x2)


def _uniform_system(n, diag, face, boundary=(0, 0, 0, 0, 0, 0), active=None, rhs=None):
    nx, ny, nz = n
    faces = tuple(workloads.uniform_faces(m) for m in n)
    fx = np.full((nz, ny, nx + 1), face)
    fy = np.full((nz, ny + 1, nx), face)
    fz = np.full((nz + 1, ny, nx), face)
    d = np.full((nz, ny, nx), diag)
    if rhs is None:
        rhs = np.zeros((nz, ny, nx))
    return workloads.PressureSystem("uniform", (nx, ny, nz), faces, tuple(boundary),
                                    np.ones((nz, ny, nx)), d, fx, fy, fz, active, rhs)


def test_diagonal_shortcut_known_answer():
    """Strong diagonal dominance takes the masked diagonal inverse instead of
    a cycle (tests/unit/solver_mg_chebyshev_test.cpp:1250-1300): on 8^3 cells
    with diagonal 100, unit faces and a solid corner cell, the correction is
    r / 100, r / 99 on the three cells that lost a face to the solid, 0 on the
    solid; a weakly dominant diagonal (7) runs the cycle again.  The
    restatement and, when built, the compiled reference."""
    import ref_oracle
    rng = np.random.default_rng(17)
    active = np.ones((8, 8, 8), np.uint8)
    active[0, 0, 0] = 0
    pol = ref_oracle.MgPolicy(smoother=1, cycle=0, pre=2, post=2, diagonal_shortcut=0.1)
    k, j, i = np.meshgrid(np.arange(8), np.arange(8), np.arange(8), indexing="ij")
    expected_divisor = np.where(i + j + k == 1, 99.0, 100.0)
    r = rng.standard_normal((8, 8, 8)) * active
    sessions = [lambda s: _oracle(s, pol)]
    if ref_oracle.available():
        sessions.append(lambda s: ref_oracle.RefSession(s, pol, algorithm="pcg"))
    for make in sessions:
        strong = make(_uniform_system((8, 8, 8), 100.0, 1.0, active=active))
        z = strong.apply_mg(r)
        assert np.array_equal(z, np.where(active == 1, r / expected_divisor, 0.0))
        weak = make(_uniform_system((8, 8, 8), 7.0, 1.0, active=active))
        zw = weak.apply_mg(r)
        assert np.all(np.isfinite(zw)) and not np.allclose(zw, r / 7.0)


def test_mg_correction_scales_with_the_residual():
    """The MG correction of 1e-12 r is 1e-12 times that of r to 1e-12
    relative (tests/unit/solver_mg_chebyshev_test.cpp:1358-1383: Chebyshev,
    diagonal 7, unit faces, r = 1), for both correction scalings."""
    import ref_oracle
    pol = ref_oracle.MgPolicy(smoother=1, cycle=0, pre=2, post=2)
    s = _uniform_system((8, 8, 8), 7.0, 1.0)
    r = np.ones((8, 8, 8))
    for unit_linear in (True, False):
        o = _oracle(s, pol, unit_linear=unit_linear)
        z = o.apply_mg(r)
        zs = o.apply_mg(1e-12 * r)
        magnitude = np.max(np.abs(z))
        assert magnitude > 0.0
        assert np.max(np.abs(zs / 1e-12 - z)) < 1e-12 * magnitude


@pytest.mark.parametrize("algorithm", ["pcg", "fgmres", "bicgstab"])
def test_iteration_cap_publishes_nothing(algorithm):
    """An iteration cap cannot masquerade as convergence
    (tests/mpi/solver_krylov_mpi_test.cpp:1474-1487): one iteration allowed,
    status rejected_step, termination maximum_iterations, and the caller's
    solution untouched; the compiled reference (PCG, FGMRES) does the same."""
    import ref_oracle
    s = workloads.make("sphere64", n=(12, 10, 9), spheres=((0.5, 0.5, 0.5, 0.2),), seed=2)
    x0 = 0.1 * np.ones_like(s.rhs)
    o = _oracle(s, ref_oracle.MgPolicy(), unit_linear=algorithm != "fgmres")
    x, info = o.solve(s.rhs, x0=x0, rtol=1e-12, maxit=1, algorithm=algorithm)
    assert info["status"] == 6 and info["termination"] == "maximum_iterations"
    assert info["iterations"] == 1 and np.array_equal(x, x0)
    if ref_oracle.available() and algorithm != "bicgstab":
        xr, ir = ref_oracle.RefSession(s, ref_oracle.MgPolicy(), algorithm=algorithm).solve(
            s.rhs, x0=x0, rtol=1e-12, maxit=1)
        assert ir["termination"] == "maximum_iterations" and ir["iterations"] == 1
        assert np.array_equal(xr, x0)


def test_ibm_coarse_rows_exclude_the_solid_identity():
    """Coarse rows of a masked hierarchy hold only the fluid cells' reaction
    and the open faces leaving the aggregate; a fully solid aggregate is an
    identity row (tests/unit/solver_mg_reuse_test.cpp:334-418: 16x12x8
    cells, faces 1e-9, diagonal 7e-9, one solid cell and a solid 2x2x2
    block)."""
    import ref_oracle
    nx, ny, nz = 16, 12, 8
    scale = 1e-9
    active = np.ones((nz, ny, nx), np.uint8)
    active[1, 1, 1] = 0
    active[2:4, 2:4, 2:4] = 0
    s = _uniform_system((nx, ny, nz), 7.0 * scale, scale, active=active)
    o = _oracle(s, ref_oracle.MgPolicy())
    levels = o.levels()
    if ref_oracle.available():
        assert ref_oracle.RefSession(s, ref_oracle.MgPolicy()).levels() == levels

    def open_cell(c):
        i, j, k = c
        inside = 0 <= i < nx and 0 <= j < ny and 0 <= k < nz
        return not inside or active[k, j, i] != 0

    width = [1, 1, 1]
    previous = (nx, ny, nz)
    assert len(levels) > 2
    for level in range(1, len(levels)):
        shape = levels[level][:3]
        width = [w * (2 if shape[a] != previous[a] else 1) for a, w in enumerate(width)]
        previous = shape
        diagonal = o.level_coefficients(level)[0]
        for x, y, z in np.ndindex(*shape):
            parent = (x, y, z)
            lo = [parent[a] * width[a] for a in range(3)]
            hi = [min((parent[a] + 1) * width[a], (nx, ny, nz)[a]) for a in range(3)]
            fluid = external = 0
            for i, j, k in np.ndindex(hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]):
                cell = (lo[0] + i, lo[1] + j, lo[2] + k)
                if not active[cell[2], cell[1], cell[0]]:
                    continue
                fluid += 1
                for a in range(3):
                    for step in (-1, 1):
                        nb = list(cell)
                        nb[a] += step
                        if not lo[a] <= nb[a] < hi[a] and open_cell(nb):
                            external += 1
            expected = 1.0 if fluid == 0 else (fluid + external) * scale
            assert abs(diagonal[z, y, x] - expected) <= 1e-14 * max(scale, expected)


def _box_system(n, lengths):
    """Uniform cells on a box, Dirichlet sides, faces area / distance."""
    nx, ny, nz = n
    faces = tuple(np.linspace(0.0, length, m + 1) for m, length in zip(n, lengths))
    hx, hy, hz = (length / m for m, length in zip(n, lengths))
    fx = np.full((nz, ny, nx + 1), hy * hz / hx)
    fy = np.full((nz, ny + 1, nx), hx * hz / hy)
    fz = np.full((nz + 1, ny, nx), hx * hy / hz)
    diagonal = fx[:, :, :-1] + fx[:, :, 1:] + fy[:, :-1] + fy[:, 1:] + fz[:-1] + fz[1:]
    return workloads.PressureSystem("box", tuple(n), faces, (0,) * 6, np.ones((nz, ny, nx)),
                                    diagonal, fx, fy, fz, None, np.zeros((nz, ny, nx)))


def test_coarsening_selection():
    """Strategy selection (tests/unit/solver_mg_reuse_test.cpp:414-470):
    16x12x8 cells on the unit cube coarsen in x, y and z with point
    smoothing; 64x48x8 cells on 1 x 1 x 4 (x and y strong) keep full
    coarsening with alternating x/y lines down to a terminal grid of at
    most 3 x 3 in the strong plane.  The compiled reference, when built,
    selects the same hierarchy."""
    import ref_oracle
    for n, lengths in (((16, 12, 8), (1.0, 1.0, 1.0)), ((64, 48, 8), (1.0, 1.0, 4.0))):
        s = _box_system(n, lengths)
        levels = _oracle(s, ref_oracle.MgPolicy()).levels()
        assert len(levels) > 1
        assert levels[1][:3] == tuple((m + 1) // 2 for m in n)  # full x/y/z coarsening
        if n == (16, 12, 8):
            assert all(level[3] == 0 for level in levels)
        else:
            assert all(level[3] == 3 for level in levels)
            assert levels[-1][0] <= 3 and levels[-1][1] <= 3
        if ref_oracle.available():
            assert ref_oracle.RefSession(s, ref_oracle.MgPolicy()).levels() == levels


def _scalar_chebyshev(rhs, diagonal, eigenvalue, stages, fraction):
    beta = 2.0
    alpha = fraction * beta
    theta = (beta + alpha) * 0.5
    delta = (beta - alpha) * 0.5
    sigma = theta / delta
    x = 0.0
    d = 0.0
    prev = 1.0 / sigma
    for s in range(stages):
        defect = rhs - eigenvalue * x
        if s == 0:
            d = defect / (theta * diagonal)
        else:
            rho = 1.0 / (2.0 * sigma - prev)
            d = rho * prev * d + (2.0 * rho / delta) * defect / diagonal
            prev = rho
        x += d
    return x


@pytest.mark.parametrize("degree", [1, 2, 3, 4])
def test_chebyshev_known_answer(degree):
    """Degree-d Chebyshev pre/post smoothing on A = 2I with alternating rhs
    has a closed form: the coarse correction of the alternating field is 0
    (solver_mg_chebyshev_test.cpp:797-841)."""
    import ref_oracle
    n = (8, 8, 8)
    i, j, k = np.meshgrid(np.arange(8), np.arange(8), np.arange(8), indexing="ij")
    sign = np.where(((i + j + k) & 1) == 0, 1.0, -1.0).transpose(2, 1, 0)
    s = _uniform_system(n, 2.0, 0.0, rhs=np.ascontiguousarray(sign))
    pol = ref_oracle.MgPolicy(smoother=1, pre=degree, post=degree)
    o = _oracle(s, pol)
    z = o.apply_mg(s.rhs)
    pre = _scalar_chebyshev(1.0, 2.0, 2.0, degree, 0.3)
    post = _scalar_chebyshev(1.0 - 2.0 * pre, 2.0, 2.0, degree, 0.3)
    assert np.max(np.abs(z - sign * (pre + post))) < 2e-12


def test_ibm_decoration_equals_masked_operator():
    """Decorated regular operator == compact operator with removed faces
    (solver_ibm_pressure_operator_test.cpp:131-233, tolerance 2e-12)."""
    s = workloads.make("sphere64", n=(18, 16, 14), spheres=((0.45, 0.5, 0.5, 0.25),))
    o = _oracle(s, None)
    v = golden_cases.probe(s)
    decorated = o.apply_operator(v)
    masked = o.apply_level(0, v)
    scale = np.max(np.abs(decorated))
    assert np.max(np.abs(decorated - masked)) <= 2e-12 * scale
    solid = s.active == 0
    assert np.array_equal(decorated[solid], v[solid])


def test_mg_cycles_contract_monotonically():
    """Residual-minimising MG as a stationary iteration reduces the true
    residual monotonically (solver_mg_convergence_test.cpp:630-800)."""
    import ref_oracle
    s = workloads.make("wrinkled256", n=(16, 12, 8), stretch_y=None, seed=3)
    o = _oracle(s, ref_oracle.MgPolicy(), unit_linear=False)
    x = np.zeros_like(s.rhs)
    r = s.rhs - o.apply_operator(x)
    norms = [np.linalg.norm(r)]
    for _ in range(10):
        x = x + o.apply_mg(r)
        r = s.rhs - o.apply_operator(x)
        norms.append(np.linalg.norm(r))
    assert all(b <= a * (1 + 1e-12) for a, b in zip(norms, norms[1:]))
    assert norms[-1] <= 0.5 * norms[0]


@pytest.mark.parametrize("line_order", [0, 1])
def test_line_relaxation_outperforms_point_smoothing(line_order):
    """One MG application from zero on the strongly x-coupled 64x12x8 mesh
    (tests/numerical/solver_mg_line_relaxation_test.cpp:316-335): x-lines are
    selected, the cycle leaves at most 0.10 of the initial residual, and at
    most 0.70 of what point-only smoothing leaves.  Lexicographic (the
    reference's) and zebra (the CUDA path's) line orders."""
    s = golden_cases.anisotropic_x_system()
    residual = {}
    for lines in (True, False):
        o = _oracle(s, golden_cases.line_relaxation_policy(lines), line_order=line_order)
        assert o.levels()[0][3] == (1 if lines else 0)
        z = o.apply_mg(s.rhs)
        assert np.all(np.isfinite(z))
        residual[lines] = np.linalg.norm(s.rhs - o.apply_operator(z))
    assert residual[True] <= 0.10 * np.linalg.norm(s.rhs)
    assert residual[True] <= 0.70 * residual[False]


def test_pcg_matches_direct_solve():
    """solve_pcg with MG against an independent sparse direct solve
    (solver_krylov_mpi_test.cpp:1141-1193: error < 1e-8)."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    s = workloads.make("sphere64", n=(12, 10, 9), spheres=((0.5, 0.5, 0.5, 0.2),), seed=2)
    o = _oracle(s, None)
    n = s.cells
    cols = []
    for c in range(n):
        e = np.zeros(n)
        e[c] = 1.0
        cols.append(sp.csc_matrix(o.apply_operator(e.reshape(s.rhs.shape)).reshape(-1, 1)))
    A = sp.hstack(cols).tocsc()
    exact = spla.spsolve(A, s.rhs.reshape(-1)).reshape(s.rhs.shape)
    x, info = o.solve(s.rhs, rtol=1e-13)
    assert info["termination"] == "converged"
    assert np.linalg.norm(x - exact) / np.linalg.norm(exact) < 1e-8


def test_zero_rhs_and_converged_guess():
    s = workloads.make("sphere64", n=(8, 8, 8))
    o = _oracle(s, None)
    x, info = o.solve(np.zeros_like(s.rhs))
    assert info["termination"] == "zero_rhs" and not np.any(x)
    x1, _ = o.solve(s.rhs, rtol=1e-12)
    x2, info2 = o.solve(s.rhs, x0=x1, rtol=1e-10)
    assert info2["iterations"] == 0 and info2["termination"] == "converged"


@pytest.mark.parametrize("name", ["sphere_24x20x16_rbV22", "wrinkled_16x40x12_lineF"])
def test_cold_path_restatement_reproduces_reference_golden(name):
    """Diagonal IC(0) in lexicographic order (ColdPressureIccg,
    src/solver_iccg.hpp:224-293; ColdPressureDilu, src/solver_cold.hpp:
    484-560, identical on the symmetric pressure rows) with solve_pcg and
    solve_bicgstab (src/solver_krylov.cpp:2651-3090), bit for bit."""
    import c_oracle
    s = golden_cases.system(name)
    meta = golden_cases.index()[name]["cold"]
    gold = np.load(os.path.join(golden_cases.GOLDEN, "cold_path.npz"))
    o = c_oracle.OracleSession(s, golden_cases.policy(name), preconditioner="dic")
    v = golden_cases.probe(s)
    z = o.apply_preconditioner(v)
    assert np.array_equal(z, gold[f"{name}_iccg_apply"])
    assert np.array_equal(z, gold[f"{name}_dilu_apply"])
    for algorithm, pc in (("pcg", "iccg"), ("bicgstab", "dilu")):
        x, info = o.solve(s.rhs, rtol=1e-12, maxit=8000, algorithm=algorithm)
        assert info["iterations"] == meta[f"{algorithm}_{pc}"]["iterations"]
        assert info["operator_applies"] == meta[f"{algorithm}_{pc}"]["operator_applies"]
        assert np.array_equal(x, gold[f"{name}_{algorithm}_{pc}_x"])


def test_cold_path_matches_live_reference_with_ibm():
    import c_oracle
    import ref_oracle
    if not ref_oracle.available():
        pytest.skip("compiled reference not built (make -C oracle ref)")
    s = workloads.make("sphere64", n=(15, 12, 10), seed=12)
    pol = ref_oracle.MgPolicy()
    o = c_oracle.OracleSession(s, pol, preconditioner="dic")
    for algorithm, pc in (("pcg", "iccg"), ("bicgstab", "dilu")):
        r = ref_oracle.RefSession(s, pol, algorithm=algorithm, preconditioner=pc)
        x1, i1 = r.solve(s.rhs, rtol=1e-9, maxit=3000)
        x2, i2 = o.solve(s.rhs, rtol=1e-9, maxit=3000, algorithm=algorithm)
        assert i1["iterations"] == i2["iterations"]
        assert np.array_equal(x1, x2)


def test_cold_bicgstab_restatement_at_64_cubed():
    """The C restatement's solve_bicgstab + DILU on the 64^3 spherical flame
    takes the reference's recorded 518 iterations and lands on its solution
    bit for bit on the seeded sample (tests/golden/cold_path_64.*), so the
    iteration spread recorded beside it (make_golden.py --cold64-spread,
    seed 0 of which is this run) is measured around the reference's own
    trajectory."""
    import json
    import c_oracle
    meta = json.load(open(os.path.join(golden_cases.GOLDEN, "cold_path_64.json")))
    gold = np.load(os.path.join(golden_cases.GOLDEN, "cold_path_64.npz"))
    s = workloads.make("sphere64")
    assert golden_cases.digest(s) == meta["digest"]
    o = c_oracle.OracleSession(s, preconditioner="dic")
    x, info = o.solve(s.rhs, rtol=1e-12, maxit=8000, algorithm="bicgstab")
    o.close()
    assert info["iterations"] == meta["bicgstab_dilu"]["iterations"]
    assert np.array_equal(x.reshape(-1)[gold["cells"]], gold["bicgstab_dilu_x"])
    spread = meta["bicgstab_dilu_ulp_spread"]["iterations"]
    assert len(spread) >= 8 and min(spread) < info["iterations"] < max(spread)


@pytest.mark.parametrize("name", ["sphere_24x20x16_rbV22", "wrinkled_16x40x12_lineF"])
def test_ulp_spread_replica_follows_the_restatement(name):
    """The Python BiCGSTAB that measures the one-ulp iteration spread
    (make_golden.py _bicgstab_ulp_iterations) takes, unperturbed, the
    reference's recorded iteration count on the small cold-path cases, so
    its control flow is the restatement's (hfo_solve_bicgstab)."""
    from golden import make_golden
    meta = golden_cases.index()[name]
    count = make_golden._bicgstab_ulp_iterations(0, spec=meta["spec"])
    assert count == meta["cold"]["bicgstab_dilu"]["iterations"]
