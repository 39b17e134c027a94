"""Parity of the CUDA path (through the C ABI) with the oracle.

Bars:
* level coefficients and point-smoother MG corrections (red-black,
  Chebyshev, V and F cycles): bit-identical to the C restatement, which is
  itself bit-identical to the reference;
* line relaxation (chunked scan on large levels, PCR on small ones):
  1e-11 relative;
* exact operator: 1e-15 relative (IBM faces folded into the coefficients
  instead of applied as link corrections);
* solves: same iteration count as the restatement run in the same line
  order, solution within 1e-12; against the reference's own solve (golden
  fixtures) iterations within +-20% and p within 1e-9 relative L2 at 1e-13.
"""
import numpy as np
import pytest

import golden_cases
from hfps import workloads

pytestmark = [pytest.mark.gpu, pytest.mark.usefixtures("oracle_built")]


@pytest.fixture(scope="module")
def hfps_mod(cuda_library):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    import hfps
    return hfps


def gpu_policy(hfps, p):
    return hfps.Policy.default().replace(
        point_smoother=p.smoother, cycle=p.cycle, pre_sweeps=p.pre, post_sweeps=p.post,
        coarse_sweeps=p.coarse_sweeps, maximum_levels=p.max_levels,
        minimum_coarse_extent=p.min_coarse_extent,
        chebyshev_lower_spectrum_fraction=p.chebyshev_fraction,
        anisotropy_threshold=p.anisotropy_threshold,
        diagonal_shortcut_maximum_ratio=p.diagonal_shortcut)


def oracle(system, policy, line_order=1, unit_linear=True):
    import c_oracle
    return c_oracle.OracleSession(system, policy, unit_linear=unit_linear, line_order=line_order)


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


CASES = sorted(golden_cases.index())


@pytest.mark.parametrize("name", CASES)
def test_level_coefficients_bitwise(hfps_mod, name):
    s = golden_cases.system(name)
    pol = golden_cases.policy(name)
    o = oracle(s, pol)
    g = hfps_mod.PressureSolver.from_system(s, gpu_policy(hfps_mod, pol))
    assert g.levels() == o.levels()
    for level in range(len(o.levels())):
        for a, b in zip(g.level_coefficients(level), o.level_coefficients(level)):
            assert np.array_equal(a, b), level


@pytest.mark.parametrize("name", CASES)
def test_operator_matches(hfps_mod, name):
    s = golden_cases.system(name)
    g = hfps_mod.PressureSolver.from_system(s, gpu_policy(hfps_mod, golden_cases.policy(name)))
    v = golden_cases.probe(s)
    ref = golden_cases.arrays(name)["op"]
    assert rel(g.apply_operator(v), ref) <= 1e-15


@pytest.mark.parametrize("name", CASES)
def test_mg_correction_matches(hfps_mod, name):
    s = golden_cases.system(name)
    pol = golden_cases.policy(name)
    g = hfps_mod.PressureSolver.from_system(s, gpu_policy(hfps_mod, pol))
    o = oracle(s, pol, line_order=1)
    v = golden_cases.probe(s)
    z = g.apply_preconditioner(v)
    line_mode = any(l[3] for l in o.levels())
    if line_mode:
        assert rel(z, o.apply_mg(v)) <= 1e-11
    else:
        assert np.array_equal(z, o.apply_mg(v))
        # the point-smoother cycle equals the reference's own output bit for bit
        assert np.array_equal(z, golden_cases.arrays(name)["mg"])


@pytest.mark.parametrize("shape", [(128, 96, 96), (73, 150, 40)])
def test_mg_scan_lines_match(hfps_mod, shape):
    """Line colours with many lines use the chunked-scan solve (chunks of 16
    rows per thread combined through shared memory): the zebra cycle matches
    the restatement's serial Thomas solves to rounding."""
    import ref_oracle
    s = workloads.make("wrinkled256", n=shape, stretch_y=1.05, seed=4)
    pol = ref_oracle.MgPolicy(cycle=0, pre=1, post=1, coarse_sweeps=2, max_levels=2)
    g = hfps_mod.PressureSolver.from_system(s, gpu_policy(hfps_mod, pol))
    o = oracle(s, pol, line_order=1)
    assert o.levels()[0][3] == 2
    v = golden_cases.probe(s)
    assert rel(g.apply_preconditioner(v), o.apply_mg(v)) <= 1e-13


def test_line_relaxation_outperforms_point_smoothing(hfps_mod):
    """The reference's line-relaxation fixture (tests/numerical/
    solver_mg_line_relaxation_test.cpp:316-335) on the GPU: x-lines (PCR
    colour passes) match the restatement's zebra cycle to line-mode rounding,
    point-only smoothing matches it bit for bit, and the line cycle keeps the
    reference test's bounds (<= 0.10 of the initial residual, <= 0.70 of the
    point-only residual)."""
    s = golden_cases.anisotropic_x_system()
    residual = {}
    for lines in (True, False):
        pol = golden_cases.line_relaxation_policy(lines)
        g = hfps_mod.PressureSolver.from_system(s, gpu_policy(hfps_mod, pol))
        o = oracle(s, pol, line_order=1)
        assert g.levels()[0][3] == (1 if lines else 0)
        z = g.apply_preconditioner(s.rhs)
        zo = o.apply_mg(s.rhs)
        if lines:
            assert rel(z, zo) <= 1e-11
        else:
            assert np.array_equal(z, zo)
        residual[lines] = np.linalg.norm(s.rhs - o.apply_operator(z))
        g.close()
    assert residual[True] <= 0.10 * np.linalg.norm(s.rhs)
    assert residual[True] <= 0.70 * residual[False]


def stretched_front(n, axis, ratio=1.05):
    """A wrinkled density front on a grid stretched along `axis` (0 x, 2 z)."""
    faces = [workloads.uniform_faces(m) for m in n]
    faces[axis] = workloads.stretched_faces(n[axis], ratio)
    faces = tuple(faces)
    z, y, x = workloads._grid(faces)
    front = (y - 0.4 - 0.05 * np.sin(8.0 * np.pi * x) * np.sin(8.0 * np.pi * z)) / 0.01
    rho = workloads._tanh_front(front) * np.ones(n[::-1])
    solid = np.broadcast_to((x - 0.2) ** 2 + (z - 0.5) ** 2 <= 0.08 * 0.08, n[::-1]).copy()
    return workloads._build("stretched_front", faces, rho, solid, workloads.PISO_BOUNDARY, 4)


@pytest.mark.parametrize("axis,shape", [(0, (96, 64, 48)), (2, (64, 48, 96))])
def test_mg_scan_lines_other_axes(hfps_mod, axis, shape):
    """x- and z-line relaxation with the chunked scan (z-lines with split-row
    vectors) against the restatement's serial Thomas solves."""
    s = stretched_front(shape, axis)
    pol = ref_oracle_policy()
    g = hfps_mod.PressureSolver.from_system(s, gpu_policy(hfps_mod, pol))
    o = oracle(s, pol, line_order=1)
    assert o.levels()[0][3] == 1 << axis
    assert g.levels()[0][3] == 1 << axis
    v = golden_cases.probe(s)
    assert rel(g.apply_preconditioner(v), o.apply_mg(v)) <= 1e-13


def ref_oracle_policy():
    import ref_oracle
    return ref_oracle.MgPolicy(cycle=0, pre=1, post=1, coarse_sweeps=2, max_levels=2)


@pytest.mark.parametrize("name", CASES)
def test_solve_parity_with_reference(hfps_mod, name):
    s = golden_cases.system(name)
    pol = golden_cases.policy(name)
    meta = golden_cases.index()[name]
    gold = golden_cases.arrays(name)
    g = hfps_mod.PressureSolver.from_system(s, gpu_policy(hfps_mod, pol))
    x, info = g.solve(s.rhs, rtol=1e-13, maxit=400)
    assert info["termination"] == "converged"
    ref_it = meta["iterations_1e13"]
    assert abs(info["iterations"] - ref_it) <= max(1, int(0.2 * ref_it))
    assert np.linalg.norm(x - gold["x"]) / np.linalg.norm(gold["x"]) <= 1e-9
    o = oracle(s, pol, line_order=1)
    xo, io = o.solve(s.rhs, rtol=1e-13, maxit=400)
    assert info["iterations"] == io["iterations"]
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= 1e-12
    hist = info["history"]
    assert len(hist) == info["iterations"] and np.all(np.isfinite(hist))


def test_sphere64_full_case(hfps_mod):
    """The 64^3 spherical-flame case against the reference solve (recorded
    when the reference is present, else the restatement)."""
    import ref_oracle
    s = workloads.make("sphere64")
    pol = ref_oracle.MgPolicy.production()
    g = hfps_mod.PressureSolver.from_system(s, hfps_mod.Policy.production())
    x, info = g.solve(s.rhs, rtol=1e-13, maxit=400)
    o = oracle(s, pol, line_order=0)
    xo, io = o.solve(s.rhs, rtol=1e-13, maxit=400)
    assert info["termination"] == "converged"
    assert abs(info["iterations"] - io["iterations"]) <= max(1, int(0.2 * io["iterations"]))
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= 1e-9
    r = s.rhs - o.apply_operator(x)
    assert np.linalg.norm(r) <= 1e-13 * np.linalg.norm(s.rhs) * 1.01


def test_mixed_precision_reaches_fp64_tolerance(hfps_mod):
    s = workloads.make("sphere64", n=(48, 40, 36))
    g = hfps_mod.PressureSolver.from_system(s, hfps_mod.Policy.production())
    x64, i64 = g.solve(s.rhs, rtol=1e-12)
    xm, im = g.solve(s.rhs, rtol=1e-12, precision=hfps_mod.MIXED)
    assert im["termination"] == "converged"
    assert im["final_true_residual"] <= 1e-12 * im["rhs_norm"]
    assert np.linalg.norm(xm - x64) / np.linalg.norm(x64) <= 1e-9
    assert abs(im["iterations"] - i64["iterations"]) <= max(2, int(0.2 * i64["iterations"]))


def test_device_and_host_memory_agree(hfps_mod):
    import torch
    s = workloads.make("sphere64", n=(32, 24, 20))
    g = hfps_mod.PressureSolver.from_system(s, hfps_mod.Policy.production())
    xh, ih = g.solve(s.rhs, rtol=1e-11)
    rd = torch.from_numpy(s.rhs.reshape(-1)).cuda()
    xd, idv = g.solve(rd, rtol=1e-11)
    assert ih["iterations"] == idv["iterations"]
    assert np.array_equal(xh.reshape(-1), xd.cpu().numpy())


def test_warm_start_and_termination_codes(hfps_mod):
    s = workloads.make("sphere64", n=(24, 24, 24))
    g = hfps_mod.PressureSolver.from_system(s, hfps_mod.Policy.production())
    x, info = g.solve(s.rhs, rtol=1e-11)
    assert info["termination"] == "converged"
    _, again = g.solve(s.rhs, x0=x, rtol=1e-10)
    assert again["iterations"] == 0 and again["termination"] == "converged"
    zero, zinfo = g.solve(np.zeros_like(s.rhs))
    assert zinfo["termination"] == "zero_rhs" and not np.any(zero)
    with pytest.raises(hfps_mod.SolverError) as err:
        g.solve(s.rhs, rtol=1e-14, maxit=3)
    assert err.value.status == 6 and err.value.result["termination"] == "maximum_iterations"
    bad = s.rhs.copy()
    bad.reshape(-1)[5] = np.nan
    with pytest.raises(hfps_mod.SolverError) as err:
        g.solve(bad)
    assert err.value.status == 5


def test_invalid_coefficients_rejected(hfps_mod):
    s = workloads.make("sphere64", n=(8, 8, 8))
    g = hfps_mod.PressureSolver(s.shape, s.faces, s.boundary, s.active)
    fx = s.face_x.copy()
    fx.reshape(-1)[3] = -1.0
    with pytest.raises(hfps_mod.SolverError) as err:
        g.set_coefficients(s.diagonal, fx, s.face_y, s.face_z)
    assert err.value.status == 2
    with pytest.raises(hfps_mod.SolverError):
        g.solve(s.rhs)  # no coefficients yet


def test_beta_helper_matches_host_assembly(hfps_mod):
    s = workloads.make("wrinkled256", n=(20, 28, 12), stretch_y=1.05)
    g = hfps_mod.PressureSolver(s.shape, s.faces, s.boundary, s.active,
                                policy=hfps_mod.Policy.production())
    g.set_beta(np.ascontiguousarray(s.beta))
    h = hfps_mod.PressureSolver.from_system(s, hfps_mod.Policy.production())
    for a, b in zip(g.level_coefficients(0), h.level_coefficients(0)):
        assert rel(a, b) <= 1e-14


def test_scaled_norm_matches_global_norm(hfps_mod):
    """HFPS_NORM_SCALED forms ||b|| and every residual norm as the reference's
    global_norm (src/solver_krylov.cpp:650-711): max |v|, then
    max * sqrt(sum (v / max)^2).  The rhs norm matches that definition
    evaluated exactly (math.fsum) to a few ulps, and PCG, FGMRES and the
    BiCGSTAB cold path reach the same solutions in the same iterations as
    with the plain norm; a zero rhs still terminates as zero_rhs."""
    import math
    s = workloads.make("wrinkled256", n=(48, 64, 32))
    b = s.rhs.reshape(-1)
    m = float(np.max(np.abs(b)))
    exact = m * math.sqrt(math.fsum(float(v) * float(v) for v in (b / m)))
    runs = [(hfps_mod.Policy.production(), dict()),
            (hfps_mod.Policy.production().replace(unit_linear=0),
             dict(algorithm=hfps_mod.FGMRES, restart=12)),
            (hfps_mod.Policy.production().replace(preconditioner=hfps_mod.IC0),
             dict(algorithm=hfps_mod.BICGSTAB))]
    for policy, extra in runs:
        g = hfps_mod.PressureSolver.from_system(s, policy)
        x0, i0 = g.solve(s.rhs, rtol=1e-11, maxit=800, **extra)
        x1, i1 = g.solve(s.rhs, rtol=1e-11, maxit=800, norm=hfps_mod.NORM_SCALED, **extra)
        assert i1["termination"] == "converged"
        assert abs(i1["rhs_norm"] - exact) <= 4e-16 * 8 * exact
        assert abs(i0["rhs_norm"] - i1["rhs_norm"]) <= 1e-14 * exact
        assert abs(i1["iterations"] - i0["iterations"]) <= 1
        assert i1["final_true_residual"] <= i1["true_residual_limit"]
        assert np.linalg.norm(x1 - x0) <= 1e-9 * np.linalg.norm(x0)
        _, z = g.solve(np.zeros_like(s.rhs), norm=hfps_mod.NORM_SCALED, **extra)
        assert z["termination"] == "zero_rhs"
        g.close()
