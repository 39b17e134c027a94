"""The cold path on the GPU (through the C ABI) against the reference.

The reference's cold pressure path pairs solve_pcg with ColdPressureIccg and
solve_bicgstab with ColdPressureDilu (src/solver_iccg.hpp:224-293,
src/solver_cold.hpp:484-560; the two factorisations coincide on the
symmetric pressure rows).  The GPU evaluates the same lexicographic
factorisation and sweeps plane by plane (wavefronts i + j + k = t), each
cell with the reference's arithmetic, so:
* one preconditioner application is bit-identical to the reference's;
* solves match the reference's solution to 1e-9 and its iteration counts:
  within +-2% for PCG, within the path's +-20% bar for BiCGSTAB, whose
  irregular convergence amplifies the one difference between the two runs
  (Krylov dot products as fixed-order trees here, compensated sums there).
"""
import numpy as np
import pytest

import golden_cases

pytestmark = [pytest.mark.gpu, pytest.mark.usefixtures("oracle_built")]

CASES = ["sphere_24x20x16_rbV22", "wrinkled_16x40x12_lineF"]


@pytest.fixture(scope="module")
def hfps_mod(cuda_library):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    import hfps
    return hfps


def cold_solver(hfps, system):
    return hfps.PressureSolver.from_system(system,
                                           hfps.Policy.default().replace(preconditioner=hfps.IC0))


@pytest.mark.parametrize("name", CASES)
def test_ic0_application_is_bit_identical(hfps_mod, name):
    s = golden_cases.system(name)
    gold = np.load(golden_cases.GOLDEN + "/cold_path.npz")
    g = cold_solver(hfps_mod, s)
    z = g.apply_preconditioner(golden_cases.probe(s))
    assert np.array_equal(z, gold[f"{name}_iccg_apply"])


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("algorithm,pc", [("pcg", "iccg"), ("bicgstab", "dilu")])
def test_cold_solves_match_reference(hfps_mod, name, algorithm, pc):
    s = golden_cases.system(name)
    meta = golden_cases.index()[name]["cold"][f"{algorithm}_{pc}"]
    gold = np.load(golden_cases.GOLDEN + "/cold_path.npz")[f"{name}_{algorithm}_{pc}_x"]
    g = cold_solver(hfps_mod, s)
    alg = hfps_mod.PCG if algorithm == "pcg" else hfps_mod.BICGSTAB
    x, info = g.solve(s.rhs, rtol=1e-12, maxit=8000, algorithm=alg)
    assert info["termination"] == "converged"
    ref_it = meta["iterations"]
    bar = 0.02 if algorithm == "pcg" else 0.2
    assert abs(info["iterations"] - ref_it) <= max(1, int(bar * ref_it))
    assert np.linalg.norm(x - gold) / np.linalg.norm(gold) <= 1e-9


def test_bicgstab_needs_the_cold_preconditioner(hfps_mod):
    """solve_bicgstab demands a fixed general preconditioner
    (src/solver_krylov.cpp:972-976): the MG plan is refused, as the
    reference refuses it."""
    s = golden_cases.system(CASES[0])
    g = hfps_mod.PressureSolver.from_system(s, hfps_mod.Policy.default())
    with pytest.raises(hfps_mod.SolverError) as err:
        g.solve(s.rhs, algorithm=hfps_mod.BICGSTAB)
    assert err.value.status == 2


def test_cold_path_at_64_cubed(hfps_mod):
    """The cold path at 64^3 (spherical flame, 262,144 cells) against the
    reference's record on a seeded sample of cells (tests/golden/
    cold_path_64.*, make_golden.py --cold64): the IC(0) application is bit
    for bit the reference's, PCG + IC(0) takes the reference's 5698
    iterations within 2%, and both solutions agree with the reference's on
    the sample to 1e-9 (PCG) and 1e-8 (BiCGSTAB; the reference's own PCG
    and BiCGSTAB solutions at rtol 1e-12 differ by 1.3e-9 there).

    BiCGSTAB + DILU takes 518 iterations in the reference, but its count at
    this size is set by last-bit rounding: moving the operator's result by
    one ulp per cell moves the C restatement's count over 450-738 (16 seeds,
    make_golden.py --cold64-spread).  The CUDA operator differs from the
    reference's by rounding only, so the count is held to that spread,
    widened by 10%, not to the single 518."""
    import json
    from hfps import workloads
    meta = json.load(open(golden_cases.GOLDEN + "/cold_path_64.json"))
    gold = dict(np.load(golden_cases.GOLDEN + "/cold_path_64.npz"))
    s = workloads.make("sphere64")
    assert golden_cases.digest(s) == meta["digest"]
    cells = gold["cells"]
    g = cold_solver(hfps_mod, s)
    z = g.apply_preconditioner(golden_cases.probe(s))
    assert np.array_equal(z.reshape(-1)[cells], gold["iccg_apply"])
    spread = meta["bicgstab_dilu_ulp_spread"]["iterations"]
    for algorithm, pc, solution_bar in (("pcg", "iccg", 1e-9), ("bicgstab", "dilu", 1e-8)):
        alg = hfps_mod.PCG if algorithm == "pcg" else hfps_mod.BICGSTAB
        x, info = g.solve(s.rhs, rtol=1e-12, maxit=8000, algorithm=alg)
        ref = meta[f"{algorithm}_{pc}"]
        assert info["termination"] == "converged"
        if algorithm == "pcg":
            assert abs(info["iterations"] - ref["iterations"]) <= int(0.02 * ref["iterations"])
        else:
            assert 0.9 * min(spread) <= info["iterations"] <= 1.1 * max(spread)
        sample = x.reshape(-1)[cells]
        want = gold[f"{algorithm}_{pc}_x"]
        assert np.linalg.norm(sample - want) / np.linalg.norm(want) <= solution_bar
        assert abs(np.linalg.norm(x) - ref["x_norm"]) <= solution_bar * ref["x_norm"]
    g.close()
