"""PCG with its r.z formed in the MG exit.

With the MG preconditioner at unit scaling, the MG exit forms r.z while it
writes z (the same products, summed in the same order as the separate dot
kernel), so one pass over r and z and one launch per iteration are saved.
HFPS_KRYLOV_FUSION=0 (read when the solver is created) keeps the separate
kernel.  Solutions, iteration counts and residual histories must agree bit
for bit.
"""
import os

import numpy as np
import pytest

from hfps import workloads

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def hfps_mod(cuda_library):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    import hfps
    return hfps


def make_solver(hfps, system, policy, fused):
    saved = os.environ.get("HFPS_KRYLOV_FUSION")
    os.environ["HFPS_KRYLOV_FUSION"] = "1" if fused else "0"
    try:
        return hfps.PressureSolver.from_system(system, policy)
    finally:
        if saved is None:
            os.environ.pop("HFPS_KRYLOV_FUSION", None)
        else:
            os.environ["HFPS_KRYLOV_FUSION"] = saved


CASES = {
    "lines_production": (lambda: workloads.make("wrinkled256", n=(96, 128, 64)), "production"),
    "sphere_production": (lambda: workloads.make("sphere64"), "production"),
    "sphere_red_black": (lambda: workloads.make("sphere64"), "default"),
}


@pytest.mark.parametrize("case", sorted(CASES))
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_fused_pcg_bitwise(hfps_mod, case, precision):
    make, policy_name = CASES[case]
    s = make()
    policy = getattr(hfps_mod.Policy, policy_name)()
    prec = hfps_mod.FP64 if precision == "fp64" else hfps_mod.MIXED
    plain = make_solver(hfps_mod, s, policy, fused=False)
    fused = make_solver(hfps_mod, s, policy, fused=True)
    x0 = None
    for step in range(2):  # a cold solve, then a warm start from its solution
        a, ia = plain.solve(s.rhs, x0=x0, rtol=1e-10, precision=prec)
        b, ib = fused.solve(s.rhs, x0=x0, rtol=1e-10, precision=prec)
        assert ia["termination"] == ib["termination"] == "converged"
        assert ia["iterations"] == ib["iterations"]
        assert np.array_equal(ia["history"], ib["history"])
        assert np.array_equal(a, b)
        assert ib["kernel_launches"] < ia["kernel_launches"] or step == 1
        x0 = 0.5 * a
    plain.close()
    fused.close()
