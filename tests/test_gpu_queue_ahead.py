"""PCG queue-ahead (solver.cu krylov_pcg): the next MG application and
direction update are queued before the host reads an iteration's scalars,
in iterations that are not planned true-residual checks while the recursive
residual is far above the limit.  That is the work the iteration does next
unless its residual met the limit, and a true-residual check overwrites z,
p and r.z; so solves are bit-identical to reading the scalars first
(HFPS_QUEUE_AHEAD=0, read when the solver is created): same solution, same
residual history, same counts, in FP64 and mixed precision."""
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


def make_solver(hfps, s, ahead):
    saved = os.environ.get("HFPS_QUEUE_AHEAD")
    os.environ["HFPS_QUEUE_AHEAD"] = "1" if ahead else "0"
    try:
        return hfps.PressureSolver.from_system(s, hfps.Policy.production())
    finally:
        if saved is None:
            os.environ.pop("HFPS_QUEUE_AHEAD", None)
        else:
            os.environ["HFPS_QUEUE_AHEAD"] = saved


@pytest.mark.parametrize("case", ["sphere64", "wrinkled_64x96x48"])
def test_queue_ahead_is_bit_identical(hfps_mod, case):
    s = (workloads.make("sphere64") if case == "sphere64"
         else workloads.make("wrinkled256", n=(64, 96, 48)))
    plain = make_solver(hfps_mod, s, False)
    ahead = make_solver(hfps_mod, s, True)
    for precision in (hfps_mod.FP64, hfps_mod.MIXED):
        for rtol in (1e-10, 1e-13):
            x0, i0 = plain.solve(s.rhs, rtol=rtol, precision=precision)
            x1, i1 = ahead.solve(s.rhs, rtol=rtol, precision=precision)
            assert np.array_equal(x0, x1)
            assert np.array_equal(i0["history"], i1["history"])
            for key in ("iterations", "termination", "operator_applies",
                        "preconditioner_applies", "final_true_residual"):
                assert i0[key] == i1[key], key
    plain.close()
    ahead.close()
