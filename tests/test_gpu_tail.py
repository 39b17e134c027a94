"""The small levels of a y-line hierarchy as one persistent launch
(kernels_tail.cu, HFPS_TAIL=1) against one kernel per phase (HFPS_TAIL=0),
both read when the solver is created.

The persistent launch runs the same phase bodies in the same order with a
grid barrier between phases, and the dense coarsest map sums its partials
in the same 32-warp grouping, so MG applications are bitwise equal in FP64
and in the FP32 hierarchy, and solves take the same iterations to the same
solution.  The CTA count is varied through HFPS_TAIL_BLOCKS: a CTA that
covers several rounds of a level's lines must give the same result.
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


CASES = {
    "y_lines_96x128x64": lambda: workloads.make("wrinkled256", n=(96, 128, 64)),
    "y_lines_odd_73x150x40": lambda: workloads.make("wrinkled256", n=(73, 150, 40)),
    "y_lines_128": lambda: workloads.make("wrinkled256", n=(128, 128, 128)),
}


def make_solver(hfps, system, policy, tail, blocks=None):
    env = {"HFPS_TAIL": "1" if tail else "0", "HFPS_TAIL_BLOCKS": str(blocks or "")}
    saved = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        return hfps.PressureSolver.from_system(system, policy)
    finally:
        for k, v in saved.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


def rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.mark.parametrize("case", sorted(CASES))
@pytest.mark.parametrize("unit", [True, False])
def test_tail_launch_matches_per_phase_kernels(hfps_mod, case, unit):
    s = CASES[case]()
    policy = hfps_mod.Policy.production().replace(unit_linear=1 if unit else 0)
    plain = make_solver(hfps_mod, s, policy, tail=False)
    tail = make_solver(hfps_mod, s, policy, tail=True)
    assert plain.levels() == tail.levels()
    rng = np.random.default_rng(5)
    r = rng.standard_normal(s.cells).reshape(s.rhs.shape)
    few = make_solver(hfps_mod, s, policy, tail=True, blocks=3)
    for precision in (hfps_mod.FP64, hfps_mod.MIXED):
        for _ in range(2):
            z0 = plain.apply_preconditioner(r, precision=precision)
            z1 = tail.apply_preconditioner(r, precision=precision)
            z2 = few.apply_preconditioner(r, precision=precision)
            assert np.array_equal(z1, z0), (precision, rel(z1, z0))
            assert np.array_equal(z2, z0), (precision, rel(z2, z0))
    few.close()
    opts = dict(rtol=1e-12, maxit=400)
    if not unit:
        opts.update(algorithm=hfps_mod.FGMRES, restart=12)
    for precision in (hfps_mod.FP64, hfps_mod.MIXED):
        x0, i0 = plain.solve(s.rhs, precision=precision, **opts)
        x1, i1 = tail.solve(s.rhs, precision=precision, **opts)
        assert i0["termination"] == i1["termination"] == "converged"
        assert i0["iterations"] == i1["iterations"]
        assert np.array_equal(x1, x0)
    # the persistent launch replaces many kernels per MG application
    _, a = plain.solve(s.rhs, rtol=1e-8, maxit=400, precision=hfps_mod.FP64, **(
        {} if unit else dict(algorithm=hfps_mod.FGMRES, restart=12)))
    _, b = tail.solve(s.rhs, rtol=1e-8, maxit=400, precision=hfps_mod.FP64, **(
        {} if unit else dict(algorithm=hfps_mod.FGMRES, restart=12)))
    assert b["kernel_launches"] < a["kernel_launches"]
    plain.close()
    tail.close()


def test_barrier_timeout_reports_failure(hfps_mod):
    """HFPS_TAIL_BARRIER_TEST=1 sets every launch's first barrier target one
    arrival beyond the grid, so its bounded wait runs out (under a second):
    the kernel records flag bit 3 and returns, and the solve fails with
    numerical_failure naming the barrier.  The GPU stays usable: a solver
    made afterwards in the same process solves normally."""
    import time
    s = CASES["y_lines_96x128x64"]()
    policy = hfps_mod.Policy.production()
    saved = os.environ.get("HFPS_TAIL_BARRIER_TEST")
    os.environ["HFPS_TAIL_BARRIER_TEST"] = "1"
    try:
        stalled = make_solver(hfps_mod, s, policy, tail=True)
    finally:
        if saved is None:
            os.environ.pop("HFPS_TAIL_BARRIER_TEST", None)
        else:
            os.environ["HFPS_TAIL_BARRIER_TEST"] = saved
    t0 = time.perf_counter()
    with pytest.raises(hfps_mod.SolverError) as err:
        stalled.solve(s.rhs, rtol=1e-10, maxit=50)
    assert time.perf_counter() - t0 < 60.0
    assert "grid barrier timed out" in str(err.value)
    stalled.close()
    fresh = make_solver(hfps_mod, s, policy, tail=True)
    x, info = fresh.solve(s.rhs, rtol=1e-10, maxit=400)
    assert info["termination"] == "converged"
    plain = make_solver(hfps_mod, s, policy, tail=False)
    y, _ = plain.solve(s.rhs, rtol=1e-10, maxit=400)
    assert np.array_equal(x, y)
    fresh.close()
    plain.close()
