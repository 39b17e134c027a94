"""The Krylov operator over 3-D tiles (k_stencil_tiled: A p with p.Ap)
against the row-walking kernel (HFPS_TILED_STENCIL=0, read when the solver
is created).
Rows are evaluated in the same order, so only the grouping of the
reduction partials differs: PCG and FGMRES solves take the same iteration
count (+-1) and agree to 1e-10, on even and ragged extents (partial tiles in
x, y and z), Dirichlet and Neumann faces."""
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
    "sphere_64": lambda: workloads.make("sphere64"),
    "sphere_ragged_45x37x70": lambda: workloads.make("sphere64", n=(45, 37, 70)),
    "wrinkled_96x128x64": lambda: workloads.make("wrinkled256", n=(96, 128, 64)),
}


def solve(hfps, s, tiled, **opts):
    saved = os.environ.get("HFPS_TILED_STENCIL")
    os.environ["HFPS_TILED_STENCIL"] = "1" if tiled else "0"
    try:
        g = hfps.PressureSolver.from_system(s, hfps.Policy.production().replace(
            unit_linear=0 if opts.get("algorithm") else 1))
        x, info = g.solve(s.rhs, **opts)
        g.close()
        return x, info
    finally:
        if saved is None:
            os.environ.pop("HFPS_TILED_STENCIL", None)
        else:
            os.environ["HFPS_TILED_STENCIL"] = saved


@pytest.mark.parametrize("case", sorted(CASES))
@pytest.mark.parametrize("fgmres", [False, True])
def test_tiled_stencil_matches_rows(hfps_mod, case, fgmres):
    s = CASES[case]()
    opts = dict(rtol=1e-12, maxit=400)
    if fgmres:
        opts.update(algorithm=hfps_mod.FGMRES, restart=12)
    x0, i0 = solve(hfps_mod, s, False, **opts)
    x1, i1 = solve(hfps_mod, s, True, **opts)
    assert i0["termination"] == i1["termination"] == "converged"
    assert abs(i0["iterations"] - i1["iterations"]) <= 1
    assert np.linalg.norm(x1 - x0) <= 1e-10 * np.linalg.norm(x0)
    assert abs(i0["initial_true_residual"] - i1["initial_true_residual"]) <= \
        1e-13 * i0["initial_true_residual"]
