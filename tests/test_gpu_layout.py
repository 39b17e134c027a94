"""Split-row layout of the MG vectors against the natural order.

On every level that relaxes y- or z-lines with the chunked scan, the MG x and
b are stored in split rows (each x-row's even-i cells, then its odd-i cells),
and the first pre-smoothing sweep of the finest level reads no x instead of
the MG entry clearing it; HFPS_SPLIT_ROWS=0 (read when the solver is created)
keeps the natural order everywhere.  Both perform the same operations on the
same values, so the MG application and whole solves must agree bit for bit:
FP64 and mixed, unit and residual-minimising corrections, even and odd nx
(the odd half of a split row then has a padding slot), y- and z-lines, one
and two split levels.
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


def z_stretched(n):
    """A wrinkled front on a grid stretched along z: z-line relaxation."""
    nx, ny, nz = n
    faces = (workloads.uniform_faces(nx), workloads.uniform_faces(ny),
             workloads.stretched_faces(nz, 1.03))
    z, y, x = workloads._grid(faces)
    front = (x - 0.4 - 0.05 * np.sin(8.0 * np.pi * y) * np.sin(8.0 * np.pi * z)) / 0.01
    rho = workloads._tanh_front(front) * np.ones((nz, ny, nx))
    solid = np.broadcast_to((x - 0.2) ** 2 + (z - 0.5) ** 2 <= 0.08 * 0.08, (nz, ny, nx)).copy()
    return workloads._build("z_stretched", faces, rho, solid, workloads.PISO_BOUNDARY, 0)


CASES = {
    "y_lines": lambda: workloads.make("wrinkled256", n=(96, 128, 64)),
    "y_lines_odd_nx": lambda: workloads.make("wrinkled256", n=(73, 150, 40)),
    # levels 0 and 1 both in split rows, odd nx and nz on level 0 and odd nz on
    # level 1: the 2x2 prolongation between split levels and at odd row ends
    "y_lines_two_split_levels": lambda: workloads.make("wrinkled256", n=(131, 160, 133)),
    "z_lines": lambda: z_stretched((64, 48, 96)),
}


def make_solver(hfps, system, policy, split):
    saved = os.environ.get("HFPS_SPLIT_ROWS")
    os.environ["HFPS_SPLIT_ROWS"] = "1" if split else "0"
    try:
        return hfps.PressureSolver.from_system(system, policy)
    finally:
        if saved is None:
            os.environ.pop("HFPS_SPLIT_ROWS", None)
        else:
            os.environ["HFPS_SPLIT_ROWS"] = saved


@pytest.mark.parametrize("case", sorted(CASES))
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("unit", [True, False])
def test_split_rows_bitwise(hfps_mod, case, precision, unit):
    s = CASES[case]()
    policy = hfps_mod.Policy.production().replace(unit_linear=1 if unit else 0)
    prec = hfps_mod.FP64 if precision == "fp64" else hfps_mod.MIXED
    natural = make_solver(hfps_mod, s, policy, split=False)
    split = make_solver(hfps_mod, s, policy, split=True)
    nx, ny, nz, mask = split.levels()[0]
    axis = {2: 1, 4: 2}.get(mask)
    assert axis is not None, "finest level must relax y- or z-lines"
    assert ((nx + 1) // 2) * (nz if axis == 1 else ny) >= 1024, "finest level must use the scan"
    rng = np.random.default_rng(3)
    r = rng.standard_normal(s.cells).reshape(s.rhs.shape)
    for _ in range(2):
        z0 = natural.apply_preconditioner(r, precision=prec)
        z1 = split.apply_preconditioner(r, precision=prec)
        assert np.array_equal(z0, z1)
    opts = dict(rtol=1e-10, precision=prec)
    if not unit:
        opts.update(algorithm=hfps_mod.FGMRES, restart=12)
    x0, i0 = natural.solve(s.rhs, **opts)
    x1, i1 = split.solve(s.rhs, **opts)
    assert i0["termination"] == i1["termination"] == "converged"
    assert i0["iterations"] == i1["iterations"]
    assert np.array_equal(x0, x1)
    natural.close()
    split.close()
