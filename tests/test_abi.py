"""The C ABI surface: the library builds for sm_100a and exports exactly
what include/hf_pressure_solver.h declares.  No GPU compute is needed."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "hf_pressure_solver.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"HFPS_API\s+[\w\s\*]+?\b(hfps_\w+)\s*\(", text)))


def test_header_declares_the_entry_points():
    names = declared_symbols()
    for required in ("hfps_create", "hfps_set_coefficients", "hfps_solve", "hfps_adjoint",
                     "hfps_apply_operator", "hfps_apply_preconditioner", "hfps_destroy"):
        assert required in names


def test_library_exports_every_declared_symbol(cuda_library):
    lib = ctypes.CDLL(cuda_library)
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing
    from hfps import solver
    assert sorted(solver.EXPORTS) == declared_symbols()


def test_policies_follow_the_reference_defaults(cuda_library):
    from hfps import Policy
    d = Policy.default()
    assert (d.point_smoother, d.cycle, d.pre_sweeps, d.post_sweeps, d.coarse_sweeps) == (0, 0, 2, 2, 24)
    assert d.chebyshev_lower_spectrum_fraction == 0.3 and d.anisotropy_threshold == 4.0
    p = Policy.production()
    assert (p.point_smoother, p.cycle, p.pre_sweeps, p.post_sweeps) == (1, 1, 1, 2)
    assert p.diagonal_shortcut_maximum_ratio == 0.1 and p.unit_linear == 1


def test_invalid_plans_are_rejected_before_any_device_work(cuda_library):
    """Geometry/policy validation happens on the host and fails loudly."""
    import numpy as np
    from hfps import Policy, PressureSolver, SolverError
    faces = [np.linspace(0, 1, 5)] * 3
    with pytest.raises(SolverError, match="periodic boundaries are not supported"):
        PressureSolver((4, 4, 4), faces, (2, 2, 0, 0, 0, 0))
    with pytest.raises(SolverError, match="invalid geometry or policy"):
        PressureSolver((4, 4, 4), faces, (0,) * 6, policy=Policy.default().replace(pre_sweeps=0))
    with pytest.raises(SolverError, match="face coordinates must increase"):
        bad = [np.array([0, 0.5, 0.4, 0.8, 1.0])] * 3
        PressureSolver((4, 4, 4), bad, (0,) * 6)
    # the Chebyshev lower-spectrum fraction must lie strictly inside (0, 1)
    # (tests/unit/solver_mg_chebyshev_test.cpp:1237-1243)
    for fraction in (0.0, 1.0, float("nan")):
        with pytest.raises(SolverError, match="invalid geometry or policy"):
            PressureSolver((4, 4, 4), faces, (0,) * 6, policy=Policy.production().replace(
                chebyshev_lower_spectrum_fraction=fraction))
    # and the diagonal-shortcut ratio inside [0, 1)
    # (tests/unit/solver_mg_chebyshev_test.cpp:1307-1312)
    for ratio in (-0.1, 1.0, float("nan")):
        with pytest.raises(SolverError, match="invalid geometry or policy"):
            PressureSolver((4, 4, 4), faces, (0,) * 6, policy=Policy.production().replace(
                diagonal_shortcut_maximum_ratio=ratio))


def test_missing_gpu_fails_loudly(cuda_library):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import numpy as np
    from hfps import PressureSolver, SolverError
    faces = [np.linspace(0, 1, 9)] * 3
    with pytest.raises(SolverError):
        PressureSolver((8, 8, 8), faces, (0,) * 6)


def test_noalloc_rejects_oversize_grids_before_any_device_call(cuda_library):
    """Grids beyond HFPS_NOALLOC_MAX_CELLS (or with an empty extent) are
    refused from the sizes alone, before the entry point touches the GPU."""
    from hfps import solver as binding
    lib = binding._lib()
    v = binding.OperatorView()
    v.nx = v.ny = v.nz = 1100                      # 1.33e9 cells > 2**30
    assert lib.hfps_operator_dot_noalloc(ctypes.byref(v), None, None, None, None) == 1
    v.nx = 0
    assert lib.hfps_operator_dot_noalloc(ctypes.byref(v), None, None, None, None) == 1
    assert lib.hfps_operator_dot_noalloc(None, None, None, None, None) == 2
    header = open(HEADER).read()
    assert "#define HFPS_NOALLOC_MAX_CELLS (1LL << 30)" in header
