"""hfps_operator_dot_noalloc against the solver's own operator entry point.

The allocation-free entry point takes device arrays the caller owns and keeps
its reduction scratch in a fixed device array inside the library.  Two calls
in a row on the same device must each give the y = A x that
hfps_apply_operator gives for the same coefficients (bit-identical rows:
same arithmetic order, FMA contraction off) and x.(A x) to 1e-12 relative.
The second call must leave the device's free memory unchanged: the first
call has already loaded the module and looked up the scratch address, so
nothing is left that could allocate.  The file is named to be collected
last, so it also runs after every other GPU test in the same process.
"""
import ctypes

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


def device_view(system, arrays):
    from hfps import solver as binding
    v = binding.OperatorView()
    v.nx, v.ny, v.nz = system.shape
    for f in range(6):
        v.boundary[f] = int(system.boundary[f])
    v.diagonal, v.face_x, v.face_y, v.face_z = (a.data_ptr() for a in arrays)
    return v


def noalloc(view, x, y, dot):
    import torch
    from hfps import solver as binding
    stream = torch.cuda.current_stream().cuda_stream
    status = binding._lib().hfps_operator_dot_noalloc(
        ctypes.byref(view), ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr()),
        ctypes.c_void_p(dot.data_ptr() if dot is not None else None),
        ctypes.c_void_p(stream))
    torch.cuda.synchronize()
    return status


@pytest.mark.parametrize("shape", [(24, 20, 16), (80, 72, 64)])
def test_noalloc_matches_operator_twice(hfps_mod, shape):
    import torch
    s = workloads.make("sphere64", n=shape, seed=3)
    g = hfps_mod.PressureSolver.from_system(s, hfps_mod.Policy.production())
    diag, fx, fy, fz, _ = g.level_coefficients(0)
    arrays = [torch.from_numpy(np.ascontiguousarray(a).reshape(-1)).cuda()
              for a in (diag, fx, fy, fz)]
    view = device_view(s, arrays)
    rng = np.random.default_rng(17)
    n = int(np.prod(shape))
    for call in range(2):
        x = rng.standard_normal(n)
        expect = g.apply_operator(x.reshape(s.rhs.shape)).reshape(-1)
        xd = torch.from_numpy(x).cuda()
        yd = torch.full((n,), np.nan, dtype=torch.float64, device="cuda")
        dot = torch.full((1,), np.nan, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        assert noalloc(view, xd, yd, dot) == 0, call
        if call == 1:
            assert torch.cuda.mem_get_info()[0] == free_before
        y = yd.cpu().numpy()
        assert np.array_equal(y, expect), call
        want = float(np.dot(x, expect))
        assert abs(float(dot.item()) - want) <= 1e-12 * abs(want), call


def test_noalloc_rejects_bad_arguments(hfps_mod):
    """Host pointers, aliasing and periodic faces are refused before any
    launch; the entry point stays usable afterwards."""
    import torch
    s = workloads.make("sphere64", n=(12, 10, 8), seed=5)
    g = hfps_mod.PressureSolver.from_system(s, hfps_mod.Policy.production())
    diag, fx, fy, fz, _ = g.level_coefficients(0)
    arrays = [torch.from_numpy(np.ascontiguousarray(a).reshape(-1)).cuda()
              for a in (diag, fx, fy, fz)]
    view = device_view(s, arrays)
    n = diag.size
    xd = torch.ones(n, dtype=torch.float64, device="cuda")
    yd = torch.zeros(n, dtype=torch.float64, device="cuda")
    host = torch.zeros(n, dtype=torch.float64)
    assert noalloc(view, xd, host, None) == 2      # host output
    assert noalloc(view, xd, xd, None) == 2        # y aliases x
    assert noalloc(view, xd, yd, xd[3:4]) == 2     # dot written into x
    assert noalloc(view, xd, yd, yd[n - 1:]) == 2  # dot written into y
    view.boundary[0] = 2
    assert noalloc(view, xd, yd, None) == 2        # periodic
    view.boundary[0] = int(s.boundary[0])
    assert noalloc(view, xd, yd, None) == 0
    expect = g.apply_operator(np.ones(s.rhs.shape)).reshape(-1)
    assert np.array_equal(yd.cpu().numpy(), expect)
    assert torch.equal(xd, torch.ones(n, dtype=torch.float64, device="cuda"))
