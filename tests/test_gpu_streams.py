"""Stream ordering of device-memory calls.

A caller that produces HFPS_DEVICE inputs on the legacy default stream (the
torch default stream, handle 0) creates the solver without a stream; the
solver's own stream must then be ordered after that work.  The test delays the
default stream with a bounded spin kernel before it writes the rhs and the
zero initial guess, so an unordered solver stream would read the stale
contents (a NaN-filled rhs, a previous solution as initial guess) and give a
different answer from the host-memory solve, which is the reference result.
"""
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


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_default_stream_inputs_are_ordered(hfps_mod, precision):
    import torch
    s = workloads.make("sphere64")
    prec = hfps_mod.FP64 if precision == "fp64" else hfps_mod.MIXED
    g = hfps_mod.PressureSolver.from_system(s, hfps_mod.Policy.production(),
                                            stream=torch.cuda.current_stream())
    expected, info = g.solve(s.rhs.reshape(-1).copy(), rtol=1e-10, precision=prec)
    source = torch.from_numpy(s.rhs.reshape(-1)).cuda()
    torch.cuda.synchronize()
    for _ in range(3):
        rhs = torch.full_like(source, float("nan"))
        stale = torch.full_like(source, 1.0e6)
        torch.cuda.synchronize()
        # About 20 ms of device time at 2 GHz, ahead of the writes below.
        torch.cuda._sleep(40_000_000)
        rhs.copy_(source)
        stale.zero_()
        x, xi = g.solve(rhs, x0=None, out=stale, rtol=1e-10, precision=prec)
        assert xi["termination"] == "converged"
        assert xi["iterations"] == info["iterations"]
        assert torch.equal(x.cpu(), torch.from_numpy(expected))
    g.close()


def test_explicit_stream_is_used(hfps_mod):
    import torch
    s = workloads.make("sphere64")
    side = torch.cuda.Stream()
    g = hfps_mod.PressureSolver.from_system(s, hfps_mod.Policy.production(), stream=side)
    expected, _ = g.solve(s.rhs.reshape(-1).copy(), rtol=1e-10)
    source = torch.from_numpy(s.rhs.reshape(-1)).cuda()
    torch.cuda.synchronize()
    with torch.cuda.stream(side):
        rhs = torch.full_like(source, float("nan"))
        torch.cuda._sleep(40_000_000)
        rhs.copy_(source)
        x, xi = g.solve(rhs, rtol=1e-10)
    assert xi["termination"] == "converged"
    side.synchronize()
    assert torch.equal(x.cpu(), torch.from_numpy(expected))
    g.close()
