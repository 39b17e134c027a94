"""The C++ torch extension of the differentiable pressure solve
(hundun-flow_b200/csrc/torch_autograd.cpp, built in-tree by
hundun-flow_b200/build.py) against the Python autograd.Function
(hfps/autograd.py): both call hfps_set_coefficients / hfps_solve forward and
hfps_adjoint backward on the same handle with the same diagonal assembly,
so p and every gradient (rhs, the three face arrays, storage) agree bit for
bit; and the extension's face gradients match central finite differences
of the loss on a few faces."""
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


def _inputs(s, torch):
    dev = "cuda"
    rhs = torch.tensor(s.rhs.reshape(-1), device=dev, requires_grad=True)
    faces = [torch.tensor(f.reshape(-1), device=dev, requires_grad=True)
             for f in (s.face_x, s.face_y, s.face_z)]
    rng = np.random.default_rng(3)
    storage = torch.tensor(0.05 + 0.1 * rng.random(s.cells), device=dev, requires_grad=True)
    target = torch.tensor(workloads.normals(7, s.cells), device=dev)
    return rhs, faces, storage, target


def test_cpp_extension_matches_python_autograd(hfps_mod):
    import torch
    import build
    from hfps.autograd import pressure_solve
    ext = build.build_torch_extension()
    s = workloads.make("sphere64", n=(16, 12, 10), seed=4)
    solver = hfps_mod.PressureSolver(s.shape, s.faces, s.boundary, s.active,
                                     policy=hfps_mod.Policy.production())
    active = solver.active_tensor("cuda")
    opts = hfps_mod.SolveOptions(rtol=1e-13, maxit=400, precision=hfps_mod.FP64)
    results = []
    for use_ext in (False, True):
        rhs, faces, storage, target = _inputs(s, torch)
        if use_ext:
            p = ext.pressure_solve(solver._handle.value, list(s.shape), opts.rtol, opts.maxit,
                                   opts.precision, rhs, *faces, storage, active)
        else:
            p = pressure_solve(solver, rhs, *faces, storage, options=opts)
        loss = 0.5 * torch.sum(active * (p - target) ** 2)
        loss.backward()
        results.append([p.detach(), rhs.grad, *(f.grad for f in faces), storage.grad])
    for a, b in zip(*results):
        assert torch.equal(a, b)
    # finite differences of the loss on a few interior x-faces (the solve is
    # re-run at rtol 1e-13 for c +- h; h = 1e-4 |c| keeps solver noise small)
    rhs, faces, storage, target = _inputs(s, torch)
    grad_x = results[1][2]
    fx = faces[0].detach()
    nx, ny, nz = s.shape
    picks = [int(i) for i in np.flatnonzero(s.face_x.reshape(-1) > 0)[::97][:4]]

    def loss_at(values):
        with torch.no_grad():
            p = ext.pressure_solve(solver._handle.value, list(s.shape), opts.rtol, opts.maxit,
                                   opts.precision, rhs.detach(), values, faces[1].detach(),
                                   faces[2].detach(), storage.detach(), active)
            return float(0.5 * torch.sum(active * (p - target) ** 2))

    for f in picks:
        h = 1e-4 * float(fx[f])
        up, down = fx.clone(), fx.clone()
        up[f] += h
        down[f] -= h
        fd = (loss_at(up) - loss_at(down)) / (2.0 * h)
        assert abs(float(grad_x[f]) - fd) <= 1e-5 * max(abs(fd), 1e-12), (f, float(grad_x[f]), fd)
    solver.close()
