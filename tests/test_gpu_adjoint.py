"""Adjoint path: gradients of L = 0.5 sum_fluid (p - p_t)^2 with respect to
rhs and every face coefficient, checked against central finite differences
(step 1e-6 |c|) and an FP64 direct-solve reference gradient, relative
tolerance 1e-6.  The system is the spherical-flame case at reduced size."""
import numpy as np
import pytest

from hfps import workloads

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup(cuda_library):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    import hfps
    s = workloads.make("sphere64", n=(14, 12, 10), spheres=((0.35, 0.5, 0.5, 0.2),))
    target = workloads.normals(7, s.cells).reshape(s.rhs.shape)
    g = hfps.PressureSolver.from_system(s, hfps.Policy.production())
    return hfps, s, target, g


def loss(s, p, target):
    m = s.active.astype(bool)
    return 0.5 * float(np.sum((p[m] - target[m]) ** 2))


def assemble(s, fx, fy, fz):
    """Sparse FP64 matrix of the IBM-masked operator for face coefficients
    fx, fy, fz (unmasked input, diagonal = sum of the six faces)."""
    import scipy.sparse as sp
    nx, ny, nz = s.shape
    act = s.active.astype(bool)
    ax = np.ones((nz, ny, nx + 1), bool)
    ax[:, :, :-1] &= act
    ax[:, :, 1:] &= act
    ay = np.ones((nz, ny + 1, nx), bool)
    ay[:, :-1, :] &= act
    ay[:, 1:, :] &= act
    az = np.ones((nz + 1, ny, nx), bool)
    az[:-1, :, :] &= act
    az[1:, :, :] &= act
    mx, my, mz = fx * ax, fy * ay, fz * az
    idx = np.arange(s.cells).reshape(nz, ny, nx)
    diag = (mx[:, :, :-1] + mx[:, :, 1:] + my[:, :-1, :] + my[:, 1:, :] + mz[:-1, :, :]
            + mz[1:, :, :])
    rows, cols, vals = [], [], []
    for (lo, hi, c) in ((idx[:, :, :-1], idx[:, :, 1:], mx[:, :, 1:-1]),
                        (idx[:, :-1, :], idx[:, 1:, :], my[:, 1:-1, :]),
                        (idx[:-1, :, :], idx[1:, :, :], mz[1:-1, :, :])):
        rows += [lo.ravel(), hi.ravel()]
        cols += [hi.ravel(), lo.ravel()]
        vals += [-c.ravel(), -c.ravel()]
    # A Neumann boundary face couples its cell to itself (D x - c x): it
    # leaves the row unchanged, so it is taken back out of the diagonal.
    nb = s.boundary
    bterm = np.zeros((nz, ny, nx))
    if nb[0] == 1: bterm[:, :, 0] += mx[:, :, 0]
    if nb[1] == 1: bterm[:, :, -1] += mx[:, :, -1]
    if nb[2] == 1: bterm[:, 0, :] += my[:, 0, :]
    if nb[3] == 1: bterm[:, -1, :] += my[:, -1, :]
    if nb[4] == 1: bterm[0, :, :] += mz[0, :, :]
    if nb[5] == 1: bterm[-1, :, :] += mz[-1, :, :]
    d = np.where(act, diag - bterm, 1.0)
    rows.append(idx.ravel())
    cols.append(idx.ravel())
    vals.append(d.ravel())
    A = sp.csc_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(s.cells, s.cells))
    return A


def solve_extended(A, b):
    """FP64 LU with iterative refinement whose residuals are formed in long
    double, so that p(c+h) - p(c-h) keeps its digits at h = 1e-6 |c|."""
    import scipy.sparse.linalg as spla
    coo = A.tocoo()
    vals = coo.data.astype(np.longdouble)
    lu = spla.splu(A.tocsc())
    bl = b.astype(np.longdouble)
    x = lu.solve(b).astype(np.longdouble)
    for _ in range(4):
        ax = np.zeros_like(bl)
        np.add.at(ax, coo.row, vals * x[coo.col])
        x = x + lu.solve((bl - ax).astype(np.float64)).astype(np.longdouble)
    return x


def central_difference(s, target, solve_plus, solve_minus, h):
    """dL/dh from p(+h), p(-h) in long double: L+ - L- = 0.5 sum (p+ - p-)
    (p+ + p- - 2 t), which avoids the cancellation of L itself."""
    m = s.active.astype(bool).reshape(-1)
    t = target.reshape(-1).astype(np.longdouble)
    pp, pm = solve_plus, solve_minus
    return float(0.5 * np.sum((pp[m] - pm[m]) * (pp[m] + pm[m] - 2 * t[m])) / h)


def test_assembled_matrix_matches_gpu_operator(setup):
    hfps, s, target, g = setup
    g.set_coefficients(s.diagonal, s.face_x, s.face_y, s.face_z)
    v = np.random.default_rng(3).standard_normal(s.rhs.shape)
    A = assemble(s, s.face_x, s.face_y, s.face_z)
    y = g.apply_operator(v)
    assert np.max(np.abs(A @ v.reshape(-1) - y.reshape(-1))) <= 1e-14 * np.max(np.abs(y))


def test_adjoint_matches_finite_differences(setup):
    """Central differences with step 1e-6 |c| (faces) and 1e-6 max(1,|b|)
    (rhs) against the GPU adjoint gradient, relative tolerance 1e-6.  The
    perturbed systems are solved directly with extended-precision
    refinement: plain FP64 solves carry ~1e-12 relative error, which a
    1e-6 step would amplify to ~1e-6 in the difference quotient."""
    hfps, s, target, g = setup
    fx, fy, fz = s.face_x.copy(), s.face_y.copy(), s.face_z.copy()
    g.set_coefficients(s.diagonal, fx, fy, fz)
    p, _ = g.solve(s.rhs, rtol=1e-14, maxit=400, history=False)
    dl_dp = np.ascontiguousarray((p - target) * s.active)
    lam, (gx, gy, gz), info = g.adjoint(p, dl_dp, rtol=1e-14, maxit=400)
    assert info["termination"] == "converged"
    grads = [gx.reshape(fx.shape), gy.reshape(fy.shape), gz.reshape(fz.shape)]
    rng = np.random.default_rng(11)
    faces = [fx, fy, fz]
    b = s.rhs.reshape(-1)
    checked = 0
    for _ in range(80):
        axis = int(rng.integers(3))
        flat = int(rng.integers(faces[axis].size))
        c0 = faces[axis].reshape(-1)[flat]
        if c0 == 0.0:
            continue
        sols, steps = [], []
        for sign in (1.0, -1.0):
            pert = [f.copy() for f in faces]
            pert[axis].reshape(-1)[flat] = c0 + sign * 1e-6 * abs(c0)
            steps.append(np.longdouble(pert[axis].reshape(-1)[flat]) - np.longdouble(c0))
            sols.append(solve_extended(assemble(s, *pert), b))
        fd = central_difference(s, target, sols[0], sols[1], steps[0] - steps[1])
        an = grads[axis].reshape(-1)[flat]
        scale = max(abs(fd), abs(an), 1e-6 * np.max(np.abs(grads[axis])))
        assert abs(fd - an) <= 1e-6 * scale, (axis, flat, fd, an)
        checked += 1
    assert checked > 30
    A = assemble(s, fx, fy, fz)
    for cell in rng.integers(s.cells, size=10):
        if s.active.reshape(-1)[cell] == 0:
            continue
        sols, steps = [], []
        for sign in (1.0, -1.0):
            bp = b.copy()
            bp[cell] += sign * 1e-6 * max(1.0, abs(b[cell]))
            steps.append(np.longdouble(bp[cell]) - np.longdouble(b[cell]))
            sols.append(solve_extended(A, bp))
        fd = central_difference(s, target, sols[0], sols[1], steps[0] - steps[1])
        an = lam.reshape(-1)[cell]
        assert abs(fd - an) <= 1e-6 * max(abs(fd), abs(an)) + 1e-12


def test_adjoint_matches_direct_reference_gradient(setup):
    """FP64 reference gradient from a sparse direct solve of A^T lambda = g."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    hfps, s, target, g = setup
    g.set_coefficients(s.diagonal, s.face_x, s.face_y, s.face_z)
    n = s.cells
    cols = [sp.csc_matrix(g.apply_operator(np.eye(1, n, c).reshape(s.rhs.shape)).reshape(-1, 1))
            for c in range(n)]
    A = sp.hstack(cols).tocsc()
    p_ref = spla.spsolve(A, s.rhs.reshape(-1))
    gvec = (p_ref - target.reshape(-1)) * s.active.reshape(-1)
    lam_ref = spla.spsolve(A.T.tocsc(), gvec)
    p, _ = g.solve(s.rhs, rtol=1e-14, history=False)
    lam, (gx, _, _), info = g.adjoint(p, np.ascontiguousarray((p - target) * s.active), rtol=1e-14)
    assert np.linalg.norm(lam.reshape(-1) - lam_ref) <= 1e-9 * np.linalg.norm(lam_ref)
    nx, ny, nz = s.shape
    act = s.active.astype(bool)
    P = p_ref.reshape(nz, ny, nx)
    Lr = lam_ref.reshape(nz, ny, nx)
    ref_gx = np.zeros((nz, ny, nx + 1))
    both = act[:, :, :-1] & act[:, :, 1:]
    ref_gx[:, :, 1:-1] = np.where(both, -(Lr[:, :, :-1] - Lr[:, :, 1:]) * (P[:, :, :-1] - P[:, :, 1:]), 0.0)
    ref_gx[:, :, -1] = np.where(act[:, :, -1], -Lr[:, :, -1] * P[:, :, -1], 0.0)  # Dirichlet x-max
    assert np.linalg.norm(gx.reshape(ref_gx.shape) - ref_gx) <= 1e-8 * np.linalg.norm(ref_gx)


def test_autograd_function_backward(setup):
    import torch
    from hfps.autograd import pressure_solve
    hfps, s, target, g = setup
    dev = torch.device("cuda")
    rhs = torch.tensor(s.rhs.reshape(-1), device=dev, requires_grad=True)
    fx = torch.tensor(s.face_x.reshape(-1), device=dev, requires_grad=True)
    fy = torch.tensor(s.face_y.reshape(-1), device=dev, requires_grad=True)
    fz = torch.tensor(s.face_z.reshape(-1), device=dev, requires_grad=True)
    p = pressure_solve(g, rhs, fx, fy, fz)
    m = torch.tensor(s.active.reshape(-1), device=dev, dtype=torch.float64)
    t = torch.tensor(target.reshape(-1), device=dev)
    L = 0.5 * torch.sum(m * (p - t) ** 2)
    L.backward()
    lam, (gx, gy, gz), _ = g.adjoint(p.detach(), (m * (p - t)).detach().contiguous(), rtol=1e-13)
    assert torch.allclose(rhs.grad, lam, rtol=1e-12, atol=0)
    assert torch.allclose(fx.grad, gx, rtol=1e-12, atol=0)
