"""The larger configurations of the pressure path at full size, checked
through size-independent properties (the CPU oracle is too slow at these
sizes; the small-size parity tests pin the arithmetic).

* 512x256x256 wrinkled flame: the mixed-precision form (FP32 MG inside FP64
  PCG) reaches the FP64 tolerance, and its solution agrees with the plain
  FP64 GPU solve and, at 1e-13, with the compiled reference's FP64 solution
  (recorded sample); the refinement (outer Krylov) step counts are reported.
* 128^3 spherical flame, loss L = 0.5 sum_fluid (p - p_t)^2 with p_t from
  seed 7: adjoint gradients with respect to 200 face coefficients (seed 11)
  and to rhs agree with central finite differences of step 1e-6 |c| to 1e-6
  relative, in FP64 and in the mixed form.  A face coefficient change is a
  rank-one change of the operator, dA = dc u u^T (u = e_i - e_j inside,
  u = e_i on a Dirichlet face), so p(c +- h) = p - (+-h)(u.p) w / (1 +- h u.w)
  with w = A^-1 u exactly (Sherman-Morrison): the difference quotient is
  evaluated without re-solving the perturbed systems, whose solver noise
  would swamp a 1e-6 step.
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


def test_mixed_form_at_512x256x256(hfps_mod):
    import torch
    s = workloads.make("wrinkled512x256x256")
    g = hfps_mod.PressureSolver.from_system(s, hfps_mod.Policy.production())
    rhs = torch.from_numpy(s.rhs.reshape(-1)).cuda()
    x64, i64 = g.solve(rhs, rtol=1e-10, history=False)
    xm, im = g.solve(rhs, rtol=1e-10, precision=hfps_mod.MIXED, history=False)
    assert i64["termination"] == im["termination"] == "converged"
    assert im["final_true_residual"] <= 1e-10 * im["rhs_norm"]
    err = float(torch.linalg.vector_norm(xm - x64) / torch.linalg.vector_norm(x64))
    print(f"512x256x256: FP64 {i64['iterations']} iterations, mixed {im['iterations']} "
          f"refinement steps, mixed vs FP64 relative error {err:.3e}")
    assert err <= 1e-8
    assert abs(im["iterations"] - i64["iterations"]) <= max(2, int(0.2 * i64["iterations"]))
    # Final error against the FP64 oracle: the compiled reference's solve of
    # this system at 1e-13 (tests/golden/wrinkled512x256x256.*), on its
    # recorded sample of cells; the mixed form converged to the same FP64
    # true residual.
    import scale_cases
    entry = scale_cases.entry("wrinkled512x256x256")
    ref = scale_cases.arrays("wrinkled512x256x256")
    xr, ir = g.solve(rhs, rtol=1e-13, maxit=400, precision=hfps_mod.MIXED, history=False)
    assert ir["termination"] == "converged"
    oracle_err = scale_cases.sample_error(xr.cpu().numpy(), ref["pcg_step0_1e13"], ref["cells"])
    want = entry["pcg_step0_1e13"]["iterations"]
    print(f"512x256x256 mixed at 1e-13: {ir['iterations']} refinement steps (reference PCG "
          f"{want}), relative error vs the reference FP64 solution {oracle_err:.3e}")
    assert oracle_err <= 1e-9
    assert abs(ir["iterations"] - want) <= max(2, 0.2 * want)


def _face_vectors(s, axis, flat):
    """(cells, signs) of u for face `flat` on `axis`, or None for a face the
    operator does not see (Neumann boundary, IBM-removed)."""
    nx, ny, nz = s.shape
    shape = [(nz, ny, nx + 1), (nz, ny + 1, nx), (nz + 1, ny, nx)][axis]
    k, j, i = np.unravel_index(flat, shape)
    pos = [i, j, k][axis]
    ext = [nx, ny, nz][axis]
    hi = (k, j, i) if pos < ext else None
    lo_idx = [i, j, k]
    lo_idx[axis] -= 1
    lo = (lo_idx[2], lo_idx[1], lo_idx[0]) if pos > 0 else None
    act = s.active.astype(bool)
    if hi is not None and lo is not None:
        if not (act[hi] and act[lo]):
            return None
        return [(hi, 1.0), (lo, -1.0)]
    side = 2 * axis + (0 if lo is None else 1)
    if s.boundary[side] == 1:  # Neumann: the face does not enter the operator
        return None
    cell = hi if hi is not None else lo
    return [(cell, 1.0)] if act[cell] else None


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_adjoint_gradients_at_128(hfps_mod, precision):
    s = workloads.make("sphere128")
    g = hfps_mod.PressureSolver.from_system(s, hfps_mod.Policy.production())
    prec = hfps_mod.FP64 if precision == "fp64" else hfps_mod.MIXED
    p, info = g.solve(s.rhs, rtol=1e-13, maxit=800, precision=prec)
    target = workloads.normals(7, s.cells).reshape(s.rhs.shape)
    act = s.active.astype(bool)
    dl_dp = np.where(act, p - target, 0.0)
    lam, grads, ainfo = g.adjoint(p, dl_dp, rtol=1e-13, maxit=800, precision=prec)
    assert ainfo["termination"] == "converged"
    coefficients = (s.face_x, s.face_y, s.face_z)
    counts = [c.size for c in coefficients]
    rng = np.random.default_rng(11)
    picks = rng.choice(sum(counts), size=200, replace=False)
    adj, fd = [], []
    for flat in picks:
        axis = 0 if flat < counts[0] else (1 if flat < counts[0] + counts[1] else 2)
        local = flat - sum(counts[:axis])
        u_cells = _face_vectors(s, axis, local)
        grad = float(grads[axis].reshape(-1)[local])
        if u_cells is None:
            assert grad == 0.0
            continue
        c = float(coefficients[axis].reshape(-1)[local])
        h = 1e-6 * abs(c)
        u = np.zeros_like(s.rhs)
        for cell, sign in u_cells:
            u[cell] = sign
        w, winfo = g.solve(u, rtol=1e-13, maxit=800)
        up, uw = float(np.sum(u * p)), float(np.sum(u * w))
        deltas = []
        for sign in (1.0, -1.0):
            d = -(sign * h) * up / (1.0 + sign * h * uw) * w
            deltas.append(float(np.sum(dl_dp * d) + 0.5 * np.sum(np.where(act, d * d, 0.0))))
        fd.append((deltas[0] - deltas[1]) / (2.0 * h))
        adj.append(grad)
    adj, fd = np.array(adj), np.array(fd)
    assert len(adj) >= 150
    err = np.linalg.norm(adj - fd) / np.linalg.norm(fd)
    print(f"128^3 {precision}: {len(adj)} faces, adjoint vs finite differences {err:.3e}")
    assert err <= 1e-6
    # rhs gradient: dL/db = lambda; the difference quotient along e_k is w.dl_dp
    for k in rng.choice(s.cells, size=8, replace=False):
        e = np.zeros(s.cells)
        e[k] = 1.0
        w, _ = g.solve(e.reshape(s.rhs.shape), rtol=1e-13, maxit=800)
        fd_k = float(np.sum(dl_dp * w))
        assert abs(float(lam.reshape(-1)[k]) - fd_k) <= 1e-6 * float(np.abs(lam).max())


def test_three_spheres512_forward_adjoint_steps(hfps_mod):
    """512^3 three-sphere flame (134M cells): the first two steps of the
    warm-started sequence, each a mixed forward solve followed by a mixed
    adjoint solve of L = 0.5 sum_fluid (p - p_t)^2 (p_t from seed 7).  The
    last step is repeated in plain FP64 from the same warm start: forward
    solutions, adjoint states and face gradients of the two forms agree."""
    import torch
    s = workloads.make("three_spheres512")
    g = hfps_mod.PressureSolver.from_system(s, hfps_mod.Policy.production())
    n = s.cells
    rhs0 = torch.from_numpy(s.rhs.reshape(-1)).cuda()
    active = torch.from_numpy(s.active.reshape(-1).astype(np.bool_)).cuda()
    target = workloads.normals_torch(7, n)
    mixed = hfps_mod.SolveOptions(rtol=1e-10, maxit=400, precision=hfps_mod.MIXED)
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    start, mid, stop = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    for step in range(2):
        rhs = rhs0 + workloads.flux_divergence_rhs_torch(1 + step, s.faces, s.boundary,
                                                         s.active, 0.05)
        x_start = x.clone()
        torch.cuda.synchronize()
        start.record()
        x, info = g.solve(rhs, x0=x, out=x, options=mixed, history=False)
        mid.record()
        dl_dp = torch.where(active, x - target, torch.zeros_like(x))
        lam, grads, ainfo = g.adjoint(x, dl_dp, options=mixed)
        stop.record()
        torch.cuda.synchronize()
        assert info["termination"] == ainfo["termination"] == "converged"
        assert info["final_true_residual"] <= 1e-10 * info["rhs_norm"]
        print(f"512^3 step {step + 1}: mixed forward {start.elapsed_time(mid):.1f} ms "
              f"({info['iterations']} iterations), adjoint {mid.elapsed_time(stop):.1f} ms "
              f"({ainfo['iterations']} iterations)")
    x64, i64 = g.solve(rhs, x0=x_start, rtol=1e-10, maxit=400, history=False)
    lam64, grads64, _ = g.adjoint(x, dl_dp, rtol=1e-10, maxit=400)

    def rel(a, b):
        return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))

    forward = rel(x, x64)
    adjoint = rel(lam, lam64)
    faces = max(rel(a, b) for a, b in zip(grads, grads64))
    print(f"512^3: FP64 forward {i64['iterations']} iterations; mixed vs FP64: solution "
          f"{forward:.2e}, lambda {adjoint:.2e}, face gradients {faces:.2e}")
    assert forward <= 1e-8 and adjoint <= 1e-8 and faces <= 1e-8
