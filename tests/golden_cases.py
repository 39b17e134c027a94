"""Loader for the golden fixtures recorded from the compiled reference."""
import hashlib
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")


def index():
    with open(os.path.join(GOLDEN, "index.json")) as f:
        return json.load(f)


def system(name):
    from hfps import workloads
    spec = dict(index()[name]["spec"])
    cfg = spec.pop("config")
    if "n" in spec:
        spec["n"] = tuple(spec["n"])
    return workloads.make(cfg, **spec)


def policy(name):
    import ref_oracle
    return ref_oracle.MgPolicy(**index()[name]["policy"])


def arrays(name):
    return dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))


def probe(sys_):
    from hfps import workloads
    return np.ascontiguousarray(workloads.normals(99, sys_.cells).reshape(sys_.rhs.shape))


def digest(s):
    h = hashlib.sha256()
    for a in (s.diagonal, s.face_x, s.face_y, s.face_z, s.rhs, *s.faces):
        h.update(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    if s.active is not None:
        h.update(np.ascontiguousarray(s.active, dtype=np.uint8).tobytes())
    return h.hexdigest()


def anisotropic_x_system():
    """The line-relaxation fixture of tests/numerical/
    solver_mg_line_relaxation_test.cpp:33-44, 236-265: 64x12x8 uniform cells
    on [0, 0.05] x [0, 1] x [0, 1] (x strongly coupled), constant face
    coefficients 1/h^2 on every face, diagonal 2 (ax + ay + az), Dirichlet
    on all six sides, rhs the product of half-period sines."""
    from hfps import workloads
    nx, ny, nz = 64, 12, 8
    faces = (np.linspace(0.0, 0.05, nx + 1), np.linspace(0.0, 1.0, ny + 1),
             np.linspace(0.0, 1.0, nz + 1))
    ax, ay, az = (1.0 / (np.diff(f)[0] ** 2) for f in faces)
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    rhs = (np.sin(np.pi * (i + 0.5) / nx) * np.sin(np.pi * (j + 0.5) / ny)
           * np.sin(np.pi * (k + 0.5) / nz))
    return workloads.PressureSystem(
        "anisotropic_x", (nx, ny, nz), faces, (workloads.DIRICHLET,) * 6,
        np.ones((nz, ny, nx)), np.full((nz, ny, nx), 2.0 * (ax + ay + az)),
        np.full((nz, ny, nx + 1), ax), np.full((nz, ny + 1, nx), ay),
        np.full((nz + 1, ny, nx), az), None, np.ascontiguousarray(rhs))


def line_relaxation_policy(lines=True):
    """That test's MG spec: Chebyshev-Jacobi V(1,1), 16 coarse sweeps, at
    most 12 levels, anisotropy threshold 4.  Without lines the threshold is
    raised past any anisotropy, which also gives up semicoarsening (the
    reference test keeps the coarsening and clears only the line axes)."""
    import ref_oracle
    return ref_oracle.MgPolicy(smoother=1, cycle=0, pre=1, post=1, coarse_sweeps=16,
                               max_levels=12, anisotropy_threshold=4.0 if lines else 1e300)


# ---- steps either side of the solve (tests/golden/pressure_steps.*) -------
STEPS_CASES = {
    # name: workloads config and overrides
    "wrinkled_20x28x12": dict(config="wrinkled256", n=(20, 28, 12), stretch_y=1.05, seed=9),
    "sphere_14x11x9": dict(config="sphere64", n=(14, 11, 9), seed=6),
}


def steps_system(name):
    """The case's system with binary32-representable face coordinates (the
    reference's runtime-axes geometry rounds every coordinate to binary32)."""
    from hfps import workloads
    import ref_oracle
    spec = dict(STEPS_CASES[name])
    cfg = spec.pop("config")
    s = workloads.make(cfg, **spec)
    return s, ref_oracle.binary32_faces(s.faces)


def steps_inputs(s, seed):
    """Seeded cell states and face fluxes of one assembly / correction case."""
    rng = np.random.default_rng(seed)
    shape = s.rhs.shape
    return {
        "rho": 1.0 + rng.random(shape),
        "rho_n": 1.0 + rng.random(shape),
        "drho_dp": 0.2 + rng.random(shape),
        "rho_nm1": 1.0 + rng.random(shape),
        "mass_source": 0.1 * rng.standard_normal(shape),
        "fluxes": [rng.standard_normal(f.shape) for f in (s.face_x, s.face_y, s.face_z)],
        "correction": rng.standard_normal(shape),
    }


# (a0, a1, a2, BDF2 with a mass source)
STEPS_BDF = {"bdf1": (1.0, -1.0, 0.0, False), "bdf2_source": (1.5, -2.0, 0.5, True)}
STEPS_SCALES = (1.0, 0.7)


def steps_arrays():
    return dict(np.load(os.path.join(GOLDEN, "pressure_steps.npz")))


def null_space_index():
    with open(os.path.join(GOLDEN, "null_space.json")) as f:
        return json.load(f)


def null_space_system():
    """The pure-Neumann sphere of tests/golden/null_space.* (MgNullSpace::constant)."""
    from hfps import workloads
    spec = dict(null_space_index()["spec"])
    cfg = spec.pop("config")
    spec["n"] = tuple(spec["n"])
    spec["boundary"] = tuple(spec["boundary"])
    return workloads.make(cfg, **spec)
