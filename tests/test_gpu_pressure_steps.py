"""Pressure assembly and flux correction on the GPU against the restatement
(oracle/pressure_steps.py), bit for bit, through the C ABI.

The reference functions (assemble_pressure_system_impl,
src/solver_pressure.cpp:110-332; mass_flux_response,
src/solver_piso.cpp:1605-1653) are restated in the reference's operation
order, and the device kernels evaluate the same order with FMA contraction
off, so the float64 results agree exactly.  The face coefficients come from
beta by face_pressure_coefficient; the solver's level-0 coefficients of an
all-fluid system are exactly those faces.
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


def _inputs(s, seed, bdf2=False, source=False):
    rng = np.random.default_rng(seed)
    shape = s.rhs.shape
    d = {
        "density_trial": 1.0 + rng.random(shape),
        "density_accepted": 1.0 + rng.random(shape),
        "drho_dp": 0.2 + rng.random(shape),
        "fluxes": [rng.standard_normal(f.shape) for f in (s.face_x, s.face_y, s.face_z)],
    }
    if bdf2:
        d["density_previous"] = 1.0 + rng.random(shape)
    if source:
        d["mass_source"] = 0.1 * rng.standard_normal(shape)
    return d


@pytest.mark.parametrize("bdf2,source", [(False, False), (True, True)])
def test_assembly_matches_restatement_bitwise(hfps_mod, bdf2, source):
    import pressure_steps
    s = workloads.make("wrinkled256", n=(20, 28, 12), stretch_y=1.05, seed=9)
    g = hfps_mod.PressureSolver(s.shape, s.faces, s.boundary, None,
                                policy=hfps_mod.Policy.production())
    inp = _inputs(s, 4, bdf2, source)
    a0, a1, a2 = (1.5, -2.0, 0.5) if bdf2 else (1.0, -1.0, 0.0)
    rhs = g.assemble(np.ascontiguousarray(s.beta), inp["density_trial"], inp["density_accepted"],
                     inp["drho_dp"], inp["fluxes"], a0, a1, a2,
                     density_previous=inp.get("density_previous"),
                     mass_source=inp.get("mass_source"))
    diag, fx, fy, fz, _ = g.level_coefficients(0)
    ref_diag, ref_rhs = pressure_steps.assemble(
        s.faces, fx, fy, fz, a0, a1, a2, inp["density_trial"], inp["density_accepted"],
        inp["drho_dp"], *inp["fluxes"], rho_nm1=inp.get("density_previous"),
        mass_source=inp.get("mass_source"))
    assert np.array_equal(diag, ref_diag)
    assert np.array_equal(rhs, ref_rhs)
    # faces: face_pressure_coefficient of beta, as the host assembly forms them
    for a, b in zip((fx, fy, fz), (s.face_x, s.face_y, s.face_z)):
        assert np.max(np.abs(a - b)) <= 1e-14 * np.max(np.abs(b))
    # the assembled system solves
    x, info = g.solve(rhs, rtol=1e-11)
    assert info["termination"] == "converged"


def test_assembly_rejects_and_keeps_the_operator(hfps_mod):
    s = workloads.make("sphere64", n=(12, 10, 8), seed=3)
    g = hfps_mod.PressureSolver(s.shape, s.faces, s.boundary, s.active,
                                policy=hfps_mod.Policy.production())
    inp = _inputs(s, 5)
    g.assemble(np.ascontiguousarray(s.beta), inp["density_trial"], inp["density_accepted"],
               inp["drho_dp"], inp["fluxes"], 1.0, -1.0)
    before = g.level_coefficients(0)
    bad = inp["density_trial"].copy()
    bad.reshape(-1)[17] = -1.0
    with pytest.raises(hfps_mod.SolverError) as err:
        g.assemble(np.ascontiguousarray(s.beta), bad, inp["density_accepted"], inp["drho_dp"],
                   inp["fluxes"], 1.0, -1.0)
    assert err.value.status == 5
    for a, b in zip(before, g.level_coefficients(0)):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("scale", [1.0, 0.7])
def test_flux_correction_matches_restatement_bitwise(hfps_mod, scale):
    import pressure_steps
    s = workloads.make("sphere64", n=(14, 11, 9), seed=6)
    g = hfps_mod.PressureSolver.from_system(s, hfps_mod.Policy.production())
    rng = np.random.default_rng(8)
    p = rng.standard_normal(s.rhs.shape)
    coefficients = (s.face_x, s.face_y, s.face_z)
    fluxes = [rng.standard_normal(f.shape) for f in coefficients]
    expect = pressure_steps.correct_flux(p, coefficients, fluxes, s.boundary, scale)
    got = [f.copy() for f in fluxes]
    g.correct_flux(p, coefficients, got, scale)
    for a, b in zip(got, expect):
        assert np.array_equal(a, b)


def test_corrected_flux_closes_continuity(hfps_mod):
    """Assemble, solve, correct: the corrected fluxes' divergence balances
    the storage terms to the solve tolerance (the PISO corrector's purpose)."""
    import pressure_steps
    s = workloads.make("wrinkled256", n=(16, 24, 10), stretch_y=1.05, seed=2)
    g = hfps_mod.PressureSolver(s.shape, s.faces, s.boundary, None,
                                policy=hfps_mod.Policy.production())
    inp = _inputs(s, 7)
    rhs = g.assemble(np.ascontiguousarray(s.beta), inp["density_trial"],
                     inp["density_accepted"], inp["drho_dp"], inp["fluxes"], 1.0, -1.0)
    p, info = g.solve(rhs, rtol=1e-12)
    _, fx, fy, fz, _ = g.level_coefficients(0)
    q = [f.copy() for f in inp["fluxes"]]
    g.correct_flux(p, (fx, fy, fz), q)
    volume = pressure_steps.cell_volume(s.faces)
    storage = volume * inp["drho_dp"] * 1.0
    # continuity with the linearised density change: V (rho* - rho_n) + storage p + div q = 0
    residual = (volume * (inp["density_trial"] - inp["density_accepted"]) + storage * p +
                pressure_steps.outward_flux(*q))
    assert np.linalg.norm(residual) <= 1e-10 * np.linalg.norm(rhs)


# ---- pinned to the reference's own code (tests/golden/pressure_steps.*) ----
STEPS_NAMES = ["sphere_14x11x9", "wrinkled_20x28x12"]


@pytest.mark.parametrize("name", STEPS_NAMES)
def test_steps_match_reference_record(hfps_mod, name):
    """hfps_set_beta's faces, hfps_assemble's system and hfps_correct_flux's
    fluxes equal what the reference's face_pressure_coefficient,
    assemble_pressure_system_impl and mass_flux_response returned on the same
    binary32 mesh, bit for bit."""
    import golden_cases
    s, faces = golden_cases.steps_system(name)
    ref = golden_cases.steps_arrays()
    policy = hfps_mod.Policy.production()
    g = hfps_mod.PressureSolver(s.shape, faces, s.boundary, None, policy=policy)
    g.set_beta(np.ascontiguousarray(s.beta))
    _, fx, fy, fz, _ = g.level_coefficients(0)
    for axis, c in zip("xyz", (fx, fy, fz)):
        assert np.array_equal(c, ref[f"{name}_face_{axis}"]), axis
    inp = golden_cases.steps_inputs(s, 4)
    for tag, (a0, a1, a2, bdf2) in golden_cases.STEPS_BDF.items():
        rhs = g.assemble(np.ascontiguousarray(s.beta), inp["rho"], inp["rho_n"], inp["drho_dp"],
                         inp["fluxes"], a0, a1, a2,
                         density_previous=inp["rho_nm1"] if bdf2 else None,
                         mass_source=inp["mass_source"] if bdf2 else None)
        diag, *_ = g.level_coefficients(0)
        assert np.array_equal(diag, ref[f"{name}_{tag}_diag"]), tag
        assert np.array_equal(rhs, ref[f"{name}_{tag}_rhs"]), tag
    coefficients = tuple(ref[f"{name}_face_{axis}"] for axis in "xyz")
    for scale in golden_cases.STEPS_SCALES:
        q = [f.copy() for f in inp["fluxes"]]
        g.correct_flux(inp["correction"], coefficients, q, scale)
        for axis, f in zip("xyz", q):
            assert np.array_equal(f, ref[f"{name}_flux_{scale}_{axis}"]), (scale, axis)
    g.close()
