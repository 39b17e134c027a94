"""The steps either side of the solve pinned to the reference's own code.

tests/golden/pressure_steps.* hold what the reference returned (oracle/_ref/
libhfps_ref_steps.so, recorded by tests/golden/make_golden.py --steps) for
face_pressure_coefficient (src/solver_piso.cpp:1060-1136),
assemble_pressure_system_impl (src/solver_pressure.cpp:110-332) and
PressureCorrectionBoundaryPlan::mass_flux_response (src/solver_piso.cpp:
1642-1653) on a y-stretched wrinkled-flame grid and a uniform sphere grid,
Dirichlet on x-max and Neumann elsewhere.  The reference's runtime-axes
geometry rounds face coordinates to binary32 (src/mesh_cartesian.cpp:
344-352), so the cases use binary32-representable coordinates.

The restatement (oracle/pressure_steps.py) reproduces every array bit for
bit, and so does the live reference where its library is built.
"""
import json
import os

import numpy as np
import pytest

import golden_cases

NAMES = sorted(golden_cases.STEPS_CASES)


def _recorded(name):
    with open(os.path.join(golden_cases.GOLDEN, "pressure_steps.json")) as f:
        return json.load(f)[name]


@pytest.mark.parametrize("name", NAMES)
def test_restatement_matches_reference_record(name):
    import pressure_steps
    s, faces = golden_cases.steps_system(name)
    assert golden_cases.digest(s) == _recorded(name)["digest"]
    ref = golden_cases.steps_arrays()
    coefficients = pressure_steps.face_coefficients(s.beta, faces, s.boundary)
    for axis, c in zip("xyz", coefficients):
        assert np.array_equal(c, ref[f"{name}_face_{axis}"]), axis
    inp = golden_cases.steps_inputs(s, 4)
    for tag, (a0, a1, a2, bdf2) in golden_cases.STEPS_BDF.items():
        diag, rhs = pressure_steps.assemble(
            faces, *coefficients, a0, a1, a2, inp["rho"], inp["rho_n"], inp["drho_dp"],
            *inp["fluxes"], rho_nm1=inp["rho_nm1"] if bdf2 else None,
            mass_source=inp["mass_source"] if bdf2 else None)
        assert np.array_equal(diag, ref[f"{name}_{tag}_diag"]), tag
        assert np.array_equal(rhs, ref[f"{name}_{tag}_rhs"]), tag
    for scale in golden_cases.STEPS_SCALES:
        q = pressure_steps.correct_flux(inp["correction"], coefficients, inp["fluxes"],
                                        s.boundary, scale)
        for axis, f in zip("xyz", q):
            assert np.array_equal(f, ref[f"{name}_flux_{scale}_{axis}"]), (scale, axis)


@pytest.mark.parametrize("name", NAMES)
def test_live_reference_reproduces_record(name):
    import ref_oracle
    if not ref_oracle.steps_available():
        pytest.skip("oracle/_ref/libhfps_ref_steps.so is not built in this tree")
    s, faces = golden_cases.steps_system(name)
    ref = golden_cases.steps_arrays()
    live = ref_oracle.RefSteps(s.shape, faces, s.boundary)
    coefficients = live.face_coefficients(s.beta)
    for axis, c in zip("xyz", coefficients):
        assert np.array_equal(c, ref[f"{name}_face_{axis}"])
    # the geometry the reference's steps read is the binary32 mesh as given
    import pressure_steps
    for axis in range(3):
        f, c, w = live.axis_metrics(axis)
        cm, wm = pressure_steps.axis_metrics(faces[axis])
        assert np.array_equal(f, faces[axis]) and np.array_equal(c, cm) and np.array_equal(w, wm)


def test_reference_rounds_runtime_faces_to_binary32():
    """Why the cases use binary32 coordinates: given double coordinates the
    reference's geometry holds their binary32 roundings."""
    import ref_oracle
    if not ref_oracle.steps_available():
        pytest.skip("oracle/_ref/libhfps_ref_steps.so is not built in this tree")
    from hfps import workloads
    s = workloads.make("wrinkled256", n=(12, 10, 8), stretch_y=1.1)
    import ctypes
    lib = ref_oracle._steps_lib()
    nx, ny, nz = s.shape
    bc = (ctypes.c_int * 6)(*s.boundary)
    dp = ctypes.POINTER(ctypes.c_double)
    f, c, w = np.zeros(nx + 1), np.zeros(nx), np.zeros(nx)
    rc = lib.hfref_axis_metrics(nx, ny, nz, *(a.ctypes.data_as(dp) for a in s.faces), bc, 0,
                                f.ctypes.data_as(dp), c.ctypes.data_as(dp), w.ctypes.data_as(dp))
    assert rc == 0
    assert not np.array_equal(f, s.faces[0])
    assert np.array_equal(f, s.faces[0].astype(np.float32).astype(np.float64))
