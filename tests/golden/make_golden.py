"""Generates the golden fixtures in tests/golden/ from the compiled reference.

Run in a tree where the reference sources are present:

    make -C oracle ref && python tests/golden/make_golden.py

For each small case the script builds the seeded system with
hfps.workloads, then records what the reference's own code returns for it
(oracle/_ref: NativeCartesianMgPlan::apply, the IBM-decorated operator,
solve_pcg with the unit-scaled MG plan and solve_fgmres(12) with the
residual-minimising one): the MG correction of a seeded vector, the operator
action, and the solutions/iteration counts at rtol 1e-13.  A checksum
of the inputs pins the generator, so a changed generator fails the tests
instead of silently comparing different systems.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "hundun-flow_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from hfps import workloads  # noqa: E402
import ref_oracle  # noqa: E402

CASES = {
    # name: (builder kwargs, policy kwargs)
    "sphere_24x20x16_rbV22": (dict(config="sphere64", n=(24, 20, 16)), dict()),
    "sphere_24x20x16_prodF": (dict(config="sphere64", n=(24, 20, 16)),
                              dict(smoother=1, cycle=1, pre=1, post=2, diagonal_shortcut=0.1)),
    "sphere_33x17x9_rbF22": (dict(config="sphere64", n=(33, 17, 9)), dict(cycle=1)),
    "wrinkled_16x40x12_lineF": (dict(config="wrinkled256", n=(16, 40, 12), stretch_y=1.1),
                                dict(smoother=1, cycle=1, pre=1, post=2)),
}


def system_for(spec):
    spec = dict(spec)
    name = spec.pop("config")
    return workloads.make(name, **spec)


def input_digest(system) -> str:
    h = hashlib.sha256()
    for a in (system.diagonal, system.face_x, system.face_y, system.face_z, system.rhs,
              *system.faces):
        h.update(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    if system.active is not None:
        h.update(np.ascontiguousarray(system.active, dtype=np.uint8).tobytes())
    return h.hexdigest()


def probe_vector(system, seed=99):
    return np.ascontiguousarray(
        workloads.normals(seed, system.cells).reshape(system.rhs.shape))


def main():
    if not ref_oracle.available():
        raise SystemExit("build oracle/_ref first: make -C oracle ref")
    index = {}
    for name, (spec, pol) in CASES.items():
        system = system_for(spec)
        policy = ref_oracle.MgPolicy(**pol)
        ref = ref_oracle.RefSession(system, policy, algorithm="pcg")
        v = probe_vector(system)
        mg = ref.apply_mg(v)
        op = ref.apply_operator(v)
        x, info = ref.solve(system.rhs, rtol=1e-13, maxit=400)
        x10, info10 = ref.solve(system.rhs, rtol=1e-10, maxit=400)
        levels = ref.levels()
        ref.close()
        fg = ref_oracle.RefSession(system, policy, algorithm="fgmres", restart=12)
        mg_rm = fg.apply_mg(v)
        xf, infof = fg.solve(system.rhs, rtol=1e-13, maxit=400)
        fg.close()
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), mg=mg, op=op, x=x, x10=x10,
                            mg_residual_minimising=mg_rm, x_fgmres=xf)
        index[name] = {
            "spec": spec, "policy": pol, "digest": input_digest(system),
            "levels": levels,
            "iterations_1e13": info["iterations"], "iterations_1e10": info10["iterations"],
            "final_true_residual_1e13": info["final_true_residual"],
            "rhs_norm": info["rhs_norm"],
            "fgmres_iterations_1e13": infof["iterations"],
            "fgmres_final_true_residual_1e13": infof["final_true_residual"],
            "fgmres_operator_applies": infof["operator_applies"],
        }
        print(name, index[name]["iterations_1e13"], index[name]["iterations_1e10"])
    # Subspace recycling across two PISO correctors: corrector 1 captures its
    # Arnoldi-cycle corrections, corrector 2 (warm-started, perturbed rhs)
    # projects them (SolverWorkspace recycle_begin_capture /
    # recycle_begin_projection, src/solver_linear_state.cpp:735-1037).
    name = "sphere_24x20x16_prodF"
    spec, pol = CASES[name]
    system = system_for(spec)
    rhs2 = workloads.warm_start_rhs(system, 1)
    recycle = {}
    arrays = {}
    for restart in (12, 4):
        ref = ref_oracle.RefSession(system, ref_oracle.MgPolicy(**pol), algorithm="fgmres",
                                    restart=restart)
        x1, i1 = ref.solve(system.rhs, rtol=1e-10, recycle="capture")
        x2, i2 = ref.solve(rhs2, x0=x1, rtol=1e-10, recycle="project")
        ref.close()
        arrays[f"x1_r{restart}"], arrays[f"x2_r{restart}"] = x1, x2
        recycle[str(restart)] = {
            "capture_iterations": i1["iterations"],
            "captured": i1["recycle_cycle_corrections"],
            "project_iterations": i2["iterations"],
            "offered": i2["recycle_offered"], "retained": i2["recycle_retained"],
            "accepted": i2["recycle_accepted"],
            "projected_residual": i2["recycle_projected_residual"],
        }
    np.savez_compressed(os.path.join(HERE, "recycle_sphere_24x20x16_prodF.npz"), **arrays)
    index[name]["recycle"] = recycle

    # Cold path: solve_pcg with ColdPressureIccg and solve_bicgstab with
    # ColdPressureDilu on the decorated operator (src/solver_iccg.hpp:224-293,
    # src/solver_cold.hpp:484-560; src/solver_krylov.cpp:2651-3090).
    cold_arrays = {}
    for name in ("sphere_24x20x16_rbV22", "wrinkled_16x40x12_lineF"):
        spec, pol = CASES[name]
        system = system_for(spec)
        v = probe_vector(system)
        entry = {}
        for algorithm, pc in (("pcg", "iccg"), ("bicgstab", "dilu")):
            ref = ref_oracle.RefSession(system, ref_oracle.MgPolicy(**pol), algorithm=algorithm,
                                        preconditioner=pc)
            cold_arrays[f"{name}_{pc}_apply"] = ref.apply_cold(v)
            x, info = ref.solve(system.rhs, rtol=1e-12, maxit=8000)
            ref.close()
            cold_arrays[f"{name}_{algorithm}_{pc}_x"] = x
            entry[f"{algorithm}_{pc}"] = {"iterations": info["iterations"],
                                         "termination": info["termination"],
                                         "operator_applies": info["operator_applies"]}
        index[name]["cold"] = entry
    np.savez_compressed(os.path.join(HERE, "cold_path.npz"), **cold_arrays)
    with open(os.path.join(HERE, "index.json"), "w") as f:
        json.dump(index, f, indent=1)


if __name__ == "__main__":
    main()
