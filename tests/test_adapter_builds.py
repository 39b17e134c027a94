"""The C++ adapter a maintainer adds to the reference
(hundun-flow_b200/adapter/b200_pressure_solve.hpp) compiles against the
reference's own headers (include/hundun/v04_linear.hpp and what it pulls
in) and links against libhfps.so: every reference type and member it names
exists with the meaning it assumes, and every C-ABI symbol it calls is
exported.  The program is built, not run (it would need a GPU).  Skipped
where the reference tree is absent."""
import os
import shutil
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REFERENCE = os.environ.get("HFPS_REFERENCE", "/root/reference/versions/v0.4")

PROGRAM = r'''
#include "b200_pressure_solve.hpp"
#include <cstdio>

int main(int argc, char**) {
  using namespace hundun::v04;
  if (argc < 2) return 0;  // built, never run on a machine without a GPU
  NativeCartesianMgSpec spec;
  spec.boundaries = {MgBoundaryKind::neumann, MgBoundaryKind::dirichlet,
                     MgBoundaryKind::neumann, MgBoundaryKind::neumann,
                     MgBoundaryKind::neumann, MgBoundaryKind::neumann};
  spec.correction_scaling = MgCorrectionScaling::residual_minimizing;
  const Int3 cells{8, 8, 8};
  std::vector<double> f(9);
  for (int i = 0; i < 9; ++i) f[i] = i / 8.0;
  B200PressureSolve solve;
  const Status st = solve.compile(spec, cells, f, f, f, {});
  if (!st) return 1;
  MgCoefficientViews views{};
  (void)solve.update(views);
  LinearSolveInvocation inv{};
  inv.control.relative_tolerance = 1e-10;
  inv.control.maximum_iterations = 100;
  inv.control.true_residual_interval = 4;
  inv.control.restart = 12;
  const LinearSolveResult r = solve.solve(inv, false, HFPS_RECYCLE_CAPTURE);
  std::printf("%u\n", r.iterations);
  return r.status ? 0 : 2;
}
'''


@pytest.mark.skipif(not os.path.isdir(os.path.join(REFERENCE, "include", "hundun")),
                    reason="reference headers not present")
def test_adapter_compiles_and_links(cuda_library):
    cxx = shutil.which("g++")
    assert cxx
    with tempfile.TemporaryDirectory() as tmp:
        src = os.path.join(tmp, "adapter_check.cpp")
        with open(src, "w") as fh:
            fh.write(PROGRAM)
        exe = os.path.join(tmp, "adapter_check")
        cmd = [cxx, "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror",
               "-I", os.path.join(ROOT, "include"),
               "-I", os.path.join(ROOT, "hundun-flow_b200", "adapter"),
               "-I", os.path.join(REFERENCE, "include"),
               "-I", os.path.join(ROOT, "oracle", "mpi_shim"),
               src, "-o", exe, "-L", os.path.dirname(cuda_library), "-lhfps",
               f"-Wl,-rpath,{os.path.dirname(cuda_library)}"]
        proc = subprocess.run(cmd, capture_output=True, text=True)
        assert proc.returncode == 0, proc.stderr[-4000:]
        assert os.path.exists(exe)
