"""hfps: B200-native pressure-coupling linear solve (Hundun-Flow hot path).

The product is the CUDA library hundun-flow_b200/libhfps.so behind the C ABI
of include/hf_pressure_solver.h; this package is its thin Python mirror
(``solver.PressureSolver``), the seeded workload generator (``workloads``)
and a torch.autograd wrapper used for gradient checks (``autograd``).
"""
from . import workloads  # noqa: F401
from .solver import (DEVICE, FGMRES, FP64, HOST, MIXED, PCG, Policy,  # noqa: F401
                     PressureSolver, SolveOptions, SolverError, library_path)
