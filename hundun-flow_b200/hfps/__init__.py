"""hfps: B200-native pressure-coupling linear solve (Hundun-Flow hot path).

The product is the CUDA library hundun-flow_b200/libhfps.so behind the C ABI
of include/hf_pressure_solver.h; this package is its thin Python mirror
(``solver.PressureSolver``), the seeded workload generator (``workloads``)
and a torch.autograd wrapper used for gradient checks (``autograd``).
"""
from . import workloads  # noqa: F401
from .solver import (BICGSTAB, DEVICE, FGMRES, FP64, HOST, IC0, MG, MIXED, NORM_PLAIN,  # noqa: F401
                     NORM_SCALED, PCG, Policy, PressureSolver, SolveOptions, SolverError,
                     library_path)
