"""Benchmark-scale parity cases: the y-stretched wrinkled flame at 128^3 and
at the benchmarked 256^3 (tests/golden/wrinkled128.*, wrinkled256.*).

The fixtures hold what the compiled reference returned for these systems
(tests/golden/make_golden.py --scale): iteration counts and a fixed seeded
sample of cells of each solution.  ``reference_solve`` runs the compiled
reference itself (oracle/_ref) in a spawned worker process, so that several
reference solves run on separate host cores beside the GPU.
"""
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
RTOLS = {"1e13": 1e-13, "1e10": 1e-10}


def entry(name):
    with open(os.path.join(GOLDEN, f"{name}.json")) as f:
        return json.load(f)


def arrays(name):
    return dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))


def system(name):
    from hfps import workloads
    spec = dict(entry(name)["spec"])
    config = spec.pop("config")
    spec["n"] = tuple(spec["n"])
    return workloads.make(config, **spec)


def rhs(sys_, step):
    from hfps import workloads
    return sys_.rhs if step == 0 else workloads.warm_start_rhs(sys_, step)


def sample_error(x, ref_sample, cells):
    """Relative L2 difference over the recorded sample of cells."""
    s = np.asarray(x).reshape(-1)[cells]
    return float(np.linalg.norm(s - ref_sample) / np.linalg.norm(ref_sample))


def _reference_worker(args):
    """(name, algorithm, step, x0 file or None, rtol, out file) -> solve
    record; the solution is written to `out file`."""
    import ref_oracle
    name, algorithm, step, x0_path, rtol, out_path = args
    sys_ = system(name)
    b = rhs(sys_, step)
    x0 = np.load(x0_path).reshape(b.shape) if x0_path else None
    ref = ref_oracle.RefSession(sys_, ref_oracle.MgPolicy.production(), algorithm=algorithm,
                                restart=12)
    x, info = ref.solve(b, x0=x0, rtol=rtol, maxit=400)
    ref.close()
    np.save(out_path, x.reshape(-1))
    return info


def reference_pool(workers):
    """A spawned pool (never forked: the parent holds a CUDA context)."""
    import multiprocessing as mp
    return mp.get_context("spawn").Pool(workers)
