"""Benchmark of the B200 pressure solve (one JSON line on rank 0).

Workload: the 256^3 pressure system with geometric y-stretching (ratio 1.02
toward y=0), a wrinkled flame density front (rho ratio 7) and a solid IBM
z-cylinder, Dirichlet p=0 on x-max and Neumann elsewhere, solved to 1e-10
relative FP64 true residual by MG-preconditioned CG (the reference's
solve_pcg control flow, true residual every 4 iterations) with the
reference's production MG policy (F-cycle, pre 1 / post 2 sweeps; the
y-strong grid selects y-line relaxation and x/z semicoarsening).  A step is
one solve of the PISO-like warm-start sequence: rhs_k = rhs_0 + 0.05 * div
(fresh N(0,1) face noise, seed k), x0 = previous solution.  Inputs are
seeded synthetic fields (no public dataset exists for this path).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

N > 1 runs N independent replicas (one per GPU, launched by torchrun): the
solve of one system does not shard across GPUs in this build.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "hundun-flow_b200"))

METRIC = "time to 1e-10 rel. residual at 256³, mixed vs FP64 MG-PCG; solves/s; HBM GB/s"
UNIT = "solves/s"
CONFIG_NAME = "wrinkled256"
RTOL = 1e-10
TRUE_RESIDUAL_INTERVAL = 4
WARM_SEQUENCE = 20
DATA = "synthetic (seeded SplitMix64/Box-Muller face-flux divergence)"


def workload_label(shape):
    """Both arms name the same workload: the stretched wrinkled-flame system
    (256^3 unless --shape overrides it) and its warm-start sequence."""
    nx, ny, nz = shape
    size = f"{nx}^3" if nx == ny == nz else f"{nx}x{ny}x{nz}"
    return f"wrinkled256 warm-start pressure solve ({size} stretched, {WARM_SEQUENCE}-step sequence)"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--shape", type=int, nargs=3, default=None,
                   help="override the grid (testing only; the bench line is the 256^3 case)")
    p.add_argument("--single", choices=["fp64", "mixed", "fgmres", "fgmres-mixed"], default=None,
                   help="profiling aid: one warm-up solve, then one solve, no timing/JSON "
                        "(PCG, or the production FGMRES(12) with the residual-minimising MG)")
    p.add_argument("--kernel", choices=["operator", "smooth_fp64", "smooth_fp32", "restrict_fp64",
                                        "prolong_fp64", "pcg_update", "mg_fp64", "mg_mixed",
                                        "residual"],
                   default=None,
                   help="profiling aid: time `--steps` launches of one level-0 kernel class "
                        "(or one MG application) with CUDA events; one JSON line, not the bench")
    p.add_argument("--config", choices=["three_spheres512"], default=None,
                   help="the 512^3 three-sphere mixed forward + adjoint sequence "
                        "(its own JSON line; not the headline metric)")
    return p.parse_args()


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    # The reference arm runs on rank 0's host cores alone and takes no
    # collective step, so its ranks join no process group.
    if world > 1 and args.impl != "reference":
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(world, value):
    """Slowest rank's time: replicas are timed on their own devices and the
    job takes as long as its slowest rank."""
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def make_system(args):
    from hfps import workloads
    kw = {}
    if args.shape:
        kw["n"] = tuple(args.shape)
    return workloads.make(CONFIG_NAME, **kw)


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.device_index = device_index
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device_index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        self.file.flush()
        self.file.seek(0)
        mhz, max_mhz, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.file.read().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                mhz.append(float(parts[1]))
                max_mhz.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower().startswith("active"):
                    reasons.add(name)
        os.unlink(self.file.name)
        if not mhz:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(mhz), "sm_max_mhz": max(max_mhz),
                "reasons": sorted(reasons), "samples": len(mhz)}


class ReferenceSampler:
    """The reference's own solve_pcg + NativeCartesianMgPlan (compiled from
    the reference sources into oracle/_ref) on the full system; the C
    restatement stands in when the compiled reference is absent."""

    def __init__(self, system):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import ref_oracle
        self.system = system
        if ref_oracle.available():
            self.session = ref_oracle.RefSession(system, ref_oracle.MgPolicy.production(),
                                                 algorithm="pcg")
            self.kind = "reference"
        else:
            import c_oracle
            self.session = c_oracle.OracleSession(system, ref_oracle.MgPolicy.production())
            self.kind = "port"

    def solve(self, rhs, x0, maxit=400):
        """One solve to the benchmark tolerance; returns (x, iterations,
        seconds inside the solve)."""
        t0 = time.perf_counter()
        x, info = self.session.solve(rhs, x0, rtol=RTOL, maxit=maxit,
                                     true_residual_interval=TRUE_RESIDUAL_INTERVAL)
        seconds = info.get("seconds") or (time.perf_counter() - t0)
        return x, info["iterations"], seconds

    def seconds_per_iteration(self, iterations: int = 2) -> float:
        """Steady-state time of one PCG iteration: a solve capped at
        1 + iterations minus one capped at 1, so the start-up work (||b||,
        the initial true residual, the check at the cap) cancels."""
        _, one, t_one = self.solve(self.system.rhs, None, maxit=1)
        _, more, t_more = self.solve(self.system.rhs, None, maxit=1 + iterations)
        return (t_more - t_one) / max(1, more - one)

    def close(self):
        self.session.close()


def _reference_sequence_worker(shape, start, conn):
    """One replica (spawned, one host core): the cold first solve of the
    warm-start sequence (x0 = 0), then, after every replica has finished its
    own, the warm second solve (rhs + 0.05 div of the seed-1 noise, x0 = the
    first solution), both to 1e-10 with the reference's solve_pcg."""
    try:
        os.environ["OMP_NUM_THREADS"] = "1"
        from hfps import workloads
        system = workloads.make(CONFIG_NAME, **({"n": tuple(shape)} if shape else {}))
        sampler = ReferenceSampler(system)
        rhs1 = workloads.warm_start_rhs(system, 1)
        start.wait()
        p0, cold_iterations, cold_seconds = sampler.solve(system.rhs, None)
        start.wait()
        _, warm_iterations, warm_seconds = sampler.solve(rhs1, p0)
        sampler.close()
        conn.send(("ok", sampler.kind, (cold_iterations, cold_seconds, warm_iterations,
                                        warm_seconds)))
    except BaseException as exc:  # report, never hang the parent
        conn.send(("error", repr(exc), None))
    finally:
        conn.close()


def _reference_iteration_worker(shape, iterations, start, conn):
    """One replica (spawned): the steady-state time of one PCG iteration."""
    try:
        os.environ["OMP_NUM_THREADS"] = "1"
        from hfps import workloads
        system = workloads.make(CONFIG_NAME, **({"n": tuple(shape)} if shape else {}))
        sampler = ReferenceSampler(system)
        start.wait()
        seconds = sampler.seconds_per_iteration(iterations)
        sampler.close()
        conn.send(("ok", sampler.kind, seconds))
    except BaseException as exc:
        conn.send(("error", repr(exc), None))
    finally:
        conn.close()


def reference_workers():
    """Host cores to use, bounded by memory: a 256^3 replica of the
    reference solver peaks near 5.5 GB of host memory."""
    cores = len(os.sched_getaffinity(0))
    available = None
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    available = int(line.split()[1]) * 1024
    except OSError:
        pass
    if available is None:
        return 1
    return max(1, min(cores, int(0.5 * available / 6.5e9)))


def run_replicas(target, workers, *args):
    """Runs `workers` spawned replicas of `target(*args, barrier, pipe)` and
    returns their (kind, result) pairs; raises if any replica failed."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    start = ctx.Barrier(workers)
    pipes, procs = [], []
    for _ in range(workers):
        parent, child = ctx.Pipe(duplex=False)
        p = ctx.Process(target=target, args=(*args, start, child))
        p.start()
        child.close()
        pipes.append(parent)
        procs.append(p)
    results = [c.recv() for c in pipes]
    for p in procs:
        p.join()
    errors = [r[1] for r in results if r[0] != "ok"]
    if errors:
        raise RuntimeError(f"reference replica failed: {errors[0]}")
    return [(r[1], r[2]) for r in results]


def reference_warm_iterations(shape):
    """Iterations the reference's solve_pcg takes on the warm second solve of
    this workload, as recorded from the compiled reference on the same inputs
    (tests/golden/wrinkled256.json, written by tests/golden/make_golden.py
    --scale); None for other shapes."""
    if shape not in (None, [256, 256, 256], (256, 256, 256)):
        return None
    path = os.path.join(ROOT, "tests", "golden", "wrinkled256.json")
    try:
        with open(path) as f:
            return int(json.load(f)["pcg_step1_1e10"]["iterations"])
    except (OSError, KeyError, ValueError):
        return None


def run_reference(args, world, rank):
    """The reference arm: the reference's own CPU MG-PCG (solve_pcg +
    NativeCartesianMgPlan compiled from its sources) on this workload, one
    single-threaded replica per host core (the reference's solve of one
    system runs on one MPI rank; the stand-in MPI has one rank).

    Every replica runs the first two solves of the warm-start sequence to
    1e-10 in full: the cold first solve (untimed warm-up, it produces the
    warm start), then, all replicas together, the warm second solve (the
    timed region).  Nothing is extrapolated: solves/s = replicas / the
    slowest replica's warm solve time, iterations are the run's own."""
    if rank != 0:
        return
    workers = reference_workers()
    results = run_replicas(_reference_sequence_worker, workers, args.shape)
    kind = results[0][0]
    cold_iterations = [r[1][0] for r in results]
    warm_iterations = [r[1][2] for r in results]
    warm_seconds = [r[1][3] for r in results]
    region = max(warm_seconds)
    value = workers / region
    shape = list(args.shape) if args.shape else [256, 256, 256]
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * region / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": DATA,
        "config": {"workload": workload_label(shape),
                   "shape": shape,
                   "algorithm": "solve_pcg + NativeCartesianMgPlan (production policy, unit_linear)",
                   "rtol": RTOL, "true_residual_interval": TRUE_RESIDUAL_INTERVAL,
                   "iterations_per_solve": warm_iterations,
                   "cold_iterations": cold_iterations,
                   "timed_region_s": region},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": workers, "kind": kind,
                         "sample": f"{workers} single-threaded replicas, each solving the warm "
                                   f"second solve of the sequence to 1e-10 in full "
                                   f"({statistics.mean(warm_iterations):.1f} iterations, "
                                   f"slowest {region:.1f} s), after its own cold first solve; "
                                   f"timed region = the warm solves, reported as {args.steps} "
                                   f"equal steps"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# DRAM bytes per level-0 cell of one zebra colour pass of the FP64 line
# kernel (split-row vectors, a pass that reads x), from one ncu capture at
# 256x256x128 (337.1 MB read + 26.1 MB written over 8,388,608 cells);
# traffic grows with the cell count.
LINE_PASS_DRAM_BYTES_PER_CELL = (303.605760e6 + 26.895872e6) / (256 * 256 * 128)

def reference_solution_errors(args, solver, rhs0):
    """Relative L2 error, over the recorded sample of cells, of the FP64 and
    mixed cold solves at rtol 1e-13 against the compiled reference's FP64
    solution of the same system; {} when no record exists for the shape."""
    import torch
    import hfps
    if args.shape not in (None, [256, 256, 256], (256, 256, 256)):
        return {}
    base = os.path.join(ROOT, "tests", "golden", "wrinkled256")
    try:
        ref = dict(np.load(base + ".npz"))
        with open(base + ".json") as f:
            entry = json.load(f)
    except OSError:
        return {}
    cells = torch.from_numpy(ref["cells"]).to(rhs0.device)
    want = torch.from_numpy(ref["pcg_step0_1e13"]).to(rhs0.device)
    out = {"reference_solution": "compiled reference solve_pcg, cold solve at 1e-13 "
                                 f"({entry['pcg_step0_1e13']['iterations']} iterations), "
                                 f"{cells.numel()} sampled cells"}
    for label, precision in (("fp64", hfps.FP64), ("mixed", hfps.MIXED)):
        o = hfps.SolveOptions(rtol=1e-13, maxit=400, true_residual_interval=TRUE_RESIDUAL_INTERVAL,
                              precision=precision)
        xs, info = solver.solve(rhs0, options=o, history=False)
        got = xs[cells]
        out[f"rel_error_vs_reference_{label}"] = float(torch.linalg.vector_norm(got - want) /
                                                       torch.linalg.vector_norm(want))
        out[f"steps_at_1e-13_{label}"] = info["iterations"]
    return out


def run_b200(args, world, rank, local):
    import numpy as np
    import torch
    import hfps
    from hfps import workloads

    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    system = make_system(args)
    stream = torch.cuda.current_stream(device)
    solver = hfps.PressureSolver.from_system(system, hfps.Policy.production(), stream=stream)
    n = system.cells
    rhs0 = torch.from_numpy(system.rhs.reshape(-1)).to(device)
    total = args.warmup + args.steps
    rhs = []
    for k in range(total):
        seed = 1 + (k % WARM_SEQUENCE)
        rhs.append(rhs0 + workloads.flux_divergence_rhs_torch(
            seed, system.faces, system.boundary, system.active, 0.05, device=device))
    opts = hfps.SolveOptions(rtol=RTOL, maxit=400, true_residual_interval=TRUE_RESIDUAL_INTERVAL)
    x = torch.zeros(n, dtype=torch.float64, device=device)

    def run_sequence(precision, steps, xbuf, offset=0, record=None):
        o = hfps.SolveOptions(rtol=RTOL, maxit=400, true_residual_interval=TRUE_RESIDUAL_INTERVAL,
                              precision=precision)
        for k in range(steps):
            _, info = solver.solve(rhs[(offset + k) % total], x0=xbuf, out=xbuf, options=o,
                                   history=False)
            if record is not None:
                record.append(info)

    # Warm-up (also instantiates the MG graphs).
    run_sequence(hfps.FP64, args.warmup, x)
    xw = x.clone()
    infos = []
    barrier(world)
    torch.cuda.synchronize()
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        start.record(stream)
        run_sequence(hfps.FP64, args.steps, x, offset=args.warmup, record=infos)
        stop.record(stream)
        torch.cuda.synchronize()
    barrier(world)
    seconds = max_over_ranks(world, start.elapsed_time(stop) / 1000.0)
    value = world * args.steps / seconds

    # Mixed precision on the same sequence (same warm-start state).
    xm = xw.clone()
    run_sequence(hfps.MIXED, 1, xm.clone(), offset=args.warmup)
    minfos = []
    torch.cuda.synchronize()
    start.record(stream)
    run_sequence(hfps.MIXED, args.steps, xm, offset=args.warmup, record=minfos)
    stop.record(stream)
    torch.cuda.synchronize()
    mixed_seconds = max_over_ranks(world, start.elapsed_time(stop) / 1000.0)
    mixed_error = float(torch.linalg.vector_norm(xm - x) / torch.linalg.vector_norm(x))
    # Error against the reference's own FP64 solution: the cold first solve
    # at 1e-13 in both forms, compared with the compiled reference's solution
    # on the recorded sample of cells (tests/golden/wrinkled256.*, written by
    # tests/golden/make_golden.py --scale).
    reference_errors = reference_solution_errors(args, solver, rhs0)

    # The reference's production pressure solve on the same sequence:
    # solve_fgmres(12) with the residual-minimising MG plan, FP64 and mixed.
    fg_solver = hfps.PressureSolver.from_system(
        system, hfps.Policy.production().replace(unit_linear=0), stream=stream)
    fg = {}
    for label, precision in (("fp64", hfps.FP64), ("mixed", hfps.MIXED)):
        o = hfps.SolveOptions(rtol=RTOL, maxit=400, true_residual_interval=TRUE_RESIDUAL_INTERVAL,
                              precision=precision, algorithm=hfps.FGMRES, restart=12)
        xf = xw.clone()
        fg_solver.solve(rhs[args.warmup % total], x0=xf.clone(), options=o, history=False)
        finfos = []
        torch.cuda.synchronize()
        start.record(stream)
        for k in range(args.steps):
            _, info = fg_solver.solve(rhs[(args.warmup + k) % total], x0=xf, out=xf, options=o,
                                      history=False)
            finfos.append(info)
        stop.record(stream)
        torch.cuda.synchronize()
        fseconds = max_over_ranks(world, start.elapsed_time(stop) / 1000.0)
        fg[label] = {"value": world * args.steps / fseconds, "unit": UNIT,
                     "iterations_per_solve": [i["iterations"] for i in finfos],
                     "rel_error_vs_pcg_fp64": float(torch.linalg.vector_norm(xf - x) /
                                                    torch.linalg.vector_norm(x))}
    fg_solver.close()

    # End to end through the C ABI with pinned host buffers: every step copies
    # rhs and x0 host->device and x device->host.
    host_rhs = [torch.empty(n, dtype=torch.float64, pin_memory=True) for _ in range(args.steps)]
    for k in range(args.steps):
        host_rhs[k].copy_(rhs[args.warmup + k])
    host_x = torch.empty(n, dtype=torch.float64, pin_memory=True)
    host_x.copy_(xw)
    torch.cuda.synchronize()
    barrier(world)
    t0 = time.perf_counter()
    for k in range(args.steps):
        solver.solve(host_rhs[k], x0=host_x, out=host_x, options=opts, history=False)
    torch.cuda.synchronize()
    e2e_seconds = max_over_ranks(world, time.perf_counter() - t0)
    e2e_value = world * args.steps / e2e_seconds

    # Dominant kernel: the level-0 zebra line-relaxation colour pass (largest
    # share of device time in the launch list).  Timed with CUDA events on
    # the solver's stream; algorithmic bytes = 28 B per level-0 cell per pass
    # (each operand of a full sweep x, b, D, fx, fy, fz and the x write read
    # or written once over the two colour passes).
    kernels = {}
    for name in ("smooth_fp64", "operator", "restrict_fp64", "prolong_fp64", "pcg_update",
                 "smooth_fp32", "mg_fp64", "mg_mixed"):
        ms, nbytes = solver.profile_kernel(name, 10)
        kernels[name] = {"ms": ms, "bytes": nbytes,
                         "gbs": (nbytes / (ms * 1e-3) / 1e9) if nbytes > 0 else None}
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        with open(peaks_path) as f:
            peak = float(json.load(f)["hbm_gbs"])
        peak_note = "measured"
    else:
        peak, peak_note = 6650.0, "fallback"
    dom = kernels["smooth_fp64"]
    roofline = {"bound": "hbm",
                "kernel": "k_line_scan_color<double,y,8,normal,split rows> level 0 "
                          "(one zebra colour)",
                "achieved": dom["gbs"], "peak": peak, "unit": "GB/s",
                "frac": dom["gbs"] / peak, "peak_source": peak_note,
                "traffic": LINE_PASS_DRAM_BYTES_PER_CELL * n,
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch at "
                                  "256x256x128, scaled by cells",
                "bytes_per_launch": dom["bytes"], "ms_per_launch": dom["ms"]}

    iterations = [i["iterations"] for i in infos]
    cpu = None
    warm_iterations = reference_warm_iterations(args.shape)
    if rank == 0 and world == 1 and not args.no_cpu_baseline and warm_iterations:
        workers = reference_workers()
        results = run_replicas(_reference_iteration_worker, workers, args.shape, 2)
        kind = results[0][0]
        t_iter = max(r[1] for r in results)
        cpu = {"value": workers / (t_iter * warm_iterations), "unit": UNIT, "cores": workers,
               "kind": kind,
               "sample": f"{workers} single-threaded replicas, each timing 2 steady-state PCG "
                         f"iterations of the 256^3 system (a 3-iteration solve minus a "
                         f"1-iteration one; slowest {t_iter:.2f} s per iteration) x "
                         f"{warm_iterations} iterations per warm solve (the reference's own "
                         f"count on these inputs, tests/golden/wrinkled256.json)"}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * seconds / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": DATA,
            "config": {"workload": workload_label(system.shape),
                       "shape": list(system.shape), "stretch_y": 1.02,
                       "algorithm": "PCG (solve_pcg control flow) + MG production policy, unit_linear",
                       "rtol": RTOL, "true_residual_interval": TRUE_RESIDUAL_INTERVAL,
                       "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (FP64 hierarchy ~2 GB per GPU)",
                       "iterations_per_solve": iterations},
            "mixed": {"value": world * args.steps / mixed_seconds, "unit": UNIT,
                      "speedup_vs_fp64": seconds / mixed_seconds,
                      "form": "FP32 MG preconditioner inside FP64 PCG (Krylov-accelerated "
                              "iterative refinement: FP64 residual, dots, norms and coarsest "
                              "solve); refinement steps = outer PCG iterations",
                      "refinement_steps_per_solve": [i["iterations"] for i in minfos],
                      "rel_error_vs_fp64_gpu": mixed_error,
                      **reference_errors},
            "fgmres": {"algorithm": "solve_fgmres(12) + residual-minimising MG (the reference's "
                                    "production pressure solve)", **fg},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 2 * n * 8,
                    "d2h_bytes_per_step": n * 8},
            "roofline": roofline,
            "kernels": kernels,
            "cpu_baseline": cpu,
            "clocks": clocks.summary(),
            "gpu_launches": int(sum(i["kernel_launches"] for i in infos)),
        }
        print(json.dumps(line), flush=True)
    solver.close()


def run_single(args):
    """One warm-up solve and one measured-by-profiler solve of step 1."""
    import torch
    import hfps
    from hfps import workloads
    system = make_system(args)
    fgmres = args.single.startswith("fgmres")
    policy = hfps.Policy.production()
    if fgmres:
        policy = policy.replace(unit_linear=0)
    solver = hfps.PressureSolver.from_system(system, policy, stream=torch.cuda.current_stream())
    rhs = torch.from_numpy(system.rhs.reshape(-1)).cuda()
    rhs1 = rhs + workloads.flux_divergence_rhs_torch(1, system.faces, system.boundary,
                                                     system.active, 0.05)
    precision = hfps.MIXED if args.single.endswith("mixed") else hfps.FP64
    extra = dict(algorithm=hfps.FGMRES, restart=12) if fgmres else {}
    opts = hfps.SolveOptions(rtol=RTOL, maxit=400, true_residual_interval=TRUE_RESIDUAL_INTERVAL,
                             precision=precision, **extra)
    x, info0 = solver.solve(rhs, options=opts, history=False)
    x, info1 = solver.solve(rhs1, x0=x, out=x, options=opts, history=False)
    torch.cuda.synchronize()
    print(json.dumps({"single": args.single, "iterations": [info0["iterations"], info1["iterations"]],
                      "kernel_launches": [info0["kernel_launches"], info1["kernel_launches"]]}))
    solver.close()


def run_kernel(args):
    """`steps` launches of one kernel class on the solver's stream (after
    hfps_profile_kernel's own warm-up launch), timed with CUDA events."""
    import hfps
    system = make_system(args)
    solver = hfps.PressureSolver.from_system(system, hfps.Policy.production())
    ms, nbytes = solver.profile_kernel(args.kernel, args.steps)
    print(json.dumps({"kernel": args.kernel, "shape": list(system.rhs.shape[::-1]),
                      "launches": args.steps, "ms_per_launch": ms,
                      "algorithmic_bytes": nbytes,
                      "gb_s": nbytes / (ms * 1e-3) / 1e9 if nbytes > 0 else None}))
    solver.close()


def run_three_spheres(args):
    """512^3 spherical flame with three IBM spheres: `steps` warm-started
    mixed-precision forward solves, each followed by a mixed adjoint solve of
    L = 0.5 sum_fluid (p - p_t)^2 (p_t from seed 7), with size-independent
    checks: the forward true residual, the adjoint identity lambda.b =
    (dL/dp).p (A is symmetric), the mixed solution against an FP64 solve, and
    the device memory in use."""
    import torch
    import hfps
    from hfps import workloads
    device = torch.device("cuda", 0)
    free0, total = torch.cuda.mem_get_info(device)
    system = workloads.make("three_spheres512")
    solver = hfps.PressureSolver.from_system(system, hfps.Policy.production(),
                                             stream=torch.cuda.current_stream(device))
    n = system.cells
    rhs0 = torch.from_numpy(system.rhs.reshape(-1)).to(device)
    active = torch.from_numpy(system.active.reshape(-1).astype(np.bool_)).to(device)
    target = workloads.normals_torch(7, n, device=device)
    opts = hfps.SolveOptions(rtol=RTOL, maxit=400, precision=hfps.MIXED)
    x = torch.zeros(n, dtype=torch.float64, device=device)
    solver.solve(rhs0, x0=x.clone(), options=opts, history=False)  # warm-up, graphs
    forward_ms, adjoint_ms, iters, adj_iters, identity, residuals = [], [], [], [], [], []
    start = torch.cuda.Event(enable_timing=True)
    mid = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    free1, _ = torch.cuda.mem_get_info(device)
    for k in range(args.steps):
        rhs = rhs0 + workloads.flux_divergence_rhs_torch(1 + k, system.faces, system.boundary,
                                                         system.active, 0.05, device=device)
        x_start = x.clone()
        torch.cuda.synchronize()
        start.record()
        x, info = solver.solve(rhs, x0=x, out=x, options=opts, history=False)
        mid.record()
        dl_dp = torch.where(active, x - target, torch.zeros_like(x))
        lam, grads, ainfo = solver.adjoint(x, dl_dp, options=opts)
        stop.record()
        torch.cuda.synchronize()
        forward_ms.append(start.elapsed_time(mid))
        adjoint_ms.append(mid.elapsed_time(stop))
        iters.append(info["iterations"])
        adj_iters.append(ainfo["iterations"])
        residuals.append(info["final_true_residual"] / info["rhs_norm"])
        lb = float(torch.dot(lam, torch.where(active, rhs, torch.zeros_like(rhs))))
        gp = float(torch.dot(dl_dp, x))
        identity.append(abs(lb - gp) / max(abs(gp), 1e-300))
    # The plain FP64 GPU forward solve of the last step (same rhs, same warm
    # start), and the FP64 adjoint of the mixed solution's loss: the gradient
    # errors compare the mixed adjoint (lambda and every face gradient) with it.
    torch.cuda.synchronize()
    start.record()
    x64, i64 = solver.solve(rhs, x0=x_start, rtol=RTOL, maxit=400, history=False)
    stop.record()
    torch.cuda.synchronize()
    fp64_ms = start.elapsed_time(stop)
    mixed_error = float(torch.linalg.vector_norm(x - x64) / torch.linalg.vector_norm(x64))
    lam64, grads64, _ = solver.adjoint(x, dl_dp, rtol=RTOL, maxit=400)

    def rel(a, b):
        return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))

    lambda_error = rel(lam, lam64)
    face_error = max(rel(g, g64) for g, g64 in zip(grads, grads64))
    ms, nbytes = solver.profile_kernel("smooth_fp32", 10)
    line = {
        "config": {"workload": "three_spheres512 (512^3 spherical flame, three IBM spheres)",
                   "cells": n, "sequence": args.steps,
                   "algorithm": "mixed MG-PCG forward + mixed adjoint per step"},
        "forward_ms": statistics.mean(forward_ms), "adjoint_ms": statistics.mean(adjoint_ms),
        "forward_iterations": iters, "adjoint_iterations": adj_iters,
        "max_relative_true_residual": max(residuals),
        "max_adjoint_identity_error": max(identity),
        "mixed_vs_fp64_relative_error": mixed_error, "fp64_iterations": i64["iterations"],
        "fp64_forward_ms": fp64_ms,
        "adjoint_lambda_vs_fp64_relative_error": lambda_error,
        "adjoint_face_gradient_vs_fp64_relative_error": face_error,
        "level0_smoother_fp32_gbs": nbytes / (ms * 1e-3) / 1e9 if ms else None,
        "device_memory_gb": (free0 - free1) / 1e9, "device_total_gb": total / 1e9,
    }
    print(json.dumps(line), flush=True)
    solver.close()


def main():
    args = parse()
    world, rank, local = dist_setup(args)
    if args.single:
        run_single(args)
        return
    if args.kernel:
        run_kernel(args)
        return
    if args.config == "three_spheres512":
        run_three_spheres(args)
        return
    if args.impl == "reference":
        run_reference(args, world, rank)
        return
    run_b200(args, world, rank, local)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
