"""Builds the sm_100a pressure-solve library in-tree: hundun-flow_b200/libhfps.so.

nvcc compiles every translation unit for sm_100a (compute_100a) with
--fmad=false, so the stencil arithmetic keeps the reference's separate
multiply/subtract rounding, then links one shared library exporting the C ABI
of include/hf_pressure_solver.h.  Objects go to hundun-flow_b200/_build/.
"""
from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIBRARY = os.path.join(HERE, "libhfps.so")
SOURCES = ["kernels.cu", "kernels_line.cu", "kernels_tail.cu", "solver.cu", "capi.cu",
           "noalloc.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC",
         "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr",
         f"-I{os.path.join(ROOT, 'include')}", f"-I{CSRC}"]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found")
    return path


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".hpp", ".cuh"))]
    headers.append(os.path.join(ROOT, "include", "hf_pressure_solver.h"))
    objects = []
    jobs = []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src.replace(".cu", ".o"))
        objects.append(obj)
        if force or _stale(obj, [path] + headers):
            cmd = [nvcc(), *ARCH, *FLAGS, "-c", path, "-o", obj]
            if verbose:
                cmd.append("-Xptxas=-v")
            jobs.append(cmd)

    def run(cmd):
        proc = subprocess.run(cmd, capture_output=True, text=True)
        if proc.returncode != 0:
            raise RuntimeError(f"nvcc failed: {' '.join(cmd)}\n{proc.stderr}")
        return proc.stderr

    with concurrent.futures.ThreadPoolExecutor(max_workers=len(SOURCES)) as pool:
        for out in pool.map(run, jobs):
            if verbose and out:
                sys.stderr.write(out)
    if force or jobs or _stale(LIBRARY, objects):
        cmd = [nvcc(), *ARCH, "-shared", "-o", LIBRARY, *objects, "-lcudart"]
        run(cmd)
    return LIBRARY


# The C++ torch extension of the differentiable solve (csrc/torch_autograd.cpp,
# used for gradient checks).  It calls only the C ABI, links libhfps.so and is
# built in-tree into hfps/_ext/ (which travels with the checkout).
TORCH_EXT_DIR = os.path.join(HERE, "hfps", "_ext")


def build_torch_extension(verbose: bool = False):
    """Compiles (when stale) and imports the extension module."""
    from torch.utils.cpp_extension import load
    os.makedirs(TORCH_EXT_DIR, exist_ok=True)
    return load(name="hfps_torch_autograd",
                sources=[os.path.join(CSRC, "torch_autograd.cpp")],
                extra_include_paths=[os.path.join(ROOT, "include")],
                extra_cflags=["-O2"],
                extra_ldflags=[f"-L{HERE}", "-lhfps", f"-Wl,-rpath,{HERE}"],
                build_directory=TORCH_EXT_DIR, verbose=verbose)


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
