"""Z-slab domain decomposition of the MG-preconditioned PCG on CPU ranks
(gloo), against the single-rank solve.

oracle/slab_oracle.py restates the partitioned solve: halo planes before
every stencil application (HaloEngine, src/parallel_halo.cpp:1208-1400),
rank-ordered global reductions in each Krylov iteration (global_dot /
global_norm, src/solver_krylov.cpp:631-711) and a replicated coarse level
(src/solver_mg.cpp:31, 1135).  On one rank it reproduces the C restatement
bit for bit (operator and MG application).  Over 2 and 4 gloo ranks the MG
application and the operator are still bit-identical to the single-rank
ones (every MG operation is element-wise over exact halo copies), and the
PCG solve takes the same iteration count and agrees to rounding (only the
reduction order differs).  Cases: y-line relaxation with x/z
semicoarsening (stretched wrinkled flame) and point Chebyshev smoothing
with full coarsening (sphere).
"""
import os
import socket
import tempfile

import numpy as np
import pytest

CASES = {
    "wrinkled_16x24x16": dict(config="wrinkled256", n=(16, 24, 16), stretch_y=1.1),
    "sphere_16x12x16": dict(config="sphere64", n=(16, 12, 16)),
}


def _system(name):
    from hfps import workloads
    spec = dict(CASES[name])
    cfg = spec.pop("config")
    return workloads.make(cfg, **spec)


def _single(name):
    import c_oracle
    import ref_oracle
    import slab_oracle
    from hfps import workloads
    s = _system(name)
    pol = ref_oracle.MgPolicy.production()
    o = c_oracle.OracleSession(s, pol, line_order=1)
    m = slab_oracle.SlabMg(s, pol, slab_oracle.LocalComm(), o)
    r = workloads.normals(5, s.cells).reshape(s.rhs.shape)
    z = m.apply_mg(r)
    y = m.apply_operator(r)
    x, info = m.solve(s.rhs, rtol=1e-12)
    return s, o, z, y, x, info, r


def _rank_main(rank, world, port, name, out_dir):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [os.path.join(root, "hundun-flow_b200"), os.path.join(root, "oracle")]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    import datetime
    import torch.distributed as dist
    import c_oracle
    import ref_oracle
    import slab_oracle
    from hfps import workloads
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        s = _system(name)
        pol = ref_oracle.MgPolicy.production()
        o = c_oracle.OracleSession(s, pol, line_order=1)
        m = slab_oracle.SlabMg(s, pol, slab_oracle.TorchComm(), o)
        L = m.levels[0]
        k0, k1 = L.k0, L.k1
        r = workloads.normals(5, s.cells).reshape(s.rhs.shape)
        z = m.apply_mg(r[k0:k1])
        y = m.apply_operator(r[k0:k1])
        x, info = m.solve(s.rhs[k0:k1], rtol=1e-12)
        depth = sum(1 for lv in m.levels if not lv.replicated)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), k0=k0, k1=k1, z=z, y=y, x=x,
                 iterations=info["iterations"], termination=info["termination"],
                 depth=depth)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as sock:
        sock.bind(("127.0.0.1", 0))
        return sock.getsockname()[1]


@pytest.mark.usefixtures("oracle_built")
@pytest.mark.parametrize("name", sorted(CASES))
def test_single_rank_restatement_matches_c_oracle(name):
    s, o, z, y, x, info, r = _single(name)
    assert np.array_equal(z, o.apply_mg(r))
    assert np.array_equal(y, o.apply_level(0, r))
    xo, io = o.solve(s.rhs, rtol=1e-12)
    assert info["termination"] == io["termination"] == "converged"
    assert info["iterations"] == io["iterations"]
    assert np.linalg.norm(x - xo) <= 1e-12 * np.linalg.norm(xo)


@pytest.mark.usefixtures("oracle_built")
@pytest.mark.parametrize("world", [2, 4])
@pytest.mark.parametrize("name", sorted(CASES))
def test_partitioned_solve_matches_single_rank(name, world):
    import torch.multiprocessing as mp
    s, _, z, y, x, info, _ = _single(name)
    with tempfile.TemporaryDirectory() as out:
        mp.start_processes(_rank_main, args=(world, _free_port(), name, out), nprocs=world,
                           start_method="spawn", join=True)
        parts = [dict(np.load(os.path.join(out, f"rank{r}.npz"))) for r in range(world)]
    assert [int(p["k0"]) for p in parts] == sorted(int(p["k0"]) for p in parts)
    assert int(parts[-1]["k1"]) == s.shape[2]
    assert all(int(p["depth"]) >= 2 for p in parts), "at least two partitioned levels"
    for a, b in zip(parts, parts[1:]):
        assert int(a["k1"]) == int(b["k0"])
    zp = np.concatenate([p["z"] for p in parts])
    yp = np.concatenate([p["y"] for p in parts])
    xp = np.concatenate([p["x"] for p in parts])
    assert np.array_equal(zp, z)
    assert np.array_equal(yp, y)
    assert all(int(p["iterations"]) == info["iterations"] for p in parts)
    assert all(str(p["termination"]) == "converged" for p in parts)
    assert np.linalg.norm(xp - x) <= 1e-12 * np.linalg.norm(x)
