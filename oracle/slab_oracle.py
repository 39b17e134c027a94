"""Z-slab domain decomposition of the pressure solve -- CPU restatement, TEST
INFRASTRUCTURE (used only by tests/ as the checker of the partitioned
algorithm).

The reference decomposes this solve over MPI ranks: a persistent halo
exchange before every stencil application (HaloEngine::begin/finish,
src/parallel_halo.cpp:1208-1400), checked global reductions in every Krylov
iteration (global_dot / global_norm, src/solver_krylov.cpp:631-711, over
ReductionEngine::checked_sum / checked_max, src/solver_reduction.cpp:
333-380 and :651) and a small coarse level replicated on every rank
(initialize_replicated_coarse, src/solver_mg.cpp:31, 1135).  This module
restates the MG-preconditioned PCG of oracle/hfps_oracle.c (zebra line
order, unit-scaled MG, the production policy) partitioned into z-slabs, one
slab per rank, with the same three kinds of communication:

* halo planes: before every defect, Chebyshev stage and zebra colour pass a
  rank sends its lowest and highest owned plane of the level's x to its
  neighbours; prolongation reads the coarse x with one halo plane;
* reductions: the reference's global_dot (rank-local Neumaier sums, added
  in rank order) and global_norm (global maximum, then rank-local scaled
  squares added in rank order);
* the coarse level: every level whose extent in z is smaller than the rank
  count, and the coarsest level, is gathered onto every rank and relaxed
  there redundantly (replicated), each rank keeping its own planes.

Slab boundaries sit on multiples of 2^m at the finest level (m = the number
of z-coarsenings out of the partitioned levels, the one into the first
replicated level included), so every restriction stays on its rank.
y- and x-lines lie inside a slab; a hierarchy that relaxes z-lines is not
partitioned along z and is rejected.  Every MG operation is element-wise
with exact halo copies, so an MG application is bit-identical to the
single-rank one; solves differ only by the reduction order.

Communication goes through a ``Comm`` object: ``LocalComm`` (one rank) or
``TorchComm`` (torch.distributed, gloo on CPU; NCCL send/recv on GPUs).
"""
from __future__ import annotations

import dataclasses
from typing import List, Optional

import numpy as np

NEUMANN = 1
OMEGA_CHEB_BETA = 2.0


# ---------------------------------------------------------------------------
# Communication


class LocalComm:
    """One rank: halo exchange fills nothing, reductions are identities."""

    rank = 0
    size = 1

    def exchange(self, lower_send, upper_send):
        return None, None

    def sum_in_rank_order(self, value: float) -> float:
        return value

    def maximum(self, value: float) -> float:
        return value

    def gather_planes(self, planes: np.ndarray, counts: List[int]) -> np.ndarray:
        return planes


class TorchComm:
    """torch.distributed point-to-point and collectives (gloo or NCCL).

    Every rank takes the same collective steps in the same order; halo
    planes travel by paired isend/irecv so that no rank waits on an
    unposted receive."""

    def __init__(self):
        import torch.distributed as dist
        self.dist = dist
        self.rank = dist.get_rank()
        self.size = dist.get_world_size()

    def exchange(self, lower_send, upper_send):
        """Sends this rank's lowest owned plane down and highest up; returns
        (plane from below, plane from above), None at the ends."""
        import torch
        dist = self.dist
        ops, recv_lo, recv_hi = [], None, None
        if self.rank > 0:
            recv_lo = torch.empty(lower_send.shape, dtype=torch.float64)
            ops.append(dist.P2POp(dist.isend, torch.from_numpy(np.ascontiguousarray(lower_send)),
                                  self.rank - 1))
            ops.append(dist.P2POp(dist.irecv, recv_lo, self.rank - 1))
        if self.rank + 1 < self.size:
            recv_hi = torch.empty(upper_send.shape, dtype=torch.float64)
            ops.append(dist.P2POp(dist.isend, torch.from_numpy(np.ascontiguousarray(upper_send)),
                                  self.rank + 1))
            ops.append(dist.P2POp(dist.irecv, recv_hi, self.rank + 1))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        return (None if recv_lo is None else recv_lo.numpy(),
                None if recv_hi is None else recv_hi.numpy())

    def _all_gather(self, value: float) -> List[float]:
        import torch
        out = [torch.zeros(1, dtype=torch.float64) for _ in range(self.size)]
        self.dist.all_gather(out, torch.tensor([value], dtype=torch.float64))
        return [float(t.item()) for t in out]

    def sum_in_rank_order(self, value: float) -> float:
        total = 0.0
        for v in self._all_gather(value):
            total += v
        return total

    def maximum(self, value: float) -> float:
        return max(self._all_gather(value))

    def gather_planes(self, planes: np.ndarray, counts: List[int]) -> np.ndarray:
        """All ranks' planes (counts[r] planes from rank r) concatenated in
        rank order, on every rank."""
        import torch
        width = max(counts)
        buf = np.zeros((width,) + planes.shape[1:])
        buf[:planes.shape[0]] = planes
        out = [torch.zeros(buf.shape, dtype=torch.float64) for _ in range(self.size)]
        self.dist.all_gather(out, torch.from_numpy(buf))
        return np.concatenate([o.numpy()[:counts[r]] for r, o in enumerate(out)], axis=0)


# ---------------------------------------------------------------------------
# Reductions (global_dot / global_norm, src/solver_krylov.cpp:631-711)


def _neumaier(values: np.ndarray) -> float:
    total = 0.0
    correction = 0.0
    for v in values.reshape(-1).tolist():
        nxt = total + v
        if abs(total) >= abs(v):
            correction += (total - nxt) + v
        else:
            correction += (v - nxt) + total
        total = nxt
    return total + correction


def global_dot(comm, a: np.ndarray, b: np.ndarray) -> float:
    return comm.sum_in_rank_order(_neumaier(a * b))


def global_norm(comm, v: np.ndarray) -> float:
    scale = comm.maximum(float(np.max(np.abs(v))) if v.size else 0.0)
    if scale == 0.0:
        return 0.0
    s = v / scale
    return scale * float(np.sqrt(comm.sum_in_rank_order(_neumaier(s * s))))


# ---------------------------------------------------------------------------
# Levels


@dataclasses.dataclass
class SlabLevel:
    """One MG level on this rank: owned planes [k0, k1) of nz (global),
    coefficients of those planes, vectors with one ghost plane each side."""

    n: tuple                      # global (nx, ny, nz)
    k0: int
    k1: int
    line_mask: int
    coarsen_mask: int
    chebyshev: bool
    replicated: bool              # every rank holds and relaxes all planes
    diag: np.ndarray
    fx: np.ndarray
    fy: np.ndarray
    fz: np.ndarray                # planes k0..k1 (k1 - k0 + 1)
    vol: np.ndarray
    counts: List[int] = dataclasses.field(default_factory=list)

    @property
    def nzl(self):
        return self.k1 - self.k0

    def zeros(self):
        nx, ny, _ = self.n
        return np.zeros((self.nzl + 2, ny, nx))


def _partitioned_depth(nz_levels, size):
    """How many leading levels are partitioned: the most that leaves the
    coarsest level replicated, keeps at least one plane per rank on every
    partitioned level and lets the finest slabs sit on multiples of 2^m (m
    z-coarsenings between partitioned levels)."""
    best = 0
    for depth in range(1, len(nz_levels)):
        # restriction out of every partitioned level stays on its rank,
        # including the one into the first replicated level
        m = sum(1 for l in range(depth) if nz_levels[l + 1] < nz_levels[l])
        unit = 1 << m
        if nz_levels[0] % (unit * size) != 0 or nz_levels[depth - 1] < size:
            break
        best = depth
    return best


def _partition(nz_fine, size, zcoarsen):
    """Owned fine planes per rank: equal slabs on multiples of 2^zcoarsen."""
    unit = 1 << zcoarsen
    blocks = nz_fine // unit
    if nz_fine % unit or blocks < size:
        raise ValueError("slab boundaries must sit on multiples of 2^m")
    base, extra = divmod(blocks, size)
    bounds = [0]
    for r in range(size):
        bounds.append(bounds[-1] + (base + (1 if r < extra else 0)) * unit)
    return bounds


class SlabMg:
    """The unit-scaled MG preconditioner and PCG of hfps_oracle.c on a
    z-slab of the system; ``levels``/``coefficients`` come from the C
    restatement (hierarchy set-up is replicated, the cycle is partitioned)."""

    def __init__(self, system, policy, comm, session):
        self.comm = comm
        self.bc = tuple(system.boundary)
        self.policy = policy
        self.active = None if system.active is None else system.active.astype(bool)
        shapes = session.levels()
        count = len(shapes)
        if any(sh[3] & 4 for sh in shapes):
            raise ValueError("z-line relaxation is not partitioned along z")
        depth = _partitioned_depth([sh[2] for sh in shapes], comm.size)
        partitioned = [l < depth for l in range(count)]
        zc = sum(1 for l in range(depth) if shapes[l + 1][2] < shapes[l][2])
        bounds0 = _partition(shapes[0][2], comm.size, zc)
        self.levels: List[SlabLevel] = []
        bounds = bounds0
        for l, (nx, ny, nz, mask) in enumerate(shapes):
            if l > 0:
                coarsened_z = nz < shapes[l - 1][2]
                if coarsened_z and partitioned[l]:
                    bounds = [b // 2 for b in bounds]
            d, fx, fy, fz, v = session.level_coefficients(l)
            cmask = 0
            if l + 1 < count:
                nxt = shapes[l + 1]
                cmask = (1 if nxt[0] < nx else 0) | (2 if nxt[1] < ny else 0) | \
                        (4 if nxt[2] < nz else 0)
            rep = not partitioned[l]
            k0, k1 = (0, nz) if rep else (bounds[comm.rank], bounds[comm.rank + 1])
            counts = [nz] * comm.size if rep else [bounds[r + 1] - bounds[r]
                                                   for r in range(comm.size)]
            cheb = l + 1 < count and mask == 0 and policy.smoother == 1
            self.levels.append(SlabLevel((nx, ny, nz), k0, k1, mask, cmask, cheb, rep,
                                         d[k0:k1], fx[k0:k1], fy[k0:k1], fz[k0:k1 + 1],
                                         v[k0:k1], counts))
        self.vec = {}  # level -> dict of x, b, r, t

    # -- halo planes -------------------------------------------------------

    def _fill_halo(self, L: SlabLevel, xg: np.ndarray):
        """Ghost planes of xg: the neighbours' owned planes inside the
        domain; at a physical z face the boundary rule (Neumann: the cell
        itself, Dirichlet: 0)."""
        if L.replicated:
            lo = hi = None
        else:
            lo, hi = self.comm.exchange(xg[1], xg[-2])
        if L.k0 == 0:
            xg[0] = xg[1] if self.bc[4] == NEUMANN else 0.0
        else:
            xg[0] = lo
        if L.k1 == L.n[2]:
            xg[-1] = xg[-2] if self.bc[5] == NEUMANN else 0.0
        else:
            xg[-1] = hi

    def _nbr(self, xg, axis, direction):
        """Neighbour values of the owned cells along x (0) or y (1), with the
        boundary rule at the domain faces; z neighbours come from the ghost
        planes (already filled)."""
        x = xg[1:-1]
        if axis == 2:
            return xg[2:] if direction > 0 else xg[:-2]
        out = np.empty_like(x)
        code = self.bc[2 * axis + (1 if direction > 0 else 0)]
        ax = 2 - axis  # numpy axis
        src = [slice(None)] * 3
        dst = [slice(None)] * 3
        edge = [slice(None)] * 3
        n = x.shape[ax]
        if direction > 0:
            dst[ax], src[ax], edge[ax] = slice(0, n - 1), slice(1, n), slice(n - 1, n)
        else:
            dst[ax], src[ax], edge[ax] = slice(1, n), slice(0, n - 1), slice(0, 1)
        out[tuple(dst)] = x[tuple(src)]
        out[tuple(edge)] = x[tuple(edge)] if code == NEUMANN else 0.0
        return out

    def _row_value(self, L, xg):
        """D x - sum c_f x_nb in point_row_value's order (xg halo-filled)."""
        x = xg[1:-1]
        v = L.diag * x
        v = v - L.fx[:, :, :-1] * self._nbr(xg, 0, -1)
        v = v - L.fx[:, :, 1:] * self._nbr(xg, 0, 1)
        v = v - L.fy[:, :-1, :] * self._nbr(xg, 1, -1)
        v = v - L.fy[:, 1:, :] * self._nbr(xg, 1, 1)
        v = v - L.fz[:-1] * self._nbr(xg, 2, -1)
        v = v - L.fz[1:] * self._nbr(xg, 2, 1)
        return v

    def _defect(self, L, xg, b):
        self._fill_halo(L, xg)
        return b - self._row_value(L, xg)

    # -- smoothers ------------------------------------------------------

    def _chebyshev(self, L, V, stages, retain):
        beta = OMEGA_CHEB_BETA
        alpha = self.policy.chebyshev_fraction * beta
        theta = (beta + alpha) * 0.5
        delta = (beta - alpha) * 0.5
        sigma = theta / delta
        previous_rho = 1.0 / sigma
        current, nxt = V["x"], V["t"]
        for s in range(stages):
            rho = 0.0 if s == 0 else 1.0 / (2.0 * sigma - previous_rho)
            previous_factor = 0.0 if s == 0 else rho * previous_rho
            residual_factor = 1.0 / theta if s == 0 else 2.0 * rho / delta
            if s != 0:
                previous_rho = rho
            defect = self._defect(L, current, V["b"])
            scaled = residual_factor * defect / L.diag
            direction = scaled if s == 0 else previous_factor * V["r"] + scaled
            V["r"] = direction
            nxt[1:-1] = current[1:-1] + direction
            current, nxt = nxt, current
        V["x"], V["t"] = current, nxt
        if retain:
            V["r"] = self._defect(L, V["x"], V["b"])

    def _red_black(self, L, V, sweeps, reverse, retain):
        """point_smooth's red-black branch (fused_point_color_update,
        omega 0.72): x += omega (b - A x) / D on one colour of (i + j + k)."""
        nx, ny, _ = L.n
        kk = np.arange(L.k0, L.k1)[:, None, None]
        jj = np.arange(ny)[None, :, None]
        ii = np.arange(nx)[None, None, :]
        parity = (ii + jj + kk) & 1
        first = 1 if reverse else 0
        for _ in range(sweeps):
            for p in range(2):
                colour = (first + p) & 1
                xg = V["x"]
                self._fill_halo(L, xg)
                value = self._row_value(L, xg)
                update = xg[1:-1] + 0.72 * (V["b"] - value) / L.diag
                xg[1:-1] = np.where(parity == colour, update, xg[1:-1])
        if retain:
            V["r"] = self._defect(L, V["x"], V["b"])

    def _line_pass(self, L, V, axis, colour):
        """One zebra colour of line relaxation along x (0) or y (1): every
        line of that colour solved by the Thomas recurrence of line_solve
        (hfps_oracle.c), vectorised across lines."""
        xg = V["x"]
        self._fill_halo(L, xg)
        nx, ny, _ = L.n
        x = xg[1:-1]
        kk = np.arange(L.k0, L.k1)[:, None, None]
        jj = np.arange(ny)[None, :, None]
        ii = np.arange(nx)[None, None, :]
        # line index pair (a, b): y-lines (i, k), x-lines (j, k)
        a = ii if axis == 1 else jj
        sel = ((a + kk) & 1) == colour
        d = V["b"].copy()
        if axis != 0:
            d = d + L.fx[:, :, :-1] * self._nbr(xg, 0, -1)
            d = d + L.fx[:, :, 1:] * self._nbr(xg, 0, 1)
        if axis != 1:
            d = d + L.fy[:, :-1, :] * self._nbr(xg, 1, -1)
            d = d + L.fy[:, 1:, :] * self._nbr(xg, 1, 1)
        d = d + L.fz[:-1] * self._nbr(xg, 2, -1)
        d = d + L.fz[1:] * self._nbr(xg, 2, 1)
        # move the line axis last
        ax = 2 - axis
        if axis == 1:
            low, high = L.fy[:, :-1, :], L.fy[:, 1:, :]
        else:
            low, high = L.fx[:, :, :-1], L.fx[:, :, 1:]
        D = np.moveaxis(L.diag, ax, -1)
        lo = np.moveaxis(low, ax, -1)
        hi = np.moveaxis(high, ax, -1)
        dd = np.moveaxis(d, ax, -1).copy()
        xs = np.moveaxis(x, ax, -1)
        mask = np.moveaxis(np.broadcast_to(sel, x.shape), ax, -1)[..., 0]
        extent = dd.shape[-1]
        # line-end terms: the neighbour beyond the line's ends
        end_lo = np.moveaxis(self._nbr(xg, axis, -1), ax, -1)[..., 0]
        end_hi = np.moveaxis(self._nbr(xg, axis, 1), ax, -1)[..., -1]
        dd[..., 0] = dd[..., 0] + lo[..., 0] * end_lo
        dd[..., -1] = dd[..., -1] + hi[..., -1] * end_hi
        work = np.empty_like(dd)
        dprime = np.empty_like(dd)
        for s in range(extent):
            a_s = 0.0 if s == 0 else -lo[..., s]
            c_s = 0.0 if s + 1 == extent else -hi[..., s]
            if s > 0:
                den = D[..., s] - a_s * work[..., s - 1]
                work[..., s] = c_s / den
                dprime[..., s] = (dd[..., s] - a_s * dprime[..., s - 1]) / den
            else:
                work[..., s] = c_s / D[..., s]
                dprime[..., s] = dd[..., s] / D[..., s]
        new = np.empty_like(dd)
        new[..., -1] = dprime[..., -1]
        for s in range(extent - 2, -1, -1):
            new[..., s] = dprime[..., s] - work[..., s] * new[..., s + 1]
        xs[mask] = new[mask]

    def _smooth(self, L, V, sweeps, reverse, retain, x_zero=False):
        if L.line_mask == 0:
            if L.chebyshev:
                self._chebyshev(L, V, sweeps, retain)
            else:
                self._red_black(L, V, sweeps, reverse, retain)
            return
        axes = [a for a in (0, 1) if L.line_mask & (1 << a)]
        if reverse:
            axes = axes[::-1]
        first = 1 if reverse else 0
        for axis in axes:
            for _ in range(sweeps):
                for p in range(2):
                    self._line_pass(L, V, axis, (first + p) & 1)

    # -- transfers --------------------------------------------------------

    def _restrict(self, F, VF, C, VC):
        """restrict_residual: coarse b = sum of the children's r (local), coarse
        x = 0; a replicated coarse level gathers the slabs' sums first."""
        mx, my, mz = F.coarsen_mask & 1, F.coarsen_mask & 2, F.coarsen_mask & 4
        r = VF["r"]
        nx, ny, _ = F.n
        cnx, cny, _ = C.n
        cnz_local = (F.nzl + 1) // 2 if mz else F.nzl
        out = np.zeros((cnz_local, cny, cnx))
        for dz in range(2 if mz else 1):
            for dy in range(2 if my else 1):
                for dx in range(2 if mx else 1):
                    zs = slice(dz, None, 2) if mz else slice(None)
                    ys = slice(dy, None, 2) if my else slice(None)
                    xs = slice(dx, None, 2) if mx else slice(None)
                    part = r[zs, ys, xs]
                    pad = np.zeros_like(out)
                    pad[:part.shape[0], :part.shape[1], :part.shape[2]] = part
                    out = out + pad
        if C.replicated and not F.replicated:
            out = self.comm.gather_planes(out, [c // 2 if mz else c for c in F.counts])
        VC["b"] = out
        VC["x"] = C.zeros()

    def _interp(self, fine, coarsened, extent):
        if not coarsened:
            return fine, fine, np.zeros(fine.shape)
        parent = fine // 2
        even = (fine & 1) == 0
        left = np.where(even, parent - 1, parent)
        right = np.where(even, parent, parent + 1)
        weight = np.where(even, 0.75, 0.25)
        low = left < 0
        high = right >= extent
        left = np.where(low, 0, np.where(high, extent - 1, left))
        right = np.where(low, 0, np.where(high, extent - 1, right))
        weight = np.where(low | high, 0.0, weight)
        return left, right, weight

    def _prolongate(self, F, VF, C, VC):
        """prolongate_add: fine x += trilinear coarse x (0 on solid cells)."""
        mx, my, mz = F.coarsen_mask & 1, F.coarsen_mask & 2, F.coarsen_mask & 4
        cx = VC["x"]
        if not C.replicated:
            self._fill_halo(C, cx)
            c_base = C.k0 - 1          # global plane of cx[0]
        else:
            c_base = -1
        nx, ny, _ = F.n
        cnx, cny, cnz = C.n
        kf = np.arange(F.k0, F.k1)
        zl, zr, zw = self._interp(kf, mz, cnz)
        yl, yr, yw = self._interp(np.arange(ny), my, cny)
        xl, xr, xw = self._interp(np.arange(nx), mx, cnx)
        value = np.zeros((F.nzl, ny, nx))
        for az in range(2):
            gz = zl if az == 0 else zr
            wz = (1.0 - zw) if az == 0 else zw
            zon = np.ones(F.nzl, bool) if az == 0 else zl != zr
            for ay in range(2):
                gy = yl if ay == 0 else yr
                wy = (1.0 - yw) if ay == 0 else yw
                yon = np.ones(ny, bool) if ay == 0 else yl != yr
                for ax in range(2):
                    gx = xl if ax == 0 else xr
                    wx = (1.0 - xw) if ax == 0 else xw
                    xon = np.ones(nx, bool) if ax == 0 else xl != xr
                    term = ((wx[None, None, :] * wy[None, :, None]) * wz[:, None, None]) * \
                        cx[(gz - c_base)[:, None, None], gy[None, :, None], gx[None, None, :]]
                    on = zon[:, None, None] & yon[None, :, None] & xon[None, None, :]
                    value = np.where(on, value + term, value)
        x = VF["x"][1:-1]
        VF["x"][1:-1] = np.where(F.vol == 0.0, 0.0, x + value)

    # -- cycle --------------------------------------------------------------

    def _vectors(self, l):
        L = self.levels[l]
        if l not in self.vec:
            self.vec[l] = {"x": L.zeros(), "t": L.zeros(), "b": np.zeros((L.nzl,) + L.n[1::-1]),
                           "r": np.zeros((L.nzl,) + L.n[1::-1])}
        return self.vec[l]

    def _cycle(self, l, counter):
        L = self.levels[l]
        V = self._vectors(l)
        if l + 1 == len(self.levels):
            self._smooth(L, V, self.policy.coarse_sweeps, False, False)
            return
        self._smooth(L, V, self.policy.pre, False, True)
        if L.line_mask != 0:
            V["r"] = self._defect(L, V["x"], V["b"])
        C = self.levels[l + 1]
        VC = self._vectors(l + 1)
        self._restrict(L, V, C, VC)
        self._cycle(l + 1, counter)
        if counter > 1:
            self._cycle(l + 1, counter - 1)
        self._prolongate(L, V, C, VC)
        self._smooth(L, V, self.policy.post, True, False)

    def apply_mg(self, r_local):
        """Unit-scaled MG correction of this rank's slab of r."""
        L = self.levels[0]
        V = self._vectors(0)
        act = self._active_slab()
        V["x"] = L.zeros()
        V["t"] = L.zeros()
        V["b"] = np.where(act, r_local, 0.0)
        self._cycle(0, 2 if self.policy.cycle == 1 else 1)
        return np.where(act, V["x"][1:-1] * 1.0, 0.0)

    def _active_slab(self):
        L = self.levels[0]
        if self.active is None:
            return np.ones((L.nzl,) + L.n[1::-1], bool)
        return self.active[L.k0:L.k1]

    def apply_operator(self, x_local):
        L = self.levels[0]
        xg = L.zeros()
        xg[1:-1] = x_local
        self._fill_halo(L, xg)
        return self._row_value(L, xg)

    # -- PCG (solve_pcg, src/solver_krylov.cpp:1299-1555) ------------------

    def solve(self, rhs_local, x_local=None, rtol=1e-10, atol=0.0, maxit=400,
              true_residual_interval=4):
        comm = self.comm
        x = np.zeros_like(rhs_local) if x_local is None else x_local.copy()
        bnorm = global_norm(comm, rhs_local)
        tol = max(atol, rtol * bnorm)
        info = {"rhs_norm": bnorm, "limit": tol, "iterations": 0}
        if bnorm == 0.0:
            info.update(termination="zero_rhs", final_true_residual=0.0)
            return np.zeros_like(x), info

        def true_residual():
            r_ = 1.0 * rhs_local + -1.0 * self.apply_operator(x)
            return r_, global_norm(comm, r_)

        r, initial = true_residual()
        final = initial
        info["initial_true_residual"] = initial
        if initial <= tol:
            info.update(termination="converged", final_true_residual=final)
            return x, info
        z = self.apply_mg(r)
        rho = global_dot(comm, r, z)
        p = z.copy()
        it = 0
        termination = "maximum_iterations"
        while it < maxit:
            ap = self.apply_operator(p)
            denominator = global_dot(comm, p, ap)
            if not (denominator > 0.0):
                termination = "breakdown"
                break
            alpha = rho / denominator
            x = x + alpha * p
            r = r + -alpha * ap
            it += 1
            recursive = global_norm(comm, r)
            if recursive <= tol or it % true_residual_interval == 0 or it == maxit:
                r, final = true_residual()
                if final <= tol:
                    termination = "converged"
                    break
                if it == maxit:
                    break
                z = self.apply_mg(r)
                rho = global_dot(comm, r, z)
                p = z.copy()
                continue
            z = self.apply_mg(r)
            rho_next = global_dot(comm, r, z)
            beta = rho_next / rho
            p = 1.0 * z + beta * p
            rho = rho_next
        info.update(iterations=it, termination=termination, final_true_residual=final)
        return x, info
