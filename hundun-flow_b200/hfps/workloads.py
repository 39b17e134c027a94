"""Seeded synthetic pressure systems with the shapes of the benchmark cases.

No public dataset exists for this path, so every input is generated here from
a counter-based SplitMix64 stream (own code) mapped to N(0,1) by Box-Muller.
The same arrays feed the CUDA solver, the C restatement and the compiled
reference, so all three see bit-identical systems.

Discretisation (follows the reference's pressure-correction assembly):

* cell beta = 1/rho; interior face coefficient
  c_f = A_f / (d_L/beta_L + d_R/beta_R)  (distance-weighted harmonic mean,
  ``face_pressure_coefficient``, src/solver_piso.cpp:1060-1136);
* Dirichlet boundary face (p'=0 on the face, ghost state = owner state):
  c_f = 2 A_f / (d/beta_o + d/beta_o) with d the owner-centre-to-face distance
  (src/solver_piso.cpp:1095-1110); Neumann boundary face: c_f = 0;
* diagonal = sum of the six face coefficients (no storage term)
  (src/solver_pressure.cpp:223-226);
* IBM solid cells are marked in ``active`` (0 = solid).  The coefficients
  stay unmasked, exactly as the reference's regular operator receives them;
  the solver removes every fluid/solid face (src/solver_ibm_pressure.cpp:
  347-385) and makes solid rows identities;
* rhs = -(sum over the cell's faces of the outward flux u_f A_f) for a face
  velocity field u_f ~ N(0,1), zeroed on Neumann faces and on faces that
  touch a solid cell; solid rows get rhs 0 (``mask_solid_rhs``,
  src/solver_ibm_pressure.cpp:387-403).

Arrays are numpy float64 in x-fastest order: a cell field has shape
(nz, ny, nx); x-faces (nz, ny, nx+1); y-faces (nz, ny+1, nx); z-faces
(nz+1, ny, nx).
"""
from __future__ import annotations

import dataclasses
import math
from typing import Dict, Optional, Sequence, Tuple

import numpy as np

DIRICHLET = 0
NEUMANN = 1

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def _splitmix64(counter: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        z = counter * _GOLDEN + _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        return z ^ (z >> np.uint64(31))


def normals(seed: int, count: int, offset: int = 0) -> np.ndarray:
    """``count`` N(0,1) deviates of stream ``seed`` starting at ``offset``.

    Deviate i uses the uniform pair (2i, 2i+1) of the stream, so any slice
    of the stream can be regenerated independently.
    """
    with np.errstate(over="ignore"):
        base = np.uint64((seed * 0x632BE59BD9B4E019 + 0x1234567) & 0xFFFFFFFFFFFFFFFF)
        index = np.arange(offset, offset + count, dtype=np.uint64)
        a = _splitmix64(base + np.uint64(2) * index)
        b = _splitmix64(base + np.uint64(2) * index + np.uint64(1))
    u1 = ((a >> np.uint64(11)).astype(np.float64) + 1.0) * (1.0 / 9007199254740992.0)
    u2 = (b >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * math.pi * u2)


def uniform_faces(n: int, length: float = 1.0) -> np.ndarray:
    return np.linspace(0.0, length, n + 1)


def stretched_faces(n: int, ratio: float) -> np.ndarray:
    """Geometric faces on [0,1] with widths growing by ``ratio`` from 0."""
    h0 = (ratio - 1.0) / (ratio ** n - 1.0)
    j = np.arange(n + 1, dtype=np.float64)
    faces = h0 * (ratio ** j - 1.0) / (ratio - 1.0)
    faces[-1] = 1.0
    return faces


@dataclasses.dataclass
class PressureSystem:
    """One pressure-correction system: geometry, coefficients, mask, rhs."""

    name: str
    shape: Tuple[int, int, int]  # (nx, ny, nz)
    faces: Tuple[np.ndarray, np.ndarray, np.ndarray]
    boundary: Tuple[int, int, int, int, int, int]
    beta: np.ndarray
    diagonal: np.ndarray
    face_x: np.ndarray
    face_y: np.ndarray
    face_z: np.ndarray
    active: Optional[np.ndarray]
    rhs: np.ndarray
    meta: Dict[str, object] = dataclasses.field(default_factory=dict)

    @property
    def cells(self) -> int:
        nx, ny, nz = self.shape
        return nx * ny * nz

    def centres(self):
        return tuple(0.5 * (f[1:] + f[:-1]) for f in self.faces)

    def widths(self):
        return tuple(np.diff(f) for f in self.faces)


def _face_coefficients(beta: np.ndarray, faces, boundary):
    """Distance-weighted harmonic face coefficients on all three axes."""
    nz, ny, nx = beta.shape
    wx, wy, wz = (np.diff(f) for f in faces)
    cx_, cy_, cz_ = (0.5 * (f[1:] + f[:-1]) for f in faces)
    inv = 1.0 / beta
    out = []
    for axis, (w, c, f) in enumerate(((wx, cx_, faces[0]), (wy, cy_, faces[1]), (wz, cz_, faces[2]))):
        n = len(w)
        # area of the face normal to `axis`: product of the other two widths
        if axis == 0:
            area = (wz[:, None] * wy[None, :])[:, :, None]
        elif axis == 1:
            area = (wz[:, None] * wx[None, :])[:, None, :]
        else:
            area = (wy[:, None] * wx[None, :])[None, :, :]
        inv_m = np.moveaxis(inv, 2 - axis, -1)  # axis last
        dl = f[1:-1] - c[:-1]
        dr = c[1:] - f[1:-1]
        interior = 1.0 / (dl * inv_m[..., :-1] + dr * inv_m[..., 1:])
        lo_d = c[0] - f[0]
        hi_d = f[-1] - c[-1]
        lo = 2.0 / (lo_d * inv_m[..., :1] + lo_d * inv_m[..., :1])
        hi = 2.0 / (hi_d * inv_m[..., -1:] + hi_d * inv_m[..., -1:])
        if boundary[2 * axis] == NEUMANN:
            lo = np.zeros_like(lo)
        if boundary[2 * axis + 1] == NEUMANN:
            hi = np.zeros_like(hi)
        coef = np.concatenate([lo, interior, hi], axis=-1)
        coef = np.moveaxis(coef, -1, 2 - axis)
        out.append(np.ascontiguousarray(coef * area))
    return out


def _diagonal(fx, fy, fz):
    return (fx[:, :, :-1] + fx[:, :, 1:] + fy[:, :-1, :] + fy[:, 1:, :]
            + fz[:-1, :, :] + fz[1:, :, :])


def face_activity(active: Optional[np.ndarray], shape):
    """Face is active iff every adjacent cell is active (fluid)."""
    nx, ny, nz = shape
    if active is None:
        return (np.ones((nz, ny, nx + 1), np.uint8), np.ones((nz, ny + 1, nx), np.uint8),
                np.ones((nz + 1, ny, nx), np.uint8))
    a = active.astype(bool)
    ax = np.ones((nz, ny, nx + 1), bool)
    ax[:, :, :-1] &= a
    ax[:, :, 1:] &= a
    ay = np.ones((nz, ny + 1, nx), bool)
    ay[:, :-1, :] &= a
    ay[:, 1:, :] &= a
    az = np.ones((nz + 1, ny, nx), bool)
    az[:-1, :, :] &= a
    az[1:, :, :] &= a
    return ax.astype(np.uint8), ay.astype(np.uint8), az.astype(np.uint8)


def flux_divergence_rhs(seed: int, faces, boundary, active, scale: float = 1.0):
    """-(outward FV flux sum) of a seeded N(0,1) face velocity field."""
    nx, ny, nz = (len(f) - 1 for f in faces)
    wx, wy, wz = (np.diff(f) for f in faces)
    n_x = (nx + 1) * ny * nz
    n_y = nx * (ny + 1) * nz
    n_z = nx * ny * (nz + 1)
    u = normals(seed, n_x + n_y + n_z)
    ux = u[:n_x].reshape(nz, ny, nx + 1) * (wz[:, None, None] * wy[None, :, None])
    uy = u[n_x:n_x + n_y].reshape(nz, ny + 1, nx) * (wz[:, None, None] * wx[None, None, :])
    uz = u[n_x + n_y:].reshape(nz + 1, ny, nx) * (wy[None, :, None] * wx[None, None, :])
    ax, ay, az = face_activity(active, (nx, ny, nz))
    ux = ux * ax
    uy = uy * ay
    uz = uz * az
    if boundary[0] == NEUMANN:
        ux[:, :, 0] = 0.0
    if boundary[1] == NEUMANN:
        ux[:, :, -1] = 0.0
    if boundary[2] == NEUMANN:
        uy[:, 0, :] = 0.0
    if boundary[3] == NEUMANN:
        uy[:, -1, :] = 0.0
    if boundary[4] == NEUMANN:
        uz[0, :, :] = 0.0
    if boundary[5] == NEUMANN:
        uz[-1, :, :] = 0.0
    outward = (ux[:, :, 1:] - ux[:, :, :-1] + uy[:, 1:, :] - uy[:, :-1, :]
               + uz[1:, :, :] - uz[:-1, :, :])
    rhs = -scale * outward
    if active is not None:
        rhs = rhs * active
    return np.ascontiguousarray(rhs)


def _tanh_front(value):
    return 1.0 + 6.0 * 0.5 * (1.0 + np.tanh(value))


def _build(name, faces, rho, solid, boundary, seed, meta=None) -> PressureSystem:
    shape = tuple(len(f) - 1 for f in faces)
    beta = 1.0 / rho
    fx, fy, fz = _face_coefficients(beta, faces, boundary)
    active = None if solid is None else np.ascontiguousarray((~solid).astype(np.uint8))
    rhs = flux_divergence_rhs(seed, faces, boundary, active)
    return PressureSystem(name, shape, tuple(faces), tuple(boundary), beta,
                          np.ascontiguousarray(_diagonal(fx, fy, fz)), fx, fy, fz,
                          active, rhs, dict(meta or {}))


def _grid(faces):
    cx, cy, cz = (0.5 * (f[1:] + f[:-1]) for f in faces)
    return cz[:, None, None], cy[None, :, None], cx[None, None, :]


PISO_BOUNDARY = (NEUMANN, DIRICHLET, NEUMANN, NEUMANN, NEUMANN, NEUMANN)


def spherical_flame(n: Sequence[int] = (64, 64, 64), thickness: float = 0.02,
                    spheres=((0.3, 0.5, 0.5, 0.1),), seed: int = 0,
                    name: str = "spherical_flame", boundary=PISO_BOUNDARY) -> PressureSystem:
    """Density-ratio-7 spherical flame with solid IBM spheres (64^3 case).
    ``boundary`` all NEUMANN gives a singular, consistent system (constant
    null space)."""
    nx, ny, nz = n
    faces = (uniform_faces(nx), uniform_faces(ny), uniform_faces(nz))
    z, y, x = _grid(faces)
    r = np.sqrt((x - 0.5) ** 2 + (y - 0.5) ** 2 + (z - 0.5) ** 2)
    rho = _tanh_front((r - 0.25) / thickness) * np.ones((nz, ny, nx))
    solid = np.zeros((nz, ny, nx), bool)
    for (sx, sy, sz, sr) in spheres:
        solid |= (x - sx) ** 2 + (y - sy) ** 2 + (z - sz) ** 2 <= sr * sr
    return _build(name, faces, rho, solid, tuple(boundary), seed,
                  {"thickness": thickness, "spheres": spheres})


def wrinkled_flame(n: Sequence[int] = (256, 256, 256), stretch_y: Optional[float] = 1.02,
                   seed: int = 0, name: str = "wrinkled_flame") -> PressureSystem:
    """Wrinkled flame front with a solid z-cylinder (256^3, y-stretched case)."""
    nx, ny, nz = n
    fy = stretched_faces(ny, stretch_y) if stretch_y else uniform_faces(ny)
    faces = (uniform_faces(nx), fy, uniform_faces(nz))
    z, y, x = _grid(faces)
    front = (x - 0.4 - 0.05 * np.sin(8.0 * math.pi * y) * np.sin(8.0 * math.pi * z)) / 0.01
    rho = _tanh_front(front) * np.ones((nz, ny, nx))
    solid = np.broadcast_to((x - 0.2) ** 2 + (y - 0.5) ** 2 <= 0.08 * 0.08, (nz, ny, nx)).copy()
    return _build(name, faces, rho, solid, PISO_BOUNDARY, seed, {"stretch_y": stretch_y})


def warm_start_rhs(system: PressureSystem, index: int, amplitude: float = 0.05) -> np.ndarray:
    """rhs of solve ``index`` (1..20) of a PISO warm-start sequence:
    b_k = b_0 + amplitude * div(fresh noise with seed k)."""
    extra = flux_divergence_rhs(index, system.faces, system.boundary, system.active, amplitude)
    return np.ascontiguousarray(system.rhs + extra)


def _logical_shift(t, bits: int):
    """Unsigned right shift of int64 tensors holding uint64 bit patterns."""
    return (t >> bits) & ((1 << (64 - bits)) - 1)


def _splitmix64_torch(counter):
    import torch
    golden = -7046029254386353131  # 0x9E3779B97F4A7C15 as int64
    m1 = -4658895280553007687      # 0xBF58476D1CE4E5B9
    m2 = -7723592293110705685      # 0x94D049BB133111EB
    z = counter * golden + golden
    z = (z ^ _logical_shift(z, 30)) * m1
    z = (z ^ _logical_shift(z, 27)) * m2
    return z ^ _logical_shift(z, 31)


def normals_torch(seed: int, count: int, offset: int = 0, device="cuda"):
    """Same stream as ``normals`` computed with torch int64 arithmetic
    (two's-complement wrap-around equals uint64 arithmetic bit for bit)."""
    import torch
    base = (seed * 0x632BE59BD9B4E019 + 0x1234567) & 0xFFFFFFFFFFFFFFFF
    if base >= 1 << 63:
        base -= 1 << 64
    index = torch.arange(offset, offset + count, dtype=torch.int64, device=device)
    a = _splitmix64_torch(base + 2 * index)
    b = _splitmix64_torch(base + 2 * index + 1)
    u1 = (_logical_shift(a, 11).to(torch.float64) + 1.0) * (1.0 / 9007199254740992.0)
    u2 = _logical_shift(b, 11).to(torch.float64) * (1.0 / 9007199254740992.0)
    return torch.sqrt(-2.0 * torch.log(u1)) * torch.cos(2.0 * math.pi * u2)


def flux_divergence_rhs_torch(seed: int, faces, boundary, active, scale: float = 1.0,
                              device="cuda"):
    """``flux_divergence_rhs`` on the GPU (same values up to the last ulp of
    log/cos); returns a flat float64 CUDA tensor."""
    import torch
    nx, ny, nz = (len(f) - 1 for f in faces)
    w = [torch.as_tensor(np.diff(f), dtype=torch.float64, device=device) for f in faces]
    wx, wy, wz = w
    n_x = (nx + 1) * ny * nz
    n_y = nx * (ny + 1) * nz
    n_z = nx * ny * (nz + 1)
    u = normals_torch(seed, n_x + n_y + n_z, device=device)
    ux = u[:n_x].reshape(nz, ny, nx + 1) * (wz[:, None, None] * wy[None, :, None])
    uy = u[n_x:n_x + n_y].reshape(nz, ny + 1, nx) * (wz[:, None, None] * wx[None, None, :])
    uz = u[n_x + n_y:].reshape(nz + 1, ny, nx) * (wy[None, :, None] * wx[None, None, :])
    if active is not None:
        ax, ay, az = (torch.as_tensor(t, device=device).to(torch.float64)
                      for t in face_activity(active, (nx, ny, nz)))
        ux, uy, uz = ux * ax, uy * ay, uz * az
    if boundary[0] == NEUMANN:
        ux[:, :, 0] = 0.0
    if boundary[1] == NEUMANN:
        ux[:, :, -1] = 0.0
    if boundary[2] == NEUMANN:
        uy[:, 0, :] = 0.0
    if boundary[3] == NEUMANN:
        uy[:, -1, :] = 0.0
    if boundary[4] == NEUMANN:
        uz[0, :, :] = 0.0
    if boundary[5] == NEUMANN:
        uz[-1, :, :] = 0.0
    outward = (ux[:, :, 1:] - ux[:, :, :-1] + uy[:, 1:, :] - uy[:, :-1, :]
               + uz[1:, :, :] - uz[:-1, :, :])
    rhs = -scale * outward
    if active is not None:
        rhs = rhs * torch.as_tensor(active, device=device).to(torch.float64)
    return rhs.reshape(-1).contiguous()


CONFIGS = {
    # name: (builder, kwargs)
    "sphere64": (spherical_flame, dict(n=(64, 64, 64))),
    "wrinkled256": (wrinkled_flame, dict(n=(256, 256, 256), stretch_y=1.02)),
    "wrinkled512x256x256": (wrinkled_flame, dict(n=(512, 256, 256), stretch_y=None)),
    "sphere128": (spherical_flame, dict(n=(128, 128, 128))),
    "three_spheres512": (spherical_flame, dict(
        n=(512, 512, 512), thickness=0.005,
        spheres=((0.25, 0.5, 0.5, 0.06), (0.5, 0.3, 0.5, 0.06), (0.5, 0.7, 0.5, 0.06)))),
}


def make(name: str, **overrides) -> PressureSystem:
    builder, kwargs = CONFIGS[name]
    kwargs = dict(kwargs)
    kwargs.update(overrides)
    return builder(name=name, **kwargs)
