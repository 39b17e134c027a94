// Device bodies of the multigrid phases (kernels.cu, kernels_line.cu): one
// definition per cell or line update, with the reference's arithmetic in the
// reference's order.  `Ld` says how vectors are read (PlainLoad or RoLoad,
// hfps_device.cuh).
#pragma once

#include "hfps_device.cuh"

namespace hfps {

// ---------------------------------------------------------------------------
// Line relaxation building blocks (kernels_line.cu).

__host__ __device__ __forceinline__ int line_extent(int axis, int nx, int ny,
                                                    int nz) {
  return axis == 0 ? nx : (axis == 1 ? ny : nz);
}

// Cells of one line: c = base + s * stride.
template <class T>
__device__ __forceinline__ void line_geometry(const Level<T>& L, int axis,
                                              int fa, int fb, int& base,
                                              int& stride) {
  if (axis == 0) {
    base = L.nx * (fa + L.ny * fb);
    stride = 1;
  } else if (axis == 1) {
    base = fa + L.nx * L.ny * fb;
    stride = L.nx;
  } else {
    base = fa + L.nx * fb;
    stride = L.nx * L.ny;
  }
}

// The line's own off-diagonal faces at cell c (row s).
template <class T>
__device__ __forceinline__ void line_faces(const Level<T>& L, int axis, int c,
                                           int j, int k, T& lowf, T& highf) {
  if (axis == 0) {
    const int f = face_x_index(L, c, j, k);
    lowf = L.fx[f];
    highf = L.fx[f + 1];
  } else if (axis == 1) {
    const int f = face_y_index(L, c, k);
    lowf = L.fy[f];
    highf = L.fy[f + L.nx];
  } else {
    lowf = L.fz[c];
    highf = L.fz[c + L.nx * L.ny];
  }
}

__device__ __forceinline__ void line_cell(int axis, int fa, int fb, int s,
                                          int& i, int& j, int& k) {
  i = axis == 0 ? s : fa;
  j = axis == 0 ? fa : (axis == 1 ? s : fb);
  k = axis == 2 ? s : fb;
}

// Right-hand side of row s of a line: rhs plus the transverse neighbours and
// the line-end boundary terms, in the reference's order (line_row's d).
template <class T, int AXIS, class Ld = PlainLoad>
__device__ __forceinline__ T line_rhs(const Level<T>& L, const T* x,
                                      const T* rhs, int fa, int fb, int s,
                                      int extent, int c) {
  int i, j, k;
  line_cell(AXIS, fa, fb, s, i, j, k);
  const int plane = L.nx * L.ny;
  const int fxi = face_x_index(L, c, j, k);
  const int fyi = face_y_index(L, c, k);
  T d = Ld::get(rhs + c);
  if (AXIS != 0) {
    d += L.fx[fxi] * line_neighbour<T, Ld>(L, x, i, j, k, c, 0, -1);
    d += L.fx[fxi + 1] * line_neighbour<T, Ld>(L, x, i, j, k, c, 0, 1);
  }
  if (AXIS != 1) {
    d += L.fy[fyi] * line_neighbour<T, Ld>(L, x, i, j, k, c, 1, -1);
    d += L.fy[fyi + L.nx] * line_neighbour<T, Ld>(L, x, i, j, k, c, 1, 1);
  }
  if (AXIS != 2) {
    d += L.fz[c] * line_neighbour<T, Ld>(L, x, i, j, k, c, 2, -1);
    d += L.fz[c + plane] * line_neighbour<T, Ld>(L, x, i, j, k, c, 2, 1);
  }
  if (s == 0 || s + 1 == extent) {
    T lowf, highf;
    line_faces(L, AXIS, c, j, k, lowf, highf);
    if (s == 0) d += lowf * line_neighbour<T, Ld>(L, x, i, j, k, c, AXIS, -1);
    if (s + 1 == extent) d += highf * line_neighbour<T, Ld>(L, x, i, j, k, c, AXIS, 1);
  }
  return d;
}

// Factors of one row (2*STEPS multipliers + final diagonal) in registers.
template <class T, int STEPS>
struct PcrRow {
  T k[2 * STEPS + 1];
};

template <class T, int STEPS>
__device__ __forceinline__ void pcr_load(const T* __restrict__ fac, size_t slab,
                                         size_t at, PcrRow<T, STEPS>& r) {
#pragma unroll
  for (int e = 0; e <= 2 * STEPS; ++e) r.k[e] = fac[e * slab + at];
}

// PCR right-hand-side elimination with register-held factors; returns x_s.
// sd is written by the other threads of the line between barriers, so it
// must not be __restrict__-qualified.
template <class T, int STEPS>
__device__ __forceinline__ T pcr_apply(const PcrRow<T, STEPS>& r, T* sd, int s) {
  constexpr int P = 1 << STEPS;
#pragma unroll
  for (int step = 0; step < STEPS; ++step) {
    const int h = 1 << step;
    const int lo = s - h, hi = s + h;
    const T dlo = lo >= 0 ? sd[lo] : T(0);
    const T dhi = hi < P ? sd[hi] : T(0);
    const T nd = sd[s] - dlo * r.k[2 * step] - dhi * r.k[2 * step + 1];
    __syncthreads();
    sd[s] = nd;
    __syncthreads();
  }
  return sd[s] / r.k[2 * STEPS];
}

template <class T, class Ld = PlainLoad>
__device__ __forceinline__ T line_rhs_any(const Level<T>& L, const T* x,
                                          const T* rhs, int axis, int fa,
                                          int fb, int s, int extent, int c) {
  if (axis == 0) return line_rhs<T, 0, Ld>(L, x, rhs, fa, fb, s, extent, c);
  if (axis == 1) return line_rhs<T, 1, Ld>(L, x, rhs, fa, fb, s, extent, c);
  return line_rhs<T, 2, Ld>(L, x, rhs, fa, fb, s, extent, c);
}


// One line slot of a zebra colour pass with PCR (k_line_pcr_factored_color):
// line t of colour `color`, row s of P = 2^STEPS threads, sd the slot's P
// shared-memory values.  Every thread of the CTA calls it (it synchronises
// the CTA); slots past the colour's lines do no memory writes.
template <class T, int STEPS, class Ld = PlainLoad>
__device__ __forceinline__ void pcr_line_slot(const Level<T>& L, T* x, const T* rhs,
                                              const T* __restrict__ fac, int axis,
                                              int color, int t, int s, T* sd) {
  constexpr int P = 1 << STEPS;
  const int a_extent = axis == 0 ? L.ny : L.nx;
  const int b_extent = axis == 2 ? L.ny : L.nz;
  const int ha = (a_extent + 1) >> 1;
  const int extent = line_extent(axis, L.nx, L.ny, L.nz);
  const int fb = t / ha;
  const int fa = 2 * (t - fb * ha) + ((fb + color) & 1);
  const bool valid = t < ha * b_extent && fa < a_extent;
  const size_t slab = static_cast<size_t>(a_extent) * b_extent * P;
  const size_t at = static_cast<size_t>(valid ? fa + a_extent * fb : 0) * P + s;
  PcrRow<T, STEPS> r;
  pcr_load(fac, slab, at, r);
  int c = 0;
  T d = T(0);
  if (valid && s < extent) {
    int i, j, k;
    line_cell(axis, fa, fb, s, i, j, k);
    c = i + L.nx * (j + L.ny * k);
    d = line_rhs_any<T, Ld>(L, x, rhs, axis, fa, fb, s, extent, c);
  }
  sd[s] = d;
  __syncthreads();
  const T value = pcr_apply(r, sd, s);
  if (valid && s < extent) x[c] = value;
}

// ---------------------------------------------------------------------------
// Point smoothers (kernels.cu).

// Damped red-black Gauss-Seidel update of colour slot t, omega = 0.72
// (fused_point_color_update, src/solver_mg.cpp:3149-3223).
template <class T, class Ld = PlainLoad>
__device__ __forceinline__ void rb_slot(const Level<T>& L, T* x, const T* b, int color,
                                        int t) {
  const int hx = (L.nx + 1) >> 1;
  const int row = t / hx;
  const int ih = t - row * hx;
  const int k = row / L.ny;
  const int j = row - k * L.ny;
  const int i = 2 * ih + ((j + k + color) & 1);
  if (i >= L.nx) return;
  const int c = i + L.nx * row;
  const T omega = T(0.72);
  const T value = row_value<T, Ld>(L, x, i, j, k, c);
  x[c] = Ld::get(x + c) + omega * (Ld::get(b + c) - value) / L.diag[c];
}

// One Chebyshev-Jacobi stage at cell c (chebyshev_stream_bulk_kernel,
// src/solver_mg.cpp:2464-2490): d = f_prev d + f_res (b - A x)/D, x' = x + d.
template <class T, class Ld = PlainLoad>
__device__ __forceinline__ void chebyshev_cell(const Level<T>& L, const T* x, const T* b,
                                               T* direction, T* next, T previous_factor,
                                               T residual_factor, int first, int c) {
  int i, j, k;
  cell_coords(c, L.nx, L.ny, i, j, k);
  const T value = row_value<T, Ld>(L, x, i, j, k, c);
  const T defect = Ld::get(b + c) - value;
  const T scaled = residual_factor * defect / L.diag[c];
  const T d = first ? scaled : previous_factor * Ld::get(direction + c) + scaled;
  direction[c] = d;
  next[c] = Ld::get(x + c) + d;
}

// ---------------------------------------------------------------------------
// Transfers (kernels.cu).

// Retained defect + restriction at coarse cell (ci, cj, ck)
// (apply_level_defect followed by restrict_residual, src/solver_mg.cpp:
// 3633-3721): the defects of the children summed in dz, dy, dx order.
// MASK >= 0 fixes the coarsening mask at compile time (the child loops then
// unroll, in the same order).
template <class T, class Ld = PlainLoad, class Pos = NaturalPos, int MASK = -1>
__device__ __forceinline__ T defect_restrict_at(const Level<T>& F, const T* x, const T* b,
                                                int mask, int ci, int cj, int ck, Pos pos) {
  const int m = MASK >= 0 ? MASK : mask;
  const int mx = m & 1, my = (m >> 1) & 1, mz = (m >> 2) & 1;
  const int xb = mx ? 2 * ci : ci, yb = my ? 2 * cj : cj, zb = mz ? 2 * ck : ck;
  T sum = T(0);
  for (int dz = 0; dz <= mz; ++dz)
    for (int dy = 0; dy <= my; ++dy)
      for (int dx = 0; dx <= mx; ++dx) {
        const int fi = xb + dx, fj = yb + dy, fk = zb + dz;
        if (fi >= F.nx || fj >= F.ny || fk >= F.nz) continue;
        const int fc = fi + F.nx * (fj + F.ny * fk);
        sum += Ld::get(b + pos(fc, fi, fj, fk)) - row_value<T, Ld>(F, x, fi, fj, fk, fc, pos);
      }
  return sum;
}

__device__ __forceinline__ void interp_axis(int fine, int coarsened,
                                            int extent, int& left, int& right,
                                            double& weight) {
  if (!coarsened) {
    left = right = fine;
    weight = 0.0;
    return;
  }
  const int parent = fine >> 1;
  if ((fine & 1) == 0) {
    left = parent - 1;
    right = parent;
    weight = 0.75;
  } else {
    left = parent;
    right = parent + 1;
    weight = 0.25;
  }
  if (left < 0) {
    left = right = 0;
    weight = 0.0;
  } else if (right >= extent) {
    left = right = extent - 1;
    weight = 0.0;
  }
}

// Trilinear prolongation and add at fine cell c, zero on solid cells
// (prolongate_add, src/solver_mg.cpp:3893-3994); returns the new x_c.
// Weights are formed in double exactly as the reference does and rounded
// once to T.  Branch-free: the up to 2x2x2 coarse candidates are loaded
// unconditionally (a degenerate axis repeats its one index) and the terms
// are added in the reference's order (z outer, x inner) with the absent
// ones skipped by selects, so all loads of a cell are in flight together.
// LdC reads the coarse correction, which is stored in layout CPos; the
// cell's x sits at x[at].
// MASK >= 0 fixes the coarsening mask at compile time, so the terms of an
// axis that is not coarsened (and their loads) drop out.
template <class T, class Ld = PlainLoad, class LdC = PlainLoad, int MASK = -1,
          class CPos = NaturalPos>
__device__ __forceinline__ T prolongate_cell(const Level<T>& F, const T* x, const Level<T>& C,
                                             const T* cx, int mask, int c, int i, int j, int k,
                                             int at, CPos cpos = CPos()) {
  const int m = MASK >= 0 ? MASK : mask;
  const int mx = m & 1, my = (m >> 1) & 1, mz = (m >> 2) & 1;
  const bool fluid = F.fluid[c] != 0;
  const T old = Ld::get(x + at);
  int xi[2], yi[2], zi[2];
  double xw, yw, zw;
  interp_axis(i, mx, C.nx, xi[0], xi[1], xw);
  interp_axis(j, my, C.ny, yi[0], yi[1], yw);
  interp_axis(k, mz, C.nz, zi[0], zi[1], zw);
  const bool two_x = xi[0] != xi[1], two_y = yi[0] != yi[1], two_z = zi[0] != zi[1];
  T term[2][2][2];
#pragma unroll
  for (int az = 0; az < 2; ++az)
#pragma unroll
    for (int ay = 0; ay < 2; ++ay)
#pragma unroll
      for (int ax = 0; ax < 2; ++ax) {
        const double wz = az == 0 ? 1.0 - zw : zw;
        const double wy = ay == 0 ? 1.0 - yw : yw;
        const double wx = ax == 0 ? 1.0 - xw : xw;
        const T w = static_cast<T>(wx * wy * wz);
        term[az][ay][ax] =
            w * LdC::get(cx + cpos(xi[ax] + C.nx * (yi[ay] + C.ny * zi[az]), xi[ax], yi[ay],
                                   zi[az]));
      }
  T value = T(0);
#pragma unroll
  for (int az = 0; az < 2; ++az)
#pragma unroll
    for (int ay = 0; ay < 2; ++ay)
#pragma unroll
      for (int ax = 0; ax < 2; ++ax) {
        const bool on = (az == 0 || two_z) && (ay == 0 || two_y) && (ax == 0 || two_x);
        const T sum = value + term[az][ay][ax];
        value = on ? sum : value;
      }
  return fluid ? old + value : T(0);
}

// ---------------------------------------------------------------------------
// Coarsest level.

// Red-black sweeps of the coarsest level in one CTA (the point branch of
// k_coarse_solve): x/b are already in the working precision and written
// only by this CTA.
template <class TC>
__device__ __forceinline__ void coarse_point_sweeps(const Level<TC>& L, TC* xw, const TC* bw,
                                                    int sweeps, int tid, int nthreads) {
  const TC omega = TC(0.72);
  const int hx = (L.nx + 1) >> 1;
  const int half = hx * L.ny * L.nz;
  for (int s = 0; s < sweeps; ++s) {
    for (int color = 0; color < 2; ++color) {
      for (int t = tid; t < half; t += nthreads) {
        const int row = t / hx;
        const int ih = t - row * hx;
        const int k = row / L.ny;
        const int j = row - k * L.ny;
        const int i = 2 * ih + ((j + k + color) & 1);
        if (i >= L.nx) continue;
        const int c = i + L.nx * row;
        const TC value = row_value(L, xw, i, j, k, c);
        xw[c] += omega * (bw[c] - value) / L.diag[c];
      }
      __syncthreads();
    }
  }
}

// Dense coarsest-level map out = P x + M b (k_coarse_dense): a block of 32
// rows, one per lane; warp w takes every kDenseWarps-th column from w with
// kDenseUnroll column loads in flight, and the row's warp partial sums are
// added in warp order.  With x_zero the P columns are skipped: their terms
// are exact zeros, so the sums are unchanged bit for bit.  v holds x then b
// widened to double; part has kDenseWarps * 32 doubles.  Every thread of
// the CTA calls it.
constexpr int kDenseWarps = 32;
constexpr int kDenseUnroll = 8;

// WARPS: the CTA's warps (kDenseWarps for k_coarse_dense; the persistent
// small-level kernel runs it with fewer).  part has WARPS * 32 doubles; the
// CTA is synchronised again before return, so part may be reused at once.
template <class T, int WARPS = kDenseWarps>
__device__ __forceinline__ void dense_rows(int n, const double* __restrict__ op,
                                           const double* v, double* part, int vblock,
                                           int lane, int warp, bool x_zero, T* out) {
  const int row = min(vblock * 32 + lane, n - 1);
  const int cols = 2 * n;
  int first = warp;
  if (x_zero && n > warp) first += ((n - warp + WARPS - 1) / WARPS) * WARPS;
  double acc = 0.0;
  for (int j0 = first; j0 < cols; j0 += WARPS * kDenseUnroll) {
    double m[kDenseUnroll];
#pragma unroll
    for (int u = 0; u < kDenseUnroll; ++u) {
      const int j = min(j0 + u * WARPS, cols - 1);
      m[u] = __ldg(op + static_cast<size_t>(j) * n + row);
    }
#pragma unroll
    for (int u = 0; u < kDenseUnroll; ++u)
      if (j0 + u * WARPS < cols) acc += m[u] * v[j0 + u * WARPS];
  }
  part[warp * 32 + lane] = acc;
  __syncthreads();
  if (warp == 0 && vblock * 32 + lane < n) {
    double sum = part[lane];
    for (int w = 1; w < WARPS; ++w) sum += part[w * 32 + lane];
    out[vblock * 32 + lane] = static_cast<T>(sum);
  }
  __syncthreads();
}

}  // namespace hfps
