// Zebra line relaxation (y-line relaxation for stretched grids) on sm_100a.
//
// The reference relaxes strong-axis lines by lexicographic line Gauss-Seidel
// with one Thomas solve per line (line_smooth_axis, src/solver_mg.cpp:
// 3352-3539).  Here lines are coloured by the parity of their transverse
// index (zebra): a colour's lines couple only to the other colour, so all of
// them are solved at once.  The line matrices depend only on the level
// coefficients, so every factorisation is computed once per coefficient
// update and each sweep does only right-hand-side work:
//   * many lines per colour: the partition method.  Each line is cut into
//     S segments; a warp solves one segment of 32 lines (lanes run across
//     lines, so loads coalesce along x), the S segment solutions are
//     coupled through a 2S x 2S interface system whose inverse is stored
//     per line, and the segment-local Thomas factors and the two spike
//     vectors of every segment are stored per cell;
//   * few lines per colour (coarse levels): one CTA row per line runs
//     parallel cyclic reduction with precomputed elimination factors held
//     in registers;
//   * the coarsest level keeps x and rhs in shared memory for all of its
//     coarse sweeps in one launch.
#include "kernels.hpp"

#include <algorithm>

namespace hfps {
namespace {

constexpr int kLanes = 32;
constexpr int kMaxSegments = 8;
constexpr int kChunk = 4;

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
template <class T, int AXIS>
__device__ __forceinline__ T line_rhs(const Level<T>& L, const T* x,
                                      const T* rhs, int fa, int fb, int s,
                                      int extent, int c) {
  int i, j, k;
  line_cell(AXIS, fa, fb, s, i, j, k);
  const int plane = L.nx * L.ny;
  const int fxi = face_x_index(L, c, j, k);
  const int fyi = face_y_index(L, c, k);
  T d = rhs[c];
  if (AXIS != 0) {
    d += L.fx[fxi] * line_neighbour(L, x, i, j, k, c, 0, -1);
    d += L.fx[fxi + 1] * line_neighbour(L, x, i, j, k, c, 0, 1);
  }
  if (AXIS != 1) {
    d += L.fy[fyi] * line_neighbour(L, x, i, j, k, c, 1, -1);
    d += L.fy[fyi + L.nx] * line_neighbour(L, x, i, j, k, c, 1, 1);
  }
  if (AXIS != 2) {
    d += L.fz[c] * line_neighbour(L, x, i, j, k, c, 2, -1);
    d += L.fz[c + plane] * line_neighbour(L, x, i, j, k, c, 2, 1);
  }
  if (s == 0 || s + 1 == extent) {
    T lowf, highf;
    line_faces(L, AXIS, c, j, k, lowf, highf);
    if (s == 0) d += lowf * line_neighbour(L, x, i, j, k, c, AXIS, -1);
    if (s + 1 == extent) d += highf * line_neighbour(L, x, i, j, k, c, AXIS, 1);
  }
  return d;
}

// ---------------------------------------------------------------------------
// Partition method.
//
// Segment q holds rows [r0, r1].  With its couplings to x_{r0-1} and
// x_{r1+1} moved to the right-hand side, T_q x = d - a_{r0} x_{r0-1} e_0 -
// c_{r1} x_{r1+1} e_m, so x = y - v x_{r0-1} - w x_{r1+1} with y = T_q^-1 d
// and the spikes v = T_q^-1 a_{r0} e_0, w = T_q^-1 c_{r1} e_m.  The first
// and last unknowns F_q, L_q of all segments solve a 2S x 2S system whose
// inverse R is stored per line.
//
// Factor layout is colour-packed so that the 32 lanes of a warp (32 lines
// of one colour, consecutive along the transverse index) read consecutive
// addresses: array e of row s of colour line t sits at
//   ((e * 2 + colour) * extent + s) * colour_lines + t,
// e = 0 local denominator, 1 local c', 2 spike v, 3 spike w, 4 sub-diagonal
// a; and R entry (r, c) of that line at
//   ((r * 2S + c) * 2 + colour) * colour_lines + t.

__host__ __device__ __forceinline__ void segment_rows(int extent, int S, int q,
                                                      int& r0, int& r1) {
  const int m = extent / S;
  r0 = q * m;
  r1 = q + 1 == S ? extent - 1 : r0 + m - 1;
}

__host__ __device__ __forceinline__ int segments_for(int extent) {
  int S = kMaxSegments;
  while (S > 1 && extent / S < 8) S >>= 1;
  return S;
}

constexpr int kSegmentArrays = 5;

struct SegmentLayout {
  int extent;
  int colour_lines;
  __host__ __device__ size_t cell(int e, int colour, int s, int t) const {
    return ((static_cast<size_t>(e) * 2 + colour) * extent + s) * colour_lines + t;
  }
  __host__ __device__ size_t cell_values() const {
    return static_cast<size_t>(kSegmentArrays) * 2 * extent * colour_lines;
  }
  __host__ __device__ size_t rinv(int n2, int r, int c, int colour, int t) const {
    return ((static_cast<size_t>(r) * n2 + c) * 2 + colour) * colour_lines + t;
  }
};

template <class T>
__global__ void k_segment_factors(Level<T> L, int axis, int S, T* __restrict__ fac) {
  const int a_extent = axis == 0 ? L.ny : L.nx;
  const int b_extent = axis == 2 ? L.ny : L.nz;
  const int lines = a_extent * b_extent;
  const int extent = line_extent(axis, L.nx, L.ny, L.nz);
  const int ha = (a_extent + 1) >> 1;
  const SegmentLayout lay{extent, ha * b_extent};
  T* rinv = fac + lay.cell_values();
  const int n2 = 2 * S;
  for (int line = blockIdx.x * blockDim.x + threadIdx.x; line < lines;
       line += gridDim.x * blockDim.x) {
    const int fb = line / a_extent;
    const int fa = line - fb * a_extent;
    const int colour = (fa + fb) & 1;
    const int t = fb * ha + (fa >> 1);
    int base, stride;
    line_geometry(L, axis, fa, fb, base, stride);
    for (int q = 0; q < S; ++q) {
      int r0, r1;
      segment_rows(extent, S, q, r0, r1);
      // Local Thomas factorisation and the forward pass of spike v.
      T prev_cl = T(0), prev_v = T(0), c_last = T(0);
      for (int s = r0; s <= r1; ++s) {
        const int c = base + s * stride;
        int i, j, k;
        line_cell(axis, fa, fb, s, i, j, k);
        T lowf, highf;
        line_faces(L, axis, c, j, k, lowf, highf);
        const T a = s == 0 ? T(0) : -lowf;
        const T cc = s + 1 == extent ? T(0) : -highf;
        const T bb = L.diag[c];
        const T d = s == r0 ? bb : bb - a * prev_cl;
        const T w_local = cc / d;
        const T vp = s == r0 ? a / d : (T(0) - a * prev_v) / d;
        if (s == r1) c_last = cc;
        fac[lay.cell(0, colour, s, t)] = d;
        fac[lay.cell(1, colour, s, t)] = w_local;
        fac[lay.cell(2, colour, s, t)] = vp;
        fac[lay.cell(4, colour, s, t)] = a;
        prev_cl = w_local;
        prev_v = vp;
      }
      // Backward passes: v = v' - c' v_next; w' is zero but for the last row.
      T next_v = T(0), next_w = T(0);
      for (int s = r1; s >= r0; --s) {
        const T cls = fac[lay.cell(1, colour, s, t)];
        const T v = s == r1 ? fac[lay.cell(2, colour, s, t)]
                            : fac[lay.cell(2, colour, s, t)] - cls * next_v;
        const T w = s == r1 ? c_last / fac[lay.cell(0, colour, s, t)] : -cls * next_w;
        fac[lay.cell(2, colour, s, t)] = v;
        fac[lay.cell(3, colour, s, t)] = w;
        next_v = v;
        next_w = w;
      }
    }
    // Interface matrix M u = y_I with u = (F_0, L_0, ..., F_{S-1}, L_{S-1}):
    //   F_q + v_{r0} L_{q-1} + w_{r0} F_{q+1} = y_{r0}
    //   L_q + v_{r1} L_{q-1} + w_{r1} F_{q+1} = y_{r1}
    T m[4 * kMaxSegments * kMaxSegments];
    T inv[4 * kMaxSegments * kMaxSegments];
    for (int e = 0; e < n2 * n2; ++e) {
      m[e] = T(0);
      inv[e] = T(0);
    }
    for (int q = 0; q < S; ++q) {
      int r0, r1;
      segment_rows(extent, S, q, r0, r1);
      const int rf = 2 * q, rl = 2 * q + 1;
      m[rf * n2 + rf] = T(1);
      m[rl * n2 + rl] = T(1);
      if (q > 0) {
        m[rf * n2 + 2 * (q - 1) + 1] += fac[lay.cell(2, colour, r0, t)];
        m[rl * n2 + 2 * (q - 1) + 1] += fac[lay.cell(2, colour, r1, t)];
      }
      if (q + 1 < S) {
        m[rf * n2 + 2 * (q + 1)] += fac[lay.cell(3, colour, r0, t)];
        m[rl * n2 + 2 * (q + 1)] += fac[lay.cell(3, colour, r1, t)];
      }
    }
    for (int e = 0; e < n2; ++e) inv[e * n2 + e] = T(1);
    // Gauss-Jordan with partial pivoting (2S <= 16 unknowns).
    for (int col = 0; col < n2; ++col) {
      int piv = col;
      T best = fabs(static_cast<double>(m[col * n2 + col]));
      for (int r = col + 1; r < n2; ++r) {
        const T mag = fabs(static_cast<double>(m[r * n2 + col]));
        if (mag > best) {
          best = mag;
          piv = r;
        }
      }
      if (piv != col) {
        for (int e = 0; e < n2; ++e) {
          T tmp = m[col * n2 + e]; m[col * n2 + e] = m[piv * n2 + e]; m[piv * n2 + e] = tmp;
          tmp = inv[col * n2 + e]; inv[col * n2 + e] = inv[piv * n2 + e]; inv[piv * n2 + e] = tmp;
        }
      }
      const T p = m[col * n2 + col];
      for (int e = 0; e < n2; ++e) {
        m[col * n2 + e] /= p;
        inv[col * n2 + e] /= p;
      }
      for (int r = 0; r < n2; ++r) {
        if (r == col) continue;
        const T f = m[r * n2 + col];
        if (f == T(0)) continue;
        for (int e = 0; e < n2; ++e) {
          m[r * n2 + e] -= f * m[col * n2 + e];
          inv[r * n2 + e] -= f * inv[col * n2 + e];
        }
      }
    }
    for (int r = 0; r < n2; ++r)
      for (int c = 0; c < n2; ++c) rinv[lay.rinv(n2, r, c, colour, t)] = inv[r * n2 + c];
  }
}

// One zebra colour with the partition method: blockDim = (32 lines, S).
template <class T, int AXIS, int S>
__global__ void __launch_bounds__(32 * S)
    k_line_segment_color(Level<T> L, T* __restrict__ x,
                         const T* __restrict__ rhs, const T* __restrict__ fac,
                         int color) {
  extern __shared__ unsigned char segment_smem[];
  T* Y = reinterpret_cast<T*>(segment_smem);           // [extent][32]
  const int extent = line_extent(AXIS, L.nx, L.ny, L.nz);
  T* UI = Y + static_cast<size_t>(extent) * kLanes;     // [2S][32]
  T* YI = UI + 2 * S * kLanes;                          // [2S][32]
  const int a_extent = AXIS == 0 ? L.ny : L.nx;
  const int b_extent = AXIS == 2 ? L.ny : L.nz;
  const int ha = (a_extent + 1) >> 1;
  const SegmentLayout lay{extent, ha * b_extent};
  const T* rinv = fac + lay.cell_values();
  const int lane = threadIdx.x;
  const int q = threadIdx.y;
  const int t = blockIdx.x * kLanes + lane;
  const int fb = t / ha;
  const int fa = 2 * (t - fb * ha) + ((fb + color) & 1);
  const bool valid = t < ha * b_extent && fa < a_extent;
  int base = 0, stride = 0;
  if (valid) line_geometry(L, AXIS, fa, fb, base, stride);
  int r0, r1;
  segment_rows(extent, S, q, r0, r1);
  const T* den = fac + lay.cell(0, color, 0, t);
  const T* cl = fac + lay.cell(1, color, 0, t);
  const T* vv = fac + lay.cell(2, color, 0, t);
  const T* ww = fac + lay.cell(3, color, 0, t);
  const T* aa = fac + lay.cell(4, color, 0, t);
  const size_t row = static_cast<size_t>(lay.colour_lines);
  // Forward local elimination y' = (d - a y'_prev) / den, loads in chunks.
  if (valid) {
    T prev = T(0);
    for (int s0 = r0; s0 <= r1; s0 += kChunk) {
      T dv[kChunk], av[kChunk], dn[kChunk];
#pragma unroll
      for (int u = 0; u < kChunk; ++u) {
        const int s = s0 + u;
        if (s <= r1) {
          av[u] = aa[s * row];
          dn[u] = den[s * row];
          dv[u] = line_rhs<T, AXIS>(L, x, rhs, fa, fb, s, extent, base + s * stride);
        }
      }
#pragma unroll
      for (int u = 0; u < kChunk; ++u) {
        const int s = s0 + u;
        if (s <= r1) {
          const T v = s == r0 ? dv[u] / dn[u] : (dv[u] - av[u] * prev) / dn[u];
          Y[s * kLanes + lane] = v;
          prev = v;
        }
      }
    }
    T next = T(0);
    for (int s = r1; s >= r0; --s) {
      const T yp = Y[s * kLanes + lane];
      const T v = s == r1 ? yp : yp - cl[s * row] * next;
      Y[s * kLanes + lane] = v;
      next = v;
    }
    YI[(2 * q) * kLanes + lane] = Y[r0 * kLanes + lane];
    YI[(2 * q + 1) * kLanes + lane] = Y[r1 * kLanes + lane];
  }
  __syncthreads();
  // Interface unknowns F_q, L_q = rows 2q, 2q+1 of R applied to y_I.
  if (valid) {
    constexpr int n2 = 2 * S;
    T f = T(0), l = T(0);
#pragma unroll
    for (int e = 0; e < n2; ++e) {
      const T y = YI[e * kLanes + lane];
      f += rinv[lay.rinv(n2, 2 * q, e, color, t)] * y;
      l += rinv[lay.rinv(n2, 2 * q + 1, e, color, t)] * y;
    }
    UI[(2 * q) * kLanes + lane] = f;
    UI[(2 * q + 1) * kLanes + lane] = l;
  }
  __syncthreads();
  if (valid) {
    const T left = q > 0 ? UI[(2 * (q - 1) + 1) * kLanes + lane] : T(0);
    const T right = q + 1 < S ? UI[(2 * (q + 1)) * kLanes + lane] : T(0);
    for (int s = r0; s <= r1; ++s)
      x[base + s * stride] = Y[s * kLanes + lane] - vv[s * row] * left - ww[s * row] * right;
  }
}

// ---------------------------------------------------------------------------
// PCR elimination factors of every line: per halving step the multipliers
// k1 = a_s / b_{s-h}, k2 = c_s / b_{s+h}, then the final diagonal.  Layout
// [2*steps+1][lines][P] so a line's threads read consecutive addresses.
template <class T>
__global__ void __launch_bounds__(1024) k_pcr_factors(Level<T> L, int axis, int P, T* __restrict__ fac) {
  extern __shared__ unsigned char pcr_factor_smem[];
  T* sa = reinterpret_cast<T*>(pcr_factor_smem) + threadIdx.y * 3 * P;
  T* sb = sa + P;
  T* sc = sb + P;
  const int a_extent = axis == 0 ? L.ny : L.nx;
  const int b_extent = axis == 2 ? L.ny : L.nz;
  const int lines = a_extent * b_extent;
  const int extent = line_extent(axis, L.nx, L.ny, L.nz);
  const int line = blockIdx.x * blockDim.y + threadIdx.y;
  const bool valid = line < lines;
  const int fb = valid ? line / a_extent : 0;
  const int fa = valid ? line - fb * a_extent : 0;
  const int s = threadIdx.x;
  T a = T(0), bb = T(1), cc = T(0);
  if (valid && s < extent) {
    int i, j, k;
    line_cell(axis, fa, fb, s, i, j, k);
    const int c = i + L.nx * (j + L.ny * k);
    T lowf, highf;
    line_faces(L, axis, c, j, k, lowf, highf);
    a = s == 0 ? T(0) : -lowf;
    bb = L.diag[c];
    cc = s + 1 == extent ? T(0) : -highf;
  }
  sa[s] = a;
  sb[s] = bb;
  sc[s] = cc;
  __syncthreads();
  const size_t slab = static_cast<size_t>(lines) * P;
  const size_t at = static_cast<size_t>(valid ? line : 0) * P + s;
  int step = 0;
  for (int h = 1; h < P; h <<= 1, ++step) {
    const int lo = s - h, hi = s + h;
    const T as = sa[s], bs = sb[s], cs = sc[s];
    T k1 = T(0), k2 = T(0), alo = T(0), clo = T(0), ahi = T(0), chi = T(0);
    if (lo >= 0) {
      k1 = as / sb[lo];
      alo = sa[lo];
      clo = sc[lo];
    }
    if (hi < P) {
      k2 = cs / sb[hi];
      ahi = sa[hi];
      chi = sc[hi];
    }
    const T na = -alo * k1;
    const T nc = -chi * k2;
    const T nb = bs - clo * k1 - ahi * k2;
    if (valid) {
      fac[(2 * step) * slab + at] = k1;
      fac[(2 * step + 1) * slab + at] = k2;
    }
    __syncthreads();
    sa[s] = na;
    sb[s] = nb;
    sc[s] = nc;
    __syncthreads();
  }
  if (valid) fac[(2 * step) * slab + at] = sb[s];
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

template <class T>
__device__ __forceinline__ T line_rhs_any(const Level<T>& L, const T* x,
                                          const T* rhs, int axis, int fa,
                                          int fb, int s, int extent, int c) {
  if (axis == 0) return line_rhs<T, 0>(L, x, rhs, fa, fb, s, extent, c);
  if (axis == 1) return line_rhs<T, 1>(L, x, rhs, fa, fb, s, extent, c);
  return line_rhs<T, 2>(L, x, rhs, fa, fb, s, extent, c);
}

// One zebra colour with PCR: blockDim = (P, lines per block), P = 2^STEPS.
template <class T, int STEPS>
__global__ void __launch_bounds__(1024) k_line_pcr_factored_color(Level<T> L, T* __restrict__ x,
                                          const T* __restrict__ rhs,
                                          const T* __restrict__ fac, int axis,
                                          int color) {
  constexpr int P = 1 << STEPS;
  extern __shared__ unsigned char pcr_rhs_smem[];
  T* sd = reinterpret_cast<T*>(pcr_rhs_smem) + threadIdx.y * P;
  const int a_extent = axis == 0 ? L.ny : L.nx;
  const int b_extent = axis == 2 ? L.ny : L.nz;
  const int ha = (a_extent + 1) >> 1;
  const int extent = line_extent(axis, L.nx, L.ny, L.nz);
  const int t = blockIdx.x * blockDim.y + threadIdx.y;
  const int fb = t / ha;
  const int fa = 2 * (t - fb * ha) + ((fb + color) & 1);
  const bool valid = t < ha * b_extent && fa < a_extent;
  const int s = threadIdx.x;
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
    d = line_rhs_any(L, x, rhs, axis, fa, fb, s, extent, c);
  }
  sd[s] = d;
  __syncthreads();
  const T value = pcr_apply(r, sd, s);
  if (valid && s < extent) x[c] = value;
}

// One zebra colour pass of the coarsest-level kernel for the lines handled
// by this thread row (factors already in registers).
template <class TC, int STEPS>
__device__ __forceinline__ void coarse_line_pass(const Level<TC>& L, TC* xs,
                                                 const TC* bs, TC* sd, int axis,
                                                 int fa, int fb, bool valid,
                                                 int c, int s, int extent,
                                                 const PcrRow<TC, STEPS>& r) {
  TC d = TC(0);
  if (valid && s < extent) d = line_rhs_any(L, xs, bs, axis, fa, fb, s, extent, c);
  sd[s] = d;
  __syncthreads();
  const TC value = pcr_apply(r, sd, s);
  if (valid && s < extent) xs[c] = value;
  __syncthreads();
}

// Coarsest level, line mode: all sweeps in one CTA with x and rhs resident
// in shared memory (widened to TC).  When each colour's lines fit the CTA's
// thread rows, both colours' PCR factors stay in registers for all sweeps.
template <class T, class TC, int STEPS>
__global__ void __launch_bounds__(512)
    k_coarse_line_smem(Level<TC> L, T* __restrict__ x, const T* __restrict__ b,
                       const TC* __restrict__ fac, int sweeps, int axis) {
  constexpr int P = 1 << STEPS;
  extern __shared__ unsigned char coarse_smem[];
  const int n = L.nx * L.ny * L.nz;
  TC* xs = reinterpret_cast<TC*>(coarse_smem);
  TC* bs = xs + n;
  TC* sd = bs + n + threadIdx.y * P;
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  const int nthreads = blockDim.x * blockDim.y;
  for (int c = tid; c < n; c += nthreads) {
    xs[c] = static_cast<TC>(x[c]);
    bs[c] = static_cast<TC>(b[c]);
  }
  __syncthreads();
  const int extent = line_extent(axis, L.nx, L.ny, L.nz);
  const int a_extent = axis == 0 ? L.ny : L.nx;
  const int b_extent = axis == 2 ? L.ny : L.nz;
  const int ha = (a_extent + 1) >> 1;
  const int lines = ha * b_extent;
  const size_t slab = static_cast<size_t>(a_extent) * b_extent * P;
  const int s = threadIdx.x;
  const auto locate = [&](int t, int color, int& fa, int& fb, bool& valid, int& c,
                          size_t& at) {
    fb = t / ha;
    fa = 2 * (t - fb * ha) + ((fb + color) & 1);
    valid = t < lines && fa < a_extent;
    at = static_cast<size_t>(valid ? fa + a_extent * fb : 0) * P + s;
    c = 0;
    if (valid && s < extent) {
      int i, j, k;
      line_cell(axis, fa, fb, s, i, j, k);
      c = i + L.nx * (j + L.ny * k);
    }
  };
  if (lines <= static_cast<int>(blockDim.y)) {
    int fa0, fb0, c0, fa1, fb1, c1;
    bool v0, v1;
    size_t at0, at1;
    locate(threadIdx.y, 0, fa0, fb0, v0, c0, at0);
    locate(threadIdx.y, 1, fa1, fb1, v1, c1, at1);
    PcrRow<TC, STEPS> r0, r1;
    pcr_load(fac, slab, at0, r0);
    pcr_load(fac, slab, at1, r1);
    for (int sweep = 0; sweep < sweeps; ++sweep) {
      coarse_line_pass(L, xs, bs, sd, axis, fa0, fb0, v0, c0, s, extent, r0);
      coarse_line_pass(L, xs, bs, sd, axis, fa1, fb1, v1, c1, s, extent, r1);
    }
  } else {
    for (int sweep = 0; sweep < sweeps; ++sweep) {
      for (int color = 0; color < 2; ++color) {
        for (int base = 0; base < lines; base += blockDim.y) {
          int fa, fb, c;
          bool valid;
          size_t at;
          locate(base + threadIdx.y, color, fa, fb, valid, c, at);
          PcrRow<TC, STEPS> r;
          pcr_load(fac, slab, at, r);
          coarse_line_pass(L, xs, bs, sd, axis, fa, fb, valid, c, s, extent, r);
        }
      }
    }
  }
  for (int c = tid; c < n; c += nthreads) x[c] = static_cast<T>(xs[c]);
}

void pcr_shape(int extent, int& P, int& lines_per_block, int& steps) {
  P = 1;
  steps = 0;
  while (P < extent) {
    P <<= 1;
    ++steps;
  }
  lines_per_block = std::max(1, std::min(1024 / P, 4));
}

template <class T, int AXIS, int S>
void launch_segment(cudaStream_t s, const Level<T>& L, T* x, const T* b,
                    const T* fac, int color, int blocks, size_t smem) {
  if (smem > 48 * 1024)
    cudaFuncSetAttribute(k_line_segment_color<T, AXIS, S>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  k_line_segment_color<T, AXIS, S><<<blocks, dim3(kLanes, S), smem, s>>>(L, x, b, fac, color);
}

template <class T, int AXIS>
void launch_segment_axis(cudaStream_t s, const Level<T>& L, T* x, const T* b,
                         const T* fac, int color, int S, int blocks, size_t smem) {
  switch (S) {
    case 1: launch_segment<T, AXIS, 1>(s, L, x, b, fac, color, blocks, smem); break;
    case 2: launch_segment<T, AXIS, 2>(s, L, x, b, fac, color, blocks, smem); break;
    case 4: launch_segment<T, AXIS, 4>(s, L, x, b, fac, color, blocks, smem); break;
    default: launch_segment<T, AXIS, 8>(s, L, x, b, fac, color, blocks, smem); break;
  }
}

}  // namespace

int line_kind(int nx, int ny, int nz, int axis) {
  const int extent = line_extent(axis, nx, ny, nz);
  const int a_extent = axis == 0 ? ny : nx;
  const int b_extent = axis == 2 ? ny : nz;
  const long long per_color = static_cast<long long>((a_extent + 1) / 2) * b_extent;
  if (per_color < kLinePcrThreshold && extent <= 1024) return kLinePcr;
  return kLineSegment;
}

size_t line_factor_values(int nx, int ny, int nz, int axis) {
  const int extent = line_extent(axis, nx, ny, nz);
  const int a_extent = axis == 0 ? ny : nx;
  const int b_extent = axis == 2 ? ny : nz;
  const size_t lines = static_cast<size_t>(a_extent) * b_extent;
  if (line_kind(nx, ny, nz, axis) == kLineSegment) {
    const size_t S = static_cast<size_t>(segments_for(extent));
    const SegmentLayout lay{extent, ((a_extent + 1) / 2) * b_extent};
    // 5 colour-packed arrays per row, plus the interface inverse per line.
    return lay.cell_values() + 2 * static_cast<size_t>(lay.colour_lines) * 4 * S * S;
  }
  int P, lpb, steps;
  pcr_shape(extent, P, lpb, steps);
  return static_cast<size_t>(2 * steps + 1) * lines * P;
}

template <class T>
void launch_line_factors(cudaStream_t s, const Level<T>& L, int axis, T* fac) {
  const int extent = line_extent(axis, L.nx, L.ny, L.nz);
  const int a_extent = axis == 0 ? L.ny : L.nx;
  const int b_extent = axis == 2 ? L.ny : L.nz;
  const int lines = a_extent * b_extent;
  if (line_kind(L.nx, L.ny, L.nz, axis) == kLineSegment) {
    const int S = segments_for(extent);
    k_segment_factors<T><<<(lines + 63) / 64, 64, 0, s>>>(L, axis, S, fac);
    return;
  }
  int P, lpb, steps;
  pcr_shape(extent, P, lpb, steps);
  const size_t smem = static_cast<size_t>(3) * P * lpb * sizeof(T);
  k_pcr_factors<T><<<(lines + lpb - 1) / lpb, dim3(P, lpb), smem, s>>>(L, axis, P, fac);
}

template <class T>
void launch_line_pass(cudaStream_t s, const Level<T>& L, T* x, const T* b,
                      const T* fac, T* scratch, int axis, int color) {
  (void)scratch;
  const int extent = line_extent(axis, L.nx, L.ny, L.nz);
  const int a_extent = axis == 0 ? L.ny : L.nx;
  const int b_extent = axis == 2 ? L.ny : L.nz;
  const long long per_color = static_cast<long long>((a_extent + 1) / 2) * b_extent;
  if (line_kind(L.nx, L.ny, L.nz, axis) == kLineSegment) {
    const int S = segments_for(extent);
    const int blocks = static_cast<int>((per_color + kLanes - 1) / kLanes);
    const size_t smem = (static_cast<size_t>(extent) + 4 * S) * kLanes * sizeof(T);
    if (axis == 0) launch_segment_axis<T, 0>(s, L, x, b, fac, color, S, blocks, smem);
    else if (axis == 1) launch_segment_axis<T, 1>(s, L, x, b, fac, color, S, blocks, smem);
    else launch_segment_axis<T, 2>(s, L, x, b, fac, color, S, blocks, smem);
    return;
  }
  int P, lpb, steps;
  pcr_shape(extent, P, lpb, steps);
  const size_t smem = static_cast<size_t>(P) * lpb * sizeof(T);
  const int blocks = static_cast<int>((per_color + lpb - 1) / lpb);
  const dim3 block(P, lpb);
  switch (steps) {
#define HFPS_PCR_CASE(N)                                                        \
  case N:                                                                       \
    k_line_pcr_factored_color<T, N><<<blocks, block, smem, s>>>(L, x, b, fac, axis, \
                                                                 color);        \
    break;
    HFPS_PCR_CASE(0) HFPS_PCR_CASE(1) HFPS_PCR_CASE(2) HFPS_PCR_CASE(3) HFPS_PCR_CASE(4)
    HFPS_PCR_CASE(5) HFPS_PCR_CASE(6) HFPS_PCR_CASE(7) HFPS_PCR_CASE(8) HFPS_PCR_CASE(9)
    HFPS_PCR_CASE(10)
#undef HFPS_PCR_CASE
    default: break;
  }
}

template <class T, class TC>
bool launch_coarse_line(cudaStream_t s, const Level<TC>& L, T* x, const T* b,
                        const TC* fac, int sweeps, int axis) {
  const int extent = line_extent(axis, L.nx, L.ny, L.nz);
  if (line_kind(L.nx, L.ny, L.nz, axis) != kLinePcr) return false;
  int P, lpb, steps;
  pcr_shape(extent, P, lpb, steps);
  const int a_extent = axis == 0 ? L.ny : L.nx;
  const int b_extent = axis == 2 ? L.ny : L.nz;
  if (P > 512) return false;
  lpb = std::max(1, std::min({512 / P, 4, ((a_extent + 1) / 2) * b_extent}));
  const size_t cells = static_cast<size_t>(L.nx) * L.ny * L.nz;
  const size_t smem = (2 * cells + static_cast<size_t>(P) * lpb) * sizeof(TC);
  if (smem > 200 * 1024) return false;
  const dim3 block(P, lpb);
  switch (steps) {
#define HFPS_COARSE_CASE(N)                                                      \
  case N:                                                                        \
    if (smem > 48 * 1024)                                                        \
      cudaFuncSetAttribute(k_coarse_line_smem<T, TC, N>,                         \
                           cudaFuncAttributeMaxDynamicSharedMemorySize,          \
                           static_cast<int>(smem));                              \
    k_coarse_line_smem<T, TC, N><<<1, block, smem, s>>>(L, x, b, fac, sweeps, axis); \
    break;
    HFPS_COARSE_CASE(0) HFPS_COARSE_CASE(1) HFPS_COARSE_CASE(2) HFPS_COARSE_CASE(3)
    HFPS_COARSE_CASE(4) HFPS_COARSE_CASE(5) HFPS_COARSE_CASE(6) HFPS_COARSE_CASE(7)
    HFPS_COARSE_CASE(8) HFPS_COARSE_CASE(9)
#undef HFPS_COARSE_CASE
    default: return false;
  }
  return true;
}

template void launch_line_factors<double>(cudaStream_t, const Level<double>&, int, double*);
template void launch_line_factors<float>(cudaStream_t, const Level<float>&, int, float*);
template void launch_line_pass<double>(cudaStream_t, const Level<double>&, double*,
                                       const double*, const double*, double*, int, int);
template void launch_line_pass<float>(cudaStream_t, const Level<float>&, float*, const float*,
                                      const float*, float*, int, int);
template bool launch_coarse_line<double, double>(cudaStream_t, const Level<double>&, double*,
                                                 const double*, const double*, int, int);
template bool launch_coarse_line<float, double>(cudaStream_t, const Level<double>&, float*,
                                                const float*, const double*, int, int);

}  // namespace hfps
