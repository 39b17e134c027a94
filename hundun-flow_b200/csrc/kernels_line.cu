// Zebra line relaxation (y-line relaxation for stretched grids) on sm_100a.
//
// The reference relaxes strong-axis lines by lexicographic line Gauss-Seidel
// with one Thomas solve per line (line_smooth_axis, src/solver_mg.cpp:
// 3352-3539).  Here lines are coloured by the parity of their transverse
// index (zebra): a colour's lines couple only to the other colour, so all of
// them are solved at once.  The line matrices depend only on the level
// coefficients, so every factorisation is computed once per coefficient
// update and each sweep does only right-hand-side work:
//   * many lines per colour: a chunked scan over precomputed Thomas
//     factors.  Lanes run across lines (loads coalesce along x), each
//     thread owns a chunk of up to 16 rows of its line, and the chunks of a
//     line combine the affine maps of the forward and backward recurrences
//     through shared memory;
//   * few lines per colour (coarse levels): one CTA row per line runs
//     parallel cyclic reduction with precomputed elimination factors held
//     in registers;
//   * the coarsest level keeps x and rhs in shared memory for all of its
//     coarse sweeps in one launch.
#include "kernels.hpp"
#include "phase_device.cuh"

#include <algorithm>

namespace hfps {
namespace {


// Right-hand side of the rows of one line with everything that is constant
// along the line hoisted: the transverse neighbours' offsets (0 where the
// neighbour is outside the level, read as 0 for Dirichlet and as the cell
// itself for Neumann), the face arrays with their index at row 0 and stride
// per row, and the line-end boundary faces.  Every load of a row is
// unconditional, so a thread can keep many rows' loads in flight.  The
// arithmetic and its order are line_rhs's.  Transverse neighbours belong to
// the other colour, which a colour pass never writes, so they are read
// through the read-only path.  With hx > 0 the vectors are in split rows
// (SplitPos): an x neighbour sits in the other half of the row, a y or z
// neighbour in the same half of the previous or next row.  A neighbour
// outside the level reads the cell itself (Neumann), so it counts as this
// colour's value for the zero flags of the first sweep.
// Variants of a scan colour pass by what is known of x (LineRhs::row).
enum ScanMode : int { kScanNormal = 0, kScanOwnZero = 1, kScanFresh = 2 };

template <class T, int AXIS, bool SPLIT>
struct LineRhs {
  static constexpr int kA0 = AXIS == 0 ? 1 : 0;  // first transverse axis
  static constexpr int kA1 = AXIS == 2 ? 1 : 2;  // second transverse axis
  const T* face[2];
  int fbase[2], fstride[2], fhigh[2];
  int off[4];
  bool keep[4];
  bool self[4];   // the neighbour is the cell itself (outside the level)
  T end_low, end_high;   // line-end boundary faces (rows 0 and extent-1)
  bool lkeep_low, lkeep_high;

  __device__ static void axis_faces(const Level<T>& L, int axis, int i, int j,
                                    int k, int line_axis, const T*& f,
                                    int& b, int& st, int& hi) {
    // Face index of cell (i, j, k) on `axis`, its step per row along
    // line_axis, and the offset of the cell's high face.
    const int nx = L.nx, ny = L.ny, nz = L.nz;
    if (axis == 0) {
      f = L.fx;
      b = i + (nx + 1) * (j + ny * k);
      st = line_axis == 0 ? 1 : (line_axis == 1 ? nx + 1 : (nx + 1) * ny);
      hi = 1;
    } else if (axis == 1) {
      f = L.fy;
      b = i + nx * (j + (ny + 1) * k);
      st = line_axis == 0 ? 1 : (line_axis == 1 ? nx : nx * (ny + 1));
      hi = nx;
    } else {
      f = L.fz;
      b = i + nx * (j + ny * k);
      st = line_axis == 0 ? 1 : (line_axis == 1 ? nx : nx * ny);
      hi = nx * ny;
    }
    (void)nz;
  }

  __device__ LineRhs(const Level<T>& L, int fa, int fb, int hx) {
    int i0, j0, k0;
    line_cell(AXIS, fa, fb, 0, i0, j0, k0);
    const int idx[3] = {i0, j0, k0};
    const int ext[3] = {L.nx, L.ny, L.nz};
    const int step[3] = {1, L.nx, L.nx * L.ny};
    const int axes[2] = {kA0, kA1};
#pragma unroll
    for (int n = 0; n < 2; ++n) {
      const int a = axes[n];
      axis_faces(L, a, i0, j0, k0, AXIS, face[n], fbase[n], fstride[n], fhigh[n]);
      const bool low_in = idx[a] > 0, high_in = idx[a] + 1 < ext[a];
      int lo = -step[a], hi = step[a];
      if (SPLIT) {
        const int odd = i0 & 1;
        lo = a == 0 ? (odd ? -hx : hx - 1) : (a == 1 ? -2 * hx : -2 * hx * L.ny);
        hi = a == 0 ? (odd ? 1 - hx : hx) : (a == 1 ? 2 * hx : 2 * hx * L.ny);
      }
      off[2 * n] = low_in ? lo : 0;
      off[2 * n + 1] = high_in ? hi : 0;
      self[2 * n] = !low_in;
      self[2 * n + 1] = !high_in;
      keep[2 * n] = low_in || ((L.neumann >> (2 * a)) & 1u);
      keep[2 * n + 1] = high_in || ((L.neumann >> (2 * a + 1)) & 1u);
    }
    const T* lface;
    int lbase, lstride, lhigh;
    axis_faces(L, AXIS, i0, j0, k0, AXIS, lface, lbase, lstride, lhigh);
    end_low = __ldg(lface + lbase);
    end_high = __ldg(lface + lbase + (ext[AXIS] - 1) * lstride + lhigh);
    lkeep_low = (L.neumann >> (2 * AXIS)) & 1u;
    lkeep_high = (L.neumann >> (2 * AXIS + 1)) & 1u;
  }

  // Row s, c its vector index.  MODE kScanFresh: x is zero everywhere and
  // not read.  kScanOwnZero: this colour's x is zero; its values (the cell
  // itself, read where a neighbour lies outside the level) are still loaded,
  // so that every load stays unconditional, and then replaced by zero.
  template <int MODE>
  __device__ __forceinline__ T row(const T* x, const T* __restrict__ rhs, int c,
                                   int s, int extent) const {
    T d = __ldg(rhs + c);
#pragma unroll
    for (int n = 0; n < 2; ++n) {
      const int f = fbase[n] + s * fstride[n];
      T lo = T(0), hi = T(0);
      if (MODE != kScanFresh) {
        lo = __ldg(x + c + off[2 * n]);
        hi = __ldg(x + c + off[2 * n + 1]);
      }
      if (MODE == kScanOwnZero) {
        lo = self[2 * n] ? T(0) : lo;
        hi = self[2 * n + 1] ? T(0) : hi;
      }
      d += __ldg(face[n] + f) * (keep[2 * n] ? lo : T(0));
      d += __ldg(face[n] + f + fhigh[n]) * (keep[2 * n + 1] ? hi : T(0));
    }
    const T self_value = MODE == kScanNormal ? x[c] : T(0);
    const T dl = d + end_low * (lkeep_low ? self_value : T(0));
    d = s == 0 ? dl : d;
    const T dh = d + end_high * (lkeep_high ? self_value : T(0));
    return s + 1 == extent ? dh : d;
  }
};

// ---------------------------------------------------------------------------
// Chunked-scan line solve.
//
// Each line's matrix is factorised once (full-line Thomas, in FP64): for row
// s, den_s = b_s - a_s c'_{s-1}, and the sweep needs
//   inv_s = 1 / den_s,   l_s = a_s / den_s,   u_s = c'_s = c_s / den_s.
// A sweep is then two first-order linear recurrences,
//   forward   y_s = d_s inv_s - l_s y_{s-1},
//   backward  x_s = y_s - u_s x_{s+1}.
// The line matrix is symmetric (a_s and c_{s-1} are the same face), so
// a_s / den_{s-1} = u_{s-1}, and the LDL^T form of the forward recurrence
//   z_s = d_s - u_{s-1} z_{s-1},   y_s = z_s inv_s
// needs no l array.  FP64 sweeps use it (one stream of 8 B per row less);
// FP32 sweeps keep the l array, because the extra load in the forward
// replay costs the FP32 kernel registers and occupancy.
// Each recurrence is an affine map per row.  A thread owns a chunk of up to
// ScanConfig<T>::rows consecutive rows of one line: it composes its chunk's
// maps, the chunks of a line combine their compositions through shared
// memory, and every thread replays its chunk from the incoming value.  No spike vectors or interface
// systems are stored, no division happens in a sweep, and the right-hand
// side of a chunk (the costly part: rhs, transverse faces and neighbours)
// stays in registers between the passes.
//
// Factor layout is colour-packed so that threads with consecutive line
// indices of one colour read consecutive addresses: array e (0 inv, then
// 1 u in the symmetric form, or 1 l and 2 u) of row s of colour line t sits at
//   ((e * 2 + colour) * extent + s) * colour_lines + t.

// Rows per chunk (held in registers) and the block-size bound, per
// precision: FP64 rows take twice the registers of FP32 rows.
// Measured on B200 at 256^3 (level-0 y-line colour pass): FP64 16 rows in
// blocks of <= 128 threads (8 lines x 16 chunks), FP32 8 rows in blocks of
// <= 512 threads (16 lines x 32 chunks).
#ifndef HFPS_SCAN_ROWS_F64
#define HFPS_SCAN_ROWS_F64 16
#endif
#ifndef HFPS_SCAN_THREADS_F64
#define HFPS_SCAN_THREADS_F64 128
#endif
#ifndef HFPS_SCAN_ROWS_F32
#define HFPS_SCAN_ROWS_F32 8
#endif
#ifndef HFPS_SCAN_THREADS_F32
#define HFPS_SCAN_THREADS_F32 512
#endif
template <class T>
struct ScanConfig;
template <>
struct ScanConfig<double> {
  static constexpr int rows = HFPS_SCAN_ROWS_F64;
  static constexpr int threads = HFPS_SCAN_THREADS_F64;
  static constexpr bool symmetric = true;
  static constexpr int arrays = 2;
};
// FP32 factors in the symmetric two-array form when HFPS_SCAN_SYM_F32 is 1.
#ifndef HFPS_SCAN_SYM_F32
#define HFPS_SCAN_SYM_F32 0
#endif
template <>
struct ScanConfig<float> {
  static constexpr int rows = HFPS_SCAN_ROWS_F32;
  static constexpr int threads = HFPS_SCAN_THREADS_F32;
  static constexpr bool symmetric = HFPS_SCAN_SYM_F32 != 0;
  static constexpr int arrays = symmetric ? 2 : 3;
};
// Longest line both precisions can solve: every chunk of a line lives in
// one block.
constexpr int kScanMaxExtent =
    HFPS_SCAN_ROWS_F64 * HFPS_SCAN_THREADS_F64 < HFPS_SCAN_ROWS_F32 * HFPS_SCAN_THREADS_F32
        ? HFPS_SCAN_ROWS_F64 * HFPS_SCAN_THREADS_F64
        : HFPS_SCAN_ROWS_F32 * HFPS_SCAN_THREADS_F32;

struct ScanLayout {
  int extent;
  int colour_lines;
  __host__ __device__ size_t cell(int e, int colour, int s, int t) const {
    return ((static_cast<size_t>(e) * 2 + colour) * extent + s) * colour_lines + t;
  }
  __host__ __device__ size_t values(int arrays) const {
    return static_cast<size_t>(arrays) * 2 * extent * colour_lines;
  }
};

// Thomas factors of every line, one thread per line, in FP64 whatever T is.
template <class T>
__global__ void k_scan_factors(Level<T> L, int axis, T* __restrict__ fac) {
  grid_dependency_sync();
  const int a_extent = axis == 0 ? L.ny : L.nx;
  const int b_extent = axis == 2 ? L.ny : L.nz;
  const int lines = a_extent * b_extent;
  const int extent = line_extent(axis, L.nx, L.ny, L.nz);
  const int ha = (a_extent + 1) >> 1;
  const ScanLayout lay{extent, ha * b_extent};
  for (int line = blockIdx.x * blockDim.x + threadIdx.x; line < lines;
       line += gridDim.x * blockDim.x) {
    const int fb = line / a_extent;
    const int fa = line - fb * a_extent;
    const int colour = (fa + fb) & 1;
    const int t = fb * ha + (fa >> 1);
    int base, stride;
    line_geometry(L, axis, fa, fb, base, stride);
    double prev_u = 0.0;
    for (int s = 0; s < extent; ++s) {
      const int c = base + s * stride;
      int i, j, k;
      line_cell(axis, fa, fb, s, i, j, k);
      T lowf, highf;
      line_faces(L, axis, c, j, k, lowf, highf);
      const double a = s == 0 ? 0.0 : -static_cast<double>(lowf);
      const double cc = s + 1 == extent ? 0.0 : -static_cast<double>(highf);
      const double den = static_cast<double>(L.diag[c]) - a * prev_u;
      const double u = cc / den;
      fac[lay.cell(0, colour, s, t)] = static_cast<T>(1.0 / den);
      if constexpr (ScanConfig<T>::symmetric) {
        fac[lay.cell(1, colour, s, t)] = static_cast<T>(u);
      } else {
        fac[lay.cell(1, colour, s, t)] = static_cast<T>(a / den);
        fac[lay.cell(2, colour, s, t)] = static_cast<T>(u);
      }
      prev_u = u;
    }
  }
}

// One zebra colour: blockDim = (LPB lines, S chunks), chunk q holds rows
// [q*m, min(extent, (q+1)*m) - 1] with m <= ScanConfig<T>::rows.  Shared memory holds
// the chunk compositions: forward (A, B) and backward (A, B), S x LPB each.
template <class T, int AXIS, int LPB, int MODE, bool SPLIT>
__global__ void __launch_bounds__(ScanConfig<T>::threads)
    k_line_scan_color(Level<T> L, T* x, const T* __restrict__ rhs,
                      const T* __restrict__ fac, int color, int m, int hx) {
  grid_dependency_sync();
  extern __shared__ unsigned char scan_smem[];
  const int S = blockDim.y;
  T* fA = reinterpret_cast<T*>(scan_smem);
  T* fB = fA + S * LPB;
  T* bA = fB + S * LPB;
  T* bB = bA + S * LPB;
  const int extent = line_extent(AXIS, L.nx, L.ny, L.nz);
  const int a_extent = AXIS == 0 ? L.ny : L.nx;
  const int b_extent = AXIS == 2 ? L.ny : L.nz;
  const int ha = (a_extent + 1) >> 1;
  const ScanLayout lay{extent, ha * b_extent};
  const int lane = threadIdx.x;
  const int q = threadIdx.y;
  const int t = blockIdx.x * LPB + lane;
  const int fb = t / ha;
  const int fa = 2 * (t - fb * ha) + ((fb + color) & 1);
  const bool valid = t < ha * b_extent && fa < a_extent;
  // Vector index of row 0 and its step per row (natural or split rows).
  int base = 0, stride = 0;
  if (valid) {
    line_geometry(L, AXIS, fa, fb, base, stride);
    if (SPLIT) {
      int i0, j0, k0;
      line_cell(AXIS, fa, fb, 0, i0, j0, k0);
      base = 2 * hx * (j0 + L.ny * k0) + (i0 & 1) * hx + (i0 >> 1);
      stride = AXIS == 1 ? 2 * hx : 2 * hx * L.ny;
    }
  }
  const int r0 = q * m;
  const int rows = valid ? max(0, min(m, extent - r0)) : 0;
  const int row = lay.colour_lines;
  const int tt = valid ? t : 0;
  constexpr bool kSym = ScanConfig<T>::symmetric;
  const T* inv = fac + lay.cell(0, color, 0, tt);
  const T* lf = fac + lay.cell(1, color, 0, tt);
  const T* uf = fac + lay.cell(kSym ? 1 : 2, color, 0, tt);
  // Rows past the chunk's end (padding, and every row of an idle thread)
  // re-read the line's last row so that all loads are unconditional; their
  // values are never used.
  const auto srow = [&](int u) { return min(r0 + u, extent - 1); };
  // Forward multiplier of row s: u_{s-1} (zero on row 0), or l_s.
  const auto lower = [&](int u) -> T {
    const int s = srow(u);
    if constexpr (kSym) {
      const T g = __ldg(uf + max(s - 1, 0) * row);
      return s > 0 ? g : T(0);
    } else {
      return __ldg(lf + s * row);
    }
  };

  // Pass 1: right-hand sides (scaled by 1/den unless symmetric), and the
  // forward composition.
  const LineRhs<T, AXIS, SPLIT> lr(L, valid ? fa : 0, valid ? fb : 0, hx);
  constexpr int kScanRows = ScanConfig<T>::rows;
  T v[kScanRows];
#pragma unroll
  for (int u = 0; u < kScanRows; ++u) {
    v[u] = lr.template row<MODE>(x, rhs, base + srow(u) * stride, srow(u), extent);
    if constexpr (!kSym) v[u] = v[u] * __ldg(inv + srow(u) * row);
  }
  T A = T(1), B = T(0);
#pragma unroll
  for (int u = 0; u < kScanRows; ++u) {
    const T l = lower(u);
    const bool on = u < rows;
    B = on ? v[u] - l * B : B;
    A = on ? -l * A : A;
  }
  fA[q * LPB + lane] = A;
  fB[q * LPB + lane] = B;
  __syncthreads();
  // Forward replay from z_{r0-1} (y_{r0-1}); v becomes y.
  T z = T(0);
  for (int p = 0; p < q; ++p) z = fA[p * LPB + lane] * z + fB[p * LPB + lane];
#pragma unroll
  for (int u = 0; u < kScanRows; ++u) {
    z = v[u] - lower(u) * z;
    if constexpr (kSym) {
      v[u] = z * __ldg(inv + srow(u) * row);
    } else {
      v[u] = z;
    }
  }
  // Backward composition x_{r0} = A x_{r1+1} + B.
  A = T(1);
  B = T(0);
#pragma unroll
  for (int u = kScanRows - 1; u >= 0; --u) {
    const T uu = __ldg(uf + srow(u) * row);
    const bool on = u < rows;
    B = on ? v[u] - uu * B : B;
    A = on ? -uu * A : A;
  }
  bA[q * LPB + lane] = A;
  bB[q * LPB + lane] = B;
  __syncthreads();
  T xn = T(0);
  for (int p = S - 1; p > q; --p) xn = bA[p * LPB + lane] * xn + bB[p * LPB + lane];
#pragma unroll
  for (int u = kScanRows - 1; u >= 0; --u) {
    const T xv = v[u] - __ldg(uf + srow(u) * row) * xn;
    xn = u < rows ? xv : xn;
    if (u < rows) x[base + srow(u) * stride] = xn;
  }
}

// ---------------------------------------------------------------------------
// PCR elimination factors of every line: per halving step the multipliers
// k1 = a_s / b_{s-h}, k2 = c_s / b_{s+h}, then the final diagonal.  Layout
// [2*steps+1][lines][P] so a line's threads read consecutive addresses.
template <class T>
__global__ void __launch_bounds__(1024) k_pcr_factors(Level<T> L, int axis, int P, T* __restrict__ fac) {
  grid_dependency_sync();
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

// One zebra colour with PCR: blockDim = (P, lines per block), P = 2^STEPS.
template <class T, int STEPS>
__global__ void __launch_bounds__(1024) k_line_pcr_factored_color(Level<T> L, T* __restrict__ x,
                                          const T* __restrict__ rhs,
                                          const T* __restrict__ fac, int axis,
                                          int color) {
  grid_dependency_sync();
  extern __shared__ unsigned char pcr_rhs_smem[];
  T* sd = reinterpret_cast<T*>(pcr_rhs_smem) + threadIdx.y * (1 << STEPS);
  pcr_line_slot<T, STEPS>(L, x, rhs, fac, axis, color, blockIdx.x * blockDim.y + threadIdx.y,
                          threadIdx.x, sd);
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
//
// With `columns` set, block j instead starts from unit data, x = e_j and
// b = 0 for j < n, x = 0 and b = e_{j-n} for j >= n, and writes its result
// to x + j*n: the columns of the affine map x_out = P x_in + M b that the
// sweeps apply (coarse_dense_operator).
template <class T, class TC, int STEPS>
__global__ void __launch_bounds__(512)
    k_coarse_line_smem(Level<TC> L, T* __restrict__ x, const T* __restrict__ b,
                       const TC* __restrict__ fac, int sweeps, int axis,
                       bool columns) {
  grid_dependency_sync();
  constexpr int P = 1 << STEPS;
  extern __shared__ unsigned char coarse_smem[];
  const int n = L.nx * L.ny * L.nz;
  TC* xs = reinterpret_cast<TC*>(coarse_smem);
  TC* bs = xs + n;
  TC* sd = bs + n + threadIdx.y * P;
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  const int nthreads = blockDim.x * blockDim.y;
  if (columns) {
    const int j = blockIdx.x;
    for (int c = tid; c < n; c += nthreads) {
      xs[c] = (j < n && c == j) ? TC(1) : TC(0);
      bs[c] = (j >= n && c == j - n) ? TC(1) : TC(0);
    }
    x += static_cast<size_t>(j) * n;
  } else {
    for (int c = tid; c < n; c += nthreads) {
      xs[c] = static_cast<TC>(x[c]);
      bs[c] = static_cast<TC>(b[c]);
    }
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

// Lines per PCR block.  One line per block (P threads) spreads a colour's
// few lines over as many SMs and keeps each step's barrier to P threads:
// measured on B200 at 256^3, one MG application 3.42 ms with 4 lines per
// block, 3.18 with 2, 3.08 with 1.
#ifndef HFPS_PCR_LINES
#define HFPS_PCR_LINES 1
#endif
void pcr_shape(int extent, int& P, int& lines_per_block, int& steps) {
  P = 1;
  steps = 0;
  while (P < extent) {
    P <<= 1;
    ++steps;
  }
  lines_per_block = std::max(1, std::min(1024 / P, HFPS_PCR_LINES));
}

// Lines per block and chunks per line of the scan kernel: at least 296
// blocks (two per SM) where the level allows, at most ScanConfig<T>::threads
// threads, at least 8 lines per block while that still allows chunks of at
// most ScanConfig<T>::rows rows.
struct ScanShape {
  int lpb, chunks, rows;
};

// Lines per block are halved (down to HFPS_SCAN_MIN_LPB) while a colour has
// fewer than two blocks per SM.
#ifndef HFPS_SCAN_MIN_LPB
#define HFPS_SCAN_MIN_LPB 8
#endif
template <class T>
ScanShape scan_shape(long long per_color, int extent) {
  constexpr int rows = ScanConfig<T>::rows;
  ScanShape sh{32, (extent + rows - 1) / rows, 0};
  while (sh.lpb > HFPS_SCAN_MIN_LPB && per_color < 296LL * sh.lpb) sh.lpb >>= 1;
  while (sh.lpb > 1 && sh.lpb * sh.chunks > ScanConfig<T>::threads) sh.lpb >>= 1;
  sh.rows = (extent + sh.chunks - 1) / sh.chunks;
  return sh;
}

struct ScanFlags {
  int hx;
  bool zero_other, zero_self;
};

template <class T, int AXIS, int LPB>
void launch_scan(cudaStream_t s, const Level<T>& L, T* x, const T* b, const T* fac,
                 int color, long long per_color, const ScanShape& sh, ScanFlags f) {
  const int blocks = static_cast<int>((per_color + LPB - 1) / LPB);
  const size_t smem = static_cast<size_t>(4) * sh.chunks * LPB * sizeof(T);
  // The zero variants and split rows only on y- and z-line levels (x-line
  // levels keep the natural order and always read x, which the cycle has
  // cleared).
  const dim3 block(LPB, sh.chunks);
  constexpr bool kYZ = AXIS != 0;
  const int mode = !kYZ ? kScanNormal
                        : (f.zero_other && f.zero_self ? kScanFresh
                                                       : (f.zero_self ? kScanOwnZero : kScanNormal));
  const bool split = kYZ && f.hx != 0;
#define HFPS_SCAN_LAUNCH(MODE, SPLIT)                                                         \
  launch(k_line_scan_color<T, AXIS, LPB, kYZ ? MODE : kScanNormal, kYZ && SPLIT>, blocks, block, \
         smem, s, L, x, b, fac, color, sh.rows, f.hx)
  if (mode == kScanFresh) {
    if (split) HFPS_SCAN_LAUNCH(kScanFresh, true);
    else HFPS_SCAN_LAUNCH(kScanFresh, false);
  } else if (mode == kScanOwnZero) {
    if (split) HFPS_SCAN_LAUNCH(kScanOwnZero, true);
    else HFPS_SCAN_LAUNCH(kScanOwnZero, false);
  } else {
    if (split) HFPS_SCAN_LAUNCH(kScanNormal, true);
    else HFPS_SCAN_LAUNCH(kScanNormal, false);
  }
#undef HFPS_SCAN_LAUNCH
}

template <class T, int AXIS>
void launch_scan_axis(cudaStream_t s, const Level<T>& L, T* x, const T* b, const T* fac,
                      int color, long long per_color, const ScanShape& sh, ScanFlags f) {
  switch (sh.lpb) {
    case 32: launch_scan<T, AXIS, 32>(s, L, x, b, fac, color, per_color, sh, f); break;
    case 16: launch_scan<T, AXIS, 16>(s, L, x, b, fac, color, per_color, sh, f); break;
    case 8: launch_scan<T, AXIS, 8>(s, L, x, b, fac, color, per_color, sh, f); break;
    case 4: launch_scan<T, AXIS, 4>(s, L, x, b, fac, color, per_color, sh, f); break;
    case 2: launch_scan<T, AXIS, 2>(s, L, x, b, fac, color, per_color, sh, f); break;
    default: launch_scan<T, AXIS, 1>(s, L, x, b, fac, color, per_color, sh, f); break;
  }
}

}  // namespace

int line_kind(int nx, int ny, int nz, int axis) {
  const int extent = line_extent(axis, nx, ny, nz);
  const int a_extent = axis == 0 ? ny : nx;
  const int b_extent = axis == 2 ? ny : nz;
  const long long per_color = static_cast<long long>((a_extent + 1) / 2) * b_extent;
  const long long threshold =
      extent >= kLinePcrLongExtent ? kLinePcrThresholdLong : kLinePcrThreshold;
  if (per_color < threshold && extent <= 1024) return kLinePcr;
  return extent <= kScanMaxExtent ? kLineScan : kLineNone;
}

template <class T>
size_t line_factor_values(int nx, int ny, int nz, int axis) {
  const int extent = line_extent(axis, nx, ny, nz);
  const int a_extent = axis == 0 ? ny : nx;
  const int b_extent = axis == 2 ? ny : nz;
  const size_t lines = static_cast<size_t>(a_extent) * b_extent;
  const int kind = line_kind(nx, ny, nz, axis);
  if (kind == kLineNone) return 0;
  if (kind == kLineScan)
    return ScanLayout{extent, ((a_extent + 1) / 2) * b_extent}.values(ScanConfig<T>::arrays);
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
  const int kind = line_kind(L.nx, L.ny, L.nz, axis);
  if (kind == kLineNone) return;
  if (kind == kLineScan) {
    launch(k_scan_factors<T>, (lines + 127) / 128, 128, 0, s, L, axis, fac);
    return;
  }
  int P, lpb, steps;
  pcr_shape(extent, P, lpb, steps);
  const size_t smem = static_cast<size_t>(3) * P * lpb * sizeof(T);
  launch(k_pcr_factors<T>, (lines + lpb - 1) / lpb, dim3(P, lpb), smem, s, L, axis, P, fac);
}

template <class T>
void launch_line_pass(cudaStream_t s, const Level<T>& L, T* x, const T* b,
                      const T* fac, T* scratch, int axis, int color, int hx,
                      bool zero_other, bool zero_self) {
  (void)scratch;
  const int extent = line_extent(axis, L.nx, L.ny, L.nz);
  const int a_extent = axis == 0 ? L.ny : L.nx;
  const int b_extent = axis == 2 ? L.ny : L.nz;
  const long long per_color = static_cast<long long>((a_extent + 1) / 2) * b_extent;
  const int kind = line_kind(L.nx, L.ny, L.nz, axis);
  if (kind == kLineNone) return;
  if (kind == kLineScan) {
    const ScanShape sh = scan_shape<T>(per_color, extent);
    const ScanFlags f{axis == 0 ? 0 : hx, zero_other, zero_self};
    if (axis == 0) launch_scan_axis<T, 0>(s, L, x, b, fac, color, per_color, sh, f);
    else if (axis == 1) launch_scan_axis<T, 1>(s, L, x, b, fac, color, per_color, sh, f);
    else launch_scan_axis<T, 2>(s, L, x, b, fac, color, per_color, sh, f);
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
    launch(k_line_pcr_factored_color<T, N>, blocks, block, smem, s, L, x, b, fac, axis, \
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
                        const TC* fac, int sweeps, int axis, bool columns) {
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
    launch(k_coarse_line_smem<T, TC, N>, columns ? 2 * static_cast<int>(cells) : 1, block, smem, \
                                    s, L, x, b, fac, sweeps, axis, columns);       \
    break;
    HFPS_COARSE_CASE(0) HFPS_COARSE_CASE(1) HFPS_COARSE_CASE(2) HFPS_COARSE_CASE(3)
    HFPS_COARSE_CASE(4) HFPS_COARSE_CASE(5) HFPS_COARSE_CASE(6) HFPS_COARSE_CASE(7)
    HFPS_COARSE_CASE(8) HFPS_COARSE_CASE(9)
#undef HFPS_COARSE_CASE
    default: return false;
  }
  return true;
}

template size_t line_factor_values<double>(int, int, int, int);
template size_t line_factor_values<float>(int, int, int, int);
template void launch_line_factors<double>(cudaStream_t, const Level<double>&, int, double*);
template void launch_line_factors<float>(cudaStream_t, const Level<float>&, int, float*);
template void launch_line_pass<double>(cudaStream_t, const Level<double>&, double*,
                                       const double*, const double*, double*, int, int, int,
                                       bool, bool);
template void launch_line_pass<float>(cudaStream_t, const Level<float>&, float*, const float*,
                                      const float*, float*, int, int, int, bool, bool);
template bool launch_coarse_line<double, double>(cudaStream_t, const Level<double>&, double*,
                                                 const double*, const double*, int, int, bool);
template bool launch_coarse_line<float, double>(cudaStream_t, const Level<double>&, float*,
                                                const float*, const double*, int, int, bool);

// ---------------------------------------------------------------------------
// Coarsest level as a dense affine map: out = P x + M b, with P and M
// (n x n each, FP64) stored column-major one after the other, as the
// columns mode of k_coarse_line_smem writes them.  A block owns 32 rows (one
// per lane); its 32 warps take every 32nd column with 8 column loads in
// flight per thread, and the 32 partial sums of a row are added in warp
// order, so the result is reproducible (dense_rows).
template <class T>
__global__ void __launch_bounds__(32 * kDenseWarps)
    k_coarse_dense(int n, const double* __restrict__ op, const T* __restrict__ x,
                   const T* __restrict__ b, T* __restrict__ out, bool x_zero) {
  grid_dependency_sync();
  extern __shared__ double dense_smem[];
  double* v = dense_smem;                    // [2n]: x then b, widened
  double* part = dense_smem + 2 * n;         // [kDenseWarps][32]
  const int tid = threadIdx.y * 32 + threadIdx.x;
  for (int j = tid; j < n; j += 32 * kDenseWarps) {
    v[j] = x_zero ? 0.0 : static_cast<double>(x[j]);
    v[n + j] = static_cast<double>(b[j]);
  }
  __syncthreads();
  dense_rows<T>(n, op, v, part, blockIdx.x, threadIdx.x, threadIdx.y, x_zero, out);
}

template <class T>
void launch_coarse_dense(cudaStream_t s, int n, const double* op, const T* x,
                         const T* b, T* out, bool x_zero) {
  const size_t smem = (2 * static_cast<size_t>(n) + 32 * kDenseWarps) * sizeof(double);
  if (smem > 48 * 1024)
    cudaFuncSetAttribute(k_coarse_dense<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         static_cast<int>(smem));
  launch(k_coarse_dense<T>, (n + 31) / 32, dim3(32, kDenseWarps), smem, s, n, op, x, b, out,
         x_zero);
}

template void launch_coarse_dense<double>(cudaStream_t, int, const double*, const double*,
                                          const double*, double*, bool);
template void launch_coarse_dense<float>(cudaStream_t, int, const double*, const float*,
                                         const float*, float*, bool);

}  // namespace hfps
