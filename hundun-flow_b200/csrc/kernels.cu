// sm_100a kernels of the pressure solve: level stencils, smoothers, grid
// transfers, Krylov vector kernels with fused deterministic reductions, and
// the hierarchy setup.  Each kernel names the reference loop it replaces
// (paths relative to versions/v0.4 of the reference).
//
// All of it is HBM-bound integer-indexed stencil work (about 0.27 flop per
// byte): kernels read each operand once with coalesced x-fastest accesses,
// neighbours come from L1/L2, and reductions use warp shuffles plus one
// block pass, finished by the last block to arrive (fixed order, so every
// sum is reproducible run to run).
#include "kernels.hpp"
#include "phase_device.cuh"

#include <algorithm>
#include <cmath>

namespace hfps {
namespace {

constexpr int kThreads = 256;
// Row-per-block kernels (transfers): at most this many threads per block,
// fewer (a multiple of 32) for short rows.
constexpr int kRowThreads = 128;

dim3 row_grid(int rows, int row_length, int& threads) {
  threads = std::min(kRowThreads, (row_length + 31) / 32 * 32);
  return dim3(rows, (row_length + threads - 1) / threads);
}
constexpr int kMaxReductionBlocks = 148 * 8;

int grid_for(long long items) {
  long long blocks = (items + kThreads - 1) / kThreads;
  if (blocks < 1) blocks = 1;
  if (blocks > 148LL * 32) blocks = 148LL * 32;
  return static_cast<int>(blocks);
}

// Last block to finish reduces the per-block partials in block order and
// applies the scalar update `op`.  Returns true in every thread of the last
// block.
template <int N>
__device__ bool finish_reduction(double (&v)[N], const Reduce& red) {
  block_sum<N>(v);
  __shared__ bool last;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int n = 0; n < N; ++n) red.partials[blockIdx.x * N + n] = v[n];
    __threadfence();
    const unsigned done = atomicAdd(&red.scalars->counters[red.op], 1u);
    last = done == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  // Fixed-order final pass: thread t sums partials t, t+blockDim, ...
  double acc[N];
#pragma unroll
  for (int n = 0; n < N; ++n) acc[n] = 0.0;
  for (int b = threadIdx.x; b < static_cast<int>(gridDim.x); b += blockDim.x) {
#pragma unroll
    for (int n = 0; n < N; ++n)
      acc[n] += reinterpret_cast<volatile double*>(red.partials)[b * N + n];
  }
  block_sum<N>(acc);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int n = 0; n < N; ++n) v[n] = acc[n];
    red.scalars->counters[red.op] = 0u;
  }
  return true;
}

__device__ void apply_scalar_op(Scalars* sc, int op, double sum) {
  switch (op) {
    case kOpPap: {
      sc->pap = sum;
      const double alpha = sc->rho / sum;
      sc->alpha = alpha;
      if (!(sum > 0.0) || !isfinite(sum)) sc->flags |= 2;
      if (!isfinite(alpha)) sc->flags |= 1;
      break;
    }
    case kOpRecursive:
      sc->rr = sum;
      if (!isfinite(sum)) sc->flags |= 1;
      break;
    case kOpRhoNext: {
      sc->rho_next = sum;
      if (!(sum > 0.0) || !isfinite(sum)) sc->flags |= 2;
      sc->beta = sum / sc->rho;
      sc->rho = sum;
      break;
    }
    case kOpRhoRestart:
      sc->rho_next = sum;
      if (!(sum > 0.0) || !isfinite(sum)) sc->flags |= 2;
      sc->rho = sum;
      sc->beta = 0.0;
      break;
    case kOpScaledNorm: {
      const double scale = sc->misc[2];
      const double norm = scale == 0.0 ? 0.0 : scale * sqrt(sum);
      sc->misc[3] = norm;
      if (!(sum >= 0.0) || !isfinite(norm)) sc->flags |= 1;
      break;
    }
    default:
      sc->misc[0] = sum;
      if (!isfinite(sum)) sc->flags |= 1;
      break;
  }
}

// Grid-wide maximum of non-negative values, in finish_reduction's pattern:
// each block's maximum goes to the partials, and the last block to arrive
// (counter `counter`) takes their maximum.  Maxima do not depend on the
// order, so the result is exact and reproducible.  Returns true in the last
// block, whose thread 0 then holds the result in v.
__device__ double block_max(double v) {
  __shared__ double warp_max[32];
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) warp_max[warp] = v;
  __syncthreads();
  double m = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < static_cast<int>((blockDim.x + 31) >> 5); ++w) m = fmax(m, warp_max[w]);
  return m;
}

__device__ bool finish_max(double& v, Scalars* sc, double* partials, int counter) {
  const double m = block_max(v);
  __shared__ bool last;
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = m;
    __threadfence();
    last = atomicAdd(&sc->counters[counter], 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  double acc = 0.0;
  for (int b = threadIdx.x; b < static_cast<int>(gridDim.x); b += blockDim.x)
    acc = fmax(acc, reinterpret_cast<volatile double*>(partials)[b]);
  acc = block_max(acc);
  if (threadIdx.x == 0) {
    v = acc;
    sc->counters[counter] = 0u;
  }
  return true;
}

// Index of natural cell c in a vector of layout v.
__device__ __forceinline__ int vec_pos(const VecLayout& v, int c) {
  if (v.hx == 0) return c;
  const int row = c / v.nx;
  const int i = c - row * v.nx;
  return 2 * v.hx * row + (i & 1) * v.hx + (i >> 1);
}

// Calls f(i, j, k, c) for every cell of an nx x ny x nz level: one warp per
// x-row (rows spread over all warps of the grid), lanes along the row, so
// loads are contiguous and the row's j, k are formed once per row.
template <class F>
__device__ __forceinline__ void for_each_cell_by_rows(int nx, int ny, int nz, F f) {
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (blockDim.x >> 5);
  const int rows = ny * nz;
  for (int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); row < rows; row += warps) {
    const int k = row / ny;
    const int j = row - k * ny;
    const int base = nx * row;
#pragma unroll 4
    for (int i = lane; i < nx; i += 32) f(i, j, k, base + i);
  }
}

// ---------------------------------------------------------------------------
// Level operators: apply_level_matrix / apply_level_defect
// (src/solver_mg.cpp:2569-2767).
template <class T>
__global__ void k_level_apply(Level<T> L, const T* __restrict__ x,
                              T* __restrict__ y) {
  grid_dependency_sync();
  const int n = L.nx * L.ny * L.nz;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += gridDim.x * blockDim.x) {
    int i, j, k;
    cell_coords(c, L.nx, L.ny, i, j, k);
    y[c] = row_value(L, x, i, j, k, c);
  }
}

template <class T>
__global__ void k_level_defect(Level<T> L, const T* __restrict__ x,
                               const T* __restrict__ b, T* __restrict__ r, int hx) {
  grid_dependency_sync();
  const int n = L.nx * L.ny * L.nz;
  const SplitPos sp{L.ny, hx};
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += gridDim.x * blockDim.x) {
    int i, j, k;
    cell_coords(c, L.nx, L.ny, i, j, k);
    if (hx == 0)
      r[c] = b[c] - row_value(L, x, i, j, k, c);
    else
      r[c] = b[sp(c, i, j, k)] - row_value<T, PlainLoad, SplitPos>(L, x, i, j, k, c, sp);
  }
}

// Damped red-black Gauss-Seidel colour pass, omega = 0.72
// (fused_point_color_update, src/solver_mg.cpp:3149-3223).  Cells of one
// colour only read the other colour (and themselves), so the pass is
// order-independent and matches the reference's sequential loop exactly.
template <class T>
__global__ void k_rb_color(Level<T> L, T* __restrict__ x,
                           const T* __restrict__ b, int color) {
  grid_dependency_sync();
  const int hx = (L.nx + 1) >> 1;
  const int n = hx * L.ny * L.nz;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += gridDim.x * blockDim.x)
    rb_slot<T>(L, x, b, color, t);
}

// One Chebyshev-Jacobi stage (chebyshev_stream_bulk_kernel,
// src/solver_mg.cpp:2464-2490): d = f_prev d + f_res (b - A x)/D, x' = x + d.
template <class T>
__global__ void k_chebyshev_stage(Level<T> L, const T* __restrict__ x,
                                  const T* __restrict__ b,
                                  T* __restrict__ direction,
                                  T* __restrict__ next, T previous_factor,
                                  T residual_factor, int first) {
  grid_dependency_sync();
  const int n = L.nx * L.ny * L.nz;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += gridDim.x * blockDim.x)
    chebyshev_cell<T>(L, x, b, direction, next, previous_factor, residual_factor, first, c);
}

// Thomas solve of one line (solve_one, src/solver_mg.cpp:3388-3493).
template <class T>
__device__ void line_thomas(const Level<T>& L, T* x, const T* b, T* work,
                            T* dprime, int axis, int fa, int fb) {
  const int extent = axis == 0 ? L.nx : (axis == 1 ? L.ny : L.nz);
  const int plane = L.nx * L.ny;
  const int stride = axis == 0 ? 1 : (axis == 1 ? L.nx : plane);
  int i0, j0, k0;
  if (axis == 0) { i0 = 0; j0 = fa; k0 = fb; }
  else if (axis == 1) { i0 = fa; j0 = 0; k0 = fb; }
  else { i0 = fa; j0 = fb; k0 = 0; }
  const int c0 = i0 + L.nx * (j0 + L.ny * k0);
  T prev_work = T(0), prev_d = T(0);
  for (int s = 0; s < extent; ++s) {
    const int i = axis == 0 ? s : i0;
    const int j = axis == 1 ? s : j0;
    const int k = axis == 2 ? s : k0;
    const int c = c0 + s * stride;
    const int fxi = face_x_index(L, c, j, k);
    const int fyi = face_y_index(L, c, k);
    T lowf, highf;
    if (axis == 0) { lowf = L.fx[fxi]; highf = L.fx[fxi + 1]; }
    else if (axis == 1) { lowf = L.fy[fyi]; highf = L.fy[fyi + L.nx]; }
    else { lowf = L.fz[c]; highf = L.fz[c + plane]; }
    const T a = s == 0 ? T(0) : -lowf;
    const T bb = L.diag[c];
    const T cc = s + 1 == extent ? T(0) : -highf;
    T d = b[c];
    if (axis != 0) {
      d += L.fx[fxi] * line_neighbour(L, x, i, j, k, c, 0, -1);
      d += L.fx[fxi + 1] * line_neighbour(L, x, i, j, k, c, 0, 1);
    }
    if (axis != 1) {
      d += L.fy[fyi] * line_neighbour(L, x, i, j, k, c, 1, -1);
      d += L.fy[fyi + L.nx] * line_neighbour(L, x, i, j, k, c, 1, 1);
    }
    if (axis != 2) {
      d += L.fz[c] * line_neighbour(L, x, i, j, k, c, 2, -1);
      d += L.fz[c + plane] * line_neighbour(L, x, i, j, k, c, 2, 1);
    }
    if (s == 0) d += lowf * line_neighbour(L, x, i, j, k, c, axis, -1);
    if (s + 1 == extent) d += highf * line_neighbour(L, x, i, j, k, c, axis, 1);
    T wv, dv;
    if (s > 0) {
      const T denominator = bb - a * prev_work;
      wv = cc / denominator;
      dv = (d - a * prev_d) / denominator;
    } else {
      wv = cc / bb;
      dv = d / bb;
    }
    work[c] = wv;
    dprime[c] = dv;
    prev_work = wv;
    prev_d = dv;
  }
  T next_x = T(0);
  for (int s = extent; s-- > 0;) {
    const int c = c0 + s * stride;
    const T v = s + 1 == extent ? dprime[c] : dprime[c] - work[c] * next_x;
    x[c] = v;
    next_x = v;
  }
}

// Fused retained defect + restriction (apply_level_defect followed by
// restrict_residual, src/solver_mg.cpp:3633-3721): every coarse cell sums
// the defects of its children in dz, dy, dx order; coarse x is zeroed.
// Fused defect + restriction: one block per coarse x-row (blockIdx.x;
// blockIdx.y splits long rows), one coarse cell per thread, the coarsening
// mask fixed at compile time; coarse x is zeroed.  Fine x and b in layout hx.
template <class T, int MASK>
__global__ void __launch_bounds__(kRowThreads)
    k_defect_restrict(Level<T> F, const T* __restrict__ x, const T* __restrict__ b, Level<T> C,
                      T* __restrict__ cb, T* __restrict__ cx, int hx, int hxc) {
  grid_dependency_sync();
  const int row = blockIdx.x;
  const int ci = blockIdx.y * blockDim.x + threadIdx.x;
  if (ci >= C.nx) return;
  const int ck = row / C.ny;
  const int cj = row - ck * C.ny;
  const int cc = hxc == 0 ? ci + C.nx * row : SplitPos{C.ny, hxc}(0, ci, cj, ck);
  cb[cc] = hx == 0
               ? defect_restrict_at<T, PlainLoad, NaturalPos, MASK>(F, x, b, MASK, ci, cj, ck,
                                                                   NaturalPos())
               : defect_restrict_at<T, PlainLoad, SplitPos, MASK>(F, x, b, MASK, ci, cj, ck,
                                                                 SplitPos{F.ny, hx});
  cx[cc] = T(0);
}

// Trilinear prolongation and add, zero on solid cells (prolongate_cell).
// One block per fine x-row (blockIdx.x; blockIdx.y splits long rows), one
// vector entry per thread (natural order, or split rows walked entry by
// entry so that stores stay contiguous), the coarse correction through the
// read-only path, the coarsening mask fixed at compile time.
template <class T, int MASK>
__global__ void __launch_bounds__(kRowThreads)
    k_prolongate(Level<T> F, T* __restrict__ x, Level<T> C, const T* __restrict__ cx, int hx,
                 int hxc) {
  grid_dependency_sync();
  const int row = blockIdx.x;
  const int w = blockIdx.y * blockDim.x + threadIdx.x;
  int i = w;
  if (hx != 0) {
    const int odd = w >= hx ? 1 : 0;
    i = 2 * (w - odd * hx) + odd;
  }
  if (i >= F.nx || (hx != 0 && w >= 2 * hx)) return;  // past the row (or the odd half's padding)
  const int k = row / F.ny;
  const int j = row - k * F.ny;
  const int c = i + F.nx * row;
  const int at = hx == 0 ? c : 2 * hx * row + w;
  x[at] = hxc == 0 ? prolongate_cell<T, PlainLoad, RoLoad, MASK>(F, x, C, cx, MASK, c, i, j, k, at)
                   : prolongate_cell<T, PlainLoad, RoLoad, MASK, SplitPos>(
                         F, x, C, cx, MASK, c, i, j, k, at, SplitPos{C.ny, hxc});
}

// Prolongation for x/z coarsening (mask 5, y kept: the levels of y-line
// relaxation) into split fine rows.  A thread takes the up to 2x2 fine cells
// (2p + dx, j, 2q + dz) over coarse cell (p, j, q).  Their stencils lie in
// coarse cells p-1..p+1 x q-1..q+1, so the nine values are loaded once
// (indices clamped into the level).  Fine cell dx takes its left and right
// x-candidates from columns dx and dx+1 of that block (rows dz and dz+1 in
// z): interp_axis's candidates are p-1/p (even) and p/p+1 (odd), and where it
// clamps at a level edge the clamped load holds the same cell.  Each fine
// value is then formed exactly as prolongate_cell forms it (same weights,
// terms and order), so results are bit-identical to k_prolongate<T, 5>.
template <class T, class CPos>
__global__ void __launch_bounds__(kRowThreads)
    k_prolongate_xz(Level<T> F, T* __restrict__ x, Level<T> C, const T* __restrict__ cx,
                    int hx, CPos cpos) {
  grid_dependency_sync();
  const int crow = blockIdx.x;  // j + ny * q (the coarse level keeps ny)
  const int p = blockIdx.y * blockDim.x + threadIdx.x;
  if (p >= C.nx) return;
  const int q = crow / F.ny;
  const int j = crow - q * F.ny;
  T v[3][3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int zq = min(max(q + a - 1, 0), C.nz - 1);
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      const int xp = min(max(p + b - 1, 0), C.nx - 1);
      v[a][b] = __ldg(cx + cpos(xp + C.nx * (j + C.ny * zq), xp, j, zq));
    }
  }
  // The four fine values and flags are loaded before any store: a load
  // issued after a store to the same array cannot be hoisted above it, and
  // would otherwise wait on the previous cell's load.
  T old[2][2];
  bool fluid[2][2];
#pragma unroll
  for (int dz = 0; dz < 2; ++dz)
#pragma unroll
    for (int dx = 0; dx < 2; ++dx) {
      const int i = 2 * p + dx, k = 2 * q + dz;
      const bool in = i < F.nx && k < F.nz;
      fluid[dz][dx] = in && F.fluid[i + F.nx * (j + F.ny * k)] != 0;
      old[dz][dx] = in ? x[2 * hx * (j + F.ny * k) + dx * hx + p] : T(0);
    }
#pragma unroll
  for (int dz = 0; dz < 2; ++dz) {
    const int k = 2 * q + dz;
    if (k >= F.nz) break;
    int zl, zr;
    double zw;
    interp_axis(k, 1, C.nz, zl, zr, zw);
    const bool two_z = zl != zr;
#pragma unroll
    for (int dx = 0; dx < 2; ++dx) {
      const int i = 2 * p + dx;
      if (i >= F.nx) break;
      int xl, xr;
      double xw;
      interp_axis(i, 1, C.nx, xl, xr, xw);
      const bool two_x = xl != xr;
      const int at = 2 * hx * (j + F.ny * k) + dx * hx + p;
      T value = T(0);
#pragma unroll
      for (int az = 0; az < 2; ++az)
#pragma unroll
        for (int ax = 0; ax < 2; ++ax) {
          const double wz = az == 0 ? 1.0 - zw : zw;
          const double wy = 1.0;
          const double wx = ax == 0 ? 1.0 - xw : xw;
          const T w = static_cast<T>(wx * wy * wz);
          const T term = w * v[dz + az][dx + ax];
          const bool on = (az == 0 || two_z) && (ax == 0 || two_x);
          const T sum = value + term;
          value = on ? sum : value;
        }
      x[at] = fluid[dz][dx] ? old[dz][dx] + value : T(0);
    }
  }
}

// Coarsest level: `sweeps` smoother sweeps in one CTA (mg_cycle coarse
// branch, src/solver_mg.cpp:4210-4227).  The state is widened to TC (FP64
// in the mixed-precision hierarchy) for the duration of the solve.
template <class T, class TC>
// x / xs are updated by every thread between barriers: no __restrict__.
__global__ void k_coarse_solve(Level<TC> L, T* x, const T* b, TC* xs, TC* bs,
                               TC* work, TC* dprime, int sweeps,
                               int line_axis) {
  grid_dependency_sync();
  const int n = L.nx * L.ny * L.nz;
  TC* xw = xs;
  const TC* bw = bs;
  if (xs != nullptr) {
    for (int c = threadIdx.x; c < n; c += blockDim.x) {
      xs[c] = static_cast<TC>(x[c]);
      bs[c] = static_cast<TC>(b[c]);
    }
    __syncthreads();
  } else {
    xw = reinterpret_cast<TC*>(x);
    bw = reinterpret_cast<const TC*>(b);
  }
  if (line_axis < 0) {
    coarse_point_sweeps(L, xw, bw, sweeps, threadIdx.x, blockDim.x);
  } else {
    const int a_extent = line_axis == 0 ? L.ny : L.nx;
    const int b_extent = line_axis == 2 ? L.ny : L.nz;
    const int ha = (a_extent + 1) >> 1;
    const int lines = ha * b_extent;
    for (int s = 0; s < sweeps; ++s) {
      for (int color = 0; color < 2; ++color) {
        for (int t = threadIdx.x; t < lines; t += blockDim.x) {
          const int fb = t / ha;
          const int fa = 2 * (t - fb * ha) + ((fb + color) & 1);
          if (fa >= a_extent) continue;
          line_thomas(L, xw, bw, work, dprime, line_axis, fa, fb);
        }
        __syncthreads();
      }
    }
  }
  if (xs != nullptr) {
    for (int c = threadIdx.x; c < n; c += blockDim.x) x[c] = static_cast<T>(xs[c]);
  }
}

// ---------------------------------------------------------------------------
// MG entry/exit (apply_impl, src/solver_mg.cpp:4866-4878, 5078-5117).
template <class T>
__global__ void k_mg_enter(int n, const double* __restrict__ r,
                           const uint8_t* __restrict__ active,
                           T* __restrict__ b, T* __restrict__ x, VecLayout v, bool zero_x) {
  grid_dependency_sync();
  // A warp per x-row: the split position of a cell is then the row's base
  // plus its parity half, with no division per cell.
  for_each_cell_by_rows(v.nx, v.ny, n / (v.nx * v.ny), [&](int i, int j, int k, int c) {
    const bool on = active == nullptr || active[c] != 0;
    const int at = v.hx == 0 ? c : 2 * v.hx * (j + v.ny * k) + (i & 1) * v.hx + (i >> 1);
    b[at] = on ? static_cast<T>(r[c]) : T(0);
    if (zero_x) x[at] = T(0);
  });
}

template <class T>
__global__ void k_mg_exit(int n, const T* __restrict__ x,
                          const uint8_t* __restrict__ active,
                          const double* __restrict__ scale_ptr,
                          double* __restrict__ z, VecLayout v) {
  grid_dependency_sync();
  const double scale = scale_ptr == nullptr ? 1.0 : *scale_ptr;
  for_each_cell_by_rows(v.nx, v.ny, n / (v.nx * v.ny), [&](int i, int j, int k, int c) {
    const bool on = active == nullptr || active[c] != 0;
    const int at = v.hx == 0 ? c : 2 * v.hx * (j + v.ny * k) + (i & 1) * v.hx + (i >> 1);
    z[c] = on ? static_cast<double>(x[at]) * scale : 0.0;
  });
}

// MG exit with the PCG's r.z: z = active ? x : 0 (unit scaling) and the sum
// of r * z, accumulated in k_dot's order (same grid, same per-thread cells),
// then red.op.  Replaces k_mg_exit followed by k_dot(r, z).
template <class T>
__global__ void k_mg_exit_dot(int n, const T* __restrict__ x,
                              const uint8_t* __restrict__ active, double* __restrict__ z,
                              VecLayout v, const double* __restrict__ r, Reduce red) {
  grid_dependency_sync();
  double acc[1] = {0.0};
  // k_dot's cells per thread (grid stride), with the cell's row and x index
  // carried from step to step instead of divided out of c each time.
  const int stride = gridDim.x * blockDim.x;
  const int row_step = stride / v.nx, i_step = stride - row_step * v.nx;
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  int row = c / v.nx;
  int i = c - row * v.nx;
  for (; c < n; c += stride) {
    const bool on = active == nullptr || active[c] != 0;
    const int at = v.hx == 0 ? c : 2 * v.hx * row + (i & 1) * v.hx + (i >> 1);
    const double zc = on ? static_cast<double>(x[at]) * 1.0 : 0.0;
    z[c] = zc;
    acc[0] += r[c] * zc;
    row += row_step;
    i += i_step;
    if (i >= v.nx) {
      i -= v.nx;
      ++row;
    }
  }
  if (finish_reduction<1>(acc, red) && threadIdx.x == 0)
    apply_scalar_op(red.scalars, red.op, acc[0]);
}

template <class T>
__global__ void k_diagonal_solve(int n, const T* __restrict__ b,
                                 const T* __restrict__ diag,
                                 T* __restrict__ x, VecLayout v) {
  grid_dependency_sync();
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += gridDim.x * blockDim.x) {
    const int at = vec_pos(v, c);
    x[at] = b[at] / diag[c];
  }
}

template <class T>
__global__ void k_mg_projection(int n, const double* __restrict__ r_in,
                                const uint8_t* __restrict__ active,
                                const T* __restrict__ recursive, Reduce red) {
  grid_dependency_sync();
  double v[3] = {0.0, 0.0, 0.0};
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += gridDim.x * blockDim.x) {
    const bool on = active == nullptr || active[c] != 0;
    const double r = on ? r_in[c] : 0.0;
    const double az = r - static_cast<double>(recursive[c]);
    v[0] += r * r;
    v[1] += r * az;
    v[2] += az * az;
  }
  if (finish_reduction<3>(v, red) && threadIdx.x == 0) {
    Scalars* sc = red.scalars;
    sc->proj[0] = v[0];
    sc->proj[1] = v[1];
    sc->proj[2] = v[2];
    const double tiny = 2.220446049250313e-16 * v[0];
    sc->mg_alpha = v[2] > tiny ? v[1] / v[2] : 0.0;
    if (!isfinite(v[0]) || !isfinite(v[1]) || !isfinite(v[2]) ||
        !isfinite(sc->mg_alpha))
      sc->flags |= 1;
  }
}

// ---------------------------------------------------------------------------
// Krylov kernels (FP64).  solve_pcg's operator apply + p.Ap
// (src/solver_krylov.cpp:1426-1447), x/r update + recursive norm
// (:1448-1463), r.z (:1536-1540) and p = z + beta p (:1546).
__global__ void k_spmv_dot(Level<double> L, const double* __restrict__ x,
                           double* __restrict__ y, Reduce red) {
  grid_dependency_sync();
  double v[1] = {0.0};
  for_each_cell_by_rows(L.nx, L.ny, L.nz, [&](int i, int j, int k, int c) {
    const double a = row_value(L, x, i, j, k, c);
    y[c] = a;
    v[0] += x[c] * a;
  });
  if (finish_reduction<1>(v, red) && threadIdx.x == 0)
    apply_scalar_op(red.scalars, red.op, v[0]);
}

__global__ void k_residual_norm(Level<double> L, const double* __restrict__ x,
                                const double* __restrict__ b,
                                double* __restrict__ r, Reduce red) {
  grid_dependency_sync();
  double v[1] = {0.0};
  for_each_cell_by_rows(L.nx, L.ny, L.nz, [&](int i, int j, int k, int c) {
    const double value = b[c] - row_value(L, x, i, j, k, c);
    r[c] = value;
    v[0] += value * value;
  });
  if (finish_reduction<1>(v, red) && threadIdx.x == 0)
    apply_scalar_op(red.scalars, red.op, v[0]);
}

// The Krylov operator y = A x with x.y over 3-D tiles: a CTA of kTileX x
// kTileY threads owns those columns of (i, j) and marches up DEPTH planes.
// Each plane of x is read from HBM once: the thread keeps its column's
// x(k-1), x(k), x(k+1) in registers and publishes x(k) in a shared-memory
// tile with a one-cell ring, from which the four in-plane neighbours are
// read; the z-faces' upper value is carried to the next plane.  The row is
// evaluated as row_value evaluates it (same terms, same order), so y is
// bit-identical to k_spmv_dot's; the reduction groups its partial sums by
// tile.  (The same tiling for the true residual r = b - A x was slower than
// k_residual_norm at 256^3, 0.208 against 0.180 ms, and is not used.)
constexpr int kTileX = 32;
constexpr int kTileY = 8;
// Tiles per launch: at most one reduction partial each in the solver's
// partials block (kBasisChunk * 148 * 8 doubles and more).
constexpr long long kMaxTiledBlocks = 16384;

template <int DEPTH>  // planes a CTA marches (a compile-time trip count)
__global__ void __launch_bounds__(kTileX * kTileY)
    k_stencil_tiled(Level<double> L, const double* __restrict__ x, double* __restrict__ y,
                    Reduce red) {
  grid_dependency_sync();
  __shared__ double tile[2][kTileY + 2][kTileX + 2];
  const int nx = L.nx, ny = L.ny, nz = L.nz;
  const int tiles_x = (nx + kTileX - 1) / kTileX;
  const int tiles_y = (ny + kTileY - 1) / kTileY;
  const int bx = blockIdx.x % tiles_x;
  const int rest = blockIdx.x / tiles_x;
  const int by = rest % tiles_y;
  const int bz = rest / tiles_y;
  const int tx = threadIdx.x % kTileX, ty = threadIdx.x / kTileX;
  const int i = bx * kTileX + tx, j = by * kTileY + ty;
  const int k0 = bz * DEPTH, k1 = min(nz, k0 + DEPTH);
  const bool on = i < nx && j < ny;
  const int ic = min(i, nx - 1), jc = min(j, ny - 1);
  const int plane = nx * ny;
  const unsigned nb = L.neumann;
  // Ring loads of this thread (in-plane neighbours outside the tile).
  const bool ring_w = tx == 0 && i > 0 && on;
  const bool ring_e = (tx == kTileX - 1 || i == nx - 1) && i + 1 < nx && on;
  const bool ring_s = ty == 0 && j > 0 && on;
  const bool ring_n = (ty == kTileY - 1 || j == ny - 1) && j + 1 < ny && on;
  int c = ic + nx * (jc + ny * k0);
  double x_prev = (on && k0 > 0) ? x[c - plane] : 0.0;
  double x_cur = on ? x[c] : 0.0;
  double fz_lo = on ? L.fz[c] : 0.0;
  double acc[1] = {0.0};
  int buf = 0;
  for (int k = k0; k < k1; ++k, c += plane) {
    const double x_next = (on && k + 1 < nz) ? x[c + plane] : 0.0;
    tile[buf][ty + 1][tx + 1] = x_cur;
    if (ring_w) tile[buf][ty + 1][tx] = x[c - 1];
    if (ring_e) tile[buf][ty + 1][tx + 2] = x[c + 1];
    if (ring_s) tile[buf][ty][tx + 1] = x[c - nx];
    if (ring_n) tile[buf][ty + 2][tx + 1] = x[c + nx];
    __syncthreads();
    if (on) {
      const double xc = x_cur;
      const double xm = i > 0 ? tile[buf][ty + 1][tx] : ((nb & 1u) ? xc : 0.0);
      const double xp = i + 1 < nx ? tile[buf][ty + 1][tx + 2] : ((nb & 2u) ? xc : 0.0);
      const double ym = j > 0 ? tile[buf][ty][tx + 1] : ((nb & 4u) ? xc : 0.0);
      const double yp = j + 1 < ny ? tile[buf][ty + 2][tx + 1] : ((nb & 8u) ? xc : 0.0);
      const double zm = k > 0 ? x_prev : ((nb & 16u) ? xc : 0.0);
      const double zp = k + 1 < nz ? x_next : ((nb & 32u) ? xc : 0.0);
      const int fxi = face_x_index(L, c, j, k);
      const int fyi = face_y_index(L, c, k);
      const double fz_hi = L.fz[c + plane];
      double v = L.diag[c] * xc;
      v -= L.fx[fxi] * xm;
      v -= L.fx[fxi + 1] * xp;
      v -= L.fy[fyi] * ym;
      v -= L.fy[fyi + nx] * yp;
      v -= fz_lo * zm;
      v -= fz_hi * zp;
      y[c] = v;
      acc[0] += xc * v;
      fz_lo = fz_hi;
    }
    x_prev = x_cur;
    x_cur = x_next;
    buf ^= 1;
  }
  if (finish_reduction<1>(acc, red) && threadIdx.x == 0)
    apply_scalar_op(red.scalars, red.op, acc[0]);
}

// ---------------------------------------------------------------------------
// Cold-path diagonal IC(0) (ColdPressureIccg, src/solver_iccg.hpp:224-293;
// ColdPressureDilu, src/solver_cold.hpp:484-560, identical on the symmetric
// pressure rows).  The factorisation and both triangular sweeps follow the
// reference's lexicographic order exactly: a cell depends only on its lower
// (resp. upper) neighbours, which all lie on the previous wavefront plane
// i + j + k = t - 1 (resp. t + 1), so every plane is one parallel launch and
// each cell's arithmetic is the reference's, operation for operation.  The
// couplings are the IBM-masked level-0 face coefficients.

// Row diagonal of the decorated operator: identity on solid cells; a link to
// a solid cell or a Neumann boundary face leaves the row and its coefficient
// is subtracted from the diagonal, in face order x-, x+, y-, y+, z-, z+.
__global__ void k_dic_rows(int nx, int ny, int nz, unsigned neumann, const double* diag,
                           const double* fx, const double* fy, const double* fz,
                           const uint8_t* active, double* out) {
  grid_dependency_sync();
  const int n = nx * ny * nz;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += gridDim.x * blockDim.x) {
    int i, j, k;
    cell_coords(c, nx, ny, i, j, k);
    const auto on = [&](int q) { return active == nullptr || active[q] != 0; };
    if (!on(c)) {
      out[c] = 1.0;
      continue;
    }
    const int fxi = c + j + ny * k;
    const int fyi = c + nx * k;
    const int plane = nx * ny;
    const double face[6] = {fx[fxi], fx[fxi + 1], fy[fyi], fy[fyi + nx], fz[c], fz[c + plane]};
    const int at[3] = {i, j, k};
    const int ext[3] = {nx, ny, nz};
    const int step[3] = {1, nx, plane};
    double d = diag[c];
    for (int f = 0; f < 6; ++f) {
      const int a = f >> 1;
      const int q = at[a] + ((f & 1) ? 1 : -1);
      if (q < 0 || q >= ext[a]) {
        if ((neumann >> f) & 1u) d -= face[f];
        continue;
      }
      if (!on((f & 1) ? c + step[a] : c - step[a])) d -= face[f];
    }
    out[c] = d;
  }
}

// Cell (i, j, k) of wavefront plane t handled by this thread, or false.
__device__ __forceinline__ bool plane_cell(int t, int nx, int ny, int nz, int& i, int& j,
                                           int& k) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= ny * nz) return false;
  k = q / ny;
  j = q - k * ny;
  i = t - j - k;
  return i >= 0 && i < nx;
}

__global__ void k_dic_pivots(int t, Level<double> L, const double* rows, double* inv,
                             Scalars* scalars) {
  grid_dependency_sync();
  int i, j, k;
  if (!plane_cell(t, L.nx, L.ny, L.nz, i, j, k)) return;
  const int c = i + L.nx * (j + L.ny * k);
  const int plane = L.nx * L.ny;
  double pivot = rows[c];
  // lower couplings: the cell's own x-, y-, z- faces
  if (i > 0) {
    const double lower = L.fx[face_x_index(L, c, j, k)];
    pivot -= lower * lower * inv[c - 1];
  }
  if (j > 0) {
    const double lower = L.fy[face_y_index(L, c, k)];
    pivot -= lower * lower * inv[c - L.nx];
  }
  if (k > 0) {
    const double lower = L.fz[c];
    pivot -= lower * lower * inv[c - plane];
  }
  if (!(pivot > 0) || !isfinite(pivot)) atomicOr(&scalars->flags, 1);
  inv[c] = 1 / pivot;
}

__global__ void k_dic_forward(int t, Level<double> L, const double* in, double* out,
                              const double* inv) {
  grid_dependency_sync();
  int i, j, k;
  if (!plane_cell(t, L.nx, L.ny, L.nz, i, j, k)) return;
  const int c = i + L.nx * (j + L.ny * k);
  double value = in[c];
  if (i > 0) value += L.fx[face_x_index(L, c, j, k)] * out[c - 1];
  if (j > 0) value += L.fy[face_y_index(L, c, k)] * out[c - L.nx];
  if (k > 0) value += L.fz[c] * out[c - L.nx * L.ny];
  out[c] = value * inv[c];
}

__global__ void k_dic_backward(int t, Level<double> L, double* out, const double* inv) {
  grid_dependency_sync();
  int i, j, k;
  if (!plane_cell(t, L.nx, L.ny, L.nz, i, j, k)) return;
  const int c = i + L.nx * (j + L.ny * k);
  const int plane = L.nx * L.ny;
  double value = 0;
  // upper couplings: the lower face of the next cell along each axis
  if (i + 1 < L.nx) value += L.fx[face_x_index(L, c, j, k) + 1] * out[c + 1];
  if (j + 1 < L.ny) value += L.fy[face_y_index(L, c, k) + L.nx] * out[c + L.nx];
  if (k + 1 < L.nz) value += L.fz[c + plane] * out[c + plane];
  out[c] += value * inv[c];
}

// ---------------------------------------------------------------------------
// BiCGSTAB kernels (solve_bicgstab, src/solver_krylov.cpp:2651-3090), in the
// reference's per-cell arithmetic.

// p = 1.0 r + beta (1.0 p - omega v) (update_bicgstab_search_direction).
__global__ void k_bicg_direction(int n, double* __restrict__ p, const double* __restrict__ r,
                                 const double* __restrict__ v, double beta, double omega) {
  grid_dependency_sync();
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += gridDim.x * blockDim.x) {
    const double intermediate = 1.0 * p[c] + -omega * v[c];
    p[c] = 1.0 * r[c] + beta * intermediate;
  }
}

// s = 1.0 r - alpha v and |s|^2 (form_bicgstab_intermediate).
__global__ void k_bicg_intermediate(int n, double* __restrict__ s, const double* __restrict__ r,
                                    const double* __restrict__ v, double alpha, Reduce red) {
  grid_dependency_sync();
  double acc[1] = {0.0};
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += gridDim.x * blockDim.x) {
    const double value = 1.0 * r[c] + -alpha * v[c];
    s[c] = value;
    acc[0] += value * value;
  }
  if (finish_reduction<1>(acc, red) && threadIdx.x == 0) apply_scalar_op(red.scalars, red.op, acc[0]);
}

// x = (x + alpha ph) + omega sh, r = 1.0 s - omega t and |r|^2
// (update_bicgstab_solution_residual).
__global__ void k_bicg_update(int n, double* __restrict__ x, const double* __restrict__ ph,
                              const double* __restrict__ sh, double* __restrict__ r,
                              const double* __restrict__ s, const double* __restrict__ t,
                              double alpha, double omega, Reduce red) {
  grid_dependency_sync();
  double acc[1] = {0.0};
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += gridDim.x * blockDim.x) {
    const double intermediate = x[c] + alpha * ph[c];
    x[c] = intermediate + omega * sh[c];
    const double value = 1.0 * s[c] + -omega * t[c];
    r[c] = value;
    acc[0] += value * value;
  }
  if (finish_reduction<1>(acc, red) && threadIdx.x == 0) apply_scalar_op(red.scalars, red.op, acc[0]);
}

// ---------------------------------------------------------------------------
// FGMRES kernels (solve_fgmres, src/solver_krylov.cpp:1557-2650).

// w = A z + (-shift) v: the operator image of the preconditioned basis
// vector shifted by the basis vector itself (add_scaled(ax, -shift, v),
// :2168-2172), in one pass.
__global__ void k_operator_shift(Level<double> L, const double* __restrict__ z,
                                 const double* __restrict__ v, double shift,
                                 double* __restrict__ w) {
  grid_dependency_sync();
  for_each_cell_by_rows(L.nx, L.ny, L.nz, [&](int i, int j, int k, int c) {
    const double a = row_value(L, z, i, j, k, c);
    w[c] = a + -shift * v[c];
  });
}

// Up to kBasisChunk dot products v_r . w (and w . w when `self`), one pass
// over w; deterministic block partials finished by the last block
// (local_multidot + checked_sum, :206-244).
// COUNT basis vectors and SELF fixed at compile time: every load of a cell
// is unconditional, so they are all in flight together (a runtime count
// turned them into a chain of branches, each waiting on its load).
template <int COUNT, bool SELF>
__global__ void k_multidot(int n, BasisRefs basis, const double* __restrict__ w,
                           double* __restrict__ out, Reduce red) {
  grid_dependency_sync();
  double acc[kBasisChunk];
#pragma unroll
  for (int r = 0; r < kBasisChunk; ++r) acc[r] = 0.0;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += gridDim.x * blockDim.x) {
    const double wc = w[c];
#pragma unroll
    for (int r = 0; r < COUNT; ++r) acc[r] += __ldg(basis.v[r] + c) * wc;
    if (SELF) acc[COUNT] += wc * wc;
  }
  constexpr int kOut = COUNT + (SELF ? 1 : 0);
  if (finish_reduction<kBasisChunk>(acc, red) && threadIdx.x == 0) {
    for (int r = 0; r < kOut; ++r) out[r] = acc[r];
    int bad = 0;
    for (int r = 0; r < kOut; ++r) bad |= !isfinite(acc[r]);
    if (bad) red.scalars->flags |= 1;
  }
}

__global__ void k_difference_nonzero(int n, const double* __restrict__ x,
                                     double* __restrict__ snap, Scalars* scalars) {
  grid_dependency_sync();
  int nonzero = 0;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += gridDim.x * blockDim.x) {
    const double v = x[c] - snap[c];
    nonzero |= v != 0.0;
    snap[c] = v;
  }
  if (__any_sync(0xffffffffu, nonzero) && (threadIdx.x & 31) == 0)
    atomicOr(&scalars->marks, 1u);
}

// out = scale * (dst + s_0 v_0 + s_1 v_1 + ...), terms added per cell in
// basis order (add_scaled_basis, :510-564), then optionally scaled
// (scale_copy, :611-625); `out` may be `dst`.
template <int COUNT>
__global__ void k_basis_update(int n, const double* dst, BasisRefs basis,
                               double scale, int scaled, double* out) {
  grid_dependency_sync();
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += gridDim.x * blockDim.x) {
    double v = dst[c];
#pragma unroll
    for (int r = 0; r < COUNT; ++r) v = v + basis.s[r] * __ldg(basis.v[r] + c);
    if (scaled) v = scale * v;
    out[c] = v;
  }
}

__global__ void k_pcg_update(int n, double* __restrict__ x,
                             const double* __restrict__ p,
                             double* __restrict__ r,
                             const double* __restrict__ ap, Reduce red) {
  grid_dependency_sync();
  const double alpha = red.scalars->alpha;
  double v[1] = {0.0};
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += gridDim.x * blockDim.x) {
    x[c] = x[c] + alpha * p[c];
    const double rv = r[c] + -alpha * ap[c];
    r[c] = rv;
    v[0] += rv * rv;
  }
  if (finish_reduction<1>(v, red) && threadIdx.x == 0)
    apply_scalar_op(red.scalars, red.op, v[0]);
}

__global__ void k_dot(int n, const double* __restrict__ a,
                      const double* __restrict__ b, Reduce red) {
  grid_dependency_sync();
  double v[1] = {0.0};
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += gridDim.x * blockDim.x)
    v[0] += a[c] * b[c];
  if (finish_reduction<1>(v, red) && threadIdx.x == 0)
    apply_scalar_op(red.scalars, red.op, v[0]);
}

__global__ void k_norm2(int n, const double* __restrict__ a, Reduce red) {
  grid_dependency_sync();
  double v[1] = {0.0};
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += gridDim.x * blockDim.x)
    v[0] += a[c] * a[c];
  if (finish_reduction<1>(v, red) && threadIdx.x == 0)
    apply_scalar_op(red.scalars, red.op, v[0]);
}

// The two passes of the max-scaled norm (global_norm, src/solver_krylov.cpp:
// 650-711): max |v| into misc[2], a non-finite entry setting flag bit 0;
// then the sum of (v / max)^2, which kOpScaledNorm turns into
// misc[3] = max * sqrt(sum).  The reference sums each rank's squares with
// Neumaier compensation; here the sum is the fixed-order FP64 tree.
__global__ void k_norm_max(int n, const double* __restrict__ a, Scalars* sc,
                           double* partials) {
  grid_dependency_sync();
  double m = 0.0;
  bool bad = false;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += gridDim.x * blockDim.x) {
    const double value = a[c];
    if (!isfinite(value)) bad = true;
    else m = fmax(m, fabs(value));
  }
  if (bad) atomicOr(&sc->flags, 1);
  if (finish_max(m, sc, partials, kOpScaledNorm) && threadIdx.x == 0) sc->misc[2] = m;
}

__global__ void k_norm_scaled_sum(int n, const double* __restrict__ a, Reduce red) {
  grid_dependency_sync();
  const double scale = red.scalars->misc[2];
  double v[1] = {0.0};
  if (scale > 0.0) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n;
         c += gridDim.x * blockDim.x) {
      const double scaled = a[c] / scale;
      v[0] += scaled * scaled;
    }
  }
  if (finish_reduction<1>(v, red) && threadIdx.x == 0)
    apply_scalar_op(red.scalars, red.op, v[0]);
}

// The two passes of project_constant: the volume-weighted sums (FP64, in
// the fixed-order tree; the reference adds them cell by cell), then the
// subtraction, formed in FP64 and stored in the level's precision.
template <class T>
__global__ void k_constant_sums(int n, VecLayout lay, const T* __restrict__ v,
                                const double* __restrict__ volume, Reduce red) {
  grid_dependency_sync();
  double acc[2] = {0.0, 0.0};
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += gridDim.x * blockDim.x) {
    const double w = volume[c];
    acc[0] += w * static_cast<double>(v[vec_pos(lay, c)]);
    acc[1] += w;
  }
  if (finish_reduction<2>(acc, red) && threadIdx.x == 0) {
    Scalars* sc = red.scalars;
    sc->constant_mean = acc[0] / acc[1];
    if (!(acc[1] > 0.0) || !isfinite(acc[0]) || !isfinite(acc[1])) sc->flags |= 1;
  }
}

template <class T>
__global__ void k_constant_apply(int n, VecLayout lay, T* __restrict__ v,
                                 const double* __restrict__ volume,
                                 const Scalars* __restrict__ sc) {
  grid_dependency_sync();
  const double mean = sc->constant_mean;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += gridDim.x * blockDim.x) {
    const int at = vec_pos(lay, c);
    v[at] = volume[c] > 0.0 ? static_cast<T>(static_cast<double>(v[at]) - mean) : T(0);
  }
}

__global__ void k_p_update(int n, double* __restrict__ p,
                           const double* __restrict__ z,
                           const Scalars* __restrict__ sc) {
  grid_dependency_sync();
  const double beta = sc->beta;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += gridDim.x * blockDim.x)
    p[c] = 1.0 * z[c] + beta * p[c];
}

__global__ void k_copy(int n, const double* __restrict__ src,
                       double* __restrict__ dst) {
  grid_dependency_sync();
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += gridDim.x * blockDim.x)
    dst[c] = src[c];
}

// ---------------------------------------------------------------------------
// Setup: copy_finest_coefficients (src/solver_mg.cpp:1469-1570).  A face is
// active iff every adjacent cell is fluid; solid rows become identities; a
// fluid diagonal loses exactly the removed face coefficients.
__device__ __forceinline__ bool cell_on(const uint8_t* a, int c) {
  return a == nullptr || a[c] != 0;
}

__global__ void k_mask_faces(int nx, int ny, int nz, const double* fx_in,
                             const double* fy_in, const double* fz_in,
                             const uint8_t* active, double* fx, double* fy,
                             double* fz) {
  grid_dependency_sync();
  const int nfx = (nx + 1) * ny * nz;
  const int nfy = nx * (ny + 1) * nz;
  const int nfz = nx * ny * (nz + 1);
  const int total = nfx + nfy + nfz;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += gridDim.x * blockDim.x) {
    if (t < nfx) {
      const int row = t / (nx + 1);
      const int i = t - row * (nx + 1);
      const int base = nx * row;
      bool on = true;
      if (i > 0) on = on && cell_on(active, base + i - 1);
      if (i < nx) on = on && cell_on(active, base + i);
      fx[t] = fx_in[t] * (on ? 1.0 : 0.0);
    } else if (t < nfx + nfy) {
      const int f = t - nfx;
      const int i = f % nx;
      const int r = f / nx;  // j + (ny+1) k
      const int k = r / (ny + 1);
      const int j = r - k * (ny + 1);
      bool on = true;
      if (j > 0) on = on && cell_on(active, i + nx * (j - 1 + ny * k));
      if (j < ny) on = on && cell_on(active, i + nx * (j + ny * k));
      fy[f] = fy_in[f] * (on ? 1.0 : 0.0);
    } else {
      const int f = t - nfx - nfy;
      const int plane = nx * ny;
      const int k = f / plane;
      const int rem = f - k * plane;
      bool on = true;
      if (k > 0) on = on && cell_on(active, rem + plane * (k - 1));
      if (k < nz) on = on && cell_on(active, rem + plane * k);
      fz[f] = fz_in[f] * (on ? 1.0 : 0.0);
    }
  }
}

__global__ void k_mask_cells(int nx, int ny, int nz, const double* x_faces,
                             const double* y_faces, const double* z_faces,
                             const double* diag_in, const double* fx_in,
                             const double* fy_in, const double* fz_in,
                             const uint8_t* active, double* diag,
                             const double* fx, const double* fy,
                             const double* fz, double* volume,
                             uint8_t* fluid) {
  grid_dependency_sync();
  const int n = nx * ny * nz;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += gridDim.x * blockDim.x) {
    int i, j, k;
    cell_coords(c, nx, ny, i, j, k);
    const bool on = cell_on(active, c);
    double vol = (x_faces[i + 1] - x_faces[i]) * (y_faces[j + 1] - y_faces[j]) *
                 (z_faces[k + 1] - z_faces[k]);
    if (!on) vol = 0.0;
    volume[c] = vol;
    fluid[c] = vol > 0.0 ? 1 : 0;
    double d = diag_in[c];
    if (active != nullptr) {
      if (!on) {
        d = 1.0;
      } else {
        const int fxi = c + j + ny * k;
        const int fyi = c + nx * k;
        const int plane = nx * ny;
        const double original = fx_in[fxi] + fx_in[fxi + 1] + fy_in[fyi] +
                                fy_in[fyi + nx] + fz_in[c] + fz_in[c + plane];
        const double act = fx[fxi] + fx[fxi + 1] + fy[fyi] + fy[fyi + nx] +
                           fz[c] + fz[c + plane];
        d = d - original + act;
      }
    }
    diag[c] = d;
  }
}

// Per fine cell: max(0, diag - sum of faces) for fluid cells, the reaction
// aggregated into the coarse diagonal (src/solver_mg.cpp:1880-1894).
__global__ void k_reaction(Level<double> L, const double* volume,
                           double* reaction) {
  grid_dependency_sync();
  const int n = L.nx * L.ny * L.nz;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += gridDim.x * blockDim.x) {
    if (volume[c] == 0.0) {
      reaction[c] = 0.0;
      continue;
    }
    int i, j, k;
    cell_coords(c, L.nx, L.ny, i, j, k);
    const int fxi = face_x_index(L, c, j, k);
    const int fyi = face_y_index(L, c, k);
    const int plane = L.nx * L.ny;
    const double faces = L.fx[fxi] + L.fx[fxi + 1] + L.fy[fyi] +
                         L.fy[fyi + L.nx] + L.fz[c] + L.fz[c + plane];
    const double v = L.diag[c] - faces;
    reaction[c] = v > 0.0 ? v : 0.0;
  }
}

// One axis of aggregate_tensor_channel (src/solver_mg.cpp:1790-1838):
// normal faces copy fine face min(2c, extent); cells and tangential faces
// sum their (at most) two children.
__global__ void k_aggregate_axis(const double* src, int ex, int ey, int ez,
                                 double* dst, int dx, int dy, int dz, int axis,
                                 int face_axis, int global_extent) {
  grid_dependency_sync();
  const int n = dx * dy * dz;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += gridDim.x * blockDim.x) {
    int o[3];
    cell_coords(t, dx, dy, o[0], o[1], o[2]);
    double value = 0.0;
    if (face_axis == axis) {
      int fg = 2 * o[axis];
      if (fg > global_extent) fg = global_extent;
      int s[3] = {o[0], o[1], o[2]};
      s[axis] = fg;
      value = src[s[0] + ex * (s[1] + ey * s[2])];
    } else {
      for (int child = 0; child < 2; ++child) {
        const int fg = 2 * o[axis] + child;
        if (fg >= global_extent) continue;
        int s[3] = {o[0], o[1], o[2]};
        s[axis] = fg;
        value += src[s[0] + ex * (s[1] + ey * s[2])];
      }
    }
    dst[t] = value;
  }
  (void)ez;
}

__global__ void k_coarse_diagonal(int nx, int ny, int nz, double* diag,
                                  const double* fx, const double* fy,
                                  const double* fz, const double* volume,
                                  uint8_t* fluid) {
  grid_dependency_sync();
  const int n = nx * ny * nz;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += gridDim.x * blockDim.x) {
    int i, j, k;
    cell_coords(c, nx, ny, i, j, k);
    const int fxi = c + j + ny * k;
    const int fyi = c + nx * k;
    const int plane = nx * ny;
    double d = diag[c];
    d += fx[fxi] + fx[fxi + 1] + fy[fyi] + fy[fyi + nx] + fz[c] + fz[c + plane];
    if (volume[c] == 0.0) d = 1.0;
    diag[c] = d;
    fluid[c] = volume[c] > 0.0 ? 1 : 0;
  }
}

// face_pressure_coefficient (src/solver_piso.cpp:1060-1136) from cell beta.
__global__ void k_beta_faces(int nx, int ny, int nz, const double* xf,
                             const double* yf, const double* zf,
                             unsigned neumann, const double* beta, double* fx,
                             double* fy, double* fz) {
  grid_dependency_sync();
  const int nfx = (nx + 1) * ny * nz;
  const int nfy = nx * (ny + 1) * nz;
  const int nfz = nx * ny * (nz + 1);
  const int total = nfx + nfy + nfz;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += gridDim.x * blockDim.x) {
    int axis, f, i, j, k, n_axis;
    const double* faces;
    if (t < nfx) {
      axis = 0; f = t; n_axis = nx; faces = xf;
      const int row = f / (nx + 1);
      i = f - row * (nx + 1);
      k = row / ny;
      j = row - k * ny;
    } else if (t < nfx + nfy) {
      axis = 1; f = t - nfx; n_axis = ny; faces = yf;
      i = f % nx;
      const int r = f / nx;
      k = r / (ny + 1);
      j = r - k * (ny + 1);
    } else {
      axis = 2; f = t - nfx - nfy; n_axis = nz; faces = zf;
      const int plane = nx * ny;
      k = f / plane;
      const int rem = f - k * plane;
      j = rem / nx;
      i = rem - j * nx;
    }
    const int normal = axis == 0 ? i : (axis == 1 ? j : k);
    double area;
    if (axis == 0) area = (yf[j + 1] - yf[j]) * (zf[k + 1] - zf[k]);
    else if (axis == 1) area = (xf[i + 1] - xf[i]) * (zf[k + 1] - zf[k]);
    else area = (xf[i + 1] - xf[i]) * (yf[j + 1] - yf[j]);
    const auto cell = [&](int nn) {
      int a = i, b = j, cc = k;
      if (axis == 0) a = nn; else if (axis == 1) b = nn; else cc = nn;
      return a + nx * (b + ny * cc);
    };
    double value;
    if (normal == 0 || normal == n_axis) {
      const bool high = normal == n_axis;
      const bool is_neumann = (neumann >> (2 * axis + (high ? 1 : 0))) & 1u;
      if (is_neumann) {
        value = 0.0;
      } else {
        // Ghost state = owner state: 2 A / (d / beta_o + d / beta_g).
        const int owner = cell(high ? n_axis - 1 : 0);
        const int m = high ? n_axis - 1 : 0;
        const double centre = faces[m] + 0.5 * (faces[m + 1] - faces[m]);
        const double d = high ? faces[n_axis] - centre : centre - faces[0];
        const double b = beta[owner];
        value = 2.0 * area / (d / b + d / b);
      }
    } else {
      // Cell centres as the reference's geometry compiler forms them,
      // left + 0.5 * width (finish_axis_metrics, src/mesh_focus.cpp:584-600).
      const double cl = faces[normal - 1] + 0.5 * (faces[normal] - faces[normal - 1]);
      const double cr = faces[normal] + 0.5 * (faces[normal + 1] - faces[normal]);
      const double dl = faces[normal] - cl;
      const double dr = cr - faces[normal];
      value = area / (dl / beta[cell(normal - 1)] + dr / beta[cell(normal)]);
    }
    if (axis == 0) fx[f] = value; else if (axis == 1) fy[f] = value; else fz[f] = value;
  }
}

__global__ void k_beta_diagonal(int nx, int ny, int nz, const double* fx,
                                const double* fy, const double* fz,
                                const double* storage, double* diag) {
  grid_dependency_sync();
  const int n = nx * ny * nz;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += gridDim.x * blockDim.x) {
    int i, j, k;
    cell_coords(c, nx, ny, i, j, k);
    const int fxi = c + j + ny * k;
    const int fyi = c + nx * k;
    const int plane = nx * ny;
    double d = storage == nullptr ? 0.0 : storage[c];
    d += fx[fxi] + fx[fxi + 1] + fy[fyi] + fy[fyi + nx] + fz[c] + fz[c + plane];
    diag[c] = d;
  }
}

// Pressure-correction system (assemble_pressure_system_impl,
// src/solver_pressure.cpp:110-332), one cell per thread, in the reference's
// operation order:
//   V      = w_x w_y w_z (cell_volume, src/solver_cartesian.cpp:333-337)
//   defect = V ((a0 rho + a1 rho_n) + a2 rho_nm1 - S)
//   diag   = (a0 V) psi + face_sum (x-, x+, y-, y+, z-, z+)
//   rhs    = -(defect + outward_flux) (x+ - x- + y+ - y- + z+ - z-)
// Any input the reference rejects (non-positive density, derivative, volume
// or diagonal, a negative or non-finite face coefficient, a non-finite
// result) sets flags bit 2; nothing is published then.
__global__ void k_assemble(int nx, int ny, int nz, const double* xf, const double* yf,
                           const double* zf, double a0, double a1, double a2, int bdf2,
                           const double* rho, const double* rho_n, const double* rho_nm1,
                           const double* psi, const double* source, const double* phix,
                           const double* phiy, const double* phiz, const double* fx,
                           const double* fy, const double* fz, double* diag, double* rhs,
                           Scalars* scalars) {
  grid_dependency_sync();
  const int n = nx * ny * nz;
  int bad = 0;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += gridDim.x * blockDim.x) {
    int i, j, k;
    cell_coords(c, nx, ny, i, j, k);
    const int fxi = c + j + ny * k;
    const int fyi = c + nx * k;
    const int plane = nx * ny;
    const double volume = (xf[i + 1] - xf[i]) * (yf[j + 1] - yf[j]) * (zf[k + 1] - zf[k]);
    const double r = rho[c];
    const double rn = rho_n[c];
    const double rnm1 = bdf2 ? rho_nm1[c] : 0.0;
    const double derivative = psi[c];
    const double s = source != nullptr ? source[c] : 0.0;
    const double defect = volume * (a0 * r + a1 * rn + a2 * rnm1 - s);
    const double f0 = fx[fxi], f1 = fx[fxi + 1], f2 = fy[fyi], f3 = fy[fyi + nx];
    const double f4 = fz[c], f5 = fz[c + plane];
    const double d = a0 * volume * derivative + (f0 + f1 + f2 + f3 + f4 + f5);
    const double outward = phix[fxi + 1] - phix[fxi] + phiy[fyi + nx] - phiy[fyi] +
                           phiz[c + plane] - phiz[c];
    const double b = -(defect + outward);
    const bool faces_ok = f0 >= 0.0 && f1 >= 0.0 && f2 >= 0.0 && f3 >= 0.0 && f4 >= 0.0 &&
                          f5 >= 0.0 && isfinite(f0 + f1 + f2 + f3 + f4 + f5);
    if (!(r > 0.0) || !(rn > 0.0) || (bdf2 && !(rnm1 > 0.0)) || !(derivative > 0.0) ||
        !(volume > 0.0) || !(d > 0.0) || !isfinite(defect) || !isfinite(d) ||
        !isfinite(b) || !faces_ok)
      bad = 1;
    diag[c] = d;
    rhs[c] = b;
  }
  if (bad) atomicOr(&scalars->flags, 4);
}

// Mass-flux response of a pressure correction (mass_flux_response,
// src/solver_piso.cpp:1605-1653): flux_f += -c_f * (scale * jump_f) with
// jump = p'_right - p'_left inside, +p'_cell on a low Dirichlet boundary
// face, -p'_cell on a high one, 0 on Neumann faces; scale 1 applies the jump
// unscaled.  One face per thread over the x, y and z face arrays.
__global__ void k_correct_flux(int nx, int ny, int nz, unsigned neumann,
                               const double* p, const double* cx, const double* cy,
                               const double* cz, double scale, double* qx, double* qy,
                               double* qz, Scalars* scalars) {
  grid_dependency_sync();
  const int nfx = (nx + 1) * ny * nz;
  const int nfy = nx * (ny + 1) * nz;
  const int nfz = nx * ny * (nz + 1);
  const int total = nfx + nfy + nfz;
  int bad = 0;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += gridDim.x * blockDim.x) {
    int axis, f, face, extent, cell_hi, step;
    if (t < nfx) {
      axis = 0; f = t; extent = nx;
      const int row = f / (nx + 1);
      face = f - row * (nx + 1);
      cell_hi = face + nx * row;
      step = 1;
    } else if (t < nfx + nfy) {
      axis = 1; f = t - nfx; extent = ny;
      const int i = f % nx;
      const int r = f / nx;
      const int k = r / (ny + 1);
      face = r - k * (ny + 1);
      cell_hi = i + nx * (face + ny * k);
      step = nx;
    } else {
      axis = 2; f = t - nfx - nfy; extent = nz;
      face = f / (nx * ny);
      cell_hi = f;
      step = nx * ny;
    }
    double jump;
    if (face == 0) {
      jump = ((neumann >> (2 * axis)) & 1u) ? 0.0 : p[cell_hi];
    } else if (face == extent) {
      jump = ((neumann >> (2 * axis + 1)) & 1u) ? 0.0 : -p[cell_hi - step];
    } else {
      jump = p[cell_hi] - p[cell_hi - step];
    }
    const double applied = scale == 1.0 ? jump : scale * jump;
    double* q = axis == 0 ? qx : (axis == 1 ? qy : qz);
    const double* coefficient = axis == 0 ? cx : (axis == 1 ? cy : cz);
    const double next = q[f] + -coefficient[f] * applied;
    bad |= !isfinite(next);
    q[f] = next;
  }
  if (bad) atomicOr(&scalars->flags, 1);
}

__global__ void k_shortcut_ratio(Level<double> L, Reduce red) {
  grid_dependency_sync();
  const int n = L.nx * L.ny * L.nz;
  double v[1] = {0.0};
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += gridDim.x * blockDim.x) {
    int i, j, k;
    cell_coords(c, L.nx, L.ny, i, j, k);
    const int fxi = face_x_index(L, c, j, k);
    const int fyi = face_y_index(L, c, k);
    const int plane = L.nx * L.ny;
    const double sum = L.fx[fxi] + L.fx[fxi + 1] + L.fy[fyi] +
                       L.fy[fyi + L.nx] + L.fz[c] + L.fz[c + plane];
    v[0] = fmax(v[0], sum / L.diag[c]);
  }
  // max reduction: reuse the partial buffer with a fixed-order max.
  __shared__ double scratch[kThreads];
  scratch[threadIdx.x] = v[0];
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) scratch[threadIdx.x] = fmax(scratch[threadIdx.x], scratch[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) red.partials[blockIdx.x] = scratch[0];
}

template <class TO, class TI>
__global__ void k_convert(size_t n, const TI* __restrict__ src,
                          TO* __restrict__ dst) {
  grid_dependency_sync();
  for (size_t c = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
       c < n; c += static_cast<size_t>(gridDim.x) * blockDim.x)
    dst[c] = static_cast<TO>(src[c]);
}

// Adjoint face gradients: dL/dc_f = -(l_i - l_j)(p_i - p_j) on active
// interior faces, -l_i p_i on Dirichlet boundary faces, 0 elsewhere.
__global__ void k_face_gradients(Level<double> L, const double* lambda,
                                 const double* p, double* gx, double* gy,
                                 double* gz) {
  grid_dependency_sync();
  const int nx = L.nx, ny = L.ny, nz = L.nz;
  const int nfx = (nx + 1) * ny * nz;
  const int nfy = nx * (ny + 1) * nz;
  const int nfz = nx * ny * (nz + 1);
  const int total = nfx + nfy + nfz;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += gridDim.x * blockDim.x) {
    int axis, f, lo = -1, hi = -1, normal, n_axis;
    if (t < nfx) {
      axis = 0; f = t; n_axis = nx;
      const int row = f / (nx + 1);
      const int i = f - row * (nx + 1);
      normal = i;
      if (i > 0) lo = nx * row + i - 1;
      if (i < nx) hi = nx * row + i;
    } else if (t < nfx + nfy) {
      axis = 1; f = t - nfx; n_axis = ny;
      const int i = f % nx;
      const int r = f / nx;
      const int k = r / (ny + 1);
      const int j = r - k * (ny + 1);
      normal = j;
      if (j > 0) lo = i + nx * (j - 1 + ny * k);
      if (j < ny) hi = i + nx * (j + ny * k);
    } else {
      axis = 2; f = t - nfx - nfy; n_axis = nz;
      const int plane = nx * ny;
      const int k = f / plane;
      const int rem = f - k * plane;
      normal = k;
      if (k > 0) lo = rem + plane * (k - 1);
      if (k < nz) hi = rem + plane * k;
    }
    double g = 0.0;
    if (lo >= 0 && hi >= 0) {
      if (L.fluid[lo] && L.fluid[hi]) g = -(lambda[lo] - lambda[hi]) * (p[lo] - p[hi]);
    } else {
      const int owner = lo >= 0 ? lo : hi;
      const bool high = normal == n_axis;
      const bool is_neumann = (L.neumann >> (2 * axis + (high ? 1 : 0))) & 1u;
      if (!is_neumann && L.fluid[owner]) g = -lambda[owner] * p[owner];
    }
    if (axis == 0) gx[f] = g; else if (axis == 1) gy[f] = g; else gz[f] = g;
  }
}

__global__ void k_adjoint_source(int n, const double* dl_dp,
                                 const uint8_t* active, double* out) {
  grid_dependency_sync();
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += gridDim.x * blockDim.x)
    out[c] = cell_on(active, c) ? dl_dp[c] : 0.0;
}

}  // namespace

int reduction_blocks(long long items) {
  long long blocks = (items + kThreads - 1) / kThreads;
  if (blocks < 1) blocks = 1;
  if (blocks > kMaxReductionBlocks) blocks = kMaxReductionBlocks;
  return static_cast<int>(blocks);
}

// ---- launchers ---------------------------------------------------------------
#define HFPS_CELLS(L) (static_cast<long long>((L).nx) * (L).ny * (L).nz)

template <class T>
void launch_level_apply(cudaStream_t s, const Level<T>& L, const T* x, T* y) {
  launch(k_level_apply<T>, grid_for(HFPS_CELLS(L)), kThreads, 0, s, L, x, y);
}
template <class T>
void launch_level_defect(cudaStream_t s, const Level<T>& L, const T* x,
                         const T* b, T* r, int hx) {
  launch(k_level_defect<T>, grid_for(HFPS_CELLS(L)), kThreads, 0, s, L, x, b, r, hx);
}
template <class T>
void launch_rb_color(cudaStream_t s, const Level<T>& L, T* x, const T* b,
                     int color) {
  const long long half = static_cast<long long>((L.nx + 1) / 2) * L.ny * L.nz;
  launch(k_rb_color<T>, grid_for(half), kThreads, 0, s, L, x, b, color);
}
template <class T>
void launch_chebyshev_stage(cudaStream_t s, const Level<T>& L, const T* x,
                            const T* b, T* direction, T* next,
                            T previous_factor, T residual_factor, int first) {
  launch(k_chebyshev_stage<T>, grid_for(HFPS_CELLS(L)), kThreads, 0, s, 
      L, x, b, direction, next, previous_factor, residual_factor, first);
}
template <class T>
void launch_defect_restrict(cudaStream_t s, const Level<T>& F, const T* x,
                            const T* b, const Level<T>& C, T* cb, T* cx,
                            int mask, int hx, int hxc) {
  int threads = 0;
  const dim3 grid = row_grid(C.ny * C.nz, C.nx, threads);
  switch (mask & 7) {
#define HFPS_RESTRICT_CASE(M)                                                              \
  case M:                                                                                  \
    launch(k_defect_restrict<T, M>, grid, threads, 0, s, F, x, b, C, cb, cx, hx, hxc);     \
    break;
    HFPS_RESTRICT_CASE(0) HFPS_RESTRICT_CASE(1) HFPS_RESTRICT_CASE(2) HFPS_RESTRICT_CASE(3)
    HFPS_RESTRICT_CASE(4) HFPS_RESTRICT_CASE(5) HFPS_RESTRICT_CASE(6) HFPS_RESTRICT_CASE(7)
#undef HFPS_RESTRICT_CASE
  }
}
template <class T>
void launch_prolongate(cudaStream_t s, const Level<T>& F, T* x,
                       const Level<T>& C, const T* cx, int mask, int hx, int hxc) {
  int threads = 0;
  if ((mask & 7) == 5 && hx != 0) {
    const dim3 grid = row_grid(F.ny * C.nz, C.nx, threads);
    if (hxc != 0)
      launch(k_prolongate_xz<T, SplitPos>, grid, threads, 0, s, F, x, C, cx, hx,
             SplitPos{C.ny, hxc});
    else
      launch(k_prolongate_xz<T, NaturalPos>, grid, threads, 0, s, F, x, C, cx, hx, NaturalPos());
    return;
  }
  const dim3 grid = row_grid(F.ny * F.nz, hx == 0 ? F.nx : 2 * hx, threads);
  switch (mask & 7) {
#define HFPS_PROLONG_CASE(M)                                                              \
  case M:                                                                                 \
    launch(k_prolongate<T, M>, grid, threads, 0, s, F, x, C, cx, hx, hxc);                \
    break;
    HFPS_PROLONG_CASE(0) HFPS_PROLONG_CASE(1) HFPS_PROLONG_CASE(2) HFPS_PROLONG_CASE(3)
    HFPS_PROLONG_CASE(4) HFPS_PROLONG_CASE(5) HFPS_PROLONG_CASE(6) HFPS_PROLONG_CASE(7)
#undef HFPS_PROLONG_CASE
  }
}
template <class T, class TC>
void launch_coarse_solve(cudaStream_t s, const Level<TC>& L, T* x, const T* b,
                         TC* xs, TC* bs, TC* work, TC* dprime, int sweeps,
                         int line_axis) {
  launch(k_coarse_solve<T, TC>, 1, 512, 0, s, L, x, b, xs, bs, work, dprime, sweeps,
                                          line_axis);
}
template <class T>
void launch_mg_enter(cudaStream_t s, int n, const double* r,
                     const uint8_t* active, T* b, T* x, VecLayout v, bool zero_x) {
  launch(k_mg_enter<T>, grid_for(n), kThreads, 0, s, n, r, active, b, x, v, zero_x);
}
template <class T>
void launch_mg_exit(cudaStream_t s, int n, const T* x, const uint8_t* active,
                    const double* scale_ptr, double* z, VecLayout v) {
  launch(k_mg_exit<T>, grid_for(n), kThreads, 0, s, n, x, active, scale_ptr, z, v);
}
template <class T>
void launch_mg_exit_dot(cudaStream_t s, int n, const T* x, const uint8_t* active, double* z,
                        VecLayout v, const double* r, Reduce red) {
  launch(k_mg_exit_dot<T>, reduction_blocks(n), kThreads, 0, s, n, x, active, z, v, r, red);
}
template <class T>
void launch_diagonal_solve(cudaStream_t s, int n, const T* b, const T* diag,
                           T* x, VecLayout v) {
  launch(k_diagonal_solve<T>, grid_for(n), kThreads, 0, s, n, b, diag, x, v);
}
template <class T>
void launch_mg_projection(cudaStream_t s, int n, const double* r,
                          const uint8_t* active, const T* recursive,
                          Reduce red) {
  launch(k_mg_projection<T>, reduction_blocks(n), kThreads, 0, s, n, r, active,
                                                              recursive, red);
}

// The tiled operator serves grids whose tile count fits the reduction
// partials.
long long tile_count(const Level<double>& L, int depth) {
  return static_cast<long long>((L.nx + kTileX - 1) / kTileX) *
         ((L.ny + kTileY - 1) / kTileY) * ((L.nz + depth - 1) / depth);
}
// Planes per tile: the deepest of 64, 32, 16, 8 that still gives at least
// three quarters of a wave of resident tiles (8 per SM), so that mid-size
// grids run in about one full wave and small ones are not left to a few SMs.
int tile_depth(const Level<double>& L) {
  static const int wave = [] {
    int device = 0, sms = 0;
    cudaGetDevice(&device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    return 8 * (sms > 0 ? sms : 148);
  }();
  int depth = 64;
  while (depth > 8 && 4 * tile_count(L, depth) < 3LL * wave) depth >>= 1;
  return depth;
}

void launch_spmv_dot(cudaStream_t s, const Level<double>& L, const double* x,
                     double* y, Reduce red, bool tiled) {
  const int depth = tile_depth(L);
  const long long tiles = tile_count(L, depth);
  if (tiled && tiles <= kMaxTiledBlocks) {
    const int blocks = static_cast<int>(tiles);
    switch (depth) {
      case 64: launch(k_stencil_tiled<64>, blocks, kTileX * kTileY, 0, s, L, x, y, red); break;
      case 32: launch(k_stencil_tiled<32>, blocks, kTileX * kTileY, 0, s, L, x, y, red); break;
      case 16: launch(k_stencil_tiled<16>, blocks, kTileX * kTileY, 0, s, L, x, y, red); break;
      default: launch(k_stencil_tiled<8>, blocks, kTileX * kTileY, 0, s, L, x, y, red); break;
    }
    return;
  }
  launch(k_spmv_dot, reduction_blocks(HFPS_CELLS(L)), kThreads, 0, s, L, x, y, red);
}
void launch_residual_norm(cudaStream_t s, const Level<double>& L,
                          const double* x, const double* b, double* r,
                          Reduce red) {
  launch(k_residual_norm, reduction_blocks(HFPS_CELLS(L)), kThreads, 0, s, L, x, b, r,
                                                                       red);
}
void launch_pcg_update(cudaStream_t s, int n, double* x, const double* p,
                       double* r, const double* ap, Reduce red) {
  launch(k_pcg_update, reduction_blocks(n), kThreads, 0, s, n, x, p, r, ap, red);
}
void launch_dot(cudaStream_t s, int n, const double* a, const double* b,
                Reduce red) {
  launch(k_dot, reduction_blocks(n), kThreads, 0, s, n, a, b, red);
}
void launch_norm2(cudaStream_t s, int n, const double* v, Reduce red) {
  launch(k_norm2, reduction_blocks(n), kThreads, 0, s, n, v, red);
}
void launch_scaled_norm(cudaStream_t s, int n, const double* v, Scalars* scalars,
                        double* partials) {
  launch(k_norm_max, reduction_blocks(n), kThreads, 0, s, n, v, scalars, partials);
  launch(k_norm_scaled_sum, reduction_blocks(n), kThreads, 0, s, n, v,
         Reduce{scalars, partials, kOpScaledNorm});
}
template <class T>
void launch_project_constant(cudaStream_t s, int nx, int ny, int nz, int hx, T* v,
                             const double* volume, Scalars* scalars, double* partials) {
  const int n = nx * ny * nz;
  const VecLayout lay{nx, ny, hx};
  launch(k_constant_sums<T>, reduction_blocks(n), kThreads, 0, s, n, lay,
         static_cast<const T*>(v), volume, Reduce{scalars, partials, kCounterProjectConstant});
  launch(k_constant_apply<T>, grid_for(n), kThreads, 0, s, n, lay, v, volume,
         static_cast<const Scalars*>(scalars));
}
template void launch_project_constant<double>(cudaStream_t, int, int, int, int, double*,
                                              const double*, Scalars*, double*);
template void launch_project_constant<float>(cudaStream_t, int, int, int, int, float*,
                                             const double*, Scalars*, double*);
void launch_p_update(cudaStream_t s, int n, double* p, const double* z,
                     const Scalars* sc) {
  launch(k_p_update, grid_for(n), kThreads, 0, s, n, p, z, sc);
}
void launch_dic_rows(cudaStream_t s, int nx, int ny, int nz, unsigned neumann,
                     const double* diag, const double* fx, const double* fy, const double* fz,
                     const uint8_t* active, double* out) {
  launch(k_dic_rows, grid_for(static_cast<long long>(nx) * ny * nz), kThreads, 0, s, nx, ny, nz,
         neumann, diag, fx, fy, fz, active, out);
}
int dic_planes(const Level<double>& L) { return L.nx + L.ny + L.nz - 2; }
static int plane_blocks(const Level<double>& L) {
  return static_cast<int>((static_cast<long long>(L.ny) * L.nz + kThreads - 1) / kThreads);
}
void launch_dic_pivots(cudaStream_t s, const Level<double>& L, const double* rows, double* inv,
                       Scalars* scalars) {
  for (int t = 0; t < dic_planes(L); ++t)
    launch(k_dic_pivots, plane_blocks(L), kThreads, 0, s, t, L, rows, inv, scalars);
}
void launch_dic_apply(cudaStream_t s, const Level<double>& L, const double* in, double* out,
                      const double* inv) {
  for (int t = 0; t < dic_planes(L); ++t)
    launch(k_dic_forward, plane_blocks(L), kThreads, 0, s, t, L, in, out, inv);
  for (int t = dic_planes(L) - 1; t >= 0; --t)
    launch(k_dic_backward, plane_blocks(L), kThreads, 0, s, t, L, out, inv);
}
void launch_bicg_direction(cudaStream_t s, int n, double* p, const double* r, const double* v,
                           double beta, double omega) {
  launch(k_bicg_direction, grid_for(n), kThreads, 0, s, n, p, r, v, beta, omega);
}
void launch_bicg_intermediate(cudaStream_t s, int n, double* sv, const double* r,
                              const double* v, double alpha, Reduce red) {
  launch(k_bicg_intermediate, reduction_blocks(n), kThreads, 0, s, n, sv, r, v, alpha, red);
}
void launch_bicg_update(cudaStream_t s, int n, double* x, const double* ph, const double* sh,
                        double* r, const double* sv, const double* t, double alpha,
                        double omega, Reduce red) {
  launch(k_bicg_update, reduction_blocks(n), kThreads, 0, s, n, x, ph, sh, r, sv, t, alpha,
         omega, red);
}
void launch_operator_shift(cudaStream_t s, const Level<double>& L, const double* z,
                           const double* v, double shift, double* w) {
  launch(k_operator_shift, grid_for(HFPS_CELLS(L)), kThreads, 0, s, L, z, v, shift, w);
}
#define HFPS_BASIS_COUNTS(X)                                                             \
  X(0) X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16)

void launch_multidot(cudaStream_t s, int n, const BasisRefs& basis, const double* w,
                     bool self, double* out, Reduce red) {
  const int blocks = reduction_blocks(n);
  switch (basis.count + (self ? 100 : 0)) {
#define HFPS_MULTIDOT_CASE(C)                                                              \
  case C:                                                                                  \
    launch(k_multidot<C, false>, blocks, kThreads, 0, s, n, basis, w, out, red);            \
    break;                                                                                 \
  case 100 + C:                                                                            \
    if (C < kBasisChunk)                                                                   \
      launch(k_multidot<(C < kBasisChunk ? C : 0), true>, blocks, kThreads, 0, s, n, basis, \
             w, out, red);                                                                 \
    break;
    HFPS_BASIS_COUNTS(HFPS_MULTIDOT_CASE)
#undef HFPS_MULTIDOT_CASE
    default: break;
  }
}
void launch_difference_nonzero(cudaStream_t s, int n, const double* x, double* snap,
                               Scalars* scalars) {
  launch(k_difference_nonzero, grid_for(n), kThreads, 0, s, n, x, snap, scalars);
}
void launch_basis_update(cudaStream_t s, int n, const double* dst, const BasisRefs& basis,
                         double scale, bool scaled, double* out) {
  switch (basis.count) {
#define HFPS_BASIS_CASE(C)                                                                 \
  case C:                                                                                  \
    launch(k_basis_update<C>, grid_for(n), kThreads, 0, s, n, dst, basis, scale,           \
           scaled ? 1 : 0, out);                                                           \
    break;
    HFPS_BASIS_COUNTS(HFPS_BASIS_CASE)
#undef HFPS_BASIS_CASE
    default: break;
  }
}
void launch_copy(cudaStream_t s, int n, const double* src, double* dst) {
  launch(k_copy, grid_for(n), kThreads, 0, s, n, src, dst);
}

void launch_mask_finest(cudaStream_t s, int nx, int ny, int nz,
                        const double* x_faces, const double* y_faces,
                        const double* z_faces, const double* diag_in,
                        const double* fx_in, const double* fy_in,
                        const double* fz_in, const uint8_t* active,
                        double* diag, double* fx, double* fy, double* fz,
                        double* volume, uint8_t* fluid) {
  const long long faces = static_cast<long long>(nx + 1) * ny * nz +
                          static_cast<long long>(nx) * (ny + 1) * nz +
                          static_cast<long long>(nx) * ny * (nz + 1);
  launch(k_mask_faces, grid_for(faces), kThreads, 0, s, nx, ny, nz, fx_in, fy_in, fz_in,
                                                    active, fx, fy, fz);
  launch(k_mask_cells, grid_for(static_cast<long long>(nx) * ny * nz), kThreads, 0, s, 
      nx, ny, nz, x_faces, y_faces, z_faces, diag_in, fx_in, fy_in, fz_in, active,
      diag, fx, fy, fz, volume, fluid);
}
void launch_reaction(cudaStream_t s, const Level<double>& L,
                     const double* volume, double* reaction) {
  launch(k_reaction, grid_for(HFPS_CELLS(L)), kThreads, 0, s, L, volume, reaction);
}
void launch_aggregate_axis(cudaStream_t s, const double* src, int ex, int ey,
                           int ez, double* dst, int dx, int dy, int dz,
                           int axis, int face_axis, int global_extent) {
  launch(k_aggregate_axis, grid_for(static_cast<long long>(dx) * dy * dz), kThreads, 0, s, src, ex, ey, ez, dst, dx, dy, dz, axis, face_axis,
                          global_extent);
}
void launch_coarse_diagonal(cudaStream_t s, int nx, int ny, int nz,
                            double* diag, const double* fx, const double* fy,
                            const double* fz, const double* volume,
                            uint8_t* fluid) {
  launch(k_coarse_diagonal, grid_for(static_cast<long long>(nx) * ny * nz), kThreads, 0, s, nx, ny, nz, diag, fx, fy, fz, volume, fluid);
}
void launch_beta_coefficients(cudaStream_t s, int nx, int ny, int nz,
                              const double* x_faces, const double* y_faces,
                              const double* z_faces, unsigned neumann,
                              const double* beta, const double* storage,
                              double* diag, double* fx, double* fy,
                              double* fz) {
  const long long faces = static_cast<long long>(nx + 1) * ny * nz +
                          static_cast<long long>(nx) * (ny + 1) * nz +
                          static_cast<long long>(nx) * ny * (nz + 1);
  launch(k_beta_faces, grid_for(faces), kThreads, 0, s, nx, ny, nz, x_faces, y_faces,
                                                    z_faces, neumann, beta, fx, fy,
                                                    fz);
  launch(k_beta_diagonal, grid_for(static_cast<long long>(nx) * ny * nz), kThreads, 0, s, nx, ny, nz, fx, fy, fz, storage, diag);
}
void launch_assemble(cudaStream_t s, int nx, int ny, int nz, const double* xf,
                     const double* yf, const double* zf, double a0, double a1, double a2,
                     bool bdf2, const double* rho, const double* rho_n, const double* rho_nm1,
                     const double* psi, const double* source, const double* phix,
                     const double* phiy, const double* phiz, const double* fx,
                     const double* fy, const double* fz, double* diag, double* rhs,
                     Scalars* scalars) {
  launch(k_assemble, grid_for(static_cast<long long>(nx) * ny * nz), kThreads, 0, s, nx, ny,
         nz, xf, yf, zf, a0, a1, a2, bdf2 ? 1 : 0, rho, rho_n, rho_nm1, psi, source, phix,
         phiy, phiz, fx, fy, fz, diag, rhs, scalars);
}
void launch_correct_flux(cudaStream_t s, int nx, int ny, int nz, unsigned neumann,
                         const double* p, const double* cx, const double* cy,
                         const double* cz, double scale, double* qx, double* qy, double* qz,
                         Scalars* scalars) {
  const long long faces = static_cast<long long>(nx + 1) * ny * nz +
                          static_cast<long long>(nx) * (ny + 1) * nz +
                          static_cast<long long>(nx) * ny * (nz + 1);
  launch(k_correct_flux, grid_for(faces), kThreads, 0, s, nx, ny, nz, neumann, p, cx, cy, cz,
         scale, qx, qy, qz, scalars);
}
void launch_shortcut_ratio(cudaStream_t s, const Level<double>& L,
                           Reduce red) {
  launch(k_shortcut_ratio, reduction_blocks(HFPS_CELLS(L)), kThreads, 0, s, L, red);
}
template <class TO, class TI>
void launch_convert(cudaStream_t s, size_t n, const TI* src, TO* dst) {
  launch(k_convert<TO, TI>, grid_for(static_cast<long long>(n)), kThreads, 0, s, n, src,
                                                                           dst);
}
void launch_face_gradients(cudaStream_t s, const Level<double>& L,
                           const double* lambda, const double* p,
                           const double* fx_in, const double* fy_in,
                           const double* fz_in, double* gx, double* gy,
                           double* gz) {
  (void)fx_in;
  (void)fy_in;
  (void)fz_in;
  const long long faces = static_cast<long long>(L.nx + 1) * L.ny * L.nz +
                          static_cast<long long>(L.nx) * (L.ny + 1) * L.nz +
                          static_cast<long long>(L.nx) * L.ny * (L.nz + 1);
  launch(k_face_gradients, grid_for(faces), kThreads, 0, s, L, lambda, p, gx, gy, gz);
}
void launch_adjoint_source(cudaStream_t s, int n, const double* dl_dp,
                           const uint8_t* active, double* out) {
  launch(k_adjoint_source, grid_for(n), kThreads, 0, s, n, dl_dp, active, out);
}

#define HFPS_INSTANTIATE(T)                                                        \
  template void launch_level_apply<T>(cudaStream_t, const Level<T>&, const T*, T*); \
  template void launch_level_defect<T>(cudaStream_t, const Level<T>&, const T*,    \
                                       const T*, T*, int);                         \
  template void launch_rb_color<T>(cudaStream_t, const Level<T>&, T*, const T*,    \
                                   int);                                           \
  template void launch_chebyshev_stage<T>(cudaStream_t, const Level<T>&, const T*, \
                                          const T*, T*, T*, T, T, int);            \
  template void launch_defect_restrict<T>(cudaStream_t, const Level<T>&, const T*, \
                                          const T*, const Level<T>&, T*, T*, int,  \
                                          int, int);                               \
  template void launch_prolongate<T>(cudaStream_t, const Level<T>&, T*,            \
                                     const Level<T>&, const T*, int, int, int);    \
  template void launch_mg_enter<T>(cudaStream_t, int, const double*,               \
                                   const uint8_t*, T*, T*, VecLayout, bool);       \
  template void launch_mg_exit<T>(cudaStream_t, int, const T*, const uint8_t*,     \
                                  const double*, double*, VecLayout);              \
  template void launch_mg_exit_dot<T>(cudaStream_t, int, const T*, const uint8_t*, \
                                      double*, VecLayout, const double*, Reduce);  \
  template void launch_diagonal_solve<T>(cudaStream_t, int, const T*, const T*,    \
                                         T*, VecLayout);                           \
  template void launch_mg_projection<T>(cudaStream_t, int, const double*,          \
                                        const uint8_t*, const T*, Reduce);

HFPS_INSTANTIATE(double)
HFPS_INSTANTIATE(float)

template void launch_coarse_solve<double, double>(cudaStream_t, const Level<double>&,
                                                  double*, const double*, double*,
                                                  double*, double*, double*, int, int);
template void launch_coarse_solve<float, double>(cudaStream_t, const Level<double>&,
                                                 float*, const float*, double*,
                                                 double*, double*, double*, int, int);
template void launch_convert<float, double>(cudaStream_t, size_t, const double*, float*);
template void launch_convert<double, float>(cudaStream_t, size_t, const float*, double*);

}  // namespace hfps
