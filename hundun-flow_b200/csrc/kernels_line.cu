// Zebra line relaxation (y-line relaxation for stretched grids) on sm_100a.
//
// The reference relaxes strong-axis lines by lexicographic line Gauss-Seidel
// with one Thomas solve per line (line_smooth_axis, src/solver_mg.cpp:
// 3352-3539).  Here lines are coloured by the parity of their transverse
// index (zebra): a colour's lines couple only to the other colour, so all of
// them are solved at once.  The line matrices depend only on the level
// coefficients, so their factorisations are computed once per coefficient
// update and every sweep does only the right-hand-side work:
//   * many lines per colour: one thread per line runs the Thomas recurrence
//     with the precomputed denominators and c' values (bit-identical to the
//     reference's arithmetic) and loads its cells in chunks so memory
//     latency overlaps the serial recurrence;
//   * few lines per colour (coarse levels): one CTA row per line runs
//     parallel cyclic reduction with precomputed elimination factors;
//   * the coarsest level keeps x and rhs in shared memory for all of its
//     coarse sweeps in one launch.
#include "kernels.hpp"

#include <algorithm>

namespace hfps {
namespace {

constexpr int kChunk = 8;

__device__ __forceinline__ int line_extent(int axis, int nx, int ny, int nz) {
  return axis == 0 ? nx : (axis == 1 ? ny : nz);
}

template <class T>
__device__ __forceinline__ int line_stride(const Level<T>& L, int axis) {
  return axis == 0 ? 1 : (axis == 1 ? L.nx : L.nx * L.ny);
}

template <class T>
__device__ __forceinline__ int line_base(const Level<T>& L, int axis, int fa,
                                         int fb) {
  if (axis == 0) return L.nx * (fa + L.ny * fb);
  if (axis == 1) return fa + L.nx * L.ny * fb;
  return fa + L.nx * fb;
}

// Thomas factors of every line (forward elimination of the matrix only):
// denominators b_s - a_s c'_{s-1} and c'_s, in the reference's operation
// order (src/solver_mg.cpp:3466-3480).
template <class T>
__global__ void k_thomas_factors(Level<T> L, int axis, T* __restrict__ work,
                                 T* __restrict__ denom) {
  const int a_extent = axis == 0 ? L.ny : L.nx;
  const int b_extent = axis == 2 ? L.ny : L.nz;
  const int lines = a_extent * b_extent;
  const int extent = line_extent(axis, L.nx, L.ny, L.nz);
  const int plane = L.nx * L.ny;
  for (int line = blockIdx.x * blockDim.x + threadIdx.x; line < lines;
       line += gridDim.x * blockDim.x) {
    const int fb = line / a_extent;
    const int fa = line - fb * a_extent;
    const int base = line_base(L, axis, fa, fb);
    const int stride = line_stride(L, axis);
    T prev_work = T(0);
    for (int s = 0; s < extent; ++s) {
      const int c = base + s * stride;
      const int i = axis == 0 ? s : fa;
      const int j = axis == 0 ? fa : (axis == 1 ? s : fb);
      const int k = axis == 2 ? s : fb;
      T lowf, highf;
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
        highf = L.fz[c + plane];
      }
      (void)i;
      const T a = s == 0 ? T(0) : -lowf;
      const T bb = L.diag[c];
      const T cc = s + 1 == extent ? T(0) : -highf;
      const T den = s == 0 ? bb : bb - a * prev_work;
      const T w = cc / den;
      work[c] = w;
      denom[c] = den;
      prev_work = w;
    }
  }
}

// Right-hand side of row s of a line: rhs plus the transverse neighbours and
// the line-end boundary terms (the d of line_row, without a, b, c).
template <class T>
__device__ __forceinline__ T line_rhs(const Level<T>& L,
                                      const T* __restrict__ x,
                                      const T* __restrict__ rhs, int axis,
                                      int fa, int fb, int s, int extent,
                                      int& c, T& lowf) {
  const int plane = L.nx * L.ny;
  const int i = axis == 0 ? s : fa;
  const int j = axis == 0 ? fa : (axis == 1 ? s : fb);
  const int k = axis == 2 ? s : fb;
  c = i + L.nx * (j + L.ny * k);
  const int fxi = face_x_index(L, c, j, k);
  const int fyi = face_y_index(L, c, k);
  T highf;
  if (axis == 0) { lowf = L.fx[fxi]; highf = L.fx[fxi + 1]; }
  else if (axis == 1) { lowf = L.fy[fyi]; highf = L.fy[fyi + L.nx]; }
  else { lowf = L.fz[c]; highf = L.fz[c + plane]; }
  T d = rhs[c];
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
  return d;
}

// One zebra colour with one thread per line and precomputed Thomas factors.
// Loads of kChunk cells are issued before their serial recurrence runs.
template <class T>
__global__ void k_line_thomas_color(Level<T> L, T* __restrict__ x,
                                    const T* __restrict__ rhs,
                                    const T* __restrict__ work,
                                    const T* __restrict__ denom,
                                    T* __restrict__ dprime, int axis,
                                    int color) {
  const int a_extent = axis == 0 ? L.ny : L.nx;
  const int b_extent = axis == 2 ? L.ny : L.nz;
  const int ha = (a_extent + 1) >> 1;
  const int n = ha * b_extent;
  const int extent = line_extent(axis, L.nx, L.ny, L.nz);
  const int stride = line_stride(L, axis);
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += gridDim.x * blockDim.x) {
    const int fb = t / ha;
    const int fa = 2 * (t - fb * ha) + ((fb + color) & 1);
    if (fa >= a_extent) continue;
    const int base = line_base(L, axis, fa, fb);
    T prev = T(0);
    for (int s0 = 0; s0 < extent; s0 += kChunk) {
      T dv[kChunk], av[kChunk], den[kChunk];
#pragma unroll
      for (int u = 0; u < kChunk; ++u) {
        const int s = s0 + u;
        if (s < extent) {
          int c;
          T lowf;
          dv[u] = line_rhs(L, x, rhs, axis, fa, fb, s, extent, c, lowf);
          av[u] = -lowf;
          den[u] = denom[c];
        }
      }
#pragma unroll
      for (int u = 0; u < kChunk; ++u) {
        const int s = s0 + u;
        if (s < extent) {
          const T v = s == 0 ? dv[u] / den[u] : (dv[u] - av[u] * prev) / den[u];
          dprime[base + s * stride] = v;
          prev = v;
        }
      }
    }
    T next = T(0);
    const int last = (extent - 1) / kChunk * kChunk;
    for (int s0 = last; s0 >= 0; s0 -= kChunk) {
      T dp[kChunk], wv[kChunk];
#pragma unroll
      for (int u = 0; u < kChunk; ++u) {
        const int s = s0 + u;
        if (s < extent) {
          const int c = base + s * stride;
          dp[u] = dprime[c];
          wv[u] = work[c];
        }
      }
#pragma unroll
      for (int u = kChunk - 1; u >= 0; --u) {
        const int s = s0 + u;
        if (s < extent) {
          const T v = s + 1 == extent ? dp[u] : dp[u] - wv[u] * next;
          x[base + s * stride] = v;
          next = v;
        }
      }
    }
  }
}

// PCR elimination factors of every line: per halving step the multipliers
// k1 = a_s / b_{s-h}, k2 = c_s / b_{s+h}, then the final diagonal.  Layout
// [2*steps+1][lines][P] so a line's threads read consecutive addresses.
template <class T>
__global__ void k_pcr_factors(Level<T> L, int axis, int P, T* __restrict__ fac) {
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
    const int plane = L.nx * L.ny;
    const int i = axis == 0 ? s : fa;
    const int j = axis == 0 ? fa : (axis == 1 ? s : fb);
    const int k = axis == 2 ? s : fb;
    const int c = i + L.nx * (j + L.ny * k);
    T lowf, highf;
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
      highf = L.fz[c + plane];
    }
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

// PCR right-hand-side elimination with precomputed factors; returns x_s.
template <class T>
__device__ __forceinline__ T pcr_apply(const T* __restrict__ fac, size_t slab,
                                       size_t at, T* __restrict__ sd, int s,
                                       int P) {
  int step = 0;
  for (int h = 1; h < P; h <<= 1, ++step) {
    const T k1 = fac[(2 * step) * slab + at];
    const T k2 = fac[(2 * step + 1) * slab + at];
    const int lo = s - h, hi = s + h;
    const T dlo = lo >= 0 ? sd[lo] : T(0);
    const T dhi = hi < P ? sd[hi] : T(0);
    const T nd = sd[s] - dlo * k1 - dhi * k2;
    __syncthreads();
    sd[s] = nd;
    __syncthreads();
  }
  return sd[s] / fac[(2 * step) * slab + at];
}

// One zebra colour with PCR: blockDim = (P, lines per block).
template <class T>
__global__ void k_line_pcr_factored_color(Level<T> L, T* __restrict__ x,
                                          const T* __restrict__ rhs,
                                          const T* __restrict__ fac, int axis,
                                          int color, int P) {
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
  int c = 0;
  T d = T(0);
  if (valid && s < extent) {
    T lowf;
    d = line_rhs(L, x, rhs, axis, fa, fb, s, extent, c, lowf);
  }
  sd[s] = d;
  __syncthreads();
  const size_t slab = static_cast<size_t>(a_extent) * b_extent * P;
  const size_t at = static_cast<size_t>(valid ? fa + a_extent * fb : 0) * P + s;
  const T value = pcr_apply(fac, slab, at, sd, s, P);
  if (valid && s < extent) x[c] = value;
}

// Coarsest level, line mode: all sweeps in one CTA with x and rhs resident
// in shared memory (widened to TC) and PCR factors in TC.
template <class T, class TC>
__global__ void k_coarse_line_smem(Level<TC> L, T* __restrict__ x,
                                   const T* __restrict__ b,
                                   const TC* __restrict__ fac, int sweeps,
                                   int axis, int P) {
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
  for (int sweep = 0; sweep < sweeps; ++sweep) {
    for (int color = 0; color < 2; ++color) {
      for (int base = 0; base < lines; base += blockDim.y) {
        const int t = base + threadIdx.y;
        const int fb = t / ha;
        const int fa = 2 * (t - fb * ha) + ((fb + color) & 1);
        const bool valid = t < lines && fa < a_extent;
        int c = 0;
        TC d = TC(0);
        if (valid && s < extent) {
          TC lowf;
          d = line_rhs(L, xs, bs, axis, fa, fb, s, extent, c, lowf);
        }
        sd[s] = d;
        __syncthreads();
        const size_t at = static_cast<size_t>(valid ? fa + a_extent * fb : 0) * P + s;
        const TC value = pcr_apply(fac, slab, at, sd, s, P);
        if (valid && s < extent) xs[c] = value;
        __syncthreads();
      }
    }
  }
  for (int c = tid; c < n; c += nthreads) x[c] = static_cast<T>(xs[c]);
}

void pcr_shape(int extent, int& P, int& lines_per_block) {
  P = 1;
  while (P < extent) P <<= 1;
  lines_per_block = std::max(1, std::min(1024 / P, 4));
}

}  // namespace

int line_kind(int nx, int ny, int nz, int axis) {
  const int extent = axis == 0 ? nx : (axis == 1 ? ny : nz);
  const int a_extent = axis == 0 ? ny : nx;
  const int b_extent = axis == 2 ? ny : nz;
  const long long per_color = static_cast<long long>((a_extent + 1) / 2) * b_extent;
  if (per_color < kLinePcrThreshold && extent <= 1024) return kLinePcr;
  return kLineThomas;
}

size_t line_factor_values(int nx, int ny, int nz, int axis) {
  const int extent = axis == 0 ? nx : (axis == 1 ? ny : nz);
  const int a_extent = axis == 0 ? ny : nx;
  const int b_extent = axis == 2 ? ny : nz;
  if (line_kind(nx, ny, nz, axis) == kLineThomas)
    return 2 * static_cast<size_t>(nx) * ny * nz;
  int P, lpb;
  pcr_shape(extent, P, lpb);
  int steps = 0;
  for (int h = 1; h < P; h <<= 1) ++steps;
  return static_cast<size_t>(2 * steps + 1) * a_extent * b_extent * P;
}

template <class T>
void launch_line_factors(cudaStream_t s, const Level<T>& L, int axis, T* fac) {
  const int extent = axis == 0 ? L.nx : (axis == 1 ? L.ny : L.nz);
  const int a_extent = axis == 0 ? L.ny : L.nx;
  const int b_extent = axis == 2 ? L.ny : L.nz;
  const int lines = a_extent * b_extent;
  if (line_kind(L.nx, L.ny, L.nz, axis) == kLineThomas) {
    const int cells = L.nx * L.ny * L.nz;
    k_thomas_factors<T><<<(lines + 127) / 128, 128, 0, s>>>(L, axis, fac, fac + cells);
    return;
  }
  int P, lpb;
  pcr_shape(extent, P, lpb);
  const size_t smem = static_cast<size_t>(3) * P * lpb * sizeof(T);
  k_pcr_factors<T><<<(lines + lpb - 1) / lpb, dim3(P, lpb), smem, s>>>(L, axis, P, fac);
}

template <class T>
void launch_line_pass(cudaStream_t s, const Level<T>& L, T* x, const T* b,
                      const T* fac, T* scratch, int axis, int color) {
  const int extent = axis == 0 ? L.nx : (axis == 1 ? L.ny : L.nz);
  const int a_extent = axis == 0 ? L.ny : L.nx;
  const int b_extent = axis == 2 ? L.ny : L.nz;
  const long long per_color = static_cast<long long>((a_extent + 1) / 2) * b_extent;
  if (line_kind(L.nx, L.ny, L.nz, axis) == kLineThomas) {
    const int cells = L.nx * L.ny * L.nz;
    const int threads = 128;
    const long long blocks = (per_color + threads - 1) / threads;
    k_line_thomas_color<T><<<static_cast<int>(blocks), threads, 0, s>>>(
        L, x, b, fac, fac + cells, scratch, axis, color);
    return;
  }
  int P, lpb;
  pcr_shape(extent, P, lpb);
  const size_t smem = static_cast<size_t>(P) * lpb * sizeof(T);
  const long long blocks = (per_color + lpb - 1) / lpb;
  k_line_pcr_factored_color<T><<<static_cast<int>(blocks), dim3(P, lpb), smem, s>>>(
      L, x, b, fac, axis, color, P);
}

template <class T, class TC>
bool launch_coarse_line(cudaStream_t s, const Level<TC>& L, T* x, const T* b,
                        const TC* fac, int sweeps, int axis) {
  const int extent = axis == 0 ? L.nx : (axis == 1 ? L.ny : L.nz);
  if (line_kind(L.nx, L.ny, L.nz, axis) != kLinePcr) return false;
  int P, lpb;
  pcr_shape(extent, P, lpb);
  const size_t cells = static_cast<size_t>(L.nx) * L.ny * L.nz;
  const size_t smem = (2 * cells + static_cast<size_t>(P) * lpb) * sizeof(TC);
  if (smem > 200 * 1024) return false;
  if (smem > 48 * 1024)
    cudaFuncSetAttribute(k_coarse_line_smem<T, TC>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  k_coarse_line_smem<T, TC><<<1, dim3(P, lpb), smem, s>>>(L, x, b, fac, sweeps, axis, P);
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
