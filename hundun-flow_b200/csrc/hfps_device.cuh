// Device-side building blocks of the B200 pressure solve.
//
// Layout (shared with the host and the C ABI): cell fields are dense and
// x-fastest; x/y/z face arrays have extents (nx+1,ny,nz), (nx,ny+1,nz),
// (nx,ny,nz+1).  For a cell c = i + nx*(j + ny*k) the six faces are
//   x: c + j + ny*k  and +1        y: c + nx*k  and +nx
//   z: c             and +nx*ny
// so every kernel addresses faces from the cell index with two adds.
//
// The library is compiled with --fmad=false: the 7-point row is evaluated
// as separate IEEE multiplies and subtractions in the reference's order
// (point_row_value, src/solver_mg.cpp:2395-2414), which makes the level
// operators, smoothers and transfers bit-identical to the reference's.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

// Programmatic dependent launch: every kernel of the library is launched
// with programmatic stream serialisation (hfps::launch), so the launch of
// the next kernel in a stream or graph overlaps the drain of this one.  Each
// kernel therefore starts with grid_dependency_sync(), which waits until the
// preceding grid has completed and its writes are visible, before touching
// any memory.  Kernels launched without the attribute pass it straight
// through.  An early launch_dependents trigger (dependents scheduled while
// this grid still runs) measured slower at 256^3: 7% on the FP32 MG cycle,
// and 3% on the FP64 one when given to the FP64 kernels alone (2.79 -> 2.88
// ms), so dependents launch at grid exit.
#ifndef HFPS_USE_PDL
#define HFPS_USE_PDL 1
#endif
#ifndef HFPS_PDL_EARLY_TRIGGER
#define HFPS_PDL_EARLY_TRIGGER 0
#endif

namespace hfps {

__device__ __forceinline__ void grid_dependency_sync() {
#if HFPS_USE_PDL
#if HFPS_PDL_EARLY_TRIGGER
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
#endif
  asm volatile("griddepcontrol.wait;" ::: "memory");
#endif
}

// Launches kernel<<<grid, block, smem, stream>>>(args...) with programmatic
// stream serialisation allowed.
template <class... Params, class... Args>
inline void launch(void (*kernel)(Params...), dim3 grid, dim3 block, size_t smem,
                   cudaStream_t stream, Args&&... args) {
#if HFPS_USE_PDL
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kernel, static_cast<Params>(args)...);
#else
  kernel<<<grid, block, smem, stream>>>(static_cast<Params>(args)...);
#endif
}

// Bit f of `neumann` is set when face f (x-,x+,y-,y+,z-,z+) is Neumann; a
// clear bit is Dirichlet (neighbour value 0).  Neumann reads the cell
// itself (MgPointBoundaryMode::self, src/solver_mg.cpp:940-963).
template <class T>
struct Level {
  int nx, ny, nz;
  unsigned neumann;
  const T* __restrict__ diag;
  const T* __restrict__ fx;
  const T* __restrict__ fy;
  const T* __restrict__ fz;
  const uint8_t* __restrict__ fluid;  // 1 where the fluid volume is > 0
};

struct Index3 {
  int i, j, k;
  int c;
};

template <class T>
__device__ __forceinline__ int face_x_index(const Level<T>& L, int c, int j,
                                            int k) {
  return c + j + L.ny * k;
}
template <class T>
__device__ __forceinline__ int face_y_index(const Level<T>& L, int c, int k) {
  return c + L.nx * k;
}

// How a shared device body reads a vector: an ordinary load, or the
// read-only data path (ld.global.nc) for arrays no thread writes during the
// launch.
struct PlainLoad {
  template <class T>
  __device__ __forceinline__ static T get(const T* p) { return *p; }
};
struct RoLoad {
  template <class T>
  __device__ __forceinline__ static T get(const T* p) { return __ldg(p); }
};

__device__ __forceinline__ void cell_coords(int c, int nx, int ny, int& i,
                                            int& j, int& k) {
  const int row = c / nx;
  i = c - row * nx;
  k = row / ny;
  j = row - k * ny;
}

// Where a level's vector stores cell (i, j, k) (c = its x-fastest index).
// NaturalPos: at c.  SplitPos ("split rows", used for the finest level of a
// y- or z-line hierarchy): every x-row stores its even-i cells and then its
// odd-i cells, each half hx = (nx + 1) / 2 long, so that one zebra colour
// of a row is contiguous.
struct NaturalPos {
  __device__ __forceinline__ int operator()(int c, int, int, int) const { return c; }
};
struct SplitPos {
  int ny, hx;
  __device__ __forceinline__ int operator()(int, int i, int j, int k) const {
    return 2 * hx * (j + ny * k) + (i & 1) * hx + (i >> 1);
  }
};

// A x at one cell, in the reference's accumulation order.
template <class T, class Ld = PlainLoad, class Pos = NaturalPos>
__device__ __forceinline__ T row_value(const Level<T>& L, const T* x, int i,
                                       int j, int k, int c, Pos pos = Pos()) {
  const int plane = L.nx * L.ny;
  const T xc = Ld::get(x + pos(c, i, j, k));
  const T xm = i > 0 ? Ld::get(x + pos(c - 1, i - 1, j, k))
                     : ((L.neumann & 1u) ? xc : T(0));
  const T xp = i + 1 < L.nx ? Ld::get(x + pos(c + 1, i + 1, j, k))
                            : ((L.neumann & 2u) ? xc : T(0));
  const T ym = j > 0 ? Ld::get(x + pos(c - L.nx, i, j - 1, k))
                     : ((L.neumann & 4u) ? xc : T(0));
  const T yp = j + 1 < L.ny ? Ld::get(x + pos(c + L.nx, i, j + 1, k))
                            : ((L.neumann & 8u) ? xc : T(0));
  const T zm = k > 0 ? Ld::get(x + pos(c - plane, i, j, k - 1))
                     : ((L.neumann & 16u) ? xc : T(0));
  const T zp = k + 1 < L.nz ? Ld::get(x + pos(c + plane, i, j, k + 1))
                            : ((L.neumann & 32u) ? xc : T(0));
  const int fxi = face_x_index(L, c, j, k);
  const int fyi = face_y_index(L, c, k);
  T v = L.diag[c] * xc;
  v -= L.fx[fxi] * xm;
  v -= L.fx[fxi + 1] * xp;
  v -= L.fy[fyi] * ym;
  v -= L.fy[fyi + L.nx] * yp;
  v -= L.fz[c] * zm;
  v -= L.fz[c + plane] * zp;
  return v;
}

// Neighbour along `axis` in direction `dir` for the line smoother's
// transverse and end terms (level_neighbor, src/solver_mg.cpp:2222-2262).
// x may live in shared memory that other threads update between barriers
// (coarsest-level kernels), so it is not __restrict__-qualified.
template <class T, class Ld = PlainLoad>
__device__ __forceinline__ T line_neighbour(const Level<T>& L, const T* x,
                                            int i, int j, int k, int c,
                                            int axis, int dir) {
  if (axis == 0) {
    if (dir < 0) return i > 0 ? Ld::get(x + c - 1) : ((L.neumann & 1u) ? Ld::get(x + c) : T(0));
    return i + 1 < L.nx ? Ld::get(x + c + 1) : ((L.neumann & 2u) ? Ld::get(x + c) : T(0));
  }
  if (axis == 1) {
    if (dir < 0)
      return j > 0 ? Ld::get(x + c - L.nx) : ((L.neumann & 4u) ? Ld::get(x + c) : T(0));
    return j + 1 < L.ny ? Ld::get(x + c + L.nx) : ((L.neumann & 8u) ? Ld::get(x + c) : T(0));
  }
  const int plane = L.nx * L.ny;
  if (dir < 0)
    return k > 0 ? Ld::get(x + c - plane) : ((L.neumann & 16u) ? Ld::get(x + c) : T(0));
  return k + 1 < L.nz ? Ld::get(x + c + plane) : ((L.neumann & 32u) ? Ld::get(x + c) : T(0));
}

// Row s of the line system through cell (fa, fb) along `axis`: the same
// a, b, c, d the Thomas solve forms (src/solver_mg.cpp:3440-3478).
template <class T>
__device__ __forceinline__ void line_row(const Level<T>& L, const T* x,
                                         const T* rhs, int axis,
                                         int fa, int fb, int s, int& c, T& a,
                                         T& bb, T& cc, T& d) {
  const int extent = axis == 0 ? L.nx : (axis == 1 ? L.ny : L.nz);
  const int plane = L.nx * L.ny;
  const int i = axis == 0 ? s : fa;
  const int j = axis == 0 ? fa : (axis == 1 ? s : fb);
  const int k = axis == 2 ? s : fb;
  c = i + L.nx * (j + L.ny * k);
  const int fxi = face_x_index(L, c, j, k);
  const int fyi = face_y_index(L, c, k);
  T lowf, highf;
  if (axis == 0) { lowf = L.fx[fxi]; highf = L.fx[fxi + 1]; }
  else if (axis == 1) { lowf = L.fy[fyi]; highf = L.fy[fyi + L.nx]; }
  else { lowf = L.fz[c]; highf = L.fz[c + plane]; }
  a = s == 0 ? T(0) : -lowf;
  bb = L.diag[c];
  cc = s + 1 == extent ? T(0) : -highf;
  d = rhs[c];
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
}

// Block-wide sum of up to three doubles; result valid in thread 0.
template <int N>
__device__ __forceinline__ void block_sum(double (&v)[N]) {
  __shared__ double scratch[32][N];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int nwarps = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int n = 0; n < N; ++n) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[n] += __shfl_down_sync(0xffffffffu, v[n], o);
  }
  if (lane == 0) {
#pragma unroll
    for (int n = 0; n < N; ++n) scratch[warp][n] = v[n];
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int n = 0; n < N; ++n) {
      v[n] = lane < nwarps ? scratch[lane][n] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v[n] += __shfl_down_sync(0xffffffffu, v[n], o);
    }
  }
  __syncthreads();
}

}  // namespace hfps
