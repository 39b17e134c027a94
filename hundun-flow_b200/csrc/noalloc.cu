// Allocation-free y = A x with x.(A x): hfps_operator_dot_noalloc.
//
// The solver's own operator kernel (k_spmv_dot) keeps its per-block partial
// sums in the solver's arena.  This variant serves callers that hold no
// solver handle and may not allocate device memory at the point of the call
// (fixed memory pools, caching allocators that forbid new allocations
// mid-step).  Its partial sums live in one fixed file-scope device array of
// HFPS_NOALLOC_MAX_BLOCKS + 1 doubles (about 9.3 KB per device); the last
// slot holds the arrival counter of the last-block reduction.
//
// What must start at zero: the arrival counter.  Static device memory is
// zero at module load, the last block puts it back to zero, and every call
// also clears it on its stream before the launch, so a call never depends on
// how an earlier one ended.  The partial sums need no clearing: every block
// writes its own slot before it counts itself in.
//
// The array is shared by all calls on a device, so calls that overlap in
// time race on it; callers serialise them on one stream.
#include <cstdint>
#include <mutex>

#include "../../include/hf_pressure_solver.h"
#include "hfps_device.cuh"

namespace hfps {
namespace {

constexpr int kNoallocThreads = 256;
constexpr int kMaxDevices = 64;
constexpr int kScratchDoubles = HFPS_NOALLOC_MAX_BLOCKS + 1;

static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

// Same row, grid-stride walk and fixed-order last-block reduction as the
// solver's operator kernel (solve_pcg's A p and p.Ap,
// src/solver_krylov.cpp:1426-1447), with the partials in `scratch`.
__global__ void __launch_bounds__(kNoallocThreads)
k_operator_dot_noalloc(Level<double> L, const double* __restrict__ x,
                       double* __restrict__ y, double* __restrict__ x_dot_y,
                       double* scratch) {
  const int n = L.nx * L.ny * L.nz;
  double v[1] = {0.0};
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += gridDim.x * blockDim.x) {
    const int row = c / L.nx;
    const int i = c - row * L.nx;
    const int k = row / L.ny;
    const int j = row - k * L.ny;
    const double a = row_value(L, x, i, j, k, c);
    y[c] = a;
    v[0] += x[c] * a;
  }
  block_sum<1>(v);
  unsigned int* arrivals =
      reinterpret_cast<unsigned int*>(scratch + HFPS_NOALLOC_MAX_BLOCKS);
  __shared__ bool last;
  if (threadIdx.x == 0) {
    scratch[blockIdx.x] = v[0];
    __threadfence();
    last = atomicAdd(arrivals, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double acc[1] = {0.0};
  for (int b = threadIdx.x; b < static_cast<int>(gridDim.x); b += blockDim.x)
    acc[0] += reinterpret_cast<volatile double*>(scratch)[b];
  block_sum<1>(acc);
  if (threadIdx.x == 0) {
    if (x_dot_y != nullptr) *x_dot_y = acc[0];
    *arrivals = 0u;
  }
}

// Scratch address per device, looked up once with that device current.  The
// address belongs to the device's primary context: cudaDeviceReset discards
// it together with the module, so the cached value is void afterwards.
std::mutex g_setup_mutex;
double* g_scratch_address[kMaxDevices] = {};

int scratch_for_current_device(double** out) {
  int device = -1;
  if (cudaGetDevice(&device) != cudaSuccess || device < 0 ||
      device >= kMaxDevices) {
    cudaGetLastError();
    return HFPS_INVALID_PLAN;
  }
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (g_scratch_address[device] == nullptr) {
    void* address = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&address, g_noalloc_scratch);
    if (e != cudaSuccess || address == nullptr) {
      cudaGetLastError();
      return HFPS_INVALID_PLAN;
    }
    g_scratch_address[device] = static_cast<double*>(address);
  }
  *out = g_scratch_address[device];
  return HFPS_OK;
}

// A device (or managed) allocation on `device`, 8-byte aligned.
bool device_array(const void* p, int device) {
  if (p == nullptr || (reinterpret_cast<std::uintptr_t>(p) & 7u) != 0) return false;
  cudaPointerAttributes attr{};
  if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return (attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged) &&
         attr.device == device;
}

}  // namespace
}  // namespace hfps

extern "C" HFPS_API int hfps_operator_dot_noalloc(const hfps_operator_view* op,
                                                  const double* x, double* y,
                                                  double* x_dot_y,
                                                  void* stream) {
  using namespace hfps;
  if (op == nullptr) return HFPS_INVALID_PLAN;
  if (op->nx < 1 || op->ny < 1 || op->nz < 1) return HFPS_INVALID_CASE;
  const long long n = static_cast<long long>(op->nx) * op->ny * op->nz;
  if (n > HFPS_NOALLOC_MAX_CELLS) return HFPS_INVALID_CASE;
  unsigned neumann = 0;
  for (int f = 0; f < 6; ++f) {
    if (op->boundary[f] == HFPS_NEUMANN) neumann |= 1u << f;
    else if (op->boundary[f] != HFPS_DIRICHLET) return HFPS_INVALID_PLAN;
  }
  double* scratch = nullptr;
  const int setup = scratch_for_current_device(&scratch);
  if (setup != HFPS_OK) return setup;
  int device = -1;
  if (cudaGetDevice(&device) != cudaSuccess) {
    cudaGetLastError();
    return HFPS_INVALID_PLAN;
  }
  const void* arrays[] = {x, y, op->diagonal, op->face_x, op->face_y, op->face_z};
  for (const void* p : arrays)
    if (!device_array(p, device)) return HFPS_INVALID_PLAN;
  if (x_dot_y != nullptr && !device_array(x_dot_y, device)) return HFPS_INVALID_PLAN;
  const std::uintptr_t xb = reinterpret_cast<std::uintptr_t>(x);
  const std::uintptr_t yb = reinterpret_cast<std::uintptr_t>(y);
  const std::uintptr_t bytes = static_cast<std::uintptr_t>(n) * sizeof(double);
  if (xb < yb + bytes && yb < xb + bytes) return HFPS_INVALID_PLAN;
  // The dot is written after the sweep: inside x or y it would overwrite
  // one input value or one result row.
  if (x_dot_y != nullptr) {
    const std::uintptr_t db = reinterpret_cast<std::uintptr_t>(x_dot_y);
    const std::uintptr_t de = db + sizeof(double);
    if ((db < xb + bytes && xb < de) || (db < yb + bytes && yb < de)) return HFPS_INVALID_PLAN;
  }

  Level<double> L{op->nx, op->ny, op->nz, neumann, op->diagonal,
                  op->face_x, op->face_y, op->face_z, nullptr};
  long long blocks = (n + kNoallocThreads - 1) / kNoallocThreads;
  if (blocks > HFPS_NOALLOC_MAX_BLOCKS) blocks = HFPS_NOALLOC_MAX_BLOCKS;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(scratch + HFPS_NOALLOC_MAX_BLOCKS, 0, sizeof(unsigned int), s) !=
      cudaSuccess) {
    cudaGetLastError();
    return HFPS_INVALID_PLAN;
  }
  k_operator_dot_noalloc<<<static_cast<int>(blocks), kNoallocThreads, 0, s>>>(
      L, x, y, x_dot_y, scratch);
  if (cudaGetLastError() != cudaSuccess) return HFPS_INVALID_PLAN;
  return HFPS_OK;
}
