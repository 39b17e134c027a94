// The small levels of a line-relaxation hierarchy as one persistent launch.
//
// Below the scan levels every phase of the cycle (a PCR colour pass over a
// few hundred lines, a defect-restriction or prolongation of a few thousand
// cells, the dense coarsest map) is a few microseconds of work, and as a
// separate kernel each one pays a launch and a grid drain on top.  Here the
// host records the phases of a sub-cycle (Solver::tail_cycle, in exactly the
// order the per-kernel path launches them) into a program passed by value
// as the kernel's parameter, and one cooperative launch of at most one
// 1024-thread CTA per SM executes them in turn, every CTA taking its share
// of each phase, with a grid-wide barrier between phases.  A CTA relaxes
// 1024 / 2^STEPS lines of a PCR pass at once, so few CTAs cover a level and
// few arrive at each barrier.  Each phase body is the same device function
// the per-kernel path uses (phase_device.cuh), with the same 32-warp
// grouping of the dense map's partial sums, so the results are bitwise
// those of that path.
//
// The barrier is bounded: a CTA that waits longer than kTailSpinLimit polls
// (under a second) records the failure in the solver's scalars (flag bit 3)
// and the program ends on every CTA, so a wait can never hang the GPU; the
// solver reports a preconditioner failure at its next check.  A program with
// barrier_offset 1 never reaches its first barrier's count, which is how the
// tests exercise that path.
#include "kernels.hpp"
#include "phase_device.cuh"

namespace hfps {
namespace {

constexpr long long kTailSpinLimit = 1LL << 21;  // polls of an L2 round trip: under a second

// Grid-wide barrier over `blocks` co-resident CTAs (cooperative launch).
// tail_count only grows, by one per CTA per barrier, so it is a multiple of
// `blocks` between barriers (the solver clears it at the start of every
// solve); a CTA's arrival ticket gives the count that ends its barrier.  The
// arrival is acquire-release: it publishes this CTA's writes, and leaving
// once the count is reached makes every other CTA's writes visible.
__device__ __forceinline__ bool tail_barrier(Scalars* sc, unsigned blocks, unsigned offset) {
  __shared__ int failed;
  __syncthreads();
  if (threadIdx.x == 0) {
    int bad = 0;
    unsigned ticket;
    __threadfence();
    asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], 1;" : "=r"(ticket)
                 : "l"(&sc->tail_count) : "memory");
    const unsigned target = (ticket / blocks + 1) * blocks + offset;
    long long polls = 0;
    while (true) {
      unsigned now;
      asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(now) : "l"(&sc->tail_count)
                   : "memory");
      if (static_cast<int>(now - target) >= 0) break;
      if (++polls > kTailSpinLimit) {
        atomicOr(&sc->flags, 8);
        bad = 1;
        break;
      }
    }
    int flags;
    asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];" : "=r"(flags) : "l"(&sc->flags)
                 : "memory");
    failed = bad || (flags & 8) != 0;
    __threadfence();
  }
  __syncthreads();
  return failed == 0;
}

constexpr int kTailThreads = 1024;

template <class T, int STEPS>
__global__ void __launch_bounds__(kTailThreads, 1) k_tail(TailProgram<T> prog) {
  grid_dependency_sync();
  constexpr int P = 1 << STEPS;
  constexpr int G = kTailThreads / P;  // lines a CTA relaxes at once
  static_assert(kTailThreads / 32 == kDenseWarps, "dense map grouping");
  extern __shared__ double tail_smem[];
  T* sd = reinterpret_cast<T*>(tail_smem);                  // PCR line values, G x P
  double* v = tail_smem + kTailThreads;                      // dense map: x then b
  double* part = v + 2 * prog.dense_n;                       // dense map partials
  const unsigned blocks = gridDim.x;
  const int tid = threadIdx.x;
  const int g = tid >> STEPS;
  const int s = tid & (P - 1);
  for (int o = 0; o < prog.count; ++o) {
    const TailOp& op = prog.ops[o];
    const Level<T>& L = prog.levels[op.level];
    switch (op.kind) {
      case kTailPcr: {
        const int axis = prog.axis[op.level];
        const int a_extent = axis == 0 ? L.ny : L.nx;
        const int b_extent = axis == 2 ? L.ny : L.nz;
        const int lines = ((a_extent + 1) >> 1) * b_extent;
        // The trip count depends on the CTA only: every thread reaches the
        // barriers inside pcr_line_slot; slots past the last line write nothing.
        for (int t0 = blockIdx.x * G; t0 < lines; t0 += blocks * G)
          pcr_line_slot<T, STEPS>(L, static_cast<T*>(op.p0), static_cast<const T*>(op.p1),
                                  static_cast<const T*>(op.p2), axis, op.arg, t0 + g, s,
                                  sd + g * P);
        break;
      }
      case kTailRestrict: {
        const Level<T>& C = prog.levels[op.level + 1];
        const T* x = static_cast<const T*>(op.p0);
        const T* b = static_cast<const T*>(op.p1);
        T* cb = static_cast<T*>(op.p2);
        T* cx = static_cast<T*>(op.p3);
        const int n = C.nx * C.ny * C.nz;
        for (int cc = blockIdx.x * kTailThreads + tid; cc < n; cc += blocks * kTailThreads) {
          int ci, cj, ck;
          cell_coords(cc, C.nx, C.ny, ci, cj, ck);
          cb[cc] = defect_restrict_at<T>(L, x, b, op.arg, ci, cj, ck, NaturalPos());
          cx[cc] = T(0);
        }
        break;
      }
      case kTailProlong: {
        const Level<T>& C = prog.levels[op.level + 1];
        T* x = static_cast<T*>(op.p0);
        const T* cx = static_cast<const T*>(op.p1);
        const int n = L.nx * L.ny * L.nz;
        for (int c = blockIdx.x * kTailThreads + tid; c < n; c += blocks * kTailThreads) {
          int i, j, k;
          cell_coords(c, L.nx, L.ny, i, j, k);
          x[c] = prolongate_cell<T>(L, x, C, cx, op.arg, c, i, j, k, c);
        }
        break;
      }
      case kTailDense: {
        const int n = prog.dense_n;
        const T* x = static_cast<const T*>(op.p0);
        const T* b = static_cast<const T*>(op.p1);
        T* out = static_cast<T*>(op.p2);
        const bool x_zero = op.arg != 0;
        const int row_blocks = (n + 31) / 32;
        if (static_cast<int>(blockIdx.x) < row_blocks) {
          for (int j = tid; j < n; j += kTailThreads) {
            v[j] = x_zero ? 0.0 : static_cast<double>(x[j]);
            v[n + j] = static_cast<double>(b[j]);
          }
          __syncthreads();
          for (int rb = blockIdx.x; rb < row_blocks; rb += blocks)
            dense_rows<T, kDenseWarps>(n, prog.dense_op, v, part, rb, tid & 31, tid >> 5,
                                       x_zero, out);
        }
        break;
      }
      default:
        break;
    }
    if (!tail_barrier(prog.scalars, blocks, static_cast<unsigned>(prog.barrier_offset))) return;
  }
}

template <class T, int STEPS>
size_t tail_smem_bytes(int dense_n) {
  return (2 * static_cast<size_t>(kTailThreads) + 2 * static_cast<size_t>(dense_n)) *
         sizeof(double);
}

template <class T, int STEPS>
int tail_blocks_per_sm(int dense_n) {
  const size_t smem = tail_smem_bytes<T, STEPS>(dense_n);
  if (smem > 48 * 1024)
    cudaFuncSetAttribute(k_tail<T, STEPS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         static_cast<int>(smem));
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tail<T, STEPS>, kTailThreads,
                                                    smem) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return per_sm;
}

template <class T, int STEPS>
bool launch_tail_steps(cudaStream_t s, const TailProgram<T>& prog, int blocks) {
  const size_t smem = tail_smem_bytes<T, STEPS>(prog.dense_n);
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(blocks);
  cfg.blockDim = dim3(kTailThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_tail<T, STEPS>, prog) == cudaSuccess;
}

}  // namespace

int tail_steps(int extent) {
  int steps = 0;
  while ((1 << steps) < extent) ++steps;
  return steps >= 5 && steps <= 10 ? steps : -1;
}

int tail_lines_per_cta(int steps) { return kTailThreads >> steps; }

template <class T>
int tail_grid(int steps, int dense_n, int sms) {
  int per_sm = 0;
  switch (steps) {
    case 5: per_sm = tail_blocks_per_sm<T, 5>(dense_n); break;
    case 6: per_sm = tail_blocks_per_sm<T, 6>(dense_n); break;
    case 7: per_sm = tail_blocks_per_sm<T, 7>(dense_n); break;
    case 8: per_sm = tail_blocks_per_sm<T, 8>(dense_n); break;
    case 9: per_sm = tail_blocks_per_sm<T, 9>(dense_n); break;
    case 10: per_sm = tail_blocks_per_sm<T, 10>(dense_n); break;
    default: break;
  }
  return per_sm * sms;
}

template <class T>
bool launch_tail(cudaStream_t s, const TailProgram<T>& prog, int steps, int blocks) {
  switch (steps) {
    case 5: return launch_tail_steps<T, 5>(s, prog, blocks);
    case 6: return launch_tail_steps<T, 6>(s, prog, blocks);
    case 7: return launch_tail_steps<T, 7>(s, prog, blocks);
    case 8: return launch_tail_steps<T, 8>(s, prog, blocks);
    case 9: return launch_tail_steps<T, 9>(s, prog, blocks);
    case 10: return launch_tail_steps<T, 10>(s, prog, blocks);
    default: return false;
  }
}

template int tail_grid<double>(int, int, int);
template int tail_grid<float>(int, int, int);
template bool launch_tail<double>(cudaStream_t, const TailProgram<double>&, int, int);
template bool launch_tail<float>(cudaStream_t, const TailProgram<float>&, int, int);

}  // namespace hfps
