// Host-callable launchers for the sm_100a kernels (kernels.cu).
//
// Every launcher enqueues on the given stream and never synchronises.  Level
// operands are passed as hfps::Level<T> (hfps_device.cuh); vectors are dense
// x-fastest arrays of the level's shape.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "hfps_device.cuh"

namespace hfps {

// Device-resident Krylov scalars.  Kernels read alpha/beta from here, so a
// whole iteration runs without a host round trip; the host reads back only
// what steers control flow.
struct Scalars {
  double rho;        // r.z of the current search direction
  double pap;        // p.Ap
  double alpha;      // rho / pap
  double rr;         // last r.r (recursive or true residual)
  double rho_next;   // r.z after the preconditioner
  double beta;       // rho_next / rho (0 after a restart)
  double proj[3];    // MG projection sums r.r, r.Az, Az.Az
  double mg_alpha;   // MG correction scale
  double misc[4];
  double hcol[72];   // FGMRES: projections of the current column and |w|^2
  int flags;         // bit 0 non-finite, bit 1 breakdown, bit 2 invalid assembly input,
                     // bit 3 a grid barrier of the small-level kernel timed out
  unsigned marks;    // bit 0: a difference had a nonzero entry (recycle capture)
  unsigned counters[12];  // last-block arrival counters, one per reduction
  double constant_mean;   // volume-weighted mean of the last project_constant
  // The small-level kernel's grid barrier: arrivals (on a 128-byte line of
  // its own).
  unsigned tail_pad0[32];
  unsigned tail_count;
  unsigned tail_pad1[31];
};

enum ScalarOp : int {
  kOpPap = 0,        // pap = sum; alpha = rho / pap
  kOpRecursive = 1,  // rr = sum
  kOpRhoNext = 2,    // rho_next = sum; beta = rho_next / rho; rho = rho_next
  kOpRhoRestart = 3, // rho = sum; beta = 0
  kOpMisc = 4,       // misc[0] = sum
  kOpScaledNorm = 7, // misc[3] = misc[2] * sqrt(sum): the max-scaled norm (counter 7)
};
// Arrival counters of reductions that apply no scalar op: 5 MG projection,
// 6 FGMRES multidot, 8 project_constant.  Counter 7 serves both passes of
// the max-scaled norm.
constexpr int kCounterProjection = 5;
constexpr int kCounterMultidot = 6;
constexpr int kCounterProjectConstant = 8;
constexpr int kMaxFgmresRestart = 64;

struct Reduce {
  Scalars* scalars;
  double* partials;   // >= gridDim.x * kBasisChunk doubles
  int op;
};

int reduction_blocks(long long items);

// Layout of a level's vectors (x, b): hx == 0 the natural x-fastest order,
// otherwise split rows (SplitPos) whose even- and odd-i halves are hx cells
// long, 2 * hx * ny * nz values in all.  Coefficients and every other vector
// stay in the natural order.
struct VecLayout {
  int nx, ny, hx;
};

// ---- level operators (T = double or float) -------------------------------
template <class T>
void launch_level_apply(cudaStream_t s, const Level<T>& L, const T* x, T* y);
// r (natural order) = b - A x with x, b in layout hx.
template <class T>
void launch_level_defect(cudaStream_t s, const Level<T>& L, const T* x,
                         const T* b, T* r, int hx = 0);
template <class T>
void launch_rb_color(cudaStream_t s, const Level<T>& L, T* x, const T* b,
                     int color);
template <class T>
void launch_chebyshev_stage(cudaStream_t s, const Level<T>& L, const T* x,
                            const T* b, T* direction, T* next,
                            T previous_factor, T residual_factor, int first);
// Fine x, b in layout hx, coarse b, x in layout hxc.
template <class T>
void launch_defect_restrict(cudaStream_t s, const Level<T>& F, const T* x,
                            const T* b, const Level<T>& C, T* cb, T* cx,
                            int coarsen_mask, int hx = 0, int hxc = 0);
// Fine x in layout hx, coarse x in layout hxc.
template <class T>
void launch_prolongate(cudaStream_t s, const Level<T>& F, T* x,
                       const Level<T>& C, const T* cx, int coarsen_mask, int hx = 0,
                       int hxc = 0);
// ---- zebra line relaxation (kernels_line.cu) --------------------------------
// Line-colour passes with at least kLinePcrThreshold lines (kLinePcrThresholdLong
// for lines of kLinePcrLongExtent cells or more) run the chunked-scan solve
// (lanes across lines, warps along chunks of one line); fewer lines run PCR
// with one CTA row per line.  Lines longer than 2048 cells are not supported
// (kLineNone).  The long-line boundary is lower because PCR's factor block
// grows with the line (2 log2(extent) + 1 arrays against the scan's two):
// measured MG applications, 512 lines per colour on the scan against PCR,
// 256-cell lines (32x256x32 in the 256^3 hierarchy) 2.74 against 2.80 ms,
// 128-cell lines (32x128x32 in the 128^3 one) 0.78 against 0.75 ms; fewer
// than 512 lines leave most SMs idle on the scan (2.82 ms with 8x256x8 on
// it as well).
#ifndef HFPS_LINE_PCR_THRESHOLD
#define HFPS_LINE_PCR_THRESHOLD 1024
#endif
#ifndef HFPS_LINE_PCR_THRESHOLD_LONG
#define HFPS_LINE_PCR_THRESHOLD_LONG 512
#endif
constexpr long long kLinePcrThreshold = HFPS_LINE_PCR_THRESHOLD;
constexpr long long kLinePcrThresholdLong = HFPS_LINE_PCR_THRESHOLD_LONG;
constexpr int kLinePcrLongExtent = 256;
enum LineKind : int { kLineNone = 0, kLineScan = 1, kLinePcr = 2 };
int line_kind(int nx, int ny, int nz, int axis);
// Values of the factor block of one level and line axis in precision T: the
// Thomas reciprocal and upper multiplier (2 per cell, FP64), plus the lower
// multiplier (3 per cell, FP32), or PCR multipliers and final diagonals.
template <class T>
size_t line_factor_values(int nx, int ny, int nz, int axis);
template <class T>
void launch_line_factors(cudaStream_t s, const Level<T>& L, int axis, T* fac);
// One zebra colour of line relaxation along `axis`, x and b in layout hx
// (split rows only with the scan solve, axis 1 or 2).  zero_other: the other
// colour's x is known to be zero (not read); zero_self: this colour's x is
// (the first pass and the first sweep of a cycle started from x = 0).
template <class T>
void launch_line_pass(cudaStream_t s, const Level<T>& L, T* x, const T* b,
                      const T* fac, T* scratch, int axis, int color, int hx = 0,
                      bool zero_other = false, bool zero_self = false);
// Coarsest level in line mode with x/rhs resident in shared memory; returns
// false when the level is too large for that form.  With `columns`, launches
// 2n blocks that write the columns of the sweeps' affine map x_out = P x_in
// + M b (P then M, column-major) to x, n = cells of the level.
template <class T, class TC>
bool launch_coarse_line(cudaStream_t s, const Level<TC>& L, T* x, const T* b,
                        const TC* fac, int sweeps, int axis, bool columns = false);
// out = P x + M b with the dense coarsest-level map built by the columns
// mode above (n <= kCoarseDenseMaxCells; out must not alias x or b).  With
// x_zero (x is known to be zero) the P half is not read.
constexpr int kCoarseDenseMaxCells = 2048;
template <class T>
void launch_coarse_dense(cudaStream_t s, int n, const double* op, const T* x,
                         const T* b, T* out, bool x_zero);

// Coarsest level: `sweeps` smoother sweeps in one CTA, arithmetic in TC.
// Line mode when line_axis >= 0 (zebra line Gauss-Seidel).
template <class T, class TC>
void launch_coarse_solve(cudaStream_t s, const Level<TC>& L, T* x, const T* b,
                         TC* xs, TC* bs, TC* work, TC* dprime, int sweeps,
                         int line_axis);

// ---- small levels as one persistent launch (kernels_tail.cu) ---------------
// A program of cycle phases for the levels below the scan levels, executed
// by one cooperative launch with a bounded grid barrier between phases.
enum TailKind : int { kTailPcr = 0, kTailRestrict = 1, kTailProlong = 2, kTailDense = 3 };
struct TailOp {
  int kind;
  int level;   // index into TailProgram::levels (the fine level of a transfer)
  int arg;     // PCR: colour; transfers: coarsening mask; dense: x is zero
  int pad;
  // PCR: x, rhs, factors.  Restrict: fine x, fine b, coarse b, coarse x.
  // Prolong: fine x, coarse x.  Dense: x, b, out.
  void* p0;
  void* p1;
  void* p2;
  void* p3;
};
constexpr int kTailMaxOps = 480;
constexpr int kTailMaxLevels = 8;
// Passed by value as the kernel parameter (kept under the 32 KB limit).
template <class T>
struct TailProgram {
  int count;
  int dense_n;
  // Added to every barrier's target count: 0, or 1 to make the first
  // barrier run out its wait limit (the failure path's test).
  int barrier_offset;
  int pad;
  int axis[kTailMaxLevels];
  Level<T> levels[kTailMaxLevels];
  const double* dense_op;
  Scalars* scalars;
  TailOp ops[kTailMaxOps];
};
static_assert(sizeof(TailProgram<double>) < 32000, "kernel parameter limit");
// log2 of the PCR width for lines of `extent` cells, or -1 if unsupported.
int tail_steps(int extent);
// Lines of one PCR pass a CTA of the persistent launch relaxes at once.
int tail_lines_per_cta(int steps);
// CTAs that can be co-resident on `sms` SMs (0: cannot run).
template <class T>
int tail_grid(int steps, int dense_n, int sms);
template <class T>
bool launch_tail(cudaStream_t s, const TailProgram<T>& prog, int steps, int blocks);

// ---- MG entry/exit ------------------------------------------------------
// b = active ? r : 0 (converted to T), and x = 0 when zero_x; b and x in
// layout v, r natural.
template <class T>
void launch_mg_enter(cudaStream_t s, int n, const double* r,
                     const uint8_t* active, T* b, T* x, VecLayout v, bool zero_x);
// z = active ? x * scale : 0 (scale read from device when scale_ptr).
template <class T>
void launch_mg_exit(cudaStream_t s, int n, const T* x, const uint8_t* active,
                    const double* scale_ptr, double* z, VecLayout v);
// launch_mg_exit (unit scaling) fused with the PCG's r.z through red.
template <class T>
void launch_mg_exit_dot(cudaStream_t s, int n, const T* x, const uint8_t* active, double* z,
                        VecLayout v, const double* r, Reduce red);
template <class T>
void launch_diagonal_solve(cudaStream_t s, int n, const T* b, const T* diag,
                           T* x, VecLayout v);
// Projection sums for the residual-minimising MG scale (level-0, FP64 r).
template <class T>
void launch_mg_projection(cudaStream_t s, int n, const double* r,
                          const uint8_t* active, const T* recursive,
                          Reduce red);

// project_constant (src/solver_mg.cpp:1411-1453) on a level vector v in
// layout hx: v - mean on cells of positive volume and 0 on the others, mean
// = sum(volume v) / sum(volume) (kept in scalars->constant_mean).  A total
// volume that is not positive or a non-finite sum sets flag bit 0.
template <class T>
void launch_project_constant(cudaStream_t s, int nx, int ny, int nz, int hx, T* v,
                             const double* volume, Scalars* scalars, double* partials);

// ---- Krylov (FP64) --------------------------------------------------------
// y = A x and x.y: over 3-D shared-memory tiles when `tiled` and the tiles'
// partial sums fit the partials block, else a warp per x-row (the same rows).
void launch_spmv_dot(cudaStream_t s, const Level<double>& L, const double* x,
                     double* y, Reduce red, bool tiled = true);
void launch_residual_norm(cudaStream_t s, const Level<double>& L,
                          const double* x, const double* b, double* r,
                          Reduce red);
void launch_pcg_update(cudaStream_t s, int n, double* x, const double* p,
                       double* r, const double* ap, Reduce red);
void launch_dot(cudaStream_t s, int n, const double* a, const double* b,
                Reduce red);
void launch_p_update(cudaStream_t s, int n, double* p, const double* z,
                     const Scalars* sc);
void launch_norm2(cudaStream_t s, int n, const double* v, Reduce red);
// The max-scaled 2-norm of global_norm (src/solver_krylov.cpp:650-711) into
// scalars->misc[3]: pass 1 forms max |v| (misc[2]; a non-finite entry sets
// flag bit 0), pass 2 max * sqrt(sum of (v / max)^2), zero when max is zero.
void launch_scaled_norm(cudaStream_t s, int n, const double* v, Scalars* scalars,
                        double* partials);
void launch_copy(cudaStream_t s, int n, const double* src, double* dst);
// ---- the steps either side of the solve ----------------------------------------
// Pressure-correction system assembly (diag, rhs) from densities, the
// density derivative, the predicted face fluxes and the face coefficients.
void launch_assemble(cudaStream_t s, int nx, int ny, int nz, const double* xf,
                     const double* yf, const double* zf, double a0, double a1, double a2,
                     bool bdf2, const double* rho, const double* rho_n, const double* rho_nm1,
                     const double* psi, const double* source, const double* phix,
                     const double* phiy, const double* phiz, const double* fx,
                     const double* fy, const double* fz, double* diag, double* rhs,
                     Scalars* scalars);
// flux += mass-flux response of the correction p (in place).
void launch_correct_flux(cudaStream_t s, int nx, int ny, int nz, unsigned neumann,
                         const double* p, const double* cx, const double* cy,
                         const double* cz, double scale, double* qx, double* qy, double* qz,
                         Scalars* scalars);
// ---- cold path: diagonal IC(0) and BiCGSTAB ----------------------------------
// Decorated-row diagonal of the cold-path factorisation.
void launch_dic_rows(cudaStream_t s, int nx, int ny, int nz, unsigned neumann,
                     const double* diag, const double* fx, const double* fy, const double* fz,
                     const uint8_t* active, double* out);
// Wavefront planes i + j + k = t of a level: nx + ny + nz - 2.
int dic_planes(const Level<double>& L);
// Inverse pivots, plane by plane (flags bit 0 on a non-positive pivot).
void launch_dic_pivots(cudaStream_t s, const Level<double>& L, const double* rows, double* inv,
                       Scalars* scalars);
// out = M^{-1} in: forward then backward sweep, plane by plane.
void launch_dic_apply(cudaStream_t s, const Level<double>& L, const double* in, double* out,
                      const double* inv);
void launch_bicg_direction(cudaStream_t s, int n, double* p, const double* r, const double* v,
                           double beta, double omega);
// s = r - alpha v, with |s|^2 through red.
void launch_bicg_intermediate(cudaStream_t s, int n, double* sv, const double* r,
                              const double* v, double alpha, Reduce red);
// x = (x + alpha ph) + omega sh, r = s - omega t, with |r|^2 through red.
void launch_bicg_update(cudaStream_t s, int n, double* x, const double* ph, const double* sh,
                        double* r, const double* sv, const double* t, double alpha,
                        double omega, Reduce red);
// ---- FGMRES (solve_fgmres) ---------------------------------------------------
// Basis vectors handled by one multidot / basis-update launch.
constexpr int kBasisChunk = 16;
struct BasisRefs {
  const double* v[kBasisChunk];
  double s[kBasisChunk];
  int count;
};
// w = A z - shift v.
void launch_operator_shift(cudaStream_t s, const Level<double>& L, const double* z,
                           const double* v, double shift, double* w);
// out[r] = v_r . w for r < count, and out[count] = w . w when `self`
// (count + self <= kBasisChunk); non-finite sums set flags bit 0.
void launch_multidot(cudaStream_t s, int n, const BasisRefs& basis, const double* w,
                     bool self, double* out, Reduce red);
// snap = x - snap; marks bit 0 when any entry is nonzero
// (difference_recycle_field, src/solver_linear_state.cpp:162-181).
void launch_difference_nonzero(cudaStream_t s, int n, const double* x, double* snap,
                               Scalars* scalars);
// out = (scaled ? scale : 1) * (dst + sum_r s_r v_r), per cell in basis order.
void launch_basis_update(cudaStream_t s, int n, const double* dst, const BasisRefs& basis,
                         double scale, bool scaled, double* out);

// ---- setup (FP64) ---------------------------------------------------------
void launch_mask_finest(cudaStream_t s, int nx, int ny, int nz,
                        const double* x_faces, const double* y_faces,
                        const double* z_faces, const double* diag_in,
                        const double* fx_in, const double* fy_in,
                        const double* fz_in, const uint8_t* active,
                        double* diag, double* fx, double* fy, double* fz,
                        double* volume, uint8_t* fluid);
void launch_reaction(cudaStream_t s, const Level<double>& L,
                     const double* volume, double* reaction);
// One axis of the tensor aggregation (aggregate_tensor_channel).
void launch_aggregate_axis(cudaStream_t s, const double* src, int ex, int ey,
                           int ez, double* dst, int dx, int dy, int dz,
                           int axis, int face_axis, int global_extent);
void launch_coarse_diagonal(cudaStream_t s, int nx, int ny, int nz,
                            double* diag, const double* fx, const double* fy,
                            const double* fz, const double* volume,
                            uint8_t* fluid);
void launch_beta_coefficients(cudaStream_t s, int nx, int ny, int nz,
                              const double* x_faces, const double* y_faces,
                              const double* z_faces, unsigned neumann,
                              const double* beta, const double* storage,
                              double* diag, double* fx, double* fy,
                              double* fz);
void launch_shortcut_ratio(cudaStream_t s, const Level<double>& L,
                           Reduce red);
template <class TO, class TI>
void launch_convert(cudaStream_t s, size_t n, const TI* src, TO* dst);

// ---- adjoint ---------------------------------------------------------------
void launch_face_gradients(cudaStream_t s, const Level<double>& L,
                           const double* lambda, const double* p,
                           const double* fx_in, const double* fy_in,
                           const double* fz_in, double* gx, double* gy,
                           double* gz);
void launch_adjoint_source(cudaStream_t s, int n, const double* dl_dp,
                           const uint8_t* active, double* out);

}  // namespace hfps
