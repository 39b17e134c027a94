// Host side of the B200 pressure solve (C++17).
//
// One Solver owns the device hierarchy of one pressure system: the level
// shapes (make_mg_workspace_requirements, src/solver_mg_workspace.cpp:
// 317-452), the masked and aggregated level coefficients
// (build_coarse_coefficients, src/solver_mg.cpp:1858-1925), the MG
// workspaces and the Krylov vectors.  The MG cycle is orchestrated here and
// captured once into a CUDA graph per precision; Krylov scalars stay on the
// device, so an iteration costs one small device-to-host read.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/hf_pressure_solver.h"
#include "kernels.hpp"

namespace hfps {

template <class T>
struct DeviceLevel {
  using value_type = T;
  int nx{}, ny{}, nz{};
  int coarsen_mask{};
  int line_mask{};
  bool chebyshev{};
  T* diag{};
  T* fx{};
  T* fy{};
  T* fz{};
  const uint8_t* fluid{};
  T* x{};
  T* b{};
  T* r{};
  T* t{};
  // Line-relaxation factors per strong axis (kernels_line.cu), or null.
  T* lfac[3]{};
  // Layout of x and b (VecLayout::hx): 0 natural, else split rows with
  // halves of `split` cells (levels of a y- or z-line hierarchy that relax
  // with the chunked scan).
  int split{};
  int cells() const { return nx * ny * nz; }
  int faces_x() const { return (nx + 1) * ny * nz; }
  int faces_y() const { return nx * (ny + 1) * nz; }
  int faces_z() const { return nx * ny * (nz + 1); }
  Level<T> view(unsigned neumann) const {
    return Level<T>{nx, ny, nz, neumann, diag, fx, fy, fz, fluid};
  }
};

struct Status {
  int code{HFPS_OK};
  uint32_t detail{};
  explicit operator bool() const { return code == HFPS_OK; }
};

class Solver {
 public:
  ~Solver();
  static Status create(const hfps_geometry& geometry, const hfps_policy& policy,
                       cudaStream_t stream, Solver** out, std::string& error);

  Status set_coefficients(const double* diag, const double* fx,
                          const double* fy, const double* fz, int memory);
  Status set_beta(const double* beta, const double* storage, int memory);
  Status assemble(const hfps_assembly& in, double* rhs, int memory);
  Status correct_flux(const double* correction, const double* cx, const double* cy,
                      const double* cz, double scale, double* qx, double* qy, double* qz,
                      int memory);
  Status solve(const double* rhs, double* solution, int memory,
               const hfps_control& control, hfps_result& result,
               double* history, uint32_t history_capacity);
  Status apply_operator(const double* x, double* y, int memory);
  Status apply_preconditioner(const double* r, double* z, int memory,
                              int precision);
  Status adjoint(const double* solution, const double* dl_dp, double* lambda,
                 double* gx, double* gy, double* gz, int memory,
                 const hfps_control& control, hfps_result& result);
  int level_count() const { return static_cast<int>(l64_.size()); }
  void level_shape(int level, int* out) const;
  Status level_coefficients(int level, double* diag, double* fx, double* fy,
                            double* fz, double* volume);
  Status profile_kernel(int kernel, int repetitions, double* ms,
                        double* bytes);
  const std::string& last_error() const { return error_; }

 private:
  Solver() = default;
  Status fail(int code, uint32_t detail, const std::string& what);
  Status check(cudaError_t e, const char* what);
  Status allocate();
  Status build_hierarchy();
  Status refresh_mixed();
  void aggregate_channel(int level, int face_axis, const double* src,
                         double* dst);
  // The MG preconditioner: z = M r, by default on the internal r/z buffers.
  Status mg_apply(bool mixed, const double* r = nullptr, double* z = nullptr);
  void clear_mg_graphs();
  // z = M r on kr_/kz_ with the policy's preconditioner (MG or cold IC(0)).
  Status precondition(bool mixed);
  Status dic_apply();
  Status dic_factor();
  Status krylov_bicgstab(const hfps_control& control, hfps_result& result,
                         double* history, uint32_t capacity);
  template <class T>
  void mg_enqueue(std::vector<DeviceLevel<T>>& levels, const double* r,
                  double* z);
  template <class T>
  void cycle(std::vector<DeviceLevel<T>>& levels, int level, int counter, bool x_zero);
  template <class T>
  void smooth(std::vector<DeviceLevel<T>>& levels, int level, int sweeps,
              bool reverse, bool x_zero);
  template <class T>
  void coarse_solve(std::vector<DeviceLevel<T>>& levels, bool x_zero);
  // The small levels as one persistent launch: tail_cycle appends the
  // phases of cycle(level, counter) to `prog` exactly as cycle() would
  // launch them (same buffer roles and swaps); tail_launch runs a program.
  void select_tail();
  template <class T>
  void tail_cycle(std::vector<DeviceLevel<T>>& levels, int level, int counter, bool x_zero,
                  TailProgram<T>& prog);
  template <class T>
  void tail_launch(std::vector<DeviceLevel<T>>& levels, TailProgram<T>& prog);
  Status krylov_pcg(const hfps_control& control, hfps_result& result,
                    double* history, uint32_t capacity);
  Status krylov_fgmres(const hfps_control& control, hfps_result& result,
                       double* history, uint32_t capacity);
  Status ensure_fgmres_storage(uint32_t restart);
  Status ensure_recycle_storage();
  Status recycle_publish(const double* x, hfps_result& result);
  Status recycle_project(const hfps_control& control, double tol, hfps_result& result);
  Status sync_scalars();
  Status copy_in(double* dst, const double* src, size_t n, int memory);
  Status copy_out(double* dst, const double* src, size_t n, int memory);

  int nx_{}, ny_{}, nz_{};
  unsigned neumann_{};
  hfps_policy policy_{};
  std::vector<double> faces_[3];
  std::vector<uint8_t> active_host_;
  bool has_active_{};
  bool own_stream_{};
  cudaStream_t stream_{};
  std::string error_;

  // Device storage: one arena for everything.
  char* arena_{};
  size_t arena_bytes_{};
  double* d_faces_[3]{};
  uint8_t* d_active_{};
  std::vector<DeviceLevel<double>> l64_;
  std::vector<DeviceLevel<float>> l32_;
  std::vector<double*> volume_;
  std::vector<uint8_t*> fluid_;
  double* agg_[3]{};          // aggregation scratch (max face count each)
  double* user_[4]{};         // staging for user coefficients (diag, fx, fy, fz)
  double* kx_{};              // Krylov vectors
  double* kr_{};
  double* kz_{};
  double* kp_{};
  double* kap_{};
  double* kb_{};
  bool krylov_fusion_{true};  // PCG's r.z formed in the MG exit
  bool queue_ahead_{true};    // PCG queues the next MG before reading scalars
  bool tiled_stencil_{true};  // the Krylov operator over 3-D tiles
  cudaEvent_t scalars_ready_{};  // the scalar readback of the current step
  Scalars* d_scalars_{};
  Scalars* h_scalars_{};      // pinned
  double* d_partials_{};
  bool coefficients_ready_{};
  bool mixed_ready_{};
  bool diagonal_shortcut_{};
  // The finest level's first pre-smoothing sweep runs on the chunked scan
  // with the zero flags, so the MG entry need not clear x.
  bool first_sweep_zero_{};
  // Coarsest level in line mode with one line axis and at most
  // kCoarseDenseMaxCells cells: its coarse_sweeps zebra line sweeps are an
  // affine map x_out = P x_in + M b, recorded column by column after every
  // coefficient update and applied as one dense product (P then M, FP64,
  // column-major).
  double* coarse_op_{};
  int coarse_axis_{-1};
  bool coarse_dense_{};
  // First level of the persistent small-level launch (-1: every phase is
  // its own kernel), its PCR width and co-resident grid per precision.
  int tail_level_{-1};
  int tail_steps_{-1};
  int tail_blocks_[2]{};
  bool tail_barrier_test_{false};
  bool scaled_norm_{false};   // the current solve's hfps_control.norm is SCALED
  void queue_norm(const double* v);
  double norm_value(double plain_squares) const;
  // FGMRES basis: V_0..V_restart, Z_0..Z_{restart-1} and the operator image,
  // allocated on first use for the largest restart asked for.
  double* fg_storage_{};
  uint32_t fg_restart_{};
  std::vector<double*> fg_v_;
  std::vector<double*> fg_z_;
  double* fg_w_{};
  // FGMRES subspace recycling across solves (hfps_recycle): a ring of up to
  // four cycle corrections (oldest first from rc_oldest_) and the snapshot
  // of x at the current cycle's start.  Publishing swaps the snapshot buffer
  // into the ring instead of copying it.  The projection's images A d_i use
  // four scratch vectors of their own.
  static constexpr int kRecycleMax = 4;
  double* rc_storage_{};
  double* rc_ring_[kRecycleMax]{};
  double* rc_snapshot_{};
  double* rc_image_[kRecycleMax]{};   // projection scratch: A d_i
  bool rc_capture_{}, rc_guard_only_{}, rc_cycle_active_{}, rc_pending_{};
  int rc_count_{}, rc_oldest_{};
  // Cold-path IC(0): decorated row diagonals and inverse pivots (level 0),
  // and the captured wavefront apply (kr_ -> kz_).
  double* dic_rows_{};
  double* dic_inv_{};
  cudaGraphExec_t dic_graph_{};
  size_t dic_nodes_{};
  // The MG application captured as one CUDA graph per (precision slot,
  // input, output) buffers: the PCG uses kr_/kz_, FGMRES every basis
  // column's V_j/Z_j directly (no copies into fixed buffers).
  struct MgGraph {
    int slot;
    const double* r;
    double* z;
    cudaGraphExec_t exec;
  };
  std::vector<MgGraph> mg_graphs_;
  size_t mg_nodes_[2]{};      // kernels per MG application (graph nodes)
  uint64_t launches_{};       // kernels launched since the last reset
  bool use_graphs_{true};
};

}  // namespace hfps
