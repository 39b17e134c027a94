// B200PressureSolve: the C++ object a Hundun-Flow maintainer adds to the
// reference to route its pressure solve through this library's C ABI
// (include/hf_pressure_solver.h).  Header-only; it is compiled inside the
// reference (it includes the reference's own headers) and links against
// hundun-flow_b200/libhfps.so.
//
// It mirrors the three calls the PISO coupler makes on its MG plan and
// Krylov driver (reference paths relative to versions/v0.4):
//   compile   NativeCartesianMgPlan::compile (include/hundun/v04_linear.hpp:
//             945-953, called at src/solver_piso.cpp:7060)
//   update    NativeCartesianMgPlan::update_coefficients (v04_linear.hpp:
//             955-960, called at src/solver_piso.cpp:7116)
//   solve     solve_fgmres / solve_pcg with the plan as preconditioner
//             (v04_linear.hpp:1070-1083, called at src/solver_piso.cpp:
//             10445-10449), returning a LinearSolveResult.
// Reference field views carry ghost layers and strides (BasicFieldView,
// include/hundun/v04_execution.hpp:119-150); the C ABI takes dense
// x-fastest interiors, so the adapter packs and unpacks host copies.  A
// coupler that keeps the fields on the device passes HFPS_DEVICE pointers
// and its stream instead.
#pragma once

#include <cstdint>
#include <vector>

#include "hf_pressure_solver.h"
#include "hundun/v04_linear.hpp"

namespace hundun::v04 {

namespace b200 {

inline Status to_status(int code) noexcept {
  return code == HFPS_OK ? Status{}
                         : Status{static_cast<StatusCode>(code), 0x8200U};
}

// Dense x-fastest copy of a cell view's interior (component 0); View is
// ConstFieldView or FieldView.
template <class View>
inline void pack_interior(View v, std::vector<double>& out) {
  const Int3 n = v.interior;
  out.resize(static_cast<std::size_t>(n.x) * n.y * n.z);
  std::size_t c = 0;
  for (std::int32_t k = 0; k < n.z; ++k)
    for (std::int32_t j = 0; j < n.y; ++j)
      for (std::int32_t i = 0; i < n.x; ++i) out[c++] = v.unchecked({i, j, k}, 0U);
}

inline void unpack_interior(const std::vector<double>& in, FieldView v) {
  const Int3 n = v.interior;
  std::size_t c = 0;
  for (std::int32_t k = 0; k < n.z; ++k)
    for (std::int32_t j = 0; j < n.y; ++j)
      for (std::int32_t i = 0; i < n.x; ++i) v.unchecked({i, j, k}, 0U) = in[c++];
}

// Dense x-fastest copy of a face view (extents include the extra face).
inline void pack_faces(ConstFaceFieldView v, std::vector<double>& out) {
  const Int3 e = v.extents;
  out.resize(static_cast<std::size_t>(e.x) * e.y * e.z);
  std::size_t c = 0;
  for (std::int32_t k = 0; k < e.z; ++k)
    for (std::int32_t j = 0; j < e.y; ++j)
      for (std::int32_t i = 0; i < e.x; ++i) out[c++] = v.unchecked({i, j, k});
}

// The LinearSolveResult fields the PISO coupler reads, from hfps_result.
inline LinearSolveResult to_result(int code, const hfps_result& r) noexcept {
  LinearSolveResult out;
  out.status = code == HFPS_OK ? Status{}
                               : Status{static_cast<StatusCode>(r.status), r.detail};
  out.termination = static_cast<LinearTermination>(r.termination);
  out.iterations = r.iterations;
  out.initial_true_residual = r.initial_true_residual;
  out.final_true_residual = r.final_true_residual;
  out.recursive_residual = r.recursive_residual;
  out.operator_applies = r.operator_applies;
  out.preconditioner_applies = r.preconditioner_applies;
  out.true_residual_criterion_valid = r.rhs_norm > 0.0 || r.true_residual_limit > 0.0;
  out.rhs_norm = r.rhs_norm;
  out.true_residual_limit = r.true_residual_limit;
  out.recycle_offered_directions = r.recycle_offered;
  out.recycle_retained_directions = r.recycle_retained;
  out.recycle_projection_accepted = r.recycle_accepted != 0U;
  out.recycle_projected_true_residual = r.recycle_projected_residual;
  out.recycle_cycle_corrections = r.recycle_captured;
  return out;
}

}  // namespace b200

class B200PressureSolve {
 public:
  B200PressureSolve() = default;
  B200PressureSolve(const B200PressureSolve&) = delete;
  B200PressureSolve& operator=(const B200PressureSolve&) = delete;
  ~B200PressureSolve() {
    if (solver_ != nullptr) hfps_destroy(solver_);
  }

  // NativeCartesianMgPlan::compile: the grid's face coordinates (the
  // geometry plan's AxisMetrics::faces(), already binary32-rounded by the
  // reference's geometry compiler), the boundary kinds and scaling of the
  // spec, and the IBM cell activity (empty: all fluid).
  Status compile(const NativeCartesianMgSpec& spec, Int3 cells, const std::vector<double>& xf,
                 const std::vector<double>& yf, const std::vector<double>& zf,
                 const std::vector<std::uint8_t>& active) noexcept {
    hfps_geometry g{};
    g.nx = cells.x;
    g.ny = cells.y;
    g.nz = cells.z;
    g.x_faces = xf.data();
    g.y_faces = yf.data();
    g.z_faces = zf.data();
    const MgBoundarySet& b = spec.boundaries;
    const MgBoundaryKind kinds[6] = {b.x_min, b.x_max, b.y_min, b.y_max, b.z_min, b.z_max};
    for (int f = 0; f < 6; ++f) g.boundary[f] = static_cast<int>(kinds[f]);
    g.cell_active = active.empty() ? nullptr : active.data();
    hfps_policy p{};
    hfps_production_policy(&p);  // production_pressure_mg_policy
    p.unit_linear = spec.correction_scaling == MgCorrectionScaling::unit_linear ? 1 : 0;
    unit_linear_ = p.unit_linear != 0;
    return b200::to_status(hfps_create(&g, &p, /*stream=*/nullptr, &solver_));
  }

  // NativeCartesianMgPlan::update_coefficients with MgCoefficientViews.
  Status update(const MgCoefficientViews& v) {
    b200::pack_interior(v.diagonal, d_);
    b200::pack_faces(v.x, fx_);
    b200::pack_faces(v.y, fy_);
    b200::pack_faces(v.z, fz_);
    return b200::to_status(
        hfps_set_coefficients(solver_, d_.data(), fx_.data(), fy_.data(), fz_.data(), HFPS_HOST));
  }

  // solve_fgmres(12) with the residual-minimising plan (the reference's
  // production pressure solve, src/solver_piso.cpp:10447), or solve_pcg
  // with a unit-scaled plan; recycle as the PISO corrector selects it
  // (src/solver_piso.cpp:10410-10433).  A failed solve publishes nothing.
  LinearSolveResult solve(const LinearSolveInvocation& inv, bool mixed,
                          int recycle = HFPS_RECYCLE_NONE) {
    hfps_control c{};
    hfps_default_control(&c);
    c.relative_tolerance = inv.control.relative_tolerance;
    c.absolute_tolerance = inv.control.absolute_tolerance;
    c.maximum_iterations = inv.control.maximum_iterations;
    c.true_residual_interval = inv.control.true_residual_interval;
    c.algorithm = unit_linear_ ? HFPS_PCG : HFPS_FGMRES;
    c.restart = unit_linear_ ? 0U : inv.control.restart;
    c.precision = mixed ? HFPS_MIXED : HFPS_FP64;
    c.recycle = recycle;
    b200::pack_interior(inv.rhs, rhs_);
    b200::pack_interior(inv.solution, x_);
    hfps_result r{};
    const int s = hfps_solve(solver_, rhs_.data(), x_.data(), HFPS_HOST, &c, &r, nullptr, 0);
    if (s == HFPS_OK) b200::unpack_interior(x_, inv.solution);
    return b200::to_result(s, r);
  }

  hfps_solver* handle() const noexcept { return solver_; }

 private:
  hfps_solver* solver_{};
  bool unit_linear_{};
  std::vector<double> d_, fx_, fy_, fz_, rhs_, x_;
};

}  // namespace hundun::v04
