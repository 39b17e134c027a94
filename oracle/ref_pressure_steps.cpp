// CPU oracle harness for the steps either side of the pressure solve, around
// the UNMODIFIED reference sources.  Test infrastructure only: nothing in the
// product path links or calls this.
//
// face_pressure_coefficient has internal linkage in the reference's
// src/solver_piso.cpp, so this translation unit compiles that reference
// source file itself (included from the reference tree at build time, see
// oracle/Makefile) and calls the function from the same unit.  The other
// two steps are reached through their declared entry points:
//   * face coefficients  face_pressure_coefficient (src/solver_piso.cpp:
//     1060-1136) over every face, as fill_pressure_coefficients does;
//   * assembly           detail::assemble_pressure_system_impl
//     (src/solver_pressure.cpp:110-332);
//   * flux correction    PressureCorrectionBoundaryPlan::mass_flux_response
//     (src/solver_piso.cpp:1642-1653) over every face, as the publication
//     loop applies it (src/solver_piso.cpp:7400-7420).
// The plans they need are compiled the way the reference's own unit test
// builds them (tests/unit/solver_pressure_boundary_plan_test.cpp:28-90): a
// runtime-axes Cartesian geometry on one rank, a ValidatedModel whose
// Neumann sides are adiabatic no-slip walls and whose Dirichlet sides are
// pressure outlets (PressureCorrectionFaceKind::homogeneous_dirichlet), the
// BoundaryCompiler, PressureCorrectionBoundaryPlan::compile and
// CartesianKernelPlan::compile.  The certificate fields the assembly
// validates are filled with consistent non-zero tokens.
#include "solver_piso.cpp"

#include <memory>
#include <vector>

namespace {
using namespace hundun::v04;

struct OwnedField {
  std::vector<double> storage;
  FieldView view{};
};

OwnedField owned_field(FieldId id, Int3 cells, std::uint8_t ghosts,
                       std::uint8_t components, StorageIdentity storage,
                       RevisionDomainIdentity domain) {
  OwnedField f;
  const std::size_t sy = static_cast<std::size_t>(cells.x + 2 * ghosts);
  const std::size_t sz = sy * static_cast<std::size_t>(cells.y + 2 * ghosts);
  const std::size_t sc = sz * static_cast<std::size_t>(cells.z + 2 * ghosts);
  f.storage.assign(sc * components, 0.0);
  f.view.base = f.storage.data() + ghosts + static_cast<std::size_t>(ghosts) * (sy + sz);
  f.view.interior = cells;
  f.view.ghosts = {ghosts, ghosts, ghosts};
  f.view.components = components;
  f.view.stride_y = sy;
  f.view.stride_z = sz;
  f.view.component_stride = sc;
  f.view.field = id;
  f.view.revision = 1U;
  f.view.storage_identity = storage;
  f.view.revision_domain = domain;
  return f;
}

Int3 face_extent(Int3 cells, CartesianAxis axis) {
  Int3 e = cells;
  if (axis == CartesianAxis::x) ++e.x;
  else if (axis == CartesianAxis::y) ++e.y;
  else ++e.z;
  return e;
}

FaceFieldView face_view(double* base, Int3 cells, CartesianAxis axis,
                        StorageIdentity storage, RevisionDomainIdentity domain) {
  const Int3 e = face_extent(cells, axis);
  return {base, e, static_cast<std::size_t>(e.x),
          static_cast<std::size_t>(e.x) * static_cast<std::size_t>(e.y), axis, storage,
          domain};
}

inline std::size_t flat(Int3 s, int i, int j, int k) {
  return static_cast<std::size_t>(i) +
         static_cast<std::size_t>(s.x) *
             (static_cast<std::size_t>(j) + static_cast<std::size_t>(s.y) * static_cast<std::size_t>(k));
}

BoundaryFaceSpec wall_face() {
  BoundaryFaceSpec face;
  face.flow_kind = BoundaryKind::no_slip_wall;
  face.thermal_kind = BoundaryKind::adiabatic_wall;
  face.mach_limit = 0.95;
  return face;
}

BoundaryFaceSpec outlet_face() {
  BoundaryFaceSpec face;
  face.flow_kind = BoundaryKind::pressure_outlet;
  face.thermal_kind = BoundaryKind::none;
  face.pressure = 101325.0;
  face.temperature = 300.0;
  face.backflow_velocity = {0.0, 0.0, 0.0};
  face.backflow_temperature = 300.0;
  face.relaxation = 0.1;
  face.mach_limit = 0.9;
  face.allow_backflow = true;
  return face;
}

// The plans of one grid: geometry, boundary, kernels, pressure boundary.
struct Plans {
  Int3 cells{};
  CartesianGeometryPlan geometry;
  MeshPatch patch{};
  BoundaryPlan boundary;
  SchemePlan schemes;
  TimeSchemePlan time;
  FieldRegistry registry;
  CartesianKernelPlan kernels;
  PressureCorrectionBoundaryPlan pressure;
};

// 0 on success, else a stage code * 100000 + the status detail.
int build(int nx, int ny, int nz, const double* xf, const double* yf, const double* zf,
          const int* bc, Plans& p) {
  int initialized = 0;
  MPI_Initialized(&initialized);
  if (!initialized) MPI_Init(nullptr, nullptr);
  p.cells = {nx, ny, nz};
  CartesianMeshSpec mesh;
  mesh.kind = GeometryKind::runtime_axes_v1;
  mesh.axes_file = "synthetic-runtime-axes";
  mesh.runtime_faces[0].assign(xf, xf + nx + 1);
  mesh.runtime_faces[1].assign(yf, yf + ny + 1);
  mesh.runtime_faces[2].assign(zf, zf + nz + 1);
  mesh.lower = {xf[0], yf[0], zf[0]};
  mesh.upper = {xf[nx], yf[ny], zf[nz]};
  mesh.has_exact_cells = true;
  mesh.exact_cells = p.cells;
  mesh.minimum_spacing = {1.0e-12, 1.0e-12, 1.0e-12};
  mesh.max_growth_ratio = 1.0e9;
  mesh.limits = {UINT64_C(1) << 40, UINT64_C(1) << 50};
  Status st = CartesianGeometryCompiler::compile(MPI_COMM_SELF, mesh, GeometryBudget{},
                                                 p.geometry, p.patch);
  if (!st) return 100000 + static_cast<int>(st.detail % 100000U);
  ValidatedModel model;
  model.fingerprint = UINT64_C(0x4846505354455053);
  model.pressure_reference = PressureReferenceKind::boundary_absolute;
  for (int f = 0; f < 6; ++f) model.boundaries[f] = bc[f] == 1 ? wall_face() : outlet_face();
  model.schemes = SchemeSpec{};
  model.time = TimeControlSpec{};
  st = BoundaryCompiler::compile(MPI_COMM_SELF, model, p.geometry, p.patch, p.registry,
                                 p.boundary, p.schemes, p.time);
  if (!st) return 200000 + static_cast<int>(st.detail % 100000U);
  st = PressureCorrectionBoundaryPlan::compile(p.geometry, p.patch, p.boundary, p.pressure);
  if (!st) return 300000 + static_cast<int>(st.detail % 100000U);
  st = CartesianKernelPlan::compile(p.schemes, p.geometry, p.patch, p.boundary, p.kernels);
  if (!st) return 400000 + static_cast<int>(st.detail % 100000U);
  return 0;
}

}  // namespace

// The translation unit is compiled with hidden visibility so that the linker
// keeps only what these entry points reach; they alone are exported.
#define HFREF_EXPORT __attribute__((visibility("default")))

extern "C" {

// Face coefficients of every face from a cell mobility beta: the reference
// takes density * r_au(component) per cell, so density = 1 and every r_au
// component = beta; boundary ghosts carry the owner's state (the ghost
// state a pressure outlet's EOS closure returns for an unchanged cell).
// Outputs: x-, y-, z-face arrays in x-fastest order.
HFREF_EXPORT int hfref_face_coefficients(int nx, int ny, int nz, const double* xf, const double* yf,
                            const double* zf, const int* bc, const double* beta,
                            double* out_x, double* out_y, double* out_z) {
  auto p = std::make_unique<Plans>();
  const int rc = build(nx, ny, nz, xf, yf, zf, bc, *p);
  if (rc != 0) return rc;
  const Int3 cells = p->cells;
  OwnedField density = owned_field(51U, cells, 1U, 1U, 501U, 601U);
  OwnedField r_au = owned_field(52U, cells, 1U, 3U, 502U, 602U);
  for (int k = -1; k <= nz; ++k)
    for (int j = -1; j <= ny; ++j)
      for (int i = -1; i <= nx; ++i) {
        const int ci = std::min(std::max(i, 0), nx - 1);
        const int cj = std::min(std::max(j, 0), ny - 1);
        const int ck = std::min(std::max(k, 0), nz - 1);
        const double b = beta[flat(cells, ci, cj, ck)];
        density.view.unchecked({i, j, k}, 0U) = 1.0;
        for (std::uint8_t c = 0; c < 3U; ++c) r_au.view.unchecked({i, j, k}, c) = b;
      }
  double* outs[3] = {out_x, out_y, out_z};
  const CartesianAxis axes[3] = {CartesianAxis::x, CartesianAxis::y, CartesianAxis::z};
  for (int a = 0; a < 3; ++a) {
    const Int3 e = face_extent(cells, axes[a]);
    for (int k = 0; k < e.z; ++k)
      for (int j = 0; j < e.y; ++j)
        for (int i = 0; i < e.x; ++i)
          outs[a][flat(e, i, j, k)] = face_pressure_coefficient(
              p->kernels, as_const(density.view), as_const(r_au.view), p->geometry, p->patch,
              p->pressure, axes[a], {i, j, k});
  }
  return 0;
}

// The kernel plan's metrics along `axis` (0 x, 1 y, 2 z): face coordinates
// (cells + 1), cell centres and widths (cells), as the pressure steps read
// them (detail::face_coordinate, centre_coordinate, cell_width).
HFREF_EXPORT int hfref_axis_metrics(int nx, int ny, int nz, const double* xf, const double* yf,
                                    const double* zf, const int* bc, int axis, double* faces,
                                    double* centres, double* widths) {
  auto p = std::make_unique<Plans>();
  const int rc = build(nx, ny, nz, xf, yf, zf, bc, *p);
  if (rc != 0) return rc;
  const CartesianAxis a = axis == 0 ? CartesianAxis::x
                                    : (axis == 1 ? CartesianAxis::y : CartesianAxis::z);
  const int n = axis == 0 ? nx : (axis == 1 ? ny : nz);
  for (int i = 0; i <= n; ++i) faces[i] = detail::face_coordinate(p->kernels, a, i);
  for (int i = 0; i < n; ++i) {
    centres[i] = detail::centre_coordinate(p->kernels, a, i);
    widths[i] = detail::cell_width(p->kernels, a, i);
  }
  return 0;
}

// The pressure-correction system from face coefficients, predicted face
// fluxes and the cell states.  bdf_order 1 or 2; rho_nm1 (BDF2) and
// mass_source may be NULL.  Returns 0, or the assembly's status
// (code * 100000 + detail) with diag/rhs untouched.
HFREF_EXPORT int hfref_assemble(int nx, int ny, int nz, const double* xf, const double* yf,
                   const double* zf, const int* bc, const double* cx, const double* cy,
                   const double* cz, const double* qx, const double* qy, const double* qz,
                   int bdf_order, double a0, double a1, double a2, const double* rho,
                   const double* rho_n, const double* rho_nm1, const double* drho_dp,
                   const double* mass_source, double* diag, double* rhs) {
  auto p = std::make_unique<Plans>();
  const int rc = build(nx, ny, nz, xf, yf, zf, bc, *p);
  if (rc != 0) return rc;
  const Int3 cells = p->cells;
  const std::size_t n = static_cast<std::size_t>(nx) * ny * nz;
  // Face arrays copied into owned storage (one block per kind of data).
  const Int3 ex = face_extent(cells, CartesianAxis::x);
  const Int3 ey = face_extent(cells, CartesianAxis::y);
  const Int3 ez = face_extent(cells, CartesianAxis::z);
  const std::size_t fx = static_cast<std::size_t>(ex.x) * ex.y * ex.z;
  const std::size_t fy = static_cast<std::size_t>(ey.x) * ey.y * ey.z;
  const std::size_t fz = static_cast<std::size_t>(ez.x) * ez.y * ez.z;
  std::vector<double> coeff(fx + fy + fz), flux(fx + fy + fz);
  std::copy(cx, cx + fx, coeff.begin());
  std::copy(cy, cy + fy, coeff.begin() + fx);
  std::copy(cz, cz + fz, coeff.begin() + fx + fy);
  std::copy(qx, qx + fx, flux.begin());
  std::copy(qy, qy + fy, flux.begin() + fx);
  std::copy(qz, qz + fz, flux.begin() + fx + fy);

  const auto cell_field = [&](FieldId id, const double* values, StorageIdentity s) {
    OwnedField f = owned_field(id, cells, 0U, 1U, s, 700U + s);
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) f.view.unchecked({i, j, k}, 0U) = values[flat(cells, i, j, k)];
    return f;
  };
  OwnedField trial = cell_field(61U, rho, 611U);
  OwnedField accepted = cell_field(62U, rho_n, 612U);
  OwnedField derivative = cell_field(64U, drho_dp, 614U);
  OwnedField previous, source;
  if (bdf_order == 2) previous = cell_field(63U, rho_nm1, 613U);
  if (mass_source != nullptr) source = cell_field(65U, mass_source, 615U);
  OwnedField sys_diag = owned_field(66U, cells, 0U, 1U, 616U, 716U);
  OwnedField sys_rhs = owned_field(67U, cells, 0U, 1U, 617U, 717U);

  constexpr RevisionToken kTime = 9U;
  constexpr PlanFingerprint kCoupler = 0x70C0U;
  detail::PressureAssemblyBinding binding;
  binding.kernels = &p->kernels;
  binding.cells = cells;
  binding.coupler = kCoupler;
  binding.pressure_reference_plan = 0x70C1U;
  binding.geometry_fingerprint = p->geometry.fingerprint();
  binding.mass_source_identity = mass_source != nullptr ? 0x70C2U : 0U;
  binding.workspace.x_pressure_coefficient =
      face_view(coeff.data(), cells, CartesianAxis::x, 630U, 730U);
  binding.workspace.y_pressure_coefficient =
      face_view(coeff.data() + fx, cells, CartesianAxis::y, 630U, 730U);
  binding.workspace.z_pressure_coefficient =
      face_view(coeff.data() + fx + fy, cells, CartesianAxis::z, 630U, 730U);
  binding.workspace.phi_h_by_a.x = face_view(flux.data(), cells, CartesianAxis::x, 631U, 731U);
  binding.workspace.phi_h_by_a.y =
      face_view(flux.data() + fx, cells, CartesianAxis::y, 631U, 731U);
  binding.workspace.phi_h_by_a.z =
      face_view(flux.data() + fx + fy, cells, CartesianAxis::z, 631U, 731U);
  binding.workspace.phi_h_by_a.revision = 5U;
  PisoIntermediateCertificate intermediate;
  intermediate.plan = kCoupler;
  intermediate.r_au = 1U;
  intermediate.h_by_a = 2U;
  intermediate.pressure_face_coefficient = 3U;
  intermediate.phi_h_by_a = 5U;
  intermediate.trial_face_flux = 6U;
  intermediate.dependency = 7U;
  intermediate.corrector = 2U;
  intermediate.thermophysical_boundary_semantics = 21U;
  intermediate.thermophysical_boundary_target = 22U;
  intermediate.thermophysical_boundary_rank_local_binding = 23U;
  intermediate.thermophysical_boundary_collective_lineage = 24U;
  intermediate.thermophysical_boundary_rank_local_lineage = 25U;
  binding.current = intermediate;
  binding.thermophysical_context.target_time = kTime;
  binding.thermophysical_context.geometry = p->geometry.fingerprint();
  binding.thermophysical_context.pressure_reference = 11U;
  binding.thermophysical_context.numeric_boundary = 12U;
  binding.thermophysical_context.phase = BoundaryThermophysicalGhostPhase::corrector_two;

  PressureCorrectionInput input;
  input.intermediate = intermediate;
  input.pressure_reference.plan = 0x70C1U;
  input.pressure_reference.predictor = 0x70C3U;
  input.pressure_reference.thermodynamics = 0x70C4U;
  input.pressure_reference.closure = 0x70C5U;
  input.pressure_reference.time = kTime;
  input.pressure_reference.pressure_reference = 11U;
  input.time = kTime;
  input.geometry = 13U;
  input.numeric_boundary = 12U;
  input.bdf.order = static_cast<std::uint8_t>(bdf_order);
  input.bdf.a0 = a0;
  input.bdf.a1 = a1;
  input.bdf.a2 = a2;
  input.density_trial = as_const(trial.view);
  input.density_accepted = as_const(accepted.view);
  if (bdf_order == 2) input.density_previous = as_const(previous.view);
  input.drho_dp_h_y = as_const(derivative.view);
  if (mass_source != nullptr) {
    input.mass_source.identity = 0x70C2U;
    input.mass_source.time = kTime;
    input.mass_source.rate = as_const(source.view);
  }
  PressureCorrectionSystemView system{sys_diag.view, sys_rhs.view};
  PressureCorrectionCertificate certificate;
  const Status st = detail::assemble_pressure_system_impl(binding, input, system, certificate);
  if (!st) return static_cast<int>(st.code) * 100000 + static_cast<int>(st.detail % 100000U);
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        diag[flat(cells, i, j, k)] = sys_diag.view.unchecked({i, j, k}, 0U);
        rhs[flat(cells, i, j, k)] = sys_rhs.view.unchecked({i, j, k}, 0U);
      }
  (void)n;
  return 0;
}

// Face fluxes after a pressure correction: q_f += mass_flux_response(p', f,
// c_f, scale) on every face.  qx/qy/qz are updated in place.
HFREF_EXPORT int hfref_correct_flux(int nx, int ny, int nz, const double* xf, const double* yf,
                       const double* zf, const int* bc, const double* correction,
                       const double* cx, const double* cy, const double* cz, double scale,
                       double* qx, double* qy, double* qz) {
  auto p = std::make_unique<Plans>();
  const int rc = build(nx, ny, nz, xf, yf, zf, bc, *p);
  if (rc != 0) return rc;
  const Int3 cells = p->cells;
  OwnedField pc = owned_field(71U, cells, 1U, 1U, 621U, 721U);
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i)
        pc.view.unchecked({i, j, k}, 0U) = correction[flat(cells, i, j, k)];
  const double* coefficients[3] = {cx, cy, cz};
  double* fluxes[3] = {qx, qy, qz};
  const CartesianAxis axes[3] = {CartesianAxis::x, CartesianAxis::y, CartesianAxis::z};
  for (int a = 0; a < 3; ++a) {
    const Int3 e = face_extent(cells, axes[a]);
    for (int k = 0; k < e.z; ++k)
      for (int j = 0; j < e.y; ++j)
        for (int i = 0; i < e.x; ++i) {
          const std::size_t f = flat(e, i, j, k);
          fluxes[a][f] += p->pressure.mass_flux_response(as_const(pc.view), axes[a], {i, j, k},
                                                         coefficients[a][f], scale);
        }
  }
  return 0;
}

}  // extern "C"
