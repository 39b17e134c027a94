// CPU oracle harness around the UNMODIFIED reference pressure-solve sources.
//
// Test infrastructure only: nothing in the product path links or calls this.
// It is compiled together with the reference's own solver sources
// (versions/v0.4/src/solver_mg*.cpp, solver_krylov.cpp, ... ; see
// oracle/Makefile) against the single-rank MPI stand-in in oracle/mpi_shim,
// and exposes a flat C ABI so that tests and the CPU baseline can drive the
// reference's own NativeCartesianMgPlan, solve_pcg and solve_fgmres.
//
// The wiring follows the reference's minimal MG+Krylov integration test
// (tests/integration/solver_mg_krylov_isolation_test.cpp:113-232).  The
// linear operator is the regular 7-point pressure operator of
// PressureLinearOperator::apply_after_exchange (src/solver_pressure.cpp:
// 746-811; Dirichlet neighbour 0 and Neumann neighbour = self per
// src/solver_piso.cpp:1568-1603) decorated exactly as
// IbmPressureOperator::decorate_pressure_action does
// (src/solver_ibm_pressure.cpp:347-385): solid rows become the identity and
// every fluid/solid link adds c_f (x_solid - x_fluid) to the fluid row.
// The preconditioner receives the undecorated coefficients plus the
// cell/face activity maps (include/hundun/v04_linear.hpp:180-187), as the
// reference's PISO epoch does.
#include "hundun/v04_linear.hpp"
#include "hundun/v04_parallel.hpp"

#include <mpi.h>

#include <algorithm>
#include <memory>
#include <array>
#include <chrono>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <memory>
#include <vector>
#include "solver_iccg.hpp"  // ColdPressureIccg, ColdPressureDilu (header classes)

namespace {
using namespace hundun::v04;

struct OwnedField {
  std::vector<double> storage;
  FieldView view{};
};

OwnedField make_field(FieldId id, Int3 cells, std::uint8_t ghosts,
                      std::uint8_t components, StorageIdentity storage,
                      RevisionDomainIdentity domain) {
  OwnedField result;
  const std::size_t sy = static_cast<std::size_t>(cells.x + 2 * ghosts);
  const std::size_t sz = sy * static_cast<std::size_t>(cells.y + 2 * ghosts);
  const std::size_t sc = sz * static_cast<std::size_t>(cells.z + 2 * ghosts);
  result.storage.assign(sc * components, 0.0);
  result.view.base = result.storage.data() + ghosts +
                     static_cast<std::size_t>(ghosts) * (sy + sz);
  result.view.interior = cells;
  result.view.ghosts = {ghosts, ghosts, ghosts};
  result.view.components = components;
  result.view.stride_y = sy;
  result.view.stride_z = sz;
  result.view.component_stride = sc;
  result.view.field = id;
  result.view.revision = 1U;
  result.view.storage_identity = storage;
  result.view.revision_domain = domain;
  return result;
}

struct OwnedFace {
  std::vector<double> storage;
  ConstFaceFieldView view{};
};

OwnedFace make_face(CartesianAxis axis, Int3 cells, const double* values,
                    StorageIdentity storage) {
  OwnedFace result;
  Int3 e = cells;
  if (axis == CartesianAxis::x) ++e.x;
  else if (axis == CartesianAxis::y) ++e.y;
  else ++e.z;
  const std::size_t count = static_cast<std::size_t>(e.x) *
                            static_cast<std::size_t>(e.y) *
                            static_cast<std::size_t>(e.z);
  result.storage.assign(values, values + count);
  result.view = {result.storage.data(),
                 e,
                 static_cast<std::size_t>(e.x),
                 static_cast<std::size_t>(e.x) * static_cast<std::size_t>(e.y),
                 axis,
                 storage,
                 80U};
  return result;
}

inline std::size_t flat(Int3 s, int i, int j, int k) {
  return static_cast<std::size_t>(i) +
         static_cast<std::size_t>(s.x) *
             (static_cast<std::size_t>(j) +
              static_cast<std::size_t>(s.y) * static_cast<std::size_t>(k));
}

MgBoundaryKind boundary_kind(int code) {
  return code == 1 ? MgBoundaryKind::neumann
                   : (code == 2 ? MgBoundaryKind::periodic
                                : MgBoundaryKind::dirichlet);
}

// Regular pressure operator followed by the IBM decoration.
class HarnessOperator final : public LinearOperator {
 public:
  Int3 cells{};
  std::array<int, 6> bc{};
  const double* diagonal{};
  const double* fx{};
  const double* fy{};
  const double* fz{};
  const std::uint8_t* active{};
  LinearIdentity identity{};

  LinearOperatorCertificate certificate() const noexcept override {
    return {identity, 0x5eed5eedULL, cells, LinearOperatorClass::spd};
  }

  double neighbour(ConstFieldView x, int i, int j, int k, int axis,
                   int direction) const noexcept {
    int c[3]{i, j, k};
    const int n[3]{cells.x, cells.y, cells.z};
    c[axis] += direction;
    if (c[axis] >= 0 && c[axis] < n[axis]) {
      return x.unchecked({c[0], c[1], c[2]}, 0U);
    }
    const int code = bc[2 * axis + (direction > 0 ? 1 : 0)];
    if (code == 0) return 0.0;
    if (code == 1) return x.unchecked({i, j, k}, 0U);
    c[axis] = direction < 0 ? n[axis] - 1 : 0;
    return x.unchecked({c[0], c[1], c[2]}, 0U);
  }

  Status apply(FieldView input, FieldView output) const noexcept override {
    const ConstFieldView x = as_const(input);
    const Int3 xe{cells.x + 1, cells.y, cells.z};
    const Int3 ye{cells.x, cells.y + 1, cells.z};
    const Int3 ze{cells.x, cells.y, cells.z + 1};
    for (int k = 0; k < cells.z; ++k)
      for (int j = 0; j < cells.y; ++j)
        for (int i = 0; i < cells.x; ++i) {
          double v = diagonal[flat(cells, i, j, k)] * x.unchecked({i, j, k}, 0U);
          v -= fx[flat(xe, i, j, k)] * neighbour(x, i, j, k, 0, -1);
          v -= fx[flat(xe, i + 1, j, k)] * neighbour(x, i, j, k, 0, 1);
          v -= fy[flat(ye, i, j, k)] * neighbour(x, i, j, k, 1, -1);
          v -= fy[flat(ye, i, j + 1, k)] * neighbour(x, i, j, k, 1, 1);
          v -= fz[flat(ze, i, j, k)] * neighbour(x, i, j, k, 2, -1);
          v -= fz[flat(ze, i, j, k + 1)] * neighbour(x, i, j, k, 2, 1);
          output.unchecked({i, j, k}, 0U) = v;
        }
    if (active == nullptr) return {};
    // Decoration: identity on solid rows, links cancel the removed face.
    for (int k = 0; k < cells.z; ++k)
      for (int j = 0; j < cells.y; ++j)
        for (int i = 0; i < cells.x; ++i)
          if (active[flat(cells, i, j, k)] == 0U)
            output.unchecked({i, j, k}, 0U) = x.unchecked({i, j, k}, 0U);
    for (int k = 0; k < cells.z; ++k)
      for (int j = 0; j < cells.y; ++j)
        for (int i = 0; i < cells.x; ++i) {
          if (active[flat(cells, i, j, k)] == 0U) continue;
          const double xf = x.unchecked({i, j, k}, 0U);
          double add = 0.0;
          const auto link = [&](int a, int b, int c, double coefficient) {
            if (a < 0 || b < 0 || c < 0 || a >= cells.x || b >= cells.y ||
                c >= cells.z)
              return;
            if (active[flat(cells, a, b, c)] != 0U) return;
            add = coefficient * (x.unchecked({a, b, c}, 0U) - xf);
            output.unchecked({i, j, k}, 0U) += add;
          };
          link(i - 1, j, k, fx[flat(xe, i, j, k)]);
          link(i + 1, j, k, fx[flat(xe, i + 1, j, k)]);
          link(i, j - 1, k, fy[flat(ye, i, j, k)]);
          link(i, j + 1, k, fy[flat(ye, i, j + 1, k)]);
          link(i, j, k - 1, fz[flat(ze, i, j, k)]);
          link(i, j, k + 1, fz[flat(ze, i, j, k + 1)]);
        }
    return {};
  }
};

// Forwards to the MG plan but certifies it as the fixed SPD preconditioner
// solve_pcg demands (src/solver_krylov.cpp:962-966).  The reference itself
// has no MG-PCG route; the MG-preconditioned CG solves of this library are
// compared against this adapter.
class PcgAdapter final : public LinearPreconditioner {
 public:
  NativeCartesianMgPlan* plan{};
  LinearPreconditionerCertificate certificate() const noexcept override {
    LinearPreconditionerCertificate c = plan->certificate();
    c.preconditioner_class = LinearPreconditionerClass::fixed_spd;
    c.apply_lifecycle = LinearPreconditionerApplyLifecycle::per_call_checked;
    return c;
  }
  Status apply(ConstFieldView input, FieldView output,
               std::uint32_t iteration) noexcept override {
    return plan->apply(input, output, iteration);
  }
};

struct Session {
  Int3 cells{};
  CartesianGeometryPlan geometry;
  MeshPatch patch{};
  std::vector<double> diagonal;
  OwnedField diagonal_field;
  OwnedFace x_faces, y_faces, z_faces;
  std::vector<std::uint8_t> active_cells, active_x, active_y, active_z;
  bool has_activity{};
  HarnessOperator op;
  ReductionEngine reductions;
  HaloEngine halo;
  std::vector<HaloEngine> coarse_halos;
  std::vector<HaloEngine*> coarse_halo_pointers;
  MgWorkspaceRequirements mg_requirements{};
  OwnedField mg_vectors;
  MgWorkspace mg_workspace;
  NativeCartesianMgPlan plan;
  PcgAdapter adapter;
  LinearWorkspaceRequirements requirements{};
  OwnedField krylov_vectors;
  OwnedField krylov_scalars;
  SolverWorkspace workspace;
  LinearIdentity identity{};
  LinearAlgorithm algorithm{LinearAlgorithm::pcg};
  std::uint32_t restart{};
  double setup_seconds{};
  // Cold-path preconditioners on the decorated operator's rows.
  int preconditioner{};  // 0 MG plan, 1 ColdPressureIccg, 2 ColdPressureDilu
  std::vector<detail::ColdPressureRow> cold_rows;
  std::unique_ptr<detail::ColdPressureIccg> iccg;
  std::unique_ptr<detail::ColdPressureDilu> dilu;
};

int code_of(Status s) {
  return static_cast<int>(s.code) * 100000 + static_cast<int>(s.detail % 100000U);
}

}  // namespace

extern "C" {

// options: [algorithm(0 pcg,1 fgmres,2 bicgstab), restart, smoother(0 red-black,
//           1 chebyshev), cycle(0 V,1 F), pre, post, coarse_sweeps,
//           scaling(0 residual-minimising, 1 unit_linear), max_levels,
//           minimum_coarse_extent, preconditioner(0 MG plan, 1 ICCG, 2 DILU),
//           null_space(0 none, 1 constant)]
// reals:   [chebyshev_lower_spectrum_fraction, anisotropy_threshold,
//           diagonal_shortcut_maximum_ratio]
// Returns 0 on success, otherwise status code * 100000 + detail.
int hfref_create(int nx, int ny, int nz, const double* x_faces,
                 const double* y_faces, const double* z_faces,
                 const int* boundary_kinds, const double* diagonal,
                 const double* face_x, const double* face_y,
                 const double* face_z, const unsigned char* cell_active,
                 const int* options, const double* reals, void** out) {
  *out = nullptr;
  int initialized = 0;
  MPI_Initialized(&initialized);
  if (!initialized) MPI_Init(nullptr, nullptr);
  const auto begin = std::chrono::steady_clock::now();
  auto session = std::make_unique<Session>();
  Session& s = *session;
  s.cells = {nx, ny, nz};
  CartesianMeshSpec mesh;
  mesh.kind = GeometryKind::runtime_axes_v1;
  // The runtime-axes route requires a non-empty provenance label.
  mesh.axes_file = "synthetic-runtime-axes";
  mesh.runtime_faces[0].assign(x_faces, x_faces + nx + 1);
  mesh.runtime_faces[1].assign(y_faces, y_faces + ny + 1);
  mesh.runtime_faces[2].assign(z_faces, z_faces + nz + 1);
  mesh.lower = {x_faces[0], y_faces[0], z_faces[0]};
  mesh.upper = {x_faces[nx], y_faces[ny], z_faces[nz]};
  mesh.has_exact_cells = true;
  mesh.exact_cells = s.cells;
  mesh.minimum_spacing = {1.0e-12, 1.0e-12, 1.0e-12};
  mesh.max_growth_ratio = 1.0e9;
  mesh.limits = {UINT64_C(1) << 40, UINT64_C(1) << 50};
  Status st = CartesianGeometryCompiler::compile(
      MPI_COMM_SELF, mesh, GeometryBudget{}, s.geometry, s.patch);
  if (!st) return code_of(st);

  const std::size_t n = static_cast<std::size_t>(nx) * ny * nz;
  s.diagonal_field = make_field(1U, s.cells, 0U, 1U, 110U, 210U);
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i)
        s.diagonal_field.view.unchecked({i, j, k}, 0U) =
            diagonal[flat(s.cells, i, j, k)];
  s.x_faces = make_face(CartesianAxis::x, s.cells, face_x, 120U);
  s.y_faces = make_face(CartesianAxis::y, s.cells, face_y, 121U);
  s.z_faces = make_face(CartesianAxis::z, s.cells, face_z, 122U);

  MgBoundarySet boundaries{boundary_kind(boundary_kinds[0]),
                           boundary_kind(boundary_kinds[1]),
                           boundary_kind(boundary_kinds[2]),
                           boundary_kind(boundary_kinds[3]),
                           boundary_kind(boundary_kinds[4]),
                           boundary_kind(boundary_kinds[5])};
  s.has_activity = cell_active != nullptr;
  if (s.has_activity) {
    s.active_cells.assign(cell_active, cell_active + n);
    const Int3 xe{nx + 1, ny, nz}, ye{nx, ny + 1, nz}, ze{nx, ny, nz + 1};
    s.active_x.assign(static_cast<std::size_t>(nx + 1) * ny * nz, 0U);
    s.active_y.assign(static_cast<std::size_t>(nx) * (ny + 1) * nz, 0U);
    s.active_z.assign(static_cast<std::size_t>(nx) * ny * (nz + 1), 0U);
    const auto cell_on = [&](int i, int j, int k) {
      return s.active_cells[flat(s.cells, i, j, k)] != 0U;
    };
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i <= nx; ++i) {
          const bool left = i > 0 ? cell_on(i - 1, j, k) : cell_on(i, j, k);
          const bool right = i < nx ? cell_on(i, j, k) : cell_on(i - 1, j, k);
          s.active_x[flat(xe, i, j, k)] = left && right ? 1U : 0U;
        }
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j <= ny; ++j)
        for (int i = 0; i < nx; ++i) {
          const bool low = j > 0 ? cell_on(i, j - 1, k) : cell_on(i, j, k);
          const bool high = j < ny ? cell_on(i, j, k) : cell_on(i, j - 1, k);
          s.active_y[flat(ye, i, j, k)] = low && high ? 1U : 0U;
        }
    for (int k = 0; k <= nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          const bool low = k > 0 ? cell_on(i, j, k - 1) : cell_on(i, j, k);
          const bool high = k < nz ? cell_on(i, j, k) : cell_on(i, j, k - 1);
          s.active_z[flat(ze, i, j, k)] = low && high ? 1U : 0U;
        }
  }

  s.algorithm = options[0] == 1 ? LinearAlgorithm::fgmres
                 : options[0] == 2 ? LinearAlgorithm::bicgstab
                                   : LinearAlgorithm::pcg;
  s.preconditioner = options[10];
  s.restart = s.algorithm == LinearAlgorithm::fgmres
                  ? static_cast<std::uint32_t>(options[1])
                  : 0U;
  st = make_linear_workspace_requirements(s.algorithm, s.cells, 1U, s.restart,
                                          ReductionMode::mpi_allreduce, 701U,
                                          s.requirements);
  if (!st) return code_of(st);
  s.krylov_vectors = make_field(30U, s.cells, 1U, s.requirements.vector_slots,
                                100U, 200U);
  s.krylov_scalars = make_field(
      31U, {static_cast<std::int32_t>(s.requirements.scalar_doubles), 1, 1},
      0U, 1U, 100U, 200U);
  st = SolverWorkspace::bind(s.requirements, s.krylov_vectors.view,
                             s.krylov_scalars.view, s.workspace);
  if (!st) return code_of(st);
  s.identity = {11U, 12U, 13U, s.workspace.fingerprint(), 15U};

  NativeCartesianMgSpec spec;
  spec.communicator = MPI_COMM_SELF;
  spec.geometry = &s.geometry;
  spec.patch = s.patch;
  spec.boundaries = boundaries;
  spec.null_space = options[11] == 1 ? MgNullSpace::constant : MgNullSpace::none;
  spec.operator_class = MgOperatorClass::symmetric_diagonally_dominant_m_matrix;
  spec.policy.point_smoother = options[2] == 1
                                   ? MgPointSmootherKind::chebyshev_jacobi
                                   : MgPointSmootherKind::red_black;
  spec.policy.cycle = options[3] == 1 ? MgCycleKind::f_cycle : MgCycleKind::v_cycle;
  spec.policy.pre_sweeps = static_cast<std::uint8_t>(options[4]);
  spec.policy.post_sweeps = static_cast<std::uint8_t>(options[5]);
  spec.policy.coarse_sweeps = static_cast<std::uint16_t>(options[6]);
  spec.policy.maximum_levels = static_cast<std::uint8_t>(options[8]);
  spec.policy.minimum_coarse_extent = static_cast<std::uint8_t>(options[9]);
  spec.policy.chebyshev_lower_spectrum_fraction = reals[0];
  spec.policy.anisotropy_threshold = reals[1];
  spec.policy.diagonal_shortcut_maximum_ratio = reals[2];
  spec.correction_scaling = options[7] == 1 ? MgCorrectionScaling::unit_linear
                                            : MgCorrectionScaling::residual_minimizing;
  spec.identity = s.identity;
  spec.coefficients = {21U, 22U, 0.0};
  if (s.has_activity) {
    spec.activity.cells = {s.active_cells.data(), s.active_cells.size()};
    spec.activity.x_faces = {s.active_x.data(), s.active_x.size()};
    spec.activity.y_faces = {s.active_y.data(), s.active_y.size()};
    spec.activity.z_faces = {s.active_z.data(), s.active_z.size()};
    spec.activity.local_fingerprint = 91U;
    spec.activity.collective_fingerprint = 92U;
  }
  st = make_mg_workspace_requirements(MPI_COMM_SELF, s.geometry, s.patch,
                                      spec.policy, 702U, s.mg_requirements);
  if (!st) return code_of(st);
  s.mg_vectors = make_field(32U, s.mg_requirements.arena_shape, 0U, 1U, 101U,
                            201U);
  st = MgWorkspace::bind(s.mg_requirements, s.mg_vectors.view, s.mg_workspace);
  if (!st) return code_of(st);
  const std::array<HaloFieldSpec, 1U> halo_fields{{{32U, 1U, 1U}}};
  const HaloTopology topology{boundaries.x_min == MgBoundaryKind::periodic,
                              boundaries.y_min == MgBoundaryKind::periodic,
                              boundaries.z_min == MgBoundaryKind::periodic};
  st = ReductionEngine::compile(MPI_COMM_SELF, ReductionMode::mpi_allreduce,
                                std::max<std::size_t>(
                                    s.requirements.reduction_capacity, 8U),
                                s.reductions);
  if (!st) return code_of(st);
  st = s.halo.reserve(MPI_COMM_SELF, s.mg_requirements.levels[0U].patch,
                      {halo_fields.data(), halo_fields.size()}, topology);
  if (!st) return code_of(st);
  s.coarse_halos = std::vector<HaloEngine>(s.mg_requirements.level_count - 1U);
  s.coarse_halo_pointers.resize(s.coarse_halos.size());
  for (std::size_t level = 1U; level < s.mg_requirements.level_count; ++level) {
    st = s.coarse_halos[level - 1U].reserve(
        MPI_COMM_SELF, s.mg_requirements.levels[level].patch,
        {halo_fields.data(), halo_fields.size()}, topology);
    if (!st) return code_of(st);
    s.coarse_halo_pointers[level - 1U] = &s.coarse_halos[level - 1U];
  }
  st = NativeCartesianMgPlan::compile(
      spec,
      MgRuntimeServices{&s.halo, &s.reductions, &s.mg_workspace,
                        {s.coarse_halo_pointers.data(),
                         s.coarse_halo_pointers.size()}},
      MgCoefficientViews{as_const(s.diagonal_field.view), s.x_faces.view,
                         s.y_faces.view, s.z_faces.view},
      s.plan);
  if (!st) return code_of(st);
  s.adapter.plan = &s.plan;

  s.op.cells = s.cells;
  for (int f = 0; f < 6; ++f) s.op.bc[f] = boundary_kinds[f];
  s.op.diagonal = diagonal;
  s.diagonal.assign(diagonal, diagonal + n);
  s.op.diagonal = s.diagonal.data();
  s.op.fx = s.x_faces.storage.data();
  s.op.fy = s.y_faces.storage.data();
  s.op.fz = s.z_faces.storage.data();
  s.op.active = s.has_activity ? s.active_cells.data() : nullptr;
  s.op.identity = s.identity;
  if (s.preconditioner != 0) {
    // Rows of the decorated operator: identity rows on solid cells; a link
    // to a solid cell or a Neumann boundary face moves its coefficient out
    // of the row (the neighbour reads the cell itself); Dirichlet boundary
    // neighbours read zero.  neighbour[2a] / [2a+1] couple to the low /
    // high neighbour along axis a with the positive face coefficient.
    s.cold_rows.assign(n, detail::ColdPressureRow{});
    const Int3 xe{nx + 1, ny, nz}, ye{nx, ny + 1, nz}, ze{nx, ny, nz + 1};
    const auto on = [&](int i, int j, int k) {
      return !s.has_activity || s.active_cells[flat(s.cells, i, j, k)] != 0U;
    };
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          detail::ColdPressureRow& row = s.cold_rows[flat(s.cells, i, j, k)];
          if (!on(i, j, k)) {
            row.diagonal = 1.0;
            continue;
          }
          row.diagonal = s.diagonal[flat(s.cells, i, j, k)];
          const int c[3]{i, j, k};
          const int e[3]{nx, ny, nz};
          const double face[6]{s.op.fx[flat(xe, i, j, k)], s.op.fx[flat(xe, i + 1, j, k)],
                               s.op.fy[flat(ye, i, j, k)], s.op.fy[flat(ye, i, j + 1, k)],
                               s.op.fz[flat(ze, i, j, k)], s.op.fz[flat(ze, i, j, k + 1)]};
          for (int f = 0; f < 6; ++f) {
            const int a = f / 2;
            int nb[3]{c[0], c[1], c[2]};
            nb[a] += (f % 2) ? 1 : -1;
            if (nb[a] < 0 || nb[a] >= e[a]) {
              if (boundary_kinds[f] == 1) row.diagonal -= face[f];
              continue;
            }
            if (!on(nb[0], nb[1], nb[2])) {
              row.diagonal -= face[f];
              continue;
            }
            row.neighbour[f] = face[f];
          }
        }
    if (s.preconditioner == 1) {
      s.iccg = std::make_unique<detail::ColdPressureIccg>(s.cold_rows, s.cells, s.identity);
      st = s.iccg->prepare();
    } else {
      s.dilu = std::make_unique<detail::ColdPressureDilu>(s.cold_rows, s.cells, s.identity);
      st = s.dilu->prepare();
    }
    if (!st) return code_of(st);
  }
  s.setup_seconds = std::chrono::duration<double>(
                        std::chrono::steady_clock::now() - begin)
                        .count();
  *out = session.release();
  return 0;
}

void hfref_destroy(void* handle) { delete static_cast<Session*>(handle); }

int hfref_levels(void* handle, int* shapes, int capacity) {
  Session& s = *static_cast<Session*>(handle);
  const int count = static_cast<int>(s.plan.level_count());
  for (int l = 0; l < count && l < capacity; ++l) {
    MgLevelView view{};
    s.plan.level(static_cast<std::size_t>(l), view);
    shapes[4 * l + 0] = view.local_shape.x;
    shapes[4 * l + 1] = view.local_shape.y;
    shapes[4 * l + 2] = view.local_shape.z;
    shapes[4 * l + 3] = view.line_axis_mask;
  }
  return count;
}

// y = A x with the decorated operator (dense x-fastest arrays, no ghosts).
int hfref_apply_operator(void* handle, const double* x, double* y) {
  Session& s = *static_cast<Session*>(handle);
  OwnedField in = make_field(40U, s.cells, 1U, 1U, 300U, 400U);
  OwnedField out = make_field(41U, s.cells, 0U, 1U, 301U, 401U);
  for (int k = 0; k < s.cells.z; ++k)
    for (int j = 0; j < s.cells.y; ++j)
      for (int i = 0; i < s.cells.x; ++i)
        in.view.unchecked({i, j, k}, 0U) = x[flat(s.cells, i, j, k)];
  const Status st = s.op.apply(in.view, out.view);
  for (int k = 0; k < s.cells.z; ++k)
    for (int j = 0; j < s.cells.y; ++j)
      for (int i = 0; i < s.cells.x; ++i)
        y[flat(s.cells, i, j, k)] = out.view.unchecked({i, j, k}, 0U);
  return st ? 0 : code_of(st);
}

// z = M r, one application of the reference MG preconditioner.
int hfref_apply_mg(void* handle, const double* r, double* z) {
  Session& s = *static_cast<Session*>(handle);
  OwnedField in = make_field(42U, s.cells, 0U, 1U, 302U, 402U);
  OwnedField out = make_field(43U, s.cells, 0U, 1U, 303U, 403U);
  for (int k = 0; k < s.cells.z; ++k)
    for (int j = 0; j < s.cells.y; ++j)
      for (int i = 0; i < s.cells.x; ++i)
        in.view.unchecked({i, j, k}, 0U) = r[flat(s.cells, i, j, k)];
  const Status st = s.plan.apply(as_const(in.view), out.view, 0U);
  for (int k = 0; k < s.cells.z; ++k)
    for (int j = 0; j < s.cells.y; ++j)
      for (int i = 0; i < s.cells.x; ++i)
        z[flat(s.cells, i, j, k)] = out.view.unchecked({i, j, k}, 0U);
  return st ? 0 : code_of(st);
}

// One application of the cold-path preconditioner (ICCG or DILU).
int hfref_apply_cold(void* handle, const double* r, double* z) {
  Session& s = *static_cast<Session*>(handle);
  if (s.preconditioner == 0) return 1;
  OwnedField in = make_field(46U, s.cells, 0U, 1U, 306U, 406U);
  OwnedField out = make_field(47U, s.cells, 0U, 1U, 307U, 407U);
  for (int k = 0; k < s.cells.z; ++k)
    for (int j = 0; j < s.cells.y; ++j)
      for (int i = 0; i < s.cells.x; ++i)
        in.view.unchecked({i, j, k}, 0U) = r[flat(s.cells, i, j, k)];
  LinearPreconditioner* pc = s.preconditioner == 1
                                 ? static_cast<LinearPreconditioner*>(s.iccg.get())
                                 : static_cast<LinearPreconditioner*>(s.dilu.get());
  const Status st = pc->apply(as_const(in.view), out.view, 0U);
  for (int k = 0; k < s.cells.z; ++k)
    for (int j = 0; j < s.cells.y; ++j)
      for (int i = 0; i < s.cells.x; ++i)
        z[flat(s.cells, i, j, k)] = out.view.unchecked({i, j, k}, 0U);
  return st ? 0 : code_of(st);
}

// Runs solve_pcg (adapter-certified MG, or ICCG), solve_bicgstab (DILU) or
// solve_fgmres (MG as given).
// recycle (FGMRES): 0 none (clears any recycle session), 1 begin a capture
// session (corrector 1: SolverWorkspace::recycle_begin_capture), 2 project
// the captured corrections (corrector 2: recycle_begin_projection), 3 the
// zero-seed initial-guess guard only (recycle_begin_initial_guess_guard),
// as PressureVelocityCoupler selects them (src/solver_piso.cpp:10410-10433),
// through the reference's test-access entry points.
// outputs: [iterations, initial_true, final_true, termination, rhs_norm,
//           limit, operator_applies, preconditioner_applies, seconds,
//           setup_seconds, recycle_offered, recycle_retained,
//           recycle_accepted, recycle_projected_residual,
//           recycle_cycle_corrections]
int hfref_solve(void* handle, const double* rhs, double* solution,
                double relative_tolerance, double absolute_tolerance,
                int maximum_iterations, int true_residual_interval,
                int recycle, double* outputs) {
  Session& s = *static_cast<Session*>(handle);
  if (s.algorithm == LinearAlgorithm::fgmres) {
    Status rs{};
    if (recycle == 0) {
      s.workspace.recycle_clear_for_test();
    } else if (recycle == 1) {
      s.workspace.recycle_clear_for_test();
      rs = s.workspace.recycle_begin_capture_for_test(s.cells, s.identity.fingerprint);
    } else if (recycle == 2) {
      rs = s.workspace.recycle_begin_projection_for_test(s.cells, s.identity.fingerprint);
    } else if (recycle == 3) {
      s.workspace.recycle_clear_for_test();
      rs = s.workspace.recycle_begin_initial_guess_guard_for_test(s.cells,
                                                                  s.identity.fingerprint);
    }
    if (!rs) return code_of(rs);
  }
  OwnedField b = make_field(44U, s.cells, 0U, 1U, 304U, 404U);
  OwnedField x = make_field(45U, s.cells, 1U, 1U, 305U, 405U);
  for (int k = 0; k < s.cells.z; ++k)
    for (int j = 0; j < s.cells.y; ++j)
      for (int i = 0; i < s.cells.x; ++i) {
        b.view.unchecked({i, j, k}, 0U) = rhs[flat(s.cells, i, j, k)];
        x.view.unchecked({i, j, k}, 0U) = solution[flat(s.cells, i, j, k)];
      }
  LinearSolveInvocation invocation;
  invocation.rhs = as_const(b.view);
  invocation.solution = x.view;
  invocation.expected_identity = s.identity;
  invocation.control.absolute_tolerance = absolute_tolerance;
  invocation.control.relative_tolerance = relative_tolerance;
  invocation.control.maximum_iterations =
      static_cast<std::uint32_t>(maximum_iterations);
  invocation.control.true_residual_interval =
      static_cast<std::uint32_t>(true_residual_interval);
  invocation.control.restart = s.restart;
  const auto begin = std::chrono::steady_clock::now();
  LinearPreconditioner* pc =
      s.preconditioner == 1 ? static_cast<LinearPreconditioner*>(s.iccg.get())
      : s.preconditioner == 2 ? static_cast<LinearPreconditioner*>(s.dilu.get())
      : s.algorithm == LinearAlgorithm::pcg ? static_cast<LinearPreconditioner*>(&s.adapter)
                                            : static_cast<LinearPreconditioner*>(&s.plan);
  const LinearSolveResult result =
      s.algorithm == LinearAlgorithm::pcg
          ? solve_pcg(s.op, *pc, invocation, s.workspace, s.reductions)
      : s.algorithm == LinearAlgorithm::bicgstab
          ? solve_bicgstab(s.op, *pc, invocation, s.workspace, s.reductions)
          : solve_fgmres(s.op, *pc, invocation, s.workspace, s.reductions);
  const double seconds =
      std::chrono::duration<double>(std::chrono::steady_clock::now() - begin)
          .count();
  for (int k = 0; k < s.cells.z; ++k)
    for (int j = 0; j < s.cells.y; ++j)
      for (int i = 0; i < s.cells.x; ++i)
        solution[flat(s.cells, i, j, k)] = x.view.unchecked({i, j, k}, 0U);
  outputs[0] = result.iterations;
  outputs[1] = result.initial_true_residual;
  outputs[2] = result.final_true_residual;
  outputs[3] = static_cast<double>(result.termination);
  outputs[4] = result.rhs_norm;
  outputs[5] = result.true_residual_limit;
  outputs[6] = static_cast<double>(result.operator_applies);
  outputs[7] = static_cast<double>(result.preconditioner_applies);
  outputs[8] = seconds;
  outputs[9] = s.setup_seconds;
  outputs[10] = static_cast<double>(result.recycle_offered_directions);
  outputs[11] = static_cast<double>(result.recycle_retained_directions);
  outputs[12] = result.recycle_projection_accepted ? 1.0 : 0.0;
  outputs[13] = result.recycle_projected_true_residual;
  outputs[14] = static_cast<double>(result.recycle_cycle_corrections);
  return result.status ? 0 : code_of(result.status);
}

}  // extern "C"
