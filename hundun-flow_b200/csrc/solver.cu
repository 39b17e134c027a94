// Host orchestration of the B200 pressure solve.  See solver.hpp.
#include "solver.hpp"

#include <algorithm>
#include <cstdint>
#include <chrono>
#include <cmath>
#include <cstring>
#include <cstdlib>
#include <limits>
#include <type_traits>

namespace hfps {
namespace {

constexpr int kMaxLevels = 32;
constexpr uint32_t kDetailPlan = 9101U;
constexpr uint32_t kDetailCuda = 9102U;
constexpr uint32_t kDetailNumeric = 9103U;
constexpr uint32_t kDetailBreakdown = 9104U;
// Whether the small levels run as one persistent launch when HFPS_TAIL is unset.
constexpr bool kTailDefault = false;

size_t align_up(size_t v) { return (v + 255) & ~static_cast<size_t>(255); }

struct Shape {
  int n[3];
  int coarsen_mask;
  int line_mask;
};

// strategy_mask (src/solver_mg_workspace.cpp:113-143).
int strategy_mask(const std::vector<double> (&faces)[3], double threshold,
                  int& line_mask) {
  double mn[3], mx[3], rep[3];
  for (int a = 0; a < 3; ++a) {
    mn[a] = std::numeric_limits<double>::infinity();
    mx[a] = 0.0;
    rep[a] = 0.0;
    const int n = static_cast<int>(faces[a].size()) - 1;
    for (int c = 0; c < n; ++c) {
      const double w = faces[a][c + 1] - faces[a][c];
      mn[a] = std::min(mn[a], w);
      mx[a] = std::max(mx[a], w);
      rep[a] += w;
    }
    rep[a] /= static_cast<double>(n);
  }
  const double largest = std::max({rep[0], rep[1], rep[2]});
  line_mask = 0;
  for (int a = 0; a < 3; ++a) {
    const bool internal = mn[a] > 0.0 && mx[a] / mn[a] >= threshold;
    const bool cross = rep[a] > 0.0 && largest / rep[a] >= threshold;
    if (internal || cross) line_mask |= 1 << a;
  }
  const int all = 7;
  if ((line_mask & (line_mask - 1)) != 0) return all;
  const int candidate = all & ~line_mask;
  return candidate == 0 ? all : candidate;
}

// Level shapes (make_mg_workspace_requirements, src/solver_mg_workspace.cpp:
// 368-409): ceil-half every preferred axis whose extent exceeds the minimum
// coarse extent until no axis can coarsen.
std::vector<Shape> level_shapes(const std::vector<double> (&faces)[3],
                                const hfps_policy& policy) {
  int line_mask = 0;
  const int preferred = strategy_mask(faces, policy.anisotropy_threshold, line_mask);
  int g[3] = {static_cast<int>(faces[0].size()) - 1,
              static_cast<int>(faces[1].size()) - 1,
              static_cast<int>(faces[2].size()) - 1};
  std::vector<Shape> shapes;
  for (int l = 0; l < policy.maximum_levels; ++l) {
    Shape s{{g[0], g[1], g[2]}, 0, line_mask};
    int next[3] = {g[0], g[1], g[2]};
    for (int a = 0; a < 3; ++a) {
      if ((preferred & (1 << a)) && g[a] > policy.minimum_coarse_extent) {
        s.coarsen_mask |= 1 << a;
        next[a] = (g[a] + 1) / 2;
      }
    }
    shapes.push_back(s);
    if (s.coarsen_mask == 0 || static_cast<int>(shapes.size()) == policy.maximum_levels)
      break;
    std::copy(next, next + 3, g);
  }
  return shapes;
}

bool valid_policy(const hfps_policy& p) {
  return std::isfinite(p.anisotropy_threshold) && p.anisotropy_threshold > 1.0 &&
         p.pre_sweeps > 0 && p.pre_sweeps <= 255 && p.post_sweeps > 0 &&
         p.post_sweeps <= 255 && p.maximum_levels >= 2 &&
         p.maximum_levels <= kMaxLevels && p.coarse_sweeps > 0 &&
         p.coarse_sweeps <= 65535 && p.minimum_coarse_extent >= 2 &&
         (p.point_smoother == 0 || p.point_smoother == 1) &&
         (p.cycle == 0 || p.cycle == 1) &&
         std::isfinite(p.chebyshev_lower_spectrum_fraction) &&
         p.chebyshev_lower_spectrum_fraction > 0.0 &&
         p.chebyshev_lower_spectrum_fraction < 1.0 &&
         (p.preconditioner == HFPS_PRECONDITIONER_MG ||
          p.preconditioner == HFPS_PRECONDITIONER_IC0) &&
         std::isfinite(p.diagonal_shortcut_maximum_ratio) &&
         p.diagonal_shortcut_maximum_ratio >= 0.0 &&
         p.diagonal_shortcut_maximum_ratio < 1.0 &&
         (p.unit_linear == 0 || p.unit_linear == 1) &&
         (p.null_space == HFPS_NULL_SPACE_NONE || p.null_space == HFPS_NULL_SPACE_CONSTANT);
}

}  // namespace

Status Solver::fail(int code, uint32_t detail, const std::string& what) {
  error_ = what;
  return Status{code, detail};
}

Status Solver::check(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return {};
  error_ = std::string(what) + ": " + cudaGetErrorString(e);
  return Status{e == cudaErrorMemoryAllocation ? HFPS_ALLOCATION_FAILURE
                                                : HFPS_INVALID_PLAN,
                kDetailCuda};
}

Solver::~Solver() {
  if (stream_ != nullptr) cudaStreamSynchronize(stream_);
  clear_mg_graphs();
  if (dic_graph_ != nullptr) cudaGraphExecDestroy(dic_graph_);
  if (h_scalars_ != nullptr) cudaFreeHost(h_scalars_);
  if (scalars_ready_ != nullptr) cudaEventDestroy(scalars_ready_);
  if (arena_ != nullptr) cudaFree(arena_);
  if (fg_storage_ != nullptr) cudaFree(fg_storage_);
  if (rc_storage_ != nullptr) cudaFree(rc_storage_);
  if (own_stream_ && stream_ != nullptr) cudaStreamDestroy(stream_);
}

Status Solver::create(const hfps_geometry& g, const hfps_policy& policy,
                      cudaStream_t stream, Solver** out, std::string& error) {
  *out = nullptr;
  if (g.nx <= 0 || g.ny <= 0 || g.nz <= 0 || g.x_faces == nullptr ||
      g.y_faces == nullptr || g.z_faces == nullptr || !valid_policy(policy)) {
    error = "invalid geometry or policy";
    return Status{HFPS_INVALID_PLAN, kDetailPlan};
  }
  const long long faces =
      static_cast<long long>(g.nx + 1) * g.ny * g.nz +
      static_cast<long long>(g.nx) * (g.ny + 1) * g.nz +
      static_cast<long long>(g.nx) * g.ny * (g.nz + 1);
  if (faces >= std::numeric_limits<int>::max()) {
    error = "grid too large for 32-bit indexing";
    return Status{HFPS_INVALID_PLAN, kDetailPlan};
  }
  unsigned neumann = 0;
  for (int f = 0; f < 6; ++f) {
    if (g.boundary[f] == HFPS_NEUMANN) neumann |= 1u << f;
    else if (g.boundary[f] != HFPS_DIRICHLET) {
      error = "periodic boundaries are not supported";
      return Status{HFPS_INVALID_PLAN, kDetailPlan};
    }
  }
  Solver* s = new Solver();
  s->nx_ = g.nx;
  s->ny_ = g.ny;
  s->nz_ = g.nz;
  s->neumann_ = neumann;
  s->policy_ = policy;
  const double* src[3] = {g.x_faces, g.y_faces, g.z_faces};
  const int n[3] = {g.nx, g.ny, g.nz};
  for (int a = 0; a < 3; ++a) {
    s->faces_[a].assign(src[a], src[a] + n[a] + 1);
    for (int c = 0; c < n[a]; ++c) {
      if (!(s->faces_[a][c + 1] > s->faces_[a][c])) {
        delete s;
        error = "face coordinates must increase";
        return Status{HFPS_INVALID_PLAN, kDetailPlan};
      }
    }
  }
  const size_t cells = static_cast<size_t>(g.nx) * g.ny * g.nz;
  if (g.cell_active != nullptr) {
    s->has_active_ = true;
    s->active_host_.assign(g.cell_active, g.cell_active + cells);
    for (uint8_t v : s->active_host_) {
      if (v > 1) {
        delete s;
        error = "cell activity must be 0 or 1";
        return Status{HFPS_INVALID_PLAN, kDetailPlan};
      }
    }
  }
  if (stream == nullptr) {
    // A blocking stream: work the caller queued on the legacy default stream
    // (device inputs it produced there, a zero-filled initial guess) is
    // ordered before the solver's copies, and the caller's later work there
    // after them.  A non-blocking stream would race with both.
    Status st = s->check(cudaStreamCreateWithFlags(&s->stream_, cudaStreamDefault),
                         "stream create");
    if (!st) {
      error = s->error_;
      delete s;
      return st;
    }
    s->own_stream_ = true;
  } else {
    s->stream_ = stream;
  }
  Status st = s->allocate();
  if (!st) {
    error = s->error_;
    delete s;
    return st;
  }
  *out = s;
  return {};
}

Status Solver::allocate() {
  const std::vector<Shape> shapes = level_shapes(faces_, policy_);
  if (shapes.size() < 2) return fail(HFPS_INVALID_PLAN, kDetailPlan, "fewer than two levels");
  for (const Shape& s : shapes)
    for (int a = 0; a < 3; ++a)
      if ((s.line_mask & (1 << a)) && line_kind(s.n[0], s.n[1], s.n[2], a) == kLineNone)
        return fail(HFPS_INVALID_PLAN, kDetailPlan, "line relaxation: line longer than 2048 cells");
  const int levels = static_cast<int>(shapes.size());
  // Split rows for the MG x and b of every non-coarsest level that relaxes
  // y- or z-lines with the chunked scan: a colour pass then reads and writes
  // whole halves of rows instead of every other cell (HFPS_SPLIT_ROWS=0 keeps
  // the natural order).
  std::vector<int> split(levels, 0);
  {
    const char* env = std::getenv("HFPS_SPLIT_ROWS");
    const bool on = !(env != nullptr && env[0] == '0');
    for (int l = 0; l + 1 < levels; ++l) {
      const Shape& sl = shapes[l];
      const int axis = sl.line_mask == 2 ? 1 : (sl.line_mask == 4 ? 2 : -1);
      const bool scan = axis > 0 && line_kind(sl.n[0], sl.n[1], sl.n[2], axis) == kLineScan;
      if (scan && on) split[l] = (sl.n[0] + 1) / 2;
      if (l == 0) first_sweep_zero_ = scan && policy_.pre_sweeps >= 1;
    }
  }
  // Sizes.
  size_t bytes = 0;
  const auto add = [&](size_t b) {
    const size_t offset = bytes;
    bytes += align_up(b);
    return offset;
  };
  struct Offsets {
    size_t d, fx, fy, fz, x, b, r, t, vol, fluid;
    size_t d32, fx32, fy32, fz32, x32, b32, r32, t32;
    size_t lf64[3], lf32[3];
  };
  std::vector<Offsets> off(levels);
  size_t max_faces = 0;
  for (int l = 0; l < levels; ++l) {
    const Shape& s = shapes[l];
    const size_t c = static_cast<size_t>(s.n[0]) * s.n[1] * s.n[2];
    const size_t fx = static_cast<size_t>(s.n[0] + 1) * s.n[1] * s.n[2];
    const size_t fy = static_cast<size_t>(s.n[0]) * (s.n[1] + 1) * s.n[2];
    const size_t fz = static_cast<size_t>(s.n[0]) * s.n[1] * (s.n[2] + 1);
    max_faces = std::max({max_faces, fx, fy, fz});
    Offsets& o = off[l];
    // x and b hold 2 * hx * ny * nz values in split rows.
    const size_t cv = split[l] > 0 ? 2 * static_cast<size_t>(split[l]) * s.n[1] * s.n[2] : c;
    o.d = add(c * 8); o.fx = add(fx * 8); o.fy = add(fy * 8); o.fz = add(fz * 8);
    o.x = add(cv * 8); o.b = add(cv * 8); o.r = add(c * 8); o.t = add(c * 8);
    o.vol = add(c * 8); o.fluid = add(c);
    o.d32 = add(c * 4); o.fx32 = add(fx * 4); o.fy32 = add(fy * 4); o.fz32 = add(fz * 4);
    o.x32 = add(cv * 4); o.b32 = add(cv * 4); o.r32 = add(c * 4); o.t32 = add(c * 4);
    for (int a = 0; a < 3; ++a) {
      o.lf64[a] = o.lf32[a] = SIZE_MAX;
      if (!(s.line_mask & (1 << a))) continue;
      o.lf64[a] = add(line_factor_values<double>(s.n[0], s.n[1], s.n[2], a) * 8);
      o.lf32[a] = add(line_factor_values<float>(s.n[0], s.n[1], s.n[2], a) * 4);
    }
  }
  const size_t cells = static_cast<size_t>(nx_) * ny_ * nz_;
  size_t faces_off[3];
  faces_off[0] = add((nx_ + 1) * 8);
  faces_off[1] = add((ny_ + 1) * 8);
  faces_off[2] = add((nz_ + 1) * 8);
  const size_t active_off = add(cells);
  size_t agg_off[3];
  for (auto& a : agg_off) a = add(max_faces * 8);
  const size_t nfx = static_cast<size_t>(nx_ + 1) * ny_ * nz_;
  const size_t nfy = static_cast<size_t>(nx_) * (ny_ + 1) * nz_;
  const size_t nfz = static_cast<size_t>(nx_) * ny_ * (nz_ + 1);
  size_t user_off[4];
  user_off[0] = add(cells * 8);
  user_off[1] = add(nfx * 8);
  user_off[2] = add(nfy * 8);
  user_off[3] = add(nfz * 8);
  size_t k_off[6];
  for (auto& k : k_off) k = add(cells * 8);
  const size_t scalars_off = add(sizeof(Scalars));
  const size_t partials_off = add(sizeof(double) * kBasisChunk * 148 * 8 + 4096);
  // Dense affine map of the coarsest-level sweeps (one line axis, few cells).
  const Shape& last = shapes.back();
  const int last_cells = last.n[0] * last.n[1] * last.n[2];
  size_t dense_off = SIZE_MAX;
  coarse_axis_ = -1;
  if (last.line_mask != 0 && (last.line_mask & (last.line_mask - 1)) == 0 &&
      last_cells <= kCoarseDenseMaxCells) {
    const int axis = last.line_mask == 1 ? 0 : (last.line_mask == 2 ? 1 : 2);
    if (line_kind(last.n[0], last.n[1], last.n[2], axis) == kLinePcr) {
      coarse_axis_ = axis;
      dense_off = add(2 * static_cast<size_t>(last_cells) * last_cells * 8);
    }
  }
  size_t dic_off[2] = {SIZE_MAX, SIZE_MAX};
  if (policy_.preconditioner == HFPS_PRECONDITIONER_IC0) {
    dic_off[0] = add(cells * 8);
    dic_off[1] = add(cells * 8);
  }
  arena_bytes_ = bytes;
  Status st = check(cudaMalloc(&arena_, arena_bytes_), "device arena");
  if (!st) return st;
  st = check(cudaMemsetAsync(arena_, 0, arena_bytes_, stream_), "arena clear");
  if (!st) return st;
  st = check(cudaMallocHost(&h_scalars_, sizeof(Scalars)), "pinned scalars");
  if (!st) return st;
  std::memset(h_scalars_, 0, sizeof(Scalars));
  const auto at = [&](size_t o) { return arena_ + o; };
  for (int a = 0; a < 3; ++a) {
    d_faces_[a] = reinterpret_cast<double*>(at(faces_off[a]));
    st = check(cudaMemcpyAsync(d_faces_[a], faces_[a].data(),
                               faces_[a].size() * sizeof(double),
                               cudaMemcpyHostToDevice, stream_),
               "faces upload");
    if (!st) return st;
  }
  if (has_active_) {
    d_active_ = reinterpret_cast<uint8_t*>(at(active_off));
    st = check(cudaMemcpyAsync(d_active_, active_host_.data(), cells,
                               cudaMemcpyHostToDevice, stream_),
               "activity upload");
    if (!st) return st;
  }
  for (auto a = 0; a < 3; ++a) agg_[a] = reinterpret_cast<double*>(at(agg_off[a]));
  for (int u = 0; u < 4; ++u) user_[u] = reinterpret_cast<double*>(at(user_off[u]));
  kx_ = reinterpret_cast<double*>(at(k_off[0]));
  kr_ = reinterpret_cast<double*>(at(k_off[1]));
  kz_ = reinterpret_cast<double*>(at(k_off[2]));
  kp_ = reinterpret_cast<double*>(at(k_off[3]));
  kap_ = reinterpret_cast<double*>(at(k_off[4]));
  kb_ = reinterpret_cast<double*>(at(k_off[5]));
  {
    // PCG's r.z formed in the MG exit (HFPS_KRYLOV_FUSION=0 keeps the
    // separate dot kernel).
    const char* env = std::getenv("HFPS_KRYLOV_FUSION");
    krylov_fusion_ = !(env != nullptr && env[0] == '0');
    // PCG queue-ahead of the next MG application (HFPS_QUEUE_AHEAD=0: the
    // host reads each iteration's scalars before queueing more work).
    const char* ahead = std::getenv("HFPS_QUEUE_AHEAD");
    queue_ahead_ = !(ahead != nullptr && ahead[0] == '0');
    // The Krylov operator over 3-D tiles (HFPS_TILED_STENCIL=0: the row
    // kernel; the same rows, another grouping of the p.Ap partials).
    const char* tiled = std::getenv("HFPS_TILED_STENCIL");
    tiled_stencil_ = !(tiled != nullptr && tiled[0] == '0');
  }
  st = check(cudaEventCreateWithFlags(&scalars_ready_, cudaEventDisableTiming), "event");
  if (!st) return st;
  d_scalars_ = reinterpret_cast<Scalars*>(at(scalars_off));
  d_partials_ = reinterpret_cast<double*>(at(partials_off));
  coarse_op_ = dense_off == SIZE_MAX ? nullptr : reinterpret_cast<double*>(at(dense_off));
  if (dic_off[0] != SIZE_MAX) {
    dic_rows_ = reinterpret_cast<double*>(at(dic_off[0]));
    dic_inv_ = reinterpret_cast<double*>(at(dic_off[1]));
  }
  l64_.resize(levels);
  l32_.resize(levels);
  volume_.resize(levels);
  fluid_.resize(levels);
  for (int l = 0; l < levels; ++l) {
    const Shape& s = shapes[l];
    const Offsets& o = off[l];
    DeviceLevel<double>& a = l64_[l];
    DeviceLevel<float>& b = l32_[l];
    a.nx = b.nx = s.n[0];
    a.ny = b.ny = s.n[1];
    a.nz = b.nz = s.n[2];
    a.coarsen_mask = b.coarsen_mask = s.coarsen_mask;
    a.line_mask = b.line_mask = s.line_mask;
    a.split = b.split = split[l];
    // build_levels: Chebyshev only on non-coarsest point levels
    // (src/solver_mg.cpp:1060-1073).
    a.chebyshev = b.chebyshev =
        l + 1 < levels && s.line_mask == 0 && policy_.point_smoother == 1;
    a.diag = reinterpret_cast<double*>(at(o.d));
    a.fx = reinterpret_cast<double*>(at(o.fx));
    a.fy = reinterpret_cast<double*>(at(o.fy));
    a.fz = reinterpret_cast<double*>(at(o.fz));
    a.x = reinterpret_cast<double*>(at(o.x));
    a.b = reinterpret_cast<double*>(at(o.b));
    a.r = reinterpret_cast<double*>(at(o.r));
    a.t = reinterpret_cast<double*>(at(o.t));
    volume_[l] = reinterpret_cast<double*>(at(o.vol));
    fluid_[l] = reinterpret_cast<uint8_t*>(at(o.fluid));
    a.fluid = b.fluid = fluid_[l];
    b.diag = reinterpret_cast<float*>(at(o.d32));
    b.fx = reinterpret_cast<float*>(at(o.fx32));
    b.fy = reinterpret_cast<float*>(at(o.fy32));
    b.fz = reinterpret_cast<float*>(at(o.fz32));
    b.x = reinterpret_cast<float*>(at(o.x32));
    b.b = reinterpret_cast<float*>(at(o.b32));
    b.r = reinterpret_cast<float*>(at(o.r32));
    b.t = reinterpret_cast<float*>(at(o.t32));
    for (int ax = 0; ax < 3; ++ax) {
      if (o.lf64[ax] == SIZE_MAX) continue;
      a.lfac[ax] = reinterpret_cast<double*>(at(o.lf64[ax]));
      b.lfac[ax] = reinterpret_cast<float*>(at(o.lf32[ax]));
    }
  }
  return check(cudaStreamSynchronize(stream_), "allocation");
}

void Solver::level_shape(int level, int* out) const {
  const DeviceLevel<double>& L = l64_[level];
  out[0] = L.nx;
  out[1] = L.ny;
  out[2] = L.nz;
  out[3] = L.line_mask;
}

Status Solver::copy_in(double* dst, const double* src, size_t n, int memory) {
  return check(cudaMemcpyAsync(dst, src, n * sizeof(double),
                               memory == HFPS_DEVICE ? cudaMemcpyDeviceToDevice
                                                     : cudaMemcpyHostToDevice,
                               stream_),
               "copy in");
}

Status Solver::copy_out(double* dst, const double* src, size_t n, int memory) {
  return check(cudaMemcpyAsync(dst, src, n * sizeof(double),
                               memory == HFPS_DEVICE ? cudaMemcpyDeviceToDevice
                                                     : cudaMemcpyDeviceToHost,
                               stream_),
               "copy out");
}

// One channel of aggregate_tensor_channel over the axes the fine level
// coarsens, in x->y->z order (src/solver_mg.cpp:1706-1856).
void Solver::aggregate_channel(int level, int face_axis, const double* src,
                               double* dst) {
  const DeviceLevel<double>& F = l64_[level];
  int e[3] = {F.nx, F.ny, F.nz};
  int g[3] = {F.nx, F.ny, F.nz};
  if (face_axis >= 0) e[face_axis] += 1;
  const double* cur = src;
  int buffer = 0;
  int remaining = 0;
  for (int a = 0; a < 3; ++a)
    if (F.coarsen_mask & (1 << a)) ++remaining;
  for (int axis = 0; axis < 3; ++axis) {
    if (!(F.coarsen_mask & (1 << axis))) continue;
    --remaining;
    int ng[3] = {g[0], g[1], g[2]};
    ng[axis] = (g[axis] + 1) / 2;
    int ne[3] = {ng[0], ng[1], ng[2]};
    if (face_axis >= 0) ne[face_axis] += 1;
    double* out = remaining == 0 ? dst : agg_[buffer];
    launch_aggregate_axis(stream_, cur, e[0], e[1], e[2], out, ne[0], ne[1], ne[2],
                          axis, face_axis, g[axis]);
    cur = out;
    buffer ^= 1;
    std::copy(ng, ng + 3, g);
    std::copy(ne, ne + 3, e);
  }
}

Status Solver::build_hierarchy() {
  for (size_t l = 1; l < l64_.size(); ++l) {
    const DeviceLevel<double>& F = l64_[l - 1];
    DeviceLevel<double>& C = l64_[l];
    aggregate_channel(static_cast<int>(l - 1), -1, volume_[l - 1], volume_[l]);
    launch_reaction(stream_, F.view(neumann_), volume_[l - 1], agg_[2]);
    aggregate_channel(static_cast<int>(l - 1), -1, agg_[2], C.diag);
    aggregate_channel(static_cast<int>(l - 1), 0, F.fx, C.fx);
    aggregate_channel(static_cast<int>(l - 1), 1, F.fy, C.fy);
    aggregate_channel(static_cast<int>(l - 1), 2, F.fz, C.fz);
    launch_coarse_diagonal(stream_, C.nx, C.ny, C.nz, C.diag, C.fx, C.fy, C.fz,
                           volume_[l], fluid_[l]);
  }
  for (auto& L : l64_)
    for (int a = 0; a < 3; ++a)
      if (L.lfac[a] != nullptr) launch_line_factors<double>(stream_, L.view(neumann_), a, L.lfac[a]);
  // The coarsest level's sweeps (from any x_in and b) are one affine map;
  // record its columns once per coefficient update.
  coarse_dense_ = false;
  if (coarse_op_ != nullptr) {
    const DeviceLevel<double>& D = l64_.back();
    coarse_dense_ = launch_coarse_line<double, double>(
        stream_, D.view(neumann_), coarse_op_, nullptr, D.lfac[coarse_axis_],
        policy_.coarse_sweeps, coarse_axis_, true);
  }
  Status st = check(cudaGetLastError(), "hierarchy kernels");
  if (!st) return st;
  select_tail();
  // Diagonal shortcut (select_diagonal_shortcut, src/solver_mg.cpp:1577-1611).
  diagonal_shortcut_ = false;
  if (policy_.diagonal_shortcut_maximum_ratio != 0.0 &&
      policy_.null_space == HFPS_NULL_SPACE_NONE) {
    const Level<double> L0 = l64_[0].view(neumann_);
    launch_shortcut_ratio(stream_, L0, Reduce{d_scalars_, d_partials_, kOpMisc});
    const int blocks = reduction_blocks(static_cast<long long>(L0.nx) * L0.ny * L0.nz);
    std::vector<double> partial(blocks);
    st = check(cudaMemcpyAsync(partial.data(), d_partials_, blocks * sizeof(double),
                               cudaMemcpyDeviceToHost, stream_),
               "shortcut readback");
    if (!st) return st;
    st = check(cudaStreamSynchronize(stream_), "shortcut");
    if (!st) return st;
    double maximum = 0.0;
    for (double v : partial) maximum = std::max(maximum, v);
    diagonal_shortcut_ = maximum <= policy_.diagonal_shortcut_maximum_ratio;
  }
  // Validate the certified hierarchy: positive finite diagonals.
  std::vector<double> probe;
  for (size_t l = 0; l < l64_.size(); ++l) {
    const DeviceLevel<double>& L = l64_[l];
    if (L.cells() > (1 << 16)) continue;
    probe.resize(L.cells());
    st = check(cudaMemcpyAsync(probe.data(), L.diag, probe.size() * sizeof(double),
                               cudaMemcpyDeviceToHost, stream_),
               "diagonal probe");
    if (!st) return st;
    st = check(cudaStreamSynchronize(stream_), "diagonal probe");
    if (!st) return st;
    for (double d : probe)
      if (!(d > 0.0) || !std::isfinite(d))
        return fail(HFPS_NUMERICAL_FAILURE, kDetailNumeric,
                    "non-positive coarse diagonal");
  }
  coefficients_ready_ = true;
  mixed_ready_ = false;
  clear_mg_graphs();
  st = check(cudaStreamSynchronize(stream_), "hierarchy");
  if (!st) return st;
  return dic_factor();
}

// Cold-path IC(0) factorisation from the coefficients still staged in
// user_ (diagonal, unmasked faces): decorated row diagonals, then the
// inverse pivots plane by plane (ColdPressureIccg::prepare,
// src/solver_iccg.hpp:236-256).
Status Solver::dic_factor() {
  if (dic_rows_ == nullptr) return {};
  const Level<double> L0 = l64_[0].view(neumann_);
  Status st = check(cudaMemsetAsync(d_scalars_, 0, sizeof(Scalars), stream_), "scalars");
  if (!st) return st;
  launch_dic_rows(stream_, nx_, ny_, nz_, neumann_, user_[0], user_[1], user_[2], user_[3],
                  d_active_, dic_rows_);
  launch_dic_pivots(stream_, L0, dic_rows_, dic_inv_, d_scalars_);
  st = sync_scalars();
  if (!st) return st;
  if (h_scalars_->flags & 1) {
    coefficients_ready_ = false;
    return fail(HFPS_NUMERICAL_FAILURE, kDetailNumeric, "IC(0) pivot not positive");
  }
  return {};
}

Status Solver::refresh_mixed() {
  if (mixed_ready_) return {};
  for (size_t l = 0; l < l64_.size(); ++l) {
    const DeviceLevel<double>& a = l64_[l];
    DeviceLevel<float>& b = l32_[l];
    launch_convert<float, double>(stream_, a.cells(), a.diag, b.diag);
    launch_convert<float, double>(stream_, a.faces_x(), a.fx, b.fx);
    launch_convert<float, double>(stream_, a.faces_y(), a.fy, b.fy);
    launch_convert<float, double>(stream_, a.faces_z(), a.fz, b.fz);
  }
  for (auto& L : l32_)
    for (int a = 0; a < 3; ++a)
      if (L.lfac[a] != nullptr) launch_line_factors<float>(stream_, L.view(neumann_), a, L.lfac[a]);
  mixed_ready_ = true;
  return check(cudaGetLastError(), "mixed conversion");
}

Status Solver::set_coefficients(const double* diag, const double* fx,
                                const double* fy, const double* fz,
                                int memory) {
  if (diag == nullptr || fx == nullptr || fy == nullptr || fz == nullptr)
    return fail(HFPS_INVALID_PLAN, kDetailPlan, "null coefficient array");
  const size_t cells = static_cast<size_t>(nx_) * ny_ * nz_;
  const size_t nf[3] = {static_cast<size_t>(nx_ + 1) * ny_ * nz_,
                        static_cast<size_t>(nx_) * (ny_ + 1) * nz_,
                        static_cast<size_t>(nx_) * ny_ * (nz_ + 1)};
  if (memory == HFPS_HOST) {
    // finite_coefficients (src/solver_mg.cpp:147-177): diagonal > 0, faces >= 0.
    for (size_t c = 0; c < cells; ++c)
      if (!(diag[c] > 0.0) || !std::isfinite(diag[c]))
        return fail(HFPS_INVALID_PLAN, kDetailPlan, "diagonal must be positive and finite");
    const double* f[3] = {fx, fy, fz};
    for (int a = 0; a < 3; ++a)
      for (size_t i = 0; i < nf[a]; ++i)
        if (f[a][i] < 0.0 || !std::isfinite(f[a][i]))
          return fail(HFPS_INVALID_PLAN, kDetailPlan, "face coefficients must be finite and >= 0");
  }
  Status st = copy_in(user_[0], diag, cells, memory);
  if (st) st = copy_in(user_[1], fx, nf[0], memory);
  if (st) st = copy_in(user_[2], fy, nf[1], memory);
  if (st) st = copy_in(user_[3], fz, nf[2], memory);
  if (!st) return st;
  DeviceLevel<double>& L0 = l64_[0];
  launch_mask_finest(stream_, nx_, ny_, nz_, d_faces_[0], d_faces_[1], d_faces_[2],
                     user_[0], user_[1], user_[2], user_[3], d_active_, L0.diag,
                     L0.fx, L0.fy, L0.fz, volume_[0], fluid_[0]);
  return build_hierarchy();
}

Status Solver::set_beta(const double* beta, const double* storage, int memory) {
  if (beta == nullptr) return fail(HFPS_INVALID_PLAN, kDetailPlan, "null beta");
  const size_t cells = static_cast<size_t>(nx_) * ny_ * nz_;
  Status st = copy_in(kz_, beta, cells, memory);
  if (st && storage != nullptr) st = copy_in(kap_, storage, cells, memory);
  if (!st) return st;
  launch_beta_coefficients(stream_, nx_, ny_, nz_, d_faces_[0], d_faces_[1],
                           d_faces_[2], neumann_, kz_,
                           storage != nullptr ? kap_ : nullptr, user_[0], user_[1],
                           user_[2], user_[3]);
  DeviceLevel<double>& L0 = l64_[0];
  launch_mask_finest(stream_, nx_, ny_, nz_, d_faces_[0], d_faces_[1], d_faces_[2],
                     user_[0], user_[1], user_[2], user_[3], d_active_, L0.diag,
                     L0.fx, L0.fy, L0.fz, volume_[0], fluid_[0]);
  return build_hierarchy();
}

Status Solver::assemble(const hfps_assembly& in, double* rhs, int memory) {
  if (in.beta == nullptr || in.density_trial == nullptr || in.density_accepted == nullptr ||
      in.drho_dp == nullptr || in.flux_x == nullptr || in.flux_y == nullptr ||
      in.flux_z == nullptr || rhs == nullptr || (in.bdf_order != 1 && in.bdf_order != 2) ||
      (in.bdf_order == 2 && in.density_previous == nullptr) || !std::isfinite(in.a0) ||
      !std::isfinite(in.a1) || !std::isfinite(in.a2) || !(in.a0 > 0.0))
    return fail(HFPS_INVALID_PLAN, kDetailPlan, "invalid assembly input");
  const size_t cells = static_cast<size_t>(nx_) * ny_ * nz_;
  const size_t nf[3] = {static_cast<size_t>(nx_ + 1) * ny_ * nz_,
                        static_cast<size_t>(nx_) * (ny_ + 1) * nz_,
                        static_cast<size_t>(nx_) * ny_ * (nz_ + 1)};
  // Device staging: the Krylov vectors are free between solves.
  double* beta = kz_;
  double* rho = kx_;
  double* rho_n = kr_;
  double* rho_nm1 = in.bdf_order == 2 ? kp_ : nullptr;
  double* psi = kap_;
  double* source = in.mass_source != nullptr ? kb_ : nullptr;
  Status st = copy_in(beta, in.beta, cells, memory);
  if (st) st = copy_in(rho, in.density_trial, cells, memory);
  if (st) st = copy_in(rho_n, in.density_accepted, cells, memory);
  if (st && rho_nm1 != nullptr) st = copy_in(rho_nm1, in.density_previous, cells, memory);
  if (st) st = copy_in(psi, in.drho_dp, cells, memory);
  if (st && source != nullptr) st = copy_in(source, in.mass_source, cells, memory);
  if (!st) return st;
  // Face coefficients from beta (face_pressure_coefficient), then the
  // predicted fluxes into the aggregation scratch (free outside a rebuild).
  launch_beta_coefficients(stream_, nx_, ny_, nz_, d_faces_[0], d_faces_[1], d_faces_[2],
                           neumann_, beta, nullptr, user_[0], user_[1], user_[2], user_[3]);
  st = copy_in(agg_[0], in.flux_x, nf[0], memory);
  if (st) st = copy_in(agg_[1], in.flux_y, nf[1], memory);
  if (st) st = copy_in(agg_[2], in.flux_z, nf[2], memory);
  if (!st) return st;
  st = check(cudaMemsetAsync(d_scalars_, 0, sizeof(Scalars), stream_), "scalars");
  if (!st) return st;
  double* assembled_rhs = beta;  // beta is consumed by the face coefficients
  launch_assemble(stream_, nx_, ny_, nz_, d_faces_[0], d_faces_[1], d_faces_[2], in.a0, in.a1,
                  in.a2, in.bdf_order == 2, rho, rho_n, rho_nm1, psi, source, agg_[0], agg_[1],
                  agg_[2], user_[1], user_[2], user_[3], user_[0], assembled_rhs, d_scalars_);
  st = sync_scalars();
  if (!st) return st;
  if (h_scalars_->flags & 4)
    return fail(HFPS_NUMERICAL_FAILURE, kDetailNumeric, "pressure assembly rejected its input");
  DeviceLevel<double>& L0 = l64_[0];
  launch_mask_finest(stream_, nx_, ny_, nz_, d_faces_[0], d_faces_[1], d_faces_[2],
                     user_[0], user_[1], user_[2], user_[3], d_active_, L0.diag,
                     L0.fx, L0.fy, L0.fz, volume_[0], fluid_[0]);
  st = build_hierarchy();
  if (!st) return st;
  st = copy_out(rhs, assembled_rhs, cells, memory);
  if (!st) return st;
  return check(cudaStreamSynchronize(stream_), "assembly");
}

Status Solver::correct_flux(const double* correction, const double* cx, const double* cy,
                            const double* cz, double scale, double* qx, double* qy,
                            double* qz, int memory) {
  if (correction == nullptr || cx == nullptr || cy == nullptr || cz == nullptr ||
      qx == nullptr || qy == nullptr || qz == nullptr || !std::isfinite(scale))
    return fail(HFPS_INVALID_PLAN, kDetailPlan, "invalid flux-correction input");
  const size_t cells = static_cast<size_t>(nx_) * ny_ * nz_;
  const size_t nf[3] = {static_cast<size_t>(nx_ + 1) * ny_ * nz_,
                        static_cast<size_t>(nx_) * (ny_ + 1) * nz_,
                        static_cast<size_t>(nx_) * ny_ * (nz_ + 1)};
  const double* c[3] = {cx, cy, cz};
  double* q[3] = {qx, qy, qz};
  // Staging: correction in kp_, coefficients in user_[1..3], fluxes in agg_.
  Status st = copy_in(kp_, correction, cells, memory);
  for (int a = 0; a < 3 && st; ++a) st = copy_in(user_[1 + a], c[a], nf[a], memory);
  for (int a = 0; a < 3 && st; ++a) st = copy_in(agg_[a], q[a], nf[a], memory);
  if (!st) return st;
  st = check(cudaMemsetAsync(d_scalars_, 0, sizeof(Scalars), stream_), "scalars");
  if (!st) return st;
  launch_correct_flux(stream_, nx_, ny_, nz_, neumann_, kp_, user_[1], user_[2], user_[3],
                      scale, agg_[0], agg_[1], agg_[2], d_scalars_);
  st = sync_scalars();
  if (!st) return st;
  if (h_scalars_->flags & 1)
    return fail(HFPS_NUMERICAL_FAILURE, kDetailNumeric, "non-finite corrected flux");
  for (int a = 0; a < 3 && st; ++a) st = copy_out(q[a], agg_[a], nf[a], memory);
  if (!st) return st;
  return check(cudaStreamSynchronize(stream_), "flux correction");
}

// ---------------------------------------------------------------------------
// MG cycle (mg_cycle, src/solver_mg.cpp:4192-4338).

// x_zero: the level's x is zero on entry (a cycle's first visit), which the
// chunked scan uses to skip reading it in the first sweep.
template <class T>
void Solver::smooth(std::vector<DeviceLevel<T>>& levels, int level, int sweeps,
                    bool reverse, bool x_zero) {
  DeviceLevel<T>& L = levels[level];
  const Level<T> view = L.view(neumann_);
  if (L.line_mask == 0) {
    if (L.chebyshev) {
      // chebyshev_point_smooth_streamed (src/solver_mg.cpp:2916-3012): the
      // ping-pong partner becomes the solution after odd stage counts.
      constexpr double beta = 2.0;
      const double alpha = policy_.chebyshev_lower_spectrum_fraction * beta;
      const double theta = (beta + alpha) * 0.5;
      const double delta = (beta - alpha) * 0.5;
      const double sigma = theta / delta;
      double previous_rho = 1.0 / sigma;
      for (int s = 0; s < sweeps; ++s) {
        const double rho = s == 0 ? 0.0 : 1.0 / (2.0 * sigma - previous_rho);
        const double previous_factor = s == 0 ? 0.0 : rho * previous_rho;
        const double residual_factor = s == 0 ? 1.0 / theta : 2.0 * rho / delta;
        if (s != 0) previous_rho = rho;
        launch_chebyshev_stage<T>(stream_, view, L.x, L.b, L.r, L.t,
                                  static_cast<T>(previous_factor),
                                  static_cast<T>(residual_factor), s == 0 ? 1 : 0);
        std::swap(L.x, L.t);
      }
    } else {
      const int first = reverse ? 1 : 0;
      for (int s = 0; s < sweeps; ++s)
        for (int pass = 0; pass < 2; ++pass)
          launch_rb_color<T>(stream_, view, L.x, L.b, (first + pass) & 1);
    }
    return;
  }
  // smooth(): line relaxation along every strong axis, reversed on the way
  // up (src/solver_mg.cpp:3566-3589); zebra colour order per sweep.
  // In the first sweep from x = 0 (one line axis), the first pass reads no
  // x and the second reads only the colour the first wrote.
  const bool one_axis = (L.line_mask & (L.line_mask - 1)) == 0;
  const auto run_axis = [&](int axis) {
    const int first = reverse ? 1 : 0;
    for (int s = 0; s < sweeps; ++s)
      for (int pass = 0; pass < 2; ++pass) {
        const bool fresh = x_zero && one_axis && s == 0;
        launch_line_pass<T>(stream_, view, L.x, L.b, L.lfac[axis], L.r, axis,
                            (first + pass) & 1, L.split, fresh && pass == 0, fresh);
      }
  };
  if (reverse) {
    for (int a = 3; a-- > 0;)
      if (L.line_mask & (1 << a)) run_axis(a);
  } else {
    for (int a = 0; a < 3; ++a)
      if (L.line_mask & (1 << a)) run_axis(a);
  }
}

template <class T>
void Solver::coarse_solve(std::vector<DeviceLevel<T>>& levels, bool x_zero) {
  DeviceLevel<T>& L = levels.back();
  DeviceLevel<double>& D = l64_.back();
  const Level<double> view = D.view(neumann_);
  const bool widen = !std::is_same<T, double>::value;
  double* xs = widen ? D.x : nullptr;
  double* bs = widen ? D.b : nullptr;
  if (L.line_mask == 0) {
    launch_coarse_solve<T, double>(stream_, view, L.x, L.b, xs, bs, D.t, D.r,
                                   policy_.coarse_sweeps, -1);
    return;
  }
  if (coarse_dense_) {
    launch_coarse_dense<T>(stream_, L.cells(), coarse_op_, L.x, L.b, L.t, x_zero);
    std::swap(L.x, L.t);
    return;
  }
  for (int a = 0; a < 3; ++a) {
    if (!(L.line_mask & (1 << a))) continue;
    if (!launch_coarse_line<T, double>(stream_, view, L.x, L.b, D.lfac[a],
                                       policy_.coarse_sweeps, a))
      launch_coarse_solve<T, double>(stream_, view, L.x, L.b, xs, bs, D.t, D.r,
                                     policy_.coarse_sweeps, a);
  }
}

// The persistent small-level launch covers levels tail_level_.. when every
// non-coarsest one relaxes lines along one axis with PCR (few lines per
// colour), all have the same line length, and the coarsest is the dense
// affine map.  HFPS_TAIL=1 / 0 turns it on / off (default kTailDefault);
// HFPS_TAIL_BLOCKS overrides its CTA count (clamped to what is co-resident
// and rounded down to a power of two).
void Solver::select_tail() {
  tail_level_ = -1;
  const char* env = std::getenv("HFPS_TAIL");
  const bool on = env != nullptr && env[0] != '\0' ? env[0] != '0' : kTailDefault;
  // HFPS_TAIL_BARRIER_TEST=1: every launch's first grid barrier runs out its
  // wait limit, so the solve fails with the barrier's status (for the test of
  // that path; the GPU stays usable).
  const char* test = std::getenv("HFPS_TAIL_BARRIER_TEST");
  tail_barrier_test_ = test != nullptr && test[0] == '1';
  if (!on || !coarse_dense_ || policy_.null_space != HFPS_NULL_SPACE_NONE) return;
  const int levels = static_cast<int>(l64_.size());
  int first = levels - 1;
  int axis = -1, extent = -1;
  for (int l = levels - 2; l >= 1; --l) {
    const DeviceLevel<double>& L = l64_[l];
    const int mask = L.line_mask;
    if (mask == 0 || (mask & (mask - 1)) != 0) break;
    const int a = mask == 1 ? 0 : (mask == 2 ? 1 : 2);
    if (line_kind(L.nx, L.ny, L.nz, a) != kLinePcr) break;
    const int e = a == 0 ? L.nx : (a == 1 ? L.ny : L.nz);
    if (axis >= 0 && (a != axis || e != extent)) break;
    axis = a;
    extent = e;
    first = l;
  }
  if (first >= levels - 1 || levels - first > kTailMaxLevels) return;
  const int steps = tail_steps(extent);
  if (steps < 0) return;
  int device = 0, sms = 0;
  cudaGetDevice(&device);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const DeviceLevel<double>& top = l64_[first];
  const int a_extent = axis == 0 ? top.ny : top.nx;
  const int b_extent = axis == 2 ? top.ny : top.nz;
  const int lines = ((a_extent + 1) / 2) * b_extent;
  const int dense_n = l64_.back().cells();
  // Enough CTAs for one round of the top level's lines (tail_lines_per_cta
  // at a time) and for the dense map's 32-row blocks.
  const int per_cta = tail_lines_per_cta(steps);
  int want = std::max((lines + per_cta - 1) / per_cta, (dense_n + 31) / 32);
  const char* blocks_env = std::getenv("HFPS_TAIL_BLOCKS");
  if (blocks_env != nullptr && std::atoi(blocks_env) > 0) want = std::atoi(blocks_env);
  // One CTA count for both precisions, a power of two: the barrier's
  // arrival counter is then a multiple of it across 32-bit wrap-around.
  int blocks = std::min({tail_grid<double>(steps, dense_n, sms),
                         tail_grid<float>(steps, dense_n, sms), want});
  if (blocks < 1) return;
  while (blocks & (blocks - 1)) blocks &= blocks - 1;
  tail_blocks_[0] = tail_blocks_[1] = blocks;
  tail_level_ = first;
  tail_steps_ = steps;
}

template <class T>
void Solver::tail_cycle(std::vector<DeviceLevel<T>>& levels, int level, int counter,
                        bool x_zero, TailProgram<T>& prog) {
  const auto add = [&](int kind, int lv, int arg, const void* a, const void* b,
                       const void* c, const void* d) {
    if (prog.count >= kTailMaxOps) {
      prog.count = kTailMaxOps + 1;  // marks an overflow; tail_launch falls back
      return;
    }
    prog.ops[prog.count++] = TailOp{kind, lv - tail_level_, arg, 0, const_cast<void*>(a),
                                    const_cast<void*>(b), const_cast<void*>(c),
                                    const_cast<void*>(d)};
  };
  DeviceLevel<T>& L = levels[level];
  if (level + 1 == static_cast<int>(levels.size())) {
    // coarse_solve's dense branch: out = P x + M b into t, then x <-> t.
    add(kTailDense, level, x_zero ? 1 : 0, L.x, L.b, L.t, nullptr);
    std::swap(L.x, L.t);
    return;
  }
  const int axis = L.line_mask == 1 ? 0 : (L.line_mask == 2 ? 1 : 2);
  const auto sweeps = [&](int count, bool reverse) {
    const int first = reverse ? 1 : 0;
    for (int s = 0; s < count; ++s)
      for (int pass = 0; pass < 2; ++pass)
        add(kTailPcr, level, (first + pass) & 1, L.x, L.b, L.lfac[axis], nullptr);
  };
  DeviceLevel<T>& C = levels[level + 1];
  sweeps(policy_.pre_sweeps, false);
  add(kTailRestrict, level, L.coarsen_mask, L.x, L.b, C.b, C.x);
  tail_cycle(levels, level + 1, counter, true, prog);
  if (counter > 1) tail_cycle(levels, level + 1, counter - 1, false, prog);
  add(kTailProlong, level, L.coarsen_mask, L.x, C.x, nullptr, nullptr);
  sweeps(policy_.post_sweeps, true);
}

template <class T>
void Solver::tail_launch(std::vector<DeviceLevel<T>>& levels, TailProgram<T>& prog) {
  const int slot = std::is_same<T, float>::value ? 1 : 0;
  const int count = static_cast<int>(levels.size()) - tail_level_;
  for (int l = 0; l < count; ++l) {
    const DeviceLevel<T>& L = levels[tail_level_ + l];
    prog.levels[l] = L.view(neumann_);
    prog.axis[l] = L.line_mask == 1 ? 0 : (L.line_mask == 2 ? 1 : 2);
  }
  prog.dense_op = coarse_op_;
  prog.dense_n = levels.back().cells();
  prog.barrier_offset = tail_barrier_test_ ? 1 : 0;
  prog.pad = 0;
  prog.scalars = d_scalars_;
  launch_tail<T>(stream_, prog, tail_steps_, tail_blocks_[slot]);
  launches_ += 1;
}

template <class T>
void Solver::cycle(std::vector<DeviceLevel<T>>& levels, int level, int counter,
                   bool x_zero) {
  if (level + 1 == static_cast<int>(levels.size())) {
    coarse_solve(levels, x_zero);
    return;
  }
  DeviceLevel<T>& F = levels[level];
  DeviceLevel<T>& C = levels[level + 1];
  smooth(levels, level, policy_.pre_sweeps, false, x_zero);
  // Retained defect + restrict_residual in one pass.
  launch_defect_restrict<T>(stream_, F.view(neumann_), F.x, F.b, C.view(neumann_),
                            C.b, C.x, F.coarsen_mask, F.split, C.split);
  // restrict_residual's projection of the coarse rhs (src/solver_mg.cpp:3708-3716).
  if (policy_.null_space == HFPS_NULL_SPACE_CONSTANT)
    launch_project_constant<T>(stream_, C.nx, C.ny, C.nz, C.split, C.b, volume_[level + 1],
                               d_scalars_, d_partials_);
  if (level + 1 == tail_level_) {
    // Both visits of the level below (an F-cycle's counter 2 and 1) in one
    // persistent launch.
    TailProgram<T> prog;
    prog.count = 0;
    std::vector<std::pair<T*, T*>> saved;
    for (auto& L : levels) saved.emplace_back(L.x, L.t);
    tail_cycle(levels, level + 1, counter, true, prog);
    if (counter > 1) tail_cycle(levels, level + 1, counter - 1, false, prog);
    if (prog.count <= kTailMaxOps) {
      tail_launch(levels, prog);
    } else {
      for (size_t l = 0; l < levels.size(); ++l) {
        levels[l].x = saved[l].first;
        levels[l].t = saved[l].second;
      }
      const int tail = tail_level_;
      tail_level_ = -1;
      cycle(levels, level + 1, counter, true);
      if (counter > 1) cycle(levels, level + 1, counter - 1, false);
      tail_level_ = tail;
    }
  } else {
    cycle(levels, level + 1, counter, true);
    if (counter > 1) cycle(levels, level + 1, counter - 1, false);
  }
  launch_prolongate<T>(stream_, F.view(neumann_), F.x, C.view(neumann_), C.x,
                       F.coarsen_mask, F.split, C.split);
  smooth(levels, level, policy_.post_sweeps, true, false);
}

// NativeCartesianMgPlan::apply_impl (src/solver_mg.cpp:4814-5122).
template <class T>
void Solver::mg_enqueue(std::vector<DeviceLevel<T>>& levels, const double* r,
                        double* z) {
  // Canonical buffer roles at entry, so captured and eager runs agree.
  std::vector<std::pair<T*, T*>> saved;
  for (auto& L : levels) saved.emplace_back(L.x, L.t);
  DeviceLevel<T>& L0 = levels[0];
  const int n = L0.cells();
  const VecLayout v0{L0.nx, L0.ny, L0.split};
  // x = 0 is written here unless the diagonal shortcut or the first
  // pre-smoothing sweep (zero flags) defines every entry anyway.
  const bool zero_x = !(diagonal_shortcut_ || first_sweep_zero_);
  launch_mg_enter<T>(stream_, n, r, d_active_, L0.b, L0.x, v0, zero_x);
  // MgNullSpace::constant: the rhs, every restricted rhs and the result lose
  // their volume-weighted mean (apply_impl, src/solver_mg.cpp:4900-4960).
  const bool constant = policy_.null_space == HFPS_NULL_SPACE_CONSTANT;
  if (constant)
    launch_project_constant<T>(stream_, L0.nx, L0.ny, L0.nz, L0.split, L0.b, volume_[0],
                               d_scalars_, d_partials_);
  if (diagonal_shortcut_) {
    launch_diagonal_solve<T>(stream_, n, L0.b, L0.diag, L0.x, v0);
  } else {
    cycle(levels, 0, policy_.cycle == 1 ? 2 : 1, true);
  }
  if (constant)
    launch_project_constant<T>(stream_, L0.nx, L0.ny, L0.nz, L0.split, L0.x, volume_[0],
                               d_scalars_, d_partials_);
  if (policy_.unit_linear && krylov_fusion_) {
    // The PCG consumes r.z of every preconditioner application: formed here
    // while z is written (kOpRhoNext; the PCG's restarts use only rho).
    launch_mg_exit_dot<T>(stream_, n, L0.x, d_active_, z, v0, r,
                          Reduce{d_scalars_, d_partials_, kOpRhoNext});
  } else if (policy_.unit_linear) {
    launch_mg_exit<T>(stream_, n, L0.x, d_active_, nullptr, z, v0);
  } else {
    launch_level_defect<T>(stream_, L0.view(neumann_), L0.x, L0.b, L0.r, L0.split);
    launch_mg_projection<T>(stream_, n, r, d_active_, L0.r,
                            Reduce{d_scalars_, d_partials_, 5});
    launch_mg_exit<T>(stream_, n, L0.x, d_active_, &d_scalars_->mg_alpha, z, v0);
  }
  for (size_t l = 0; l < levels.size(); ++l) {
    levels[l].x = saved[l].first;
    levels[l].t = saved[l].second;
  }
}

void Solver::clear_mg_graphs() {
  for (MgGraph& g : mg_graphs_)
    if (g.exec != nullptr) cudaGraphExecDestroy(g.exec);
  mg_graphs_.clear();
}

Status Solver::mg_apply(bool mixed, const double* r, double* z) {
  if (mixed) {
    Status st = refresh_mixed();
    if (!st) return st;
  }
  if (r == nullptr) r = kr_;
  if (z == nullptr) z = kz_;
  const int slot = mixed ? 1 : 0;
  if (!use_graphs_) {
    if (mixed) mg_enqueue(l32_, r, z);
    else mg_enqueue(l64_, r, z);
    launches_ += mg_nodes_[slot];
    return check(cudaGetLastError(), "mg launch");
  }
  cudaGraphExec_t exec = nullptr;
  for (const MgGraph& g : mg_graphs_)
    if (g.slot == slot && g.r == r && g.z == z) exec = g.exec;
  if (exec == nullptr) {
    cudaGraph_t graph = nullptr;
    Status st = check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal),
                      "graph capture begin");
    if (!st) return st;
    if (mixed) mg_enqueue(l32_, r, z);
    else mg_enqueue(l64_, r, z);
    st = check(cudaStreamEndCapture(stream_, &graph), "graph capture end");
    if (!st) return st;
    size_t nodes = 0;
    cudaGraphGetNodes(graph, nullptr, &nodes);
    mg_nodes_[slot] = nodes;
    st = check(cudaGraphInstantiate(&exec, graph, 0), "graph instantiate");
    cudaGraphDestroy(graph);
    if (!st) return st;
    mg_graphs_.push_back(MgGraph{slot, r, z, exec});
  }
  launches_ += mg_nodes_[slot];
  return check(cudaGraphLaunch(exec, stream_), "graph launch");
}

Status Solver::dic_apply() {
  const Level<double> L0 = l64_[0].view(neumann_);
  if (!use_graphs_) {
    launch_dic_apply(stream_, L0, kr_, kz_, dic_inv_);
    launches_ += 2 * static_cast<uint64_t>(dic_planes(L0));
    return check(cudaGetLastError(), "IC(0) launch");
  }
  if (dic_graph_ == nullptr) {
    cudaGraph_t graph = nullptr;
    Status st = check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal),
                      "graph capture begin");
    if (!st) return st;
    launch_dic_apply(stream_, L0, kr_, kz_, dic_inv_);
    st = check(cudaStreamEndCapture(stream_, &graph), "graph capture end");
    if (!st) return st;
    cudaGraphGetNodes(graph, nullptr, &dic_nodes_);
    st = check(cudaGraphInstantiate(&dic_graph_, graph, 0), "graph instantiate");
    cudaGraphDestroy(graph);
    if (!st) return st;
  }
  launches_ += dic_nodes_;
  return check(cudaGraphLaunch(dic_graph_, stream_), "graph launch");
}

Status Solver::precondition(bool mixed) {
  if (policy_.preconditioner == HFPS_PRECONDITIONER_IC0) return dic_apply();
  return mg_apply(mixed);
}

Status Solver::sync_scalars() {
  Status st = check(cudaMemcpyAsync(h_scalars_, d_scalars_, sizeof(Scalars),
                                    cudaMemcpyDeviceToHost, stream_),
                    "scalar readback");
  if (!st) return st;
  st = check(cudaStreamSynchronize(stream_), "solver step");
  if (!st) return st;
  if (h_scalars_->flags & 8)
    return fail(HFPS_NUMERICAL_FAILURE, kDetailNumeric,
                "small-level kernel: a grid barrier timed out");
  return {};
}

// The solve's 2-norm of a vector whose plain sum of squares a kernel has just
// formed: queue_norm adds the two max-scaled passes when the solve asked for
// the reference's global_norm (HFPS_NORM_SCALED); norm_value reads whichever
// form after the scalars are back on the host.
void Solver::queue_norm(const double* v) {
  if (!scaled_norm_) return;
  launch_scaled_norm(stream_, nx_ * ny_ * nz_, v, d_scalars_, d_partials_);
  launches_ += 2;
}
double Solver::norm_value(double plain_squares) const {
  return scaled_norm_ ? h_scalars_->misc[3] : std::sqrt(plain_squares);
}

// solve_pcg (src/solver_krylov.cpp:1299-1555) with identical control flow:
// true residual every `true_residual_interval` iterations, at a recursive
// convergence claim and at the cap, and a restart of the search direction
// (p = z) after every verification.
Status Solver::krylov_pcg(const hfps_control& control, hfps_result& result,
                          double* history, uint32_t capacity) {
  const int n = nx_ * ny_ * nz_;
  const bool mixed = control.precision == HFPS_MIXED;
  const Level<double> A = l64_[0].view(neumann_);
  const auto red = [&](int op) { return Reduce{d_scalars_, d_partials_, op}; };
  Status st = check(cudaMemsetAsync(d_scalars_, 0, sizeof(Scalars), stream_), "scalars");
  if (!st) return st;
  launch_norm2(stream_, n, kb_, red(kOpMisc));
  launches_ += 1;
  queue_norm(kb_);
  st = sync_scalars();
  if (!st) return st;
  if (h_scalars_->flags & 1) {
    result.termination = HFPS_NON_FINITE;
    return fail(HFPS_NUMERICAL_FAILURE, kDetailNumeric, "non-finite rhs");
  }
  const double bnorm = norm_value(h_scalars_->misc[0]);
  const double tol = std::max(control.absolute_tolerance,
                              control.relative_tolerance * bnorm);
  result.rhs_norm = bnorm;
  result.true_residual_limit = tol;
  if (bnorm == 0.0) {
    st = check(cudaMemsetAsync(kx_, 0, n * sizeof(double), stream_), "zero x");
    result.termination = HFPS_ZERO_RHS;
    return st;
  }
  launch_residual_norm(stream_, A, kx_, kb_, kr_, red(kOpRecursive));
  launches_ += 1;
  ++result.operator_applies;
  queue_norm(kr_);
  st = sync_scalars();
  if (!st) return st;
  result.initial_true_residual = norm_value(h_scalars_->rr);
  result.final_true_residual = result.initial_true_residual;
  result.recursive_residual = result.initial_true_residual;
  if (!std::isfinite(result.initial_true_residual)) {
    result.termination = HFPS_NON_FINITE;
    return fail(HFPS_NUMERICAL_FAILURE, kDetailNumeric, "non-finite residual");
  }
  if (result.initial_true_residual <= tol) {
    result.termination = HFPS_CONVERGED;
    return {};
  }
  // With the MG preconditioner at unit scaling the MG exit forms r.z itself
  // (kOpRhoNext: rho = r.z; a restart uses only rho).
  const bool fused_dot = krylov_fusion_ && policy_.unit_linear &&
                         policy_.preconditioner != HFPS_PRECONDITIONER_IC0;
  const auto restart_direction = [&]() -> Status {
    Status s = precondition(mixed);
    if (!s) return s;
    ++result.preconditioner_applies;
    if (!fused_dot) {
      launch_dot(stream_, n, kr_, kz_, red(kOpRhoRestart));
      launches_ += 1;
    }
    launch_copy(stream_, n, kz_, kp_);
    launches_ += 1;
    return {};
  };
  st = restart_direction();
  if (!st) return st;
  uint32_t it = 0;
  // Queue-ahead: in an iteration that is not a planned true-residual check,
  // while the last recursive residual is far above the limit, the next MG
  // application and direction update are queued before the host reads this
  // iteration's scalars.  They are what the iteration does next unless its
  // recursive residual has met the limit, and the true-residual check that
  // then follows overwrites z, p and r.z anyway; so results are unchanged
  // and the GPU does not idle while the host reads the scalars.
  constexpr double kQueueAheadMargin = 8.0;
  double last_recursive = result.initial_true_residual;
  while (it < control.maximum_iterations) {
    launch_spmv_dot(stream_, A, kp_, kap_, red(kOpPap), tiled_stencil_);
    ++result.operator_applies;
    launch_pcg_update(stream_, n, kx_, kp_, kr_, kap_, red(kOpRecursive));
    launches_ += 2;
    queue_norm(kr_);
    ++it;
    const bool planned = it % control.true_residual_interval == 0 ||
                         it == control.maximum_iterations;
    const bool ahead = queue_ahead_ && !planned && last_recursive > kQueueAheadMargin * tol;
    st = check(cudaMemcpyAsync(h_scalars_, d_scalars_, sizeof(Scalars), cudaMemcpyDeviceToHost,
                               stream_),
               "scalar readback");
    if (!st) return st;
    st = check(cudaEventRecord(scalars_ready_, stream_), "scalar event");
    if (!st) return st;
    if (ahead) {
      st = precondition(mixed);
      if (!st) return st;
      if (!fused_dot) {
        launch_dot(stream_, n, kr_, kz_, red(kOpRhoNext));
        launches_ += 1;
      }
      launch_p_update(stream_, n, kp_, kz_, d_scalars_);
      launches_ += 1;
    }
    st = check(cudaEventSynchronize(scalars_ready_), "solver step");
    if (!st) return st;
    if (h_scalars_->flags & 8)
      return fail(HFPS_NUMERICAL_FAILURE, kDetailNumeric,
                  "small-level kernel: a grid barrier timed out");
    result.iterations = it;
    // A breakdown flag comes from p.Ap of this iteration (the reference
    // stops before counting it) or from the r.z that formed this direction
    // (counted in the previous iteration): either way the reference reports
    // one iteration fewer than this loop has taken.
    if (h_scalars_->flags & 2) {
      result.iterations = it - 1;
      result.termination = HFPS_BREAKDOWN;
      return fail(HFPS_NUMERICAL_FAILURE, kDetailBreakdown, "Krylov breakdown");
    }
    if (h_scalars_->flags & 1) {
      result.termination = HFPS_NON_FINITE;
      return fail(HFPS_NUMERICAL_FAILURE, kDetailNumeric, "non-finite Krylov scalar");
    }
    const double recursive = norm_value(h_scalars_->rr);
    result.recursive_residual = recursive;
    last_recursive = recursive;
    if (history != nullptr && it - 1 < capacity) {
      history[it - 1] = recursive;
      result.history_length = it;
    }
    const bool verify = recursive <= tol || planned;
    if (verify) {
      launch_residual_norm(stream_, A, kx_, kb_, kr_, red(kOpRecursive));
      launches_ += 1;
      ++result.operator_applies;
      queue_norm(kr_);
      st = sync_scalars();
      if (!st) return st;
      result.final_true_residual = norm_value(h_scalars_->rr);
      result.recursive_residual = result.final_true_residual;
      if (result.final_true_residual <= tol) {
        result.termination = HFPS_CONVERGED;
        return {};
      }
      if (it == control.maximum_iterations) break;
      st = restart_direction();
      if (!st) return st;
      continue;
    }
    ++result.preconditioner_applies;
    if (ahead) continue;  // already queued
    st = precondition(mixed);
    if (!st) return st;
    if (!fused_dot) {
      launch_dot(stream_, n, kr_, kz_, red(kOpRhoNext));
      launches_ += 1;
    }
    launch_p_update(stream_, n, kp_, kz_, d_scalars_);
    launches_ += 1;
  }
  result.termination = HFPS_MAXIMUM_ITERATIONS;
  return fail(HFPS_REJECTED_STEP, kDetailBreakdown, "maximum iterations reached");
}

Status Solver::ensure_fgmres_storage(uint32_t restart) {
  if (fg_storage_ != nullptr && restart <= fg_restart_) return {};
  if (fg_storage_ != nullptr) {
    Status st = check(cudaStreamSynchronize(stream_), "fgmres storage");
    if (!st) return st;
    clear_mg_graphs();  // graphs captured on the old basis buffers
    cudaFree(fg_storage_);
    fg_storage_ = nullptr;
  }
  const size_t n = static_cast<size_t>(nx_) * ny_ * nz_;
  const size_t stride = (n + 31) & ~static_cast<size_t>(31);
  const size_t vectors = 2 * static_cast<size_t>(restart) + 2;
  Status st = check(cudaMalloc(&fg_storage_, vectors * stride * sizeof(double)),
                    "fgmres basis");
  if (!st) {
    fg_storage_ = nullptr;
    return st;
  }
  fg_restart_ = restart;
  fg_v_.assign(restart + 1, nullptr);
  fg_z_.assign(restart, nullptr);
  for (uint32_t i = 0; i <= restart; ++i) fg_v_[i] = fg_storage_ + i * stride;
  for (uint32_t i = 0; i < restart; ++i) fg_z_[i] = fg_storage_ + (restart + 1 + i) * stride;
  fg_w_ = fg_storage_ + (2 * static_cast<size_t>(restart) + 1) * stride;
  return {};
}

Status Solver::ensure_recycle_storage() {
  if (rc_storage_ != nullptr) return {};
  const size_t n = static_cast<size_t>(nx_) * ny_ * nz_;
  const size_t stride = (n + 31) & ~static_cast<size_t>(31);
  Status st = check(cudaMalloc(&rc_storage_, (2 * kRecycleMax + 1) * stride * sizeof(double)),
                    "recycle storage");
  if (!st) {
    rc_storage_ = nullptr;
    return st;
  }
  for (int i = 0; i < kRecycleMax; ++i) {
    rc_ring_[i] = rc_storage_ + i * stride;
    rc_image_[i] = rc_storage_ + (kRecycleMax + 1 + i) * stride;
  }
  rc_snapshot_ = rc_storage_ + kRecycleMax * stride;
  return {};
}

// recycle_capture_cycle_publish (src/solver_linear_state.cpp:897-1017):
// the cycle's correction x - snapshot enters the ring when it has a nonzero
// entry, replacing the oldest of four.
Status Solver::recycle_publish(const double* x, hfps_result& result) {
  if (!rc_capture_ || !rc_cycle_active_) return {};
  const int n = nx_ * ny_ * nz_;
  Status st = check(cudaMemsetAsync(&d_scalars_->marks, 0, sizeof(unsigned), stream_),
                    "recycle mark");
  if (!st) return st;
  launch_difference_nonzero(stream_, n, x, rc_snapshot_, d_scalars_);
  launches_ += 1;
  st = sync_scalars();
  if (!st) return st;
  rc_cycle_active_ = false;
  if (!(h_scalars_->marks & 1u)) return {};
  ++result.recycle_captured;
  const int slot = rc_count_ < kRecycleMax ? (rc_oldest_ + rc_count_) % kRecycleMax : rc_oldest_;
  std::swap(rc_ring_[slot], rc_snapshot_);
  if (rc_count_ < kRecycleMax) ++rc_count_;
  else rc_oldest_ = (rc_oldest_ + 1) % kRecycleMax;
  return {};
}

// apply_recycle_projection (src/solver_krylov.cpp:1745-2019): images A d_i,
// a rank test against 64 eps max |A d_i|, two classical Gram-Schmidt passes
// over the retained images (the directions follow), normalisation,
// alpha_i = image_i . r and the candidate x + sum alpha_i d_i, taken when its
// true residual is below the current one.  The projection's operator
// applies are not counted as the solve's (as in the reference).
Status Solver::recycle_project(const hfps_control& control, double tol, hfps_result& result) {
  rc_pending_ = false;
  const int n = nx_ * ny_ * nz_;
  (void)control;
  const Level<double> A = l64_[0].view(neumann_);
  const auto red = [&](int op) { return Reduce{d_scalars_, d_partials_, op}; };
  const int offered = rc_count_;
  result.recycle_offered = static_cast<uint32_t>(offered);
  double* images[kRecycleMax];
  double* dirs[kRecycleMax];
  double pre[kRecycleMax];
  double max_pre = 0.0;
  Status st;
  for (int i = 0; i < offered; ++i) {
    dirs[i] = rc_ring_[(rc_oldest_ + i) % kRecycleMax];
    images[i] = rc_image_[i];
    launch_level_apply<double>(stream_, A, dirs[i], images[i]);
    launch_norm2(stream_, n, images[i], red(kOpMisc));
    launches_ += 2;
    st = sync_scalars();
    if (!st) return st;
    pre[i] = std::sqrt(h_scalars_->misc[0]);
    max_pre = std::max(max_pre, pre[i]);
  }
  rc_count_ = 0;
  rc_oldest_ = 0;
  int kept[kRecycleMax];
  int retained = 0;
  if (offered > 0 && max_pre > 0.0 && std::isfinite(max_pre)) {
    const double threshold = 64.0 * std::numeric_limits<double>::epsilon() * max_pre;
    for (int i = 0; i < offered; ++i) {
      if (!(pre[i] > threshold)) continue;
      double image_norm = pre[i];
      if (retained != 0) {
        for (int pass = 0; pass < 2; ++pass) {
          BasisRefs refs{};
          refs.count = retained;
          for (int p = 0; p < retained; ++p) refs.v[p] = images[kept[p]];
          // k_multidot reads w = images[i] against the retained images
          launch_multidot(stream_, n, refs, images[i], false, d_scalars_->hcol,
                          red(kCounterMultidot));
          launches_ += 1;
          st = sync_scalars();
          if (!st) return st;
          BasisRefs img{}, dir{};
          img.count = dir.count = retained;
          for (int p = 0; p < retained; ++p) {
            img.v[p] = images[kept[p]];
            dir.v[p] = dirs[kept[p]];
            img.s[p] = dir.s[p] = -h_scalars_->hcol[p];
          }
          launch_basis_update(stream_, n, images[i], img, 1.0, false, images[i]);
          launch_basis_update(stream_, n, dirs[i], dir, 1.0, false, dirs[i]);
          launches_ += 2;
        }
        launch_norm2(stream_, n, images[i], red(kOpMisc));
        launches_ += 1;
        st = sync_scalars();
        if (!st) return st;
        image_norm = std::sqrt(h_scalars_->misc[0]);
      }
      if (!(image_norm > threshold) || !std::isfinite(image_norm)) continue;
      BasisRefs none{};
      launch_basis_update(stream_, n, images[i], none, 1.0 / image_norm, true, images[i]);
      launch_basis_update(stream_, n, dirs[i], none, 1.0 / image_norm, true, dirs[i]);
      launches_ += 2;
      kept[retained++] = i;
    }
  }
  result.recycle_retained = static_cast<uint32_t>(retained);
  if (retained == 0) return {};
  BasisRefs refs{};
  refs.count = retained;
  for (int p = 0; p < retained; ++p) refs.v[p] = images[kept[p]];
  launch_multidot(stream_, n, refs, fg_v_[0], false, d_scalars_->hcol, red(kCounterMultidot));
  launches_ += 1;
  st = sync_scalars();
  if (!st) return st;
  BasisRefs dir{};
  dir.count = retained;
  for (int p = 0; p < retained; ++p) {
    dir.v[p] = dirs[kept[p]];
    dir.s[p] = h_scalars_->hcol[p];
  }
  double* candidate = rc_snapshot_;
  launch_basis_update(stream_, n, kx_, dir, 1.0, false, candidate);
  launch_residual_norm(stream_, A, candidate, kb_, fg_w_, red(kOpRecursive));
  launches_ += 2;
  queue_norm(fg_w_);
  st = sync_scalars();
  if (!st) return st;
  const double candidate_norm = norm_value(h_scalars_->rr);
  result.recycle_projected_residual = candidate_norm;
  if (std::isfinite(candidate_norm) && candidate_norm < result.final_true_residual) {
    launch_copy(stream_, n, candidate, kx_);
    launch_copy(stream_, n, fg_w_, fg_v_[0]);
    launches_ += 2;
    result.final_true_residual = candidate_norm;
    result.recursive_residual = candidate_norm;
    result.recycle_accepted = 1;
  }
  (void)tol;
  return {};
}

// solve_fgmres (src/solver_krylov.cpp:1557-2650), same control flow: the
// single-reduction Arnoldi step on w = A z_j - v_j (shift 1, :35) with one
// batched reduction for the projections and |w|^2, the Pythagorean norm
// (single_reduction_fgmres_norm, :565-609) with its two fallbacks (discard
// the column and restart when the recurrence turns unsafe past column 0,
// explicit re-orthogonalisation at column 0 or a zero norm), Givens
// rotations, a true-residual audit of the candidate x + Z y in the spare
// basis slot every true_residual_interval iterations (and at a recursive
// convergence claim), and a restart from the true residual at cycle ends.
// Vectors stay on the device; the (restart+1) x restart Hessenberg system,
// its rotations and back substitution run on the host from one read-back of
// the column per iteration.
Status Solver::krylov_fgmres(const hfps_control& control, hfps_result& result,
                             double* history, uint32_t capacity) {
  const int n = nx_ * ny_ * nz_;
  const uint32_t restart = control.restart;
  const bool mixed = control.precision == HFPS_MIXED;
  const Level<double> A = l64_[0].view(neumann_);
  const double kShift = 1.0;
  const auto red = [&](int op) { return Reduce{d_scalars_, d_partials_, op}; };
  Status st = ensure_fgmres_storage(restart);
  if (!st) return st;
  // Recycle session as PressureVelocityCoupler selects it per corrector
  // (src/solver_piso.cpp:10410-10433).
  if (control.recycle != HFPS_RECYCLE_NONE) {
    st = ensure_recycle_storage();
    if (!st) return st;
  }
  const auto recycle_clear = [&]() {
    rc_capture_ = rc_guard_only_ = rc_cycle_active_ = rc_pending_ = false;
    rc_count_ = rc_oldest_ = 0;
  };
  switch (control.recycle) {
    case HFPS_RECYCLE_CAPTURE: recycle_clear(); rc_capture_ = true; break;
    case HFPS_RECYCLE_PROJECT:
      if (!rc_capture_ || rc_cycle_active_ || rc_pending_)
        return fail(HFPS_INVALID_PLAN, kDetailPlan, "projection without a capture session");
      rc_capture_ = false;
      rc_pending_ = true;
      break;
    case HFPS_RECYCLE_GUARD: recycle_clear(); rc_guard_only_ = true; break;
    default: recycle_clear(); break;
  }
  st = check(cudaMemsetAsync(d_scalars_, 0, sizeof(Scalars), stream_), "scalars");
  if (!st) return st;
  launch_norm2(stream_, n, kb_, red(kOpMisc));
  launches_ += 1;
  queue_norm(kb_);
  st = sync_scalars();
  if (!st) return st;
  if (h_scalars_->flags & 1) {
    result.termination = HFPS_NON_FINITE;
    return fail(HFPS_NUMERICAL_FAILURE, kDetailNumeric, "non-finite rhs");
  }
  const double bnorm = norm_value(h_scalars_->misc[0]);
  const double tol = std::max(control.absolute_tolerance,
                              control.relative_tolerance * bnorm);
  result.rhs_norm = bnorm;
  result.true_residual_limit = tol;
  if (bnorm == 0.0) {
    st = check(cudaMemsetAsync(kx_, 0, n * sizeof(double), stream_), "zero x");
    result.termination = HFPS_ZERO_RHS;
    return st;
  }
  std::vector<double*>& V = fg_v_;
  std::vector<double*>& Z = fg_z_;
  double* w = fg_w_;
  // compute_true_residual (:1071-1092): V_0 = b - A x and its norm.
  const auto true_residual = [&](const double* x, double* r, double& norm) -> Status {
    launch_residual_norm(stream_, A, x, kb_, r, red(kOpRecursive));
    launches_ += 1;
    ++result.operator_applies;
    queue_norm(r);
    Status s = sync_scalars();
    if (!s) return s;
    norm = norm_value(h_scalars_->rr);
    if (!std::isfinite(norm)) {
      result.termination = HFPS_NON_FINITE;
      return fail(HFPS_NUMERICAL_FAILURE, kDetailNumeric, "non-finite residual");
    }
    return {};
  };
  // dst/out = scale * (dst + sum_r s_r b_r), in chunks of kBasisChunk terms
  // (the per-cell accumulation order is that of one long loop).
  const auto basis_update = [&](const double* dst, double* const* b, const double* sc,
                                int count, double scale, bool scaled, double* out) {
    int done = 0;
    do {
      BasisRefs refs{};
      refs.count = std::min(kBasisChunk, count - done);
      for (int r = 0; r < refs.count; ++r) {
        refs.v[r] = b[done + r];
        refs.s[r] = sc[done + r];
      }
      const bool last = done + refs.count >= count;
      launch_basis_update(stream_, n, done == 0 ? dst : out, refs, scale, last && scaled, out);
      launches_ += 1;
      done += refs.count;
    } while (done < count);
  };
  // hcol[r] = V_r . w (r < count) and hcol[count] = w . w when `self`.
  const auto multidot = [&](int count, bool self) -> Status {
    int done = 0;
    const int total = count + (self ? 1 : 0);
    do {
      BasisRefs refs{};
      refs.count = std::min(kBasisChunk - (self ? 1 : 0), count - done);
      if (refs.count < 0) refs.count = 0;
      for (int r = 0; r < refs.count; ++r) refs.v[r] = V[done + r];
      const bool with_self = self && done + refs.count == count;
      launch_multidot(stream_, n, refs, w, with_self, d_scalars_->hcol + done,
                      red(kCounterMultidot));
      launches_ += 1;
      done += refs.count + (with_self ? 1 : 0);
    } while (done < total);
    Status s = sync_scalars();
    if (!s) return s;
    if (h_scalars_->flags & 1) {
      result.termination = HFPS_NON_FINITE;
      return fail(HFPS_NUMERICAL_FAILURE, kDetailNumeric, "non-finite Arnoldi projection");
    }
    return {};
  };

  double initial = 0.0;
  st = true_residual(kx_, V[0], initial);
  if (!st) return st;
  // reset_to_zero_initial_guess under the recycle guard (:1673-1686).
  if ((rc_capture_ || rc_guard_only_) && initial > bnorm) {
    st = check(cudaMemsetAsync(kx_, 0, n * sizeof(double), stream_), "zero seed");
    if (!st) return st;
    launch_copy(stream_, n, kb_, V[0]);
    launches_ += 1;
    initial = bnorm;
  }
  result.initial_true_residual = initial;
  result.final_true_residual = initial;
  result.recursive_residual = initial;
  if (initial <= tol) {
    rc_pending_ = false;
    result.termination = HFPS_CONVERGED;
    return {};
  }
  if (rc_pending_) {
    st = recycle_project(control, tol, result);
    if (!st) return st;
    if (result.recycle_accepted && result.final_true_residual <= tol) {
      result.termination = HFPS_CONVERGED;
      return {};
    }
  }
  const size_t rows = restart + 1;
  std::vector<double> h(rows * restart, 0.0), cs(restart, 0.0), sn(restart, 0.0),
      g(rows, 0.0), y(restart, 0.0), scales(rows, 0.0);
  uint32_t it = 0;
  const auto record = [&](double recursive) {
    result.recursive_residual = recursive;
    if (history != nullptr && it - 1 < capacity) {
      history[it - 1] = recursive;
      result.history_length = it;
    }
  };
  // Back substitution of the rotated Hessenberg system (:2471-2486).
  const auto solve_y = [&](int count) -> Status {
    for (int row = count - 1; row >= 0; --row) {
      double value = g[row];
      for (int upper = row + 1; upper < count; ++upper)
        value -= h[static_cast<size_t>(upper) * rows + row] * y[upper];
      const double divisor = h[static_cast<size_t>(row) * rows + row];
      if (divisor == 0.0 || !std::isfinite(divisor)) {
        result.termination = HFPS_BREAKDOWN;
        return fail(HFPS_NUMERICAL_FAILURE, kDetailBreakdown, "FGMRES breakdown");
      }
      y[row] = value / divisor;
      if (!std::isfinite(y[row])) {
        result.termination = HFPS_NON_FINITE;
        return fail(HFPS_NUMERICAL_FAILURE, kDetailNumeric, "non-finite FGMRES update");
      }
    }
    return {};
  };
  while (it < control.maximum_iterations) {
    if (rc_capture_) {
      // recycle_capture_cycle_start (src/solver_linear_state.cpp:857-895)
      launch_copy(stream_, n, kx_, rc_snapshot_);
      launches_ += 1;
      rc_cycle_active_ = true;
    }
    const double beta = result.final_true_residual;
    basis_update(V[0], nullptr, nullptr, 0, 1.0 / beta, true, V[0]);
    std::fill(g.begin(), g.end(), 0.0);
    g[0] = beta;
    bool restarted = false;
    for (uint32_t column = 0; column < restart && it < control.maximum_iterations; ++column) {
      // z_j = M v_j: the MG graph of this column's buffers, or the cold
      // path through the internal r/z buffers.
      if (policy_.preconditioner != HFPS_PRECONDITIONER_IC0) {
        st = mg_apply(mixed, V[column], Z[column]);
        if (!st) return st;
      } else {
        launch_copy(stream_, n, V[column], kr_);
        launches_ += 1;
        st = precondition(mixed);
        if (!st) return st;
        launch_copy(stream_, n, kz_, Z[column]);
        launches_ += 1;
      }
      ++result.preconditioner_applies;
      launch_operator_shift(stream_, A, Z[column], V[column], kShift, w);
      launches_ += 1;
      ++result.operator_applies;
      const int count = static_cast<int>(column) + 1;
      st = multidot(count, true);
      if (!st) return st;
      double* column_h = h.data() + static_cast<size_t>(column) * rows;
      for (int r = 0; r <= count; ++r) column_h[r] = h_scalars_->hcol[r];
      const double bar_norm = column_h[count];
      for (int r = 0; r < count; ++r) scales[r] = -column_h[r];
      double t = bar_norm;
      for (int r = 0; r < count; ++r) t = t - column_h[r] * column_h[r];
      if (!std::isfinite(t)) {
        result.termination = HFPS_NON_FINITE;
        return fail(HFPS_NUMERICAL_FAILURE, kDetailNumeric, "non-finite Arnoldi norm");
      }
      const bool unsafe = t < 0.0;
      double next_norm = unsafe ? 0.0 : std::sqrt(t);
      if (unsafe && column != 0) {
        // Discard the column and finish the cycle on the previous ones.
        ++it;
        result.iterations = it;
        st = solve_y(static_cast<int>(column));
        if (!st) return st;
        basis_update(kx_, Z.data(), y.data(), static_cast<int>(column), 1.0, false, kx_);
        double norm = 0.0;
        st = true_residual(kx_, V[0], norm);
        if (!st) return st;
        st = recycle_publish(kx_, result);
        if (!st) return st;
        result.final_true_residual = norm;
        record(norm);
        if (norm <= tol) {
          result.termination = HFPS_CONVERGED;
          return {};
        }
        if (it == control.maximum_iterations) break;
        std::fill(h.begin(), h.end(), 0.0);
        std::fill(cs.begin(), cs.end(), 0.0);
        std::fill(sn.begin(), sn.end(), 0.0);
        std::fill(g.begin(), g.end(), 0.0);
        std::fill(y.begin(), y.end(), 0.0);
        restarted = true;
        break;
      }
      bool explicit_orth = false;
      if (unsafe || next_norm == 0.0) {
        // Second orthogonalisation pass, measured stably (:2330-2395).
        basis_update(w, V.data(), scales.data(), count, 1.0, false, w);
        st = multidot(count, false);
        if (!st) return st;
        for (int r = 0; r < count; ++r) {
          const double c = h_scalars_->hcol[r];
          column_h[r] += c;
          scales[r] = -c;
        }
        basis_update(w, V.data(), scales.data(), count, 1.0, false, w);
        launch_norm2(stream_, n, w, red(kOpMisc));
        launches_ += 1;
        st = sync_scalars();
        if (!st) return st;
        next_norm = std::sqrt(h_scalars_->misc[0]);
        explicit_orth = true;
      }
      column_h[column] += kShift;
      column_h[column + 1] = next_norm;
      for (uint32_t r = 0; r < column; ++r) {
        double& upper = h[static_cast<size_t>(column) * rows + r];
        double& lower = h[static_cast<size_t>(column) * rows + r + 1];
        const double rotated = cs[r] * upper + sn[r] * lower;
        lower = -sn[r] * upper + cs[r] * lower;
        upper = rotated;
      }
      double& diagonal = h[static_cast<size_t>(column) * rows + column];
      double& subdiagonal = h[static_cast<size_t>(column) * rows + column + 1];
      const double rotation_norm = std::hypot(diagonal, subdiagonal);
      if (!(rotation_norm > 0.0) || !std::isfinite(rotation_norm)) {
        result.termination = HFPS_BREAKDOWN;
        return fail(HFPS_NUMERICAL_FAILURE, kDetailBreakdown, "FGMRES rotation breakdown");
      }
      cs[column] = diagonal / rotation_norm;
      sn[column] = subdiagonal / rotation_norm;
      diagonal = rotation_norm;
      subdiagonal = 0.0;
      g[column + 1] = -sn[column] * g[column];
      g[column] = cs[column] * g[column];
      ++it;
      result.iterations = it;
      const double recursive = std::abs(g[column + 1]);
      record(recursive);
      const bool happy = next_norm == 0.0;
      const bool cycle_end = happy || column + 1 == restart || it == control.maximum_iterations;
      const bool verify = happy || recursive <= tol ||
                          it % control.true_residual_interval == 0 || cycle_end;
      if (!cycle_end) {
        // v_{j+1} = (w - sum h_r v_r) / |.|, one fused pass.
        if (explicit_orth) basis_update(w, nullptr, nullptr, 0, 1.0 / next_norm, true, V[column + 1]);
        else basis_update(w, V.data(), scales.data(), count, 1.0 / next_norm, true, V[column + 1]);
      }
      if (!verify) continue;
      st = solve_y(count);
      if (!st) return st;
      if (!cycle_end) {
        // Audit the candidate x + Z y in the unused last basis slot.
        double* trial = V[restart];
        basis_update(kx_, Z.data(), y.data(), count, 1.0, false, trial);
        double audited = 0.0;
        st = true_residual(trial, w, audited);
        if (!st) return st;
        result.final_true_residual = audited;
        if (audited <= tol) {
          st = recycle_publish(trial, result);
          if (!st) return st;
          launch_copy(stream_, n, trial, kx_);
          launches_ += 1;
          result.termination = HFPS_CONVERGED;
          return {};
        }
        continue;
      }
      basis_update(kx_, Z.data(), y.data(), count, 1.0, false, kx_);
      double norm = 0.0;
      st = true_residual(kx_, V[0], norm);
      if (!st) return st;
      st = recycle_publish(kx_, result);
      if (!st) return st;
      result.final_true_residual = norm;
      result.recursive_residual = norm;
      if (norm <= tol) {
        result.termination = HFPS_CONVERGED;
        return {};
      }
      if (it == control.maximum_iterations) break;
      if (happy) {
        const double guard = 64.0 * std::numeric_limits<double>::epsilon() * std::max(beta, tol);
        if (!(norm + guard < beta)) {
          result.termination = HFPS_BREAKDOWN;
          return fail(HFPS_NUMERICAL_FAILURE, kDetailBreakdown, "FGMRES stagnation");
        }
      }
      restarted = true;
      break;
    }
    if (!restarted) break;
  }
  result.termination = HFPS_MAXIMUM_ITERATIONS;
  return fail(HFPS_REJECTED_STEP, kDetailBreakdown, "maximum iterations reached");
}

// solve_bicgstab (src/solver_krylov.cpp:2651-3090) with the default
// control (no bounded recurrence, no maximum norm, no best-iterate
// retention): the early exit when |s| meets the tolerance, omega from the
// (t.s, t.t) pair, a true residual every true_residual_interval iterations
// and at a recursive claim, and a fresh start (r_hat = r) after every
// verification that does not converge.  The preconditioner runs on the
// kr_ -> kz_ buffers; the BiCGSTAB vectors live in the FGMRES basis block.
Status Solver::krylov_bicgstab(const hfps_control& control, hfps_result& result,
                               double* history, uint32_t capacity) {
  const int n = nx_ * ny_ * nz_;
  const Level<double> A = l64_[0].view(neumann_);
  const auto red = [&](int op) { return Reduce{d_scalars_, d_partials_, op}; };
  Status st = ensure_fgmres_storage(4);
  if (!st) return st;
  double* rh = fg_v_[0];
  double* p = fg_v_[1];
  double* sv = fg_v_[2];
  double* ph = fg_v_[3];
  double* sh = fg_v_[4];
  double* v = fg_z_[0];
  double* t = fg_z_[1];
  double* r = fg_z_[2];
  st = check(cudaMemsetAsync(d_scalars_, 0, sizeof(Scalars), stream_), "scalars");
  if (!st) return st;
  launch_norm2(stream_, n, kb_, red(kOpMisc));
  launches_ += 1;
  queue_norm(kb_);
  st = sync_scalars();
  if (!st) return st;
  if (h_scalars_->flags & 1) {
    result.termination = HFPS_NON_FINITE;
    return fail(HFPS_NUMERICAL_FAILURE, kDetailNumeric, "non-finite rhs");
  }
  const double bnorm = norm_value(h_scalars_->misc[0]);
  const double tol = std::max(control.absolute_tolerance, control.relative_tolerance * bnorm);
  result.rhs_norm = bnorm;
  result.true_residual_limit = tol;
  if (bnorm == 0.0) {
    st = check(cudaMemsetAsync(kx_, 0, n * sizeof(double), stream_), "zero x");
    result.termination = HFPS_ZERO_RHS;
    return st;
  }
  const auto true_residual = [&](double& norm) -> Status {
    launch_residual_norm(stream_, A, kx_, kb_, r, red(kOpRecursive));
    launches_ += 1;
    ++result.operator_applies;
    queue_norm(r);
    Status s2 = sync_scalars();
    if (!s2) return s2;
    norm = norm_value(h_scalars_->rr);
    if (!std::isfinite(norm)) {
      result.termination = HFPS_NON_FINITE;
      return fail(HFPS_NUMERICAL_FAILURE, kDetailNumeric, "non-finite residual");
    }
    return {};
  };
  const auto dots = [&](std::initializer_list<const double*> left, const double* w) -> Status {
    BasisRefs refs{};
    refs.count = 0;
    for (const double* l : left) refs.v[refs.count++] = l;
    launch_multidot(stream_, n, refs, w, false, d_scalars_->hcol, red(kCounterMultidot));
    launches_ += 1;
    return sync_scalars();
  };
  const auto precondition_into = [&](const double* in, double* out) -> Status {
    launch_copy(stream_, n, in, kr_);
    launches_ += 1;
    Status s2 = precondition(false);
    if (!s2) return s2;
    ++result.preconditioner_applies;
    launch_copy(stream_, n, kz_, out);
    launches_ += 1;
    return {};
  };
  const auto breakdown = [&]() {
    result.termination = HFPS_BREAKDOWN;
    return fail(HFPS_NUMERICAL_FAILURE, kDetailBreakdown, "BiCGSTAB breakdown");
  };
  double initial = 0.0;
  st = true_residual(initial);
  if (!st) return st;
  result.initial_true_residual = initial;
  result.final_true_residual = initial;
  result.recursive_residual = initial;
  if (initial <= tol) {
    result.termination = HFPS_CONVERGED;
    return {};
  }
  launch_copy(stream_, n, r, rh);
  launches_ += 1;
  double rho_prev = 1.0, alpha = 1.0, omega = 1.0;
  bool fresh = true;
  uint32_t it = 0;
  const auto record = [&](double value) {
    result.recursive_residual = value;
    if (history != nullptr && it - 1 < capacity) {
      history[it - 1] = value;
      result.history_length = it;
    }
  };
  while (it < control.maximum_iterations) {
    st = dots({rh}, r);
    if (!st) return st;
    const double rho = h_scalars_->hcol[0];
    if (rho == 0.0 || !std::isfinite(rho)) return breakdown();
    if (fresh) {
      launch_copy(stream_, n, r, p);
      launches_ += 1;
    } else {
      if (omega == 0.0 || !std::isfinite(omega)) return breakdown();
      const double beta = (rho / rho_prev) * (alpha / omega);
      launch_bicg_direction(stream_, n, p, r, v, beta, omega);
      launches_ += 1;
    }
    st = precondition_into(p, ph);
    if (!st) return st;
    launch_level_apply<double>(stream_, A, ph, v);
    launches_ += 1;
    ++result.operator_applies;
    st = dots({rh}, v);
    if (!st) return st;
    const double denominator = h_scalars_->hcol[0];
    if (denominator == 0.0 || !std::isfinite(denominator)) return breakdown();
    alpha = rho / denominator;
    launch_bicg_intermediate(stream_, n, sv, r, v, alpha, red(kOpMisc));
    launches_ += 1;
    queue_norm(sv);
    st = sync_scalars();
    if (!st) return st;
    const double s_norm = norm_value(h_scalars_->misc[0]);
    if (!std::isfinite(s_norm)) {
      result.termination = HFPS_NON_FINITE;
      return fail(HFPS_NUMERICAL_FAILURE, kDetailNumeric, "non-finite BiCGSTAB residual");
    }
    if (s_norm <= tol) {
      BasisRefs one{};
      one.count = 1;
      one.v[0] = ph;
      one.s[0] = alpha;
      launch_basis_update(stream_, n, kx_, one, 1.0, false, kx_);
      launches_ += 1;
      ++it;
      result.iterations = it;
      double norm = 0.0;
      st = true_residual(norm);
      if (!st) return st;
      result.final_true_residual = norm;
      record(norm);
      if (norm <= tol) {
        result.termination = HFPS_CONVERGED;
        return {};
      }
      if (it == control.maximum_iterations) break;
      launch_copy(stream_, n, r, rh);
      launches_ += 1;
      rho_prev = 1.0; alpha = 1.0; omega = 1.0; fresh = true;
      continue;
    }
    st = precondition_into(sv, sh);
    if (!st) return st;
    launch_level_apply<double>(stream_, A, sh, t);
    launches_ += 1;
    ++result.operator_applies;
    st = dots({sv, t}, t);
    if (!st) return st;
    const double ts = h_scalars_->hcol[0], tt = h_scalars_->hcol[1];
    if (!(tt > 0.0) || !std::isfinite(ts) || !std::isfinite(tt)) return breakdown();
    omega = ts / tt;
    if (omega == 0.0 || !std::isfinite(omega)) return breakdown();
    launch_bicg_update(stream_, n, kx_, ph, sh, r, sv, t, alpha, omega, red(kOpRecursive));
    launches_ += 1;
    queue_norm(r);
    ++it;
    result.iterations = it;
    st = sync_scalars();
    if (!st) return st;
    const double recursive = norm_value(h_scalars_->rr);
    if (!std::isfinite(recursive)) {
      result.termination = HFPS_NON_FINITE;
      return fail(HFPS_NUMERICAL_FAILURE, kDetailNumeric, "non-finite BiCGSTAB residual");
    }
    record(recursive);
    const bool verify = recursive <= tol || it % control.true_residual_interval == 0 ||
                        it == control.maximum_iterations;
    if (verify) {
      double norm = 0.0;
      st = true_residual(norm);
      if (!st) return st;
      result.final_true_residual = norm;
      result.recursive_residual = norm;
      if (norm <= tol) {
        result.termination = HFPS_CONVERGED;
        return {};
      }
      if (it == control.maximum_iterations) break;
      launch_copy(stream_, n, r, rh);
      launches_ += 1;
      rho_prev = 1.0; alpha = 1.0; omega = 1.0; fresh = true;
      continue;
    }
    rho_prev = rho;
    fresh = false;
  }
  result.termination = HFPS_MAXIMUM_ITERATIONS;
  return fail(HFPS_REJECTED_STEP, kDetailBreakdown, "maximum iterations reached");
}

Status Solver::solve(const double* rhs, double* solution, int memory,
                     const hfps_control& control, hfps_result& result,
                     double* history, uint32_t capacity) {
  const auto begin = std::chrono::steady_clock::now();
  result = hfps_result{};
  result.levels = static_cast<uint32_t>(l64_.size());
  result.termination = HFPS_TERMINATION_INVALID_PLAN;
  if (!coefficients_ready_)
    return fail(HFPS_INVALID_PLAN, kDetailPlan, "coefficients not set");
  if (rhs == nullptr || solution == nullptr || control.maximum_iterations == 0 ||
      control.true_residual_interval == 0 ||
      !std::isfinite(control.relative_tolerance) ||
      !std::isfinite(control.absolute_tolerance) ||
      control.relative_tolerance < 0.0 || control.absolute_tolerance < 0.0 ||
      (control.relative_tolerance == 0.0 && control.absolute_tolerance == 0.0) ||
      (control.precision != HFPS_FP64 && control.precision != HFPS_MIXED) ||
      (control.norm != HFPS_NORM_PLAIN && control.norm != HFPS_NORM_SCALED) ||
      control.recycle < HFPS_RECYCLE_NONE || control.recycle > HFPS_RECYCLE_GUARD ||
      (control.algorithm == HFPS_PCG && control.recycle != HFPS_RECYCLE_NONE) ||
      (control.algorithm != HFPS_FGMRES && control.recycle != HFPS_RECYCLE_NONE) ||
      !((control.algorithm == HFPS_PCG && control.restart == 0 &&
         (policy_.unit_linear || policy_.preconditioner == HFPS_PRECONDITIONER_IC0)) ||
        (control.algorithm == HFPS_BICGSTAB && control.restart == 0 &&
         policy_.preconditioner == HFPS_PRECONDITIONER_IC0) ||
        (control.algorithm == HFPS_FGMRES && control.restart >= 1 &&
         control.restart <= static_cast<uint32_t>(kMaxFgmresRestart))))
    return fail(HFPS_INVALID_PLAN, kDetailPlan, "invalid solve control");
  const size_t n = static_cast<size_t>(nx_) * ny_ * nz_;
  Status st = copy_in(kb_, rhs, n, memory);
  if (st) st = copy_in(kx_, solution, n, memory);
  if (!st) return st;
  launches_ = 0;
  scaled_norm_ = control.norm == HFPS_NORM_SCALED;
  st = control.algorithm == HFPS_FGMRES     ? krylov_fgmres(control, result, history, capacity)
       : control.algorithm == HFPS_BICGSTAB ? krylov_bicgstab(control, result, history, capacity)
                                            : krylov_pcg(control, result, history, capacity);
  result.kernel_launches = launches_;
  if (st) {
    st = copy_out(solution, kx_, n, memory);
    if (st) st = check(cudaStreamSynchronize(stream_), "solution copy");
  }
  result.status = st.code;
  result.detail = st.detail;
  result.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - begin).count();
  return st;
}

Status Solver::apply_operator(const double* x, double* y, int memory) {
  if (!coefficients_ready_) return fail(HFPS_INVALID_PLAN, kDetailPlan, "coefficients not set");
  const size_t n = static_cast<size_t>(nx_) * ny_ * nz_;
  Status st = copy_in(kp_, x, n, memory);
  if (!st) return st;
  launch_level_apply<double>(stream_, l64_[0].view(neumann_), kp_, kap_);
  st = copy_out(y, kap_, n, memory);
  if (!st) return st;
  return check(cudaStreamSynchronize(stream_), "operator");
}

Status Solver::apply_preconditioner(const double* r, double* z, int memory,
                                    int precision) {
  if (!coefficients_ready_) return fail(HFPS_INVALID_PLAN, kDetailPlan, "coefficients not set");
  const size_t n = static_cast<size_t>(nx_) * ny_ * nz_;
  Status st = copy_in(kr_, r, n, memory);
  if (!st) return st;
  st = check(cudaMemsetAsync(d_scalars_, 0, sizeof(Scalars), stream_), "scalars");
  if (!st) return st;
  st = precondition(precision == HFPS_MIXED);
  if (!st) return st;
  st = copy_out(z, kz_, n, memory);
  if (!st) return st;
  return sync_scalars();
}

Status Solver::adjoint(const double* solution, const double* dl_dp,
                       double* lambda, double* gx, double* gy, double* gz,
                       int memory, const hfps_control& control,
                       hfps_result& result) {
  if (!coefficients_ready_) return fail(HFPS_INVALID_PLAN, kDetailPlan, "coefficients not set");
  if (solution == nullptr || dl_dp == nullptr)
    return fail(HFPS_INVALID_PLAN, kDetailPlan, "null adjoint input");
  const size_t n = static_cast<size_t>(nx_) * ny_ * nz_;
  // A is symmetric (SPD operator class, src/solver_ibm_pressure.cpp:242-245),
  // so A^T lambda = dL/dp is the forward solve with rhs dL/dp masked to the
  // fluid rows (solid rows are identities with zero rhs).
  Status st = copy_in(kz_, dl_dp, n, memory);
  if (!st) return st;
  launch_adjoint_source(stream_, static_cast<int>(n), kz_, d_active_, kb_);
  st = check(cudaMemsetAsync(kx_, 0, n * sizeof(double), stream_), "lambda init");
  if (!st) return st;
  const auto begin = std::chrono::steady_clock::now();
  result = hfps_result{};
  result.levels = static_cast<uint32_t>(l64_.size());
  launches_ = 0;
  st = krylov_pcg(control, result, nullptr, 0);
  result.kernel_launches = launches_ + 1;
  result.status = st.code;
  result.detail = st.detail;
  if (!st) return st;
  // lambda now in kx_; p into kp_ (device copy of the forward solution).
  st = copy_in(kp_, solution, n, memory);
  if (!st) return st;
  const DeviceLevel<double>& L0 = l64_[0];
  const size_t nf[3] = {static_cast<size_t>(L0.faces_x()), static_cast<size_t>(L0.faces_y()),
                        static_cast<size_t>(L0.faces_z())};
  // Gradient staging: reuse the user coefficient staging buffers.
  launch_face_gradients(stream_, L0.view(neumann_), kx_, kp_, nullptr, nullptr, nullptr,
                        user_[1], user_[2], user_[3]);
  if (lambda != nullptr) st = copy_out(lambda, kx_, n, memory);
  if (st && gx != nullptr) st = copy_out(gx, user_[1], nf[0], memory);
  if (st && gy != nullptr) st = copy_out(gy, user_[2], nf[1], memory);
  if (st && gz != nullptr) st = copy_out(gz, user_[3], nf[2], memory);
  if (st) st = check(cudaStreamSynchronize(stream_), "adjoint");
  result.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - begin).count();
  return st;
}

Status Solver::level_coefficients(int level, double* diag, double* fx,
                                  double* fy, double* fz, double* volume) {
  if (level < 0 || level >= level_count())
    return fail(HFPS_INVALID_PLAN, kDetailPlan, "level out of range");
  const DeviceLevel<double>& L = l64_[level];
  Status st{};
  if (diag) st = copy_out(diag, L.diag, L.cells(), HFPS_HOST);
  if (st && fx) st = copy_out(fx, L.fx, L.faces_x(), HFPS_HOST);
  if (st && fy) st = copy_out(fy, L.fy, L.faces_y(), HFPS_HOST);
  if (st && fz) st = copy_out(fz, L.fz, L.faces_z(), HFPS_HOST);
  if (st && volume) st = copy_out(volume, volume_[level], L.cells(), HFPS_HOST);
  if (!st) return st;
  return check(cudaStreamSynchronize(stream_), "level coefficients");
}

}  // namespace hfps

namespace hfps {

// Algorithmic bytes use w = sizeof(T) per cell-stream: stencil operand set
// x, D, fx, fy, fz (5w), plus what each kernel writes or reads besides.
Status Solver::profile_kernel(int kernel, int repetitions, double* ms,
                              double* bytes) {
  if (!coefficients_ready_) return fail(HFPS_INVALID_PLAN, kDetailPlan, "coefficients not set");
  if (repetitions <= 0 || ms == nullptr || bytes == nullptr)
    return fail(HFPS_INVALID_PLAN, kDetailPlan, "invalid profile request");
  const int n = nx_ * ny_ * nz_;
  const double cells = static_cast<double>(n);
  DeviceLevel<double>& L0 = l64_[0];
  DeviceLevel<float>& F0 = l32_[0];
  const Level<double> A = L0.view(neumann_);
  if (kernel == HFPS_KERNEL_SMOOTH_FP32 || kernel == HFPS_KERNEL_MG_MIXED) {
    Status st = refresh_mixed();
    if (!st) return st;
  }
  const auto red = [&](int op) { return Reduce{d_scalars_, d_partials_, op}; };
  Status st = check(cudaMemsetAsync(d_scalars_, 0, sizeof(Scalars), stream_), "scalars");
  if (!st) return st;
  // Deterministic finite operands.
  launch_copy(stream_, n, kb_, kr_);
  launch_copy(stream_, n, kb_, kp_);
  const auto level0_smoother = [&](auto& levels) -> double {
    auto& L = levels[0];
    using T = typename std::remove_reference<decltype(L)>::type::value_type;
    const Level<T> view = L.view(neumann_);
    if (L.line_mask != 0) {
      int axis = 0;
      while (!(L.line_mask & (1 << axis))) ++axis;
      launch_line_pass<T>(stream_, view, L.x, L.b, L.lfac[axis], L.r, axis, 0, L.split);
      return 28.0 / 8.0 * sizeof(T);
    }
    if (L.chebyshev) {
      launch_chebyshev_stage<T>(stream_, view, L.x, L.b, L.r, L.t, T(0.5), T(0.5), 0);
      return 72.0 / 8.0 * sizeof(T);
    }
    launch_rb_color<T>(stream_, view, L.x, L.b, 0);
    return 28.0 / 8.0 * sizeof(T);
  };
  cudaEvent_t start, stop;
  cudaEventCreate(&start);
  cudaEventCreate(&stop);
  double per_cell = 0.0;
  const auto one = [&]() {
    switch (kernel) {
      case HFPS_KERNEL_OPERATOR:
        launch_spmv_dot(stream_, A, kp_, kap_, red(kOpMisc), tiled_stencil_);
        per_cell = 48.0;
        break;
      case HFPS_KERNEL_SMOOTH_FP64:
        per_cell = level0_smoother(l64_);
        break;
      case HFPS_KERNEL_SMOOTH_FP32:
        per_cell = level0_smoother(l32_);
        break;
      case HFPS_KERNEL_RESTRICT_FP64:
        launch_defect_restrict<double>(stream_, A, L0.x, L0.b, l64_[1].view(neumann_),
                                       l64_[1].b, l64_[1].x, L0.coarsen_mask, L0.split,
                                       l64_[1].split);
        per_cell = 48.0 + 2.0 * 8.0 / (l64_[0].cells() / static_cast<double>(l64_[1].cells()));
        break;
      case HFPS_KERNEL_PROLONG_FP64:
        launch_prolongate<double>(stream_, A, L0.x, l64_[1].view(neumann_), l64_[1].x,
                                  L0.coarsen_mask, L0.split, l64_[1].split);
        per_cell = 16.0 + 1.0 + 8.0 / (l64_[0].cells() / static_cast<double>(l64_[1].cells()));
        break;
      case HFPS_KERNEL_PCG_UPDATE:
        launch_pcg_update(stream_, n, kx_, kp_, kr_, kap_, red(kOpMisc));
        per_cell = 48.0;
        break;
      case HFPS_KERNEL_RESIDUAL:
        launch_residual_norm(stream_, A, kp_, kb_, kr_, red(kOpMisc));
        per_cell = 56.0;
        break;
      case HFPS_KERNEL_MG_FP64:
      case HFPS_KERNEL_MG_MIXED:
        mg_apply(kernel == HFPS_KERNEL_MG_MIXED);
        per_cell = 0.0;
        break;
      default:
        per_cell = -1.0;
        break;
    }
  };
  one();  // warm-up (also builds a graph when needed)
  if (per_cell < 0.0) {
    cudaEventDestroy(start);
    cudaEventDestroy(stop);
    return fail(HFPS_INVALID_PLAN, kDetailPlan, "unknown kernel class");
  }
  cudaEventRecord(start, stream_);
  for (int r = 0; r < repetitions; ++r) one();
  cudaEventRecord(stop, stream_);
  st = check(cudaEventSynchronize(stop), "profile");
  float elapsed = 0.0f;
  cudaEventElapsedTime(&elapsed, start, stop);
  cudaEventDestroy(start);
  cudaEventDestroy(stop);
  (void)F0;
  if (!st) return st;
  *ms = static_cast<double>(elapsed) / repetitions;
  *bytes = per_cell * cells;
  return check(cudaGetLastError(), "profile kernels");
}

}  // namespace hfps
