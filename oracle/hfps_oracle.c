/*
 * CPU restatement of the reference pressure solve -- TEST INFRASTRUCTURE.
 *
 * Used only by tests/, __graft_entry__.smoke() and bench.py's CPU baseline
 * leg, as the checker.  Never linked into the product library.
 *
 * Each function cites the reference code it restates (paths relative to
 * versions/v0.4 of the reference).  Arithmetic is written in the same
 * order as the reference so that the compiled reference agrees with it to
 * the last few ulps; the one deliberate option is the line-smoother order:
 * line_order 0 is the reference's lexicographic line Gauss-Seidel
 * (src/solver_mg.cpp:3352-3539), line_order 1 the zebra (two-colour by
 * line) order the CUDA path uses.
 */
#include "hfps_oracle.h"

#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define MAX_LEVELS 32
#define AXIS_X 1
#define AXIS_Y 2
#define AXIS_Z 4

enum { BC_DIRICHLET = 0, BC_NEUMANN = 1 };
enum { TERM_CONVERGED = 0, TERM_ZERO_RHS = 1, TERM_MAXIMUM = 2,
       TERM_BREAKDOWN = 3, TERM_NON_FINITE = 4 };

typedef struct {
  int n[3];
  int coarsen_mask;
  int line_mask;
  int chebyshev;
  size_t cells, fxn, fyn, fzn;
  double *diag, *fx, *fy, *fz, *vol;
  double *x, *b, *r, *t;
} level_t;

typedef struct {
  int n[3];
  int bc[6];
  double* faces[3];
  double *diag0, *fx0, *fy0, *fz0; /* caller coefficients (unmasked) */
  unsigned char* active;           /* NULL = all fluid */
  int levels;
  level_t lv[MAX_LEVELS];
  int smoother, cycle, pre, post, coarse_sweeps, unit_linear, line_order;
  int max_levels, min_extent;
  double cheb_fraction, anisotropy, shortcut_ratio;
  int diagonal_shortcut;
  double* work[6];
  /* FGMRES subspace recycling across solves (SolverWorkspace recycle state,
   * src/solver_linear_state.cpp:735-1037): a ring of up to RECYCLE_MAX
   * cycle corrections, oldest first from rc_oldest, and the cycle-start
   * snapshot of x. */
  int rc_capture, rc_guard_only, rc_cycle_active, rc_pending;
  int rc_count, rc_oldest;
  double* rc_ring[4];
  double* rc_snapshot;
  double* rc_image[4]; /* projection scratch: A d_i */
  /* Cold-path preconditioner (ColdPressureIccg / ColdPressureDilu,
   * src/solver_iccg.hpp:224-293, src/solver_cold.hpp:484-560): 0 the MG
   * plan, 1 diagonal IC(0) in the reference's lexicographic order (the two
   * classes coincide on the symmetric pressure rows). */
  int pc_kind;
  double* dic_diag;   /* decorated row diagonal */
  double* dic_nb;     /* 6 couplings per row: x-, x+, y-, y+, z-, z+ */
  double* dic_inv;    /* inverse pivots */
} oracle_t;

static size_t idx(const int* n, int i, int j, int k) {
  return (size_t)i + (size_t)n[0] * ((size_t)j + (size_t)n[1] * (size_t)k);
}
static size_t fidx_x(const int* n, int i, int j, int k) {
  return (size_t)i + (size_t)(n[0] + 1) * ((size_t)j + (size_t)n[1] * (size_t)k);
}
static size_t fidx_y(const int* n, int i, int j, int k) {
  return (size_t)i + (size_t)n[0] * ((size_t)j + (size_t)(n[1] + 1) * (size_t)k);
}
static size_t fidx_z(const int* n, int i, int j, int k) {
  return (size_t)i + (size_t)n[0] * ((size_t)j + (size_t)n[1] * (size_t)k);
}

/* ------------------------------------------------------------------ */
/* Level shapes: strategy_mask + coarsen_axis                          */
/* (src/solver_mg_workspace.cpp:113-199, 317-452)                      */
/* ------------------------------------------------------------------ */
static int strategy_mask(oracle_t* o, int* line_mask) {
  double mn[3], mx[3], rep[3];
  for (int a = 0; a < 3; ++a) {
    mn[a] = INFINITY;
    mx[a] = 0.0;
    rep[a] = 0.0;
    for (int c = 0; c < o->n[a]; ++c) {
      const double w = o->faces[a][c + 1] - o->faces[a][c];
      if (w < mn[a]) mn[a] = w;
      if (w > mx[a]) mx[a] = w;
      rep[a] += w;
    }
    rep[a] /= (double)o->n[a];
  }
  double largest = rep[0];
  if (rep[1] > largest) largest = rep[1];
  if (rep[2] > largest) largest = rep[2];
  *line_mask = 0;
  const int masks[3] = {AXIS_X, AXIS_Y, AXIS_Z};
  for (int a = 0; a < 3; ++a) {
    const int internal = mn[a] > 0.0 && mx[a] / mn[a] >= o->anisotropy;
    const int cross = rep[a] > 0.0 && largest / rep[a] >= o->anisotropy;
    if (internal || cross) *line_mask |= masks[a];
  }
  const int all = AXIS_X | AXIS_Y | AXIS_Z;
  if ((*line_mask & (*line_mask - 1)) != 0) return all;
  const int candidate = all & ~*line_mask;
  return candidate == 0 ? all : candidate;
}

static int build_shapes(oracle_t* o) {
  int line_mask = 0;
  const int preferred = strategy_mask(o, &line_mask);
  int g[3] = {o->n[0], o->n[1], o->n[2]};
  o->levels = 0;
  for (int l = 0; l < o->max_levels; ++l) {
    level_t* L = &o->lv[o->levels++];
    memset(L, 0, sizeof(*L));
    L->n[0] = g[0];
    L->n[1] = g[1];
    L->n[2] = g[2];
    L->line_mask = line_mask;
    int mask = 0;
    int next[3] = {g[0], g[1], g[2]};
    for (int a = 0; a < 3; ++a) {
      if ((preferred & (1 << a)) && g[a] > o->min_extent) {
        mask |= 1 << a;
        next[a] = (g[a] + 1) / 2;
      }
    }
    L->coarsen_mask = mask;
    if (mask == 0 || o->levels == o->max_levels) break;
    g[0] = next[0];
    g[1] = next[1];
    g[2] = next[2];
  }
  if (o->levels < 2) return -1;
  for (int l = 0; l < o->levels; ++l) {
    level_t* L = &o->lv[l];
    /* build_levels: Chebyshev on every non-coarsest level without a line
     * mask (src/solver_mg.cpp:1060-1073). */
    L->chebyshev = l + 1 < o->levels && L->line_mask == 0 && o->smoother == 1;
    L->cells = (size_t)L->n[0] * L->n[1] * L->n[2];
    L->fxn = (size_t)(L->n[0] + 1) * L->n[1] * L->n[2];
    L->fyn = (size_t)L->n[0] * (L->n[1] + 1) * L->n[2];
    L->fzn = (size_t)L->n[0] * L->n[1] * (L->n[2] + 1);
    L->diag = calloc(L->cells, sizeof(double));
    L->vol = calloc(L->cells, sizeof(double));
    L->fx = calloc(L->fxn, sizeof(double));
    L->fy = calloc(L->fyn, sizeof(double));
    L->fz = calloc(L->fzn, sizeof(double));
    L->x = calloc(L->cells, sizeof(double));
    L->b = calloc(L->cells, sizeof(double));
    L->r = calloc(L->cells, sizeof(double));
    L->t = calloc(L->cells, sizeof(double));
    if (!L->diag || !L->vol || !L->fx || !L->fy || !L->fz || !L->x || !L->b ||
        !L->r || !L->t)
      return -2;
  }
  return 0;
}

/* ------------------------------------------------------------------ */
/* Coefficients: copy_finest_coefficients + build_coarse_coefficients  */
/* (src/solver_mg.cpp:1469-1570, 1706-1963)                            */
/* ------------------------------------------------------------------ */
static int cell_active(const oracle_t* o, int i, int j, int k) {
  return o->active == NULL || o->active[idx(o->n, i, j, k)] != 0;
}

/* Face activity: a face is active iff every adjacent cell is active. */
static double face_act(const oracle_t* o, int axis, int i, int j, int k) {
  if (o->active == NULL) return 1.0;
  int lo[3] = {i, j, k};
  int hi[3] = {i, j, k};
  lo[axis] -= 1;
  const int n = o->n[axis];
  int ok = 1;
  if (lo[axis] >= 0) ok &= cell_active(o, lo[0], lo[1], lo[2]);
  if (hi[axis] < n) ok &= cell_active(o, hi[0], hi[1], hi[2]);
  return ok ? 1.0 : 0.0;
}

static void copy_finest(oracle_t* o) {
  level_t* L = &o->lv[0];
  const int* n = L->n;
  for (int k = 0; k < n[2]; ++k)
    for (int j = 0; j < n[1]; ++j)
      for (int i = 0; i < n[0]; ++i) {
        const size_t c = idx(n, i, j, k);
        L->diag[c] = o->diag0[c];
        L->vol[c] = (o->faces[0][i + 1] - o->faces[0][i]) *
                    (o->faces[1][j + 1] - o->faces[1][j]) *
                    (o->faces[2][k + 1] - o->faces[2][k]);
        if (!cell_active(o, i, j, k)) L->vol[c] = 0.0;
      }
  for (int k = 0; k < n[2]; ++k)
    for (int j = 0; j < n[1]; ++j)
      for (int i = 0; i <= n[0]; ++i) {
        const size_t f = fidx_x(n, i, j, k);
        L->fx[f] = o->fx0[f] * face_act(o, 0, i, j, k);
      }
  for (int k = 0; k < n[2]; ++k)
    for (int j = 0; j <= n[1]; ++j)
      for (int i = 0; i < n[0]; ++i) {
        const size_t f = fidx_y(n, i, j, k);
        L->fy[f] = o->fy0[f] * face_act(o, 1, i, j, k);
      }
  for (int k = 0; k <= n[2]; ++k)
    for (int j = 0; j < n[1]; ++j)
      for (int i = 0; i < n[0]; ++i) {
        const size_t f = fidx_z(n, i, j, k);
        L->fz[f] = o->fz0[f] * face_act(o, 2, i, j, k);
      }
  if (o->active == NULL) return;
  for (int k = 0; k < n[2]; ++k)
    for (int j = 0; j < n[1]; ++j)
      for (int i = 0; i < n[0]; ++i) {
        const size_t c = idx(n, i, j, k);
        if (!cell_active(o, i, j, k)) {
          L->diag[c] = 1.0;
          continue;
        }
        const double original =
            o->fx0[fidx_x(n, i, j, k)] + o->fx0[fidx_x(n, i + 1, j, k)] +
            o->fy0[fidx_y(n, i, j, k)] + o->fy0[fidx_y(n, i, j + 1, k)] +
            o->fz0[fidx_z(n, i, j, k)] + o->fz0[fidx_z(n, i, j, k + 1)];
        const double act =
            L->fx[fidx_x(n, i, j, k)] + L->fx[fidx_x(n, i + 1, j, k)] +
            L->fy[fidx_y(n, i, j, k)] + L->fy[fidx_y(n, i, j + 1, k)] +
            L->fz[fidx_z(n, i, j, k)] + L->fz[fidx_z(n, i, j, k + 1)];
        L->diag[c] = L->diag[c] - original + act;
      }
}

/* Generic tensor channel aggregation in x->y->z order over the coarsened
 * axes (aggregate_tensor_channel, src/solver_mg.cpp:1706-1856).
 * face_axis = -1 for cell channels.  `src` has the fine extents. */
static void aggregate(const level_t* fine, int face_axis, const double* src,
                      double* dst, double* buf0, double* buf1) {
  int e[3] = {fine->n[0], fine->n[1], fine->n[2]};
  int g[3] = {fine->n[0], fine->n[1], fine->n[2]};
  if (face_axis >= 0) e[face_axis] += 1;
  size_t count = (size_t)e[0] * e[1] * e[2];
  memcpy(buf0, src, count * sizeof(double));
  double* cur = buf0;
  double* nxt = buf1;
  for (int axis = 0; axis < 3; ++axis) {
    if (!(fine->coarsen_mask & (1 << axis))) continue;
    int ng[3] = {g[0], g[1], g[2]};
    ng[axis] = (g[axis] + 1) / 2;
    int ne[3] = {ng[0], ng[1], ng[2]};
    if (face_axis >= 0) ne[face_axis] += 1;
    for (int k = 0; k < ne[2]; ++k)
      for (int j = 0; j < ne[1]; ++j)
        for (int i = 0; i < ne[0]; ++i) {
          int out[3] = {i, j, k};
          double value = 0.0;
          if (face_axis == axis) {
            int fine_global = 2 * out[axis];
            if (fine_global > g[axis]) fine_global = g[axis];
            int s[3] = {i, j, k};
            s[axis] = fine_global;
            value = cur[(size_t)s[0] + (size_t)e[0] * ((size_t)s[1] + (size_t)e[1] * s[2])];
          } else {
            for (int child = 0; child < 2; ++child) {
              const int fine_global = 2 * out[axis] + child;
              if (fine_global >= g[axis]) continue;
              int s[3] = {i, j, k};
              s[axis] = fine_global;
              value += cur[(size_t)s[0] + (size_t)e[0] * ((size_t)s[1] + (size_t)e[1] * s[2])];
            }
          }
          nxt[(size_t)i + (size_t)ne[0] * ((size_t)j + (size_t)ne[1] * k)] = value;
        }
    double* swap = cur;
    cur = nxt;
    nxt = swap;
    g[0] = ng[0];
    g[1] = ng[1];
    g[2] = ng[2];
    e[0] = ne[0];
    e[1] = ne[1];
    e[2] = ne[2];
  }
  count = (size_t)e[0] * e[1] * e[2];
  memcpy(dst, cur, count * sizeof(double));
}

static int build_coarse(oracle_t* o) {
  size_t maxv = 0;
  for (int l = 0; l < o->levels; ++l) {
    const level_t* L = &o->lv[l];
    if (L->fxn > maxv) maxv = L->fxn;
    if (L->fyn > maxv) maxv = L->fyn;
    if (L->fzn > maxv) maxv = L->fzn;
  }
  double* b0 = malloc(maxv * sizeof(double));
  double* b1 = malloc(maxv * sizeof(double));
  double* reaction = malloc(maxv * sizeof(double));
  if (!b0 || !b1 || !reaction) return -2;
  copy_finest(o);
  for (int l = 1; l < o->levels; ++l) {
    const level_t* F = &o->lv[l - 1];
    level_t* C = &o->lv[l];
    const int* fs = F->n;
    aggregate(F, -1, F->vol, C->vol, b0, b1);
    for (int k = 0; k < fs[2]; ++k)
      for (int j = 0; j < fs[1]; ++j)
        for (int i = 0; i < fs[0]; ++i) {
          const size_t c = idx(fs, i, j, k);
          if (F->vol[c] == 0.0) {
            reaction[c] = 0.0;
            continue;
          }
          const double faces =
              F->fx[fidx_x(fs, i, j, k)] + F->fx[fidx_x(fs, i + 1, j, k)] +
              F->fy[fidx_y(fs, i, j, k)] + F->fy[fidx_y(fs, i, j + 1, k)] +
              F->fz[fidx_z(fs, i, j, k)] + F->fz[fidx_z(fs, i, j, k + 1)];
          const double v = F->diag[c] - faces;
          reaction[c] = v > 0.0 ? v : 0.0;
        }
    aggregate(F, -1, reaction, C->diag, b0, b1);
    aggregate(F, 0, F->fx, C->fx, b0, b1);
    aggregate(F, 1, F->fy, C->fy, b0, b1);
    aggregate(F, 2, F->fz, C->fz, b0, b1);
    const int* cs = C->n;
    for (int k = 0; k < cs[2]; ++k)
      for (int j = 0; j < cs[1]; ++j)
        for (int i = 0; i < cs[0]; ++i) {
          const size_t c = idx(cs, i, j, k);
          C->diag[c] += C->fx[fidx_x(cs, i, j, k)] + C->fx[fidx_x(cs, i + 1, j, k)] +
                        C->fy[fidx_y(cs, i, j, k)] + C->fy[fidx_y(cs, i, j + 1, k)] +
                        C->fz[fidx_z(cs, i, j, k)] + C->fz[fidx_z(cs, i, j, k + 1)];
          if (C->vol[c] == 0.0) C->diag[c] = 1.0;
        }
  }
  free(b0);
  free(b1);
  free(reaction);
  return 0;
}

/* select_diagonal_shortcut (src/solver_mg.cpp:1577-1611). */
static void select_shortcut(oracle_t* o) {
  o->diagonal_shortcut = 0;
  if (o->shortcut_ratio == 0.0) return;
  const level_t* L = &o->lv[0];
  const int* n = L->n;
  double maximum = 0.0;
  for (int k = 0; k < n[2]; ++k)
    for (int j = 0; j < n[1]; ++j)
      for (int i = 0; i < n[0]; ++i) {
        const double sum =
            L->fx[fidx_x(n, i, j, k)] + L->fx[fidx_x(n, i + 1, j, k)] +
            L->fy[fidx_y(n, i, j, k)] + L->fy[fidx_y(n, i, j + 1, k)] +
            L->fz[fidx_z(n, i, j, k)] + L->fz[fidx_z(n, i, j, k + 1)];
        const double ratio = sum / L->diag[idx(n, i, j, k)];
        if (ratio > maximum) maximum = ratio;
      }
  o->diagonal_shortcut = maximum <= o->shortcut_ratio;
}

/* ------------------------------------------------------------------ */
/* Level stencil (point_row_value, src/solver_mg.cpp:2395-2414)        */
/* Boundary neighbour: Dirichlet 0, Neumann self (:940-963).           */
/* ------------------------------------------------------------------ */
static double nb(const oracle_t* o, const level_t* L, const double* x, int i,
                 int j, int k, int axis, int dir) {
  int c[3] = {i, j, k};
  c[axis] += dir;
  if (c[axis] >= 0 && c[axis] < L->n[axis])
    return x[idx(L->n, c[0], c[1], c[2])];
  const int code = o->bc[2 * axis + (dir > 0 ? 1 : 0)];
  return code == BC_NEUMANN ? x[idx(L->n, i, j, k)] : 0.0;
}

static double row_value(const oracle_t* o, const level_t* L, const double* x,
                        int i, int j, int k) {
  const int* n = L->n;
  double v = L->diag[idx(n, i, j, k)] * x[idx(n, i, j, k)];
  v -= L->fx[fidx_x(n, i, j, k)] * nb(o, L, x, i, j, k, 0, -1);
  v -= L->fx[fidx_x(n, i + 1, j, k)] * nb(o, L, x, i, j, k, 0, 1);
  v -= L->fy[fidx_y(n, i, j, k)] * nb(o, L, x, i, j, k, 1, -1);
  v -= L->fy[fidx_y(n, i, j + 1, k)] * nb(o, L, x, i, j, k, 1, 1);
  v -= L->fz[fidx_z(n, i, j, k)] * nb(o, L, x, i, j, k, 2, -1);
  v -= L->fz[fidx_z(n, i, j, k + 1)] * nb(o, L, x, i, j, k, 2, 1);
  return v;
}

/* apply_level_defect: out = rhs - A x (src/solver_mg.cpp:2653-2767). */
static void level_defect(const oracle_t* o, const level_t* L, const double* x,
                         const double* b, double* out) {
  const int* n = L->n;
  for (int k = 0; k < n[2]; ++k)
    for (int j = 0; j < n[1]; ++j)
      for (int i = 0; i < n[0]; ++i)
        out[idx(n, i, j, k)] = b[idx(n, i, j, k)] - row_value(o, L, x, i, j, k);
}

/* fused_point_color_update (src/solver_mg.cpp:3149-3223), omega 0.72. */
static void color_update(const oracle_t* o, level_t* L, int color) {
  const int* n = L->n;
  const double omega = 0.72;
  for (int k = 0; k < n[2]; ++k)
    for (int j = 0; j < n[1]; ++j)
      for (int i = 0; i < n[0]; ++i) {
        if (((i + j + k) & 1) != color) continue;
        const size_t c = idx(n, i, j, k);
        const double value = row_value(o, L, L->x, i, j, k);
        L->x[c] += omega * (L->b[c] - value) / L->diag[c];
      }
}

/* point_smooth red-black branch (src/solver_mg.cpp:3225-3350). */
static void point_smooth(const oracle_t* o, level_t* L, int sweeps,
                         int reverse, int retain) {
  const int first = reverse ? 1 : 0;
  for (int s = 0; s < sweeps; ++s)
    for (int pass = 0; pass < 2; ++pass) color_update(o, L, (first + pass) & 1);
  if (retain) level_defect(o, L, L->x, L->b, L->r);
}

/* chebyshev_point_smooth_streamed (src/solver_mg.cpp:2916-3091). */
static void chebyshev_smooth(const oracle_t* o, level_t* L, int stages,
                             int retain) {
  const double beta = 2.0;
  const double alpha = o->cheb_fraction * beta;
  const double theta = (beta + alpha) * 0.5;
  const double delta = (beta - alpha) * 0.5;
  const double sigma = theta / delta;
  double previous_rho = 1.0 / sigma;
  double* current = L->x;
  double* next = L->t;
  const int* n = L->n;
  for (int s = 0; s < stages; ++s) {
    const double rho = s == 0 ? 0.0 : 1.0 / (2.0 * sigma - previous_rho);
    const double previous_factor = s == 0 ? 0.0 : rho * previous_rho;
    const double residual_factor = s == 0 ? 1.0 / theta : 2.0 * rho / delta;
    if (s != 0) previous_rho = rho;
    for (int k = 0; k < n[2]; ++k)
      for (int j = 0; j < n[1]; ++j)
        for (int i = 0; i < n[0]; ++i) {
          const size_t c = idx(n, i, j, k);
          const double value = row_value(o, L, current, i, j, k);
          const double defect = L->b[c] - value;
          const double scaled = residual_factor * defect / L->diag[c];
          const double direction =
              s == 0 ? scaled : previous_factor * L->r[c] + scaled;
          L->r[c] = direction;
          next[c] = current[c] + direction;
        }
    double* swap = current;
    current = next;
    next = swap;
  }
  if (current != L->x) memcpy(L->x, current, L->cells * sizeof(double));
  if (retain) level_defect(o, L, L->x, L->b, L->r);
}

/* One Thomas line solve (solve_one in line_smooth_axis,
 * src/solver_mg.cpp:3388-3493).  (a,b) index the line per the reference's
 * fixed_a/fixed_b convention. */
static void line_solve(const oracle_t* o, level_t* L, int axis, int fa,
                       int fb) {
  const int* n = L->n;
  const int extent = n[axis];
  double* work = L->t;
  double* dprime = L->r;
  for (int s = 0; s < extent; ++s) {
    int c[3];
    if (axis == 0) { c[0] = s; c[1] = fa; c[2] = fb; }
    else if (axis == 1) { c[0] = fa; c[1] = s; c[2] = fb; }
    else { c[0] = fa; c[1] = fb; c[2] = s; }
    const int i = c[0], j = c[1], k = c[2];
    const size_t cell = idx(n, i, j, k);
    double lowf, highf;
    if (axis == 0) { lowf = L->fx[fidx_x(n, i, j, k)]; highf = L->fx[fidx_x(n, i + 1, j, k)]; }
    else if (axis == 1) { lowf = L->fy[fidx_y(n, i, j, k)]; highf = L->fy[fidx_y(n, i, j + 1, k)]; }
    else { lowf = L->fz[fidx_z(n, i, j, k)]; highf = L->fz[fidx_z(n, i, j, k + 1)]; }
    const double a = s == 0 ? 0.0 : -lowf;
    const double bb = L->diag[cell];
    const double cc = s + 1 == extent ? 0.0 : -highf;
    double d = L->b[cell];
    if (axis != 0) {
      d += L->fx[fidx_x(n, i, j, k)] * nb(o, L, L->x, i, j, k, 0, -1);
      d += L->fx[fidx_x(n, i + 1, j, k)] * nb(o, L, L->x, i, j, k, 0, 1);
    }
    if (axis != 1) {
      d += L->fy[fidx_y(n, i, j, k)] * nb(o, L, L->x, i, j, k, 1, -1);
      d += L->fy[fidx_y(n, i, j + 1, k)] * nb(o, L, L->x, i, j, k, 1, 1);
    }
    if (axis != 2) {
      d += L->fz[fidx_z(n, i, j, k)] * nb(o, L, L->x, i, j, k, 2, -1);
      d += L->fz[fidx_z(n, i, j, k + 1)] * nb(o, L, L->x, i, j, k, 2, 1);
    }
    if (s == 0) d += lowf * nb(o, L, L->x, i, j, k, axis, -1);
    if (s + 1 == extent) d += highf * nb(o, L, L->x, i, j, k, axis, 1);
    if (s > 0) {
      int p[3] = {i, j, k};
      p[axis] -= 1;
      const size_t prev = idx(n, p[0], p[1], p[2]);
      const double denominator = bb - a * work[prev];
      work[cell] = cc / denominator;
      dprime[cell] = (d - a * dprime[prev]) / denominator;
    } else {
      work[cell] = cc / bb;
      dprime[cell] = d / bb;
    }
  }
  for (int s = extent; s-- > 0;) {
    int c[3];
    if (axis == 0) { c[0] = s; c[1] = fa; c[2] = fb; }
    else if (axis == 1) { c[0] = fa; c[1] = s; c[2] = fb; }
    else { c[0] = fa; c[1] = fb; c[2] = s; }
    const size_t cell = idx(n, c[0], c[1], c[2]);
    if (s + 1 == extent) {
      L->x[cell] = dprime[cell];
    } else {
      int q[3] = {c[0], c[1], c[2]};
      q[axis] += 1;
      L->x[cell] = dprime[cell] - work[cell] * L->x[idx(n, q[0], q[1], q[2])];
    }
  }
}

/* line_smooth_axis sweep loop (src/solver_mg.cpp:3495-3520); zebra order
 * when line_order == 1. */
static void line_smooth_axis(const oracle_t* o, level_t* L, int axis,
                             int sweeps, int reverse) {
  const int a_extent = axis == 0 ? L->n[1] : L->n[0];
  const int b_extent = axis == 2 ? L->n[1] : L->n[2];
  for (int s = 0; s < sweeps; ++s) {
    if (o->line_order == 0) {
      if (reverse) {
        for (int b = b_extent; b-- > 0;)
          for (int a = a_extent; a-- > 0;) line_solve(o, L, axis, a, b);
      } else {
        for (int b = 0; b < b_extent; ++b)
          for (int a = 0; a < a_extent; ++a) line_solve(o, L, axis, a, b);
      }
    } else {
      const int first = reverse ? 1 : 0;
      for (int pass = 0; pass < 2; ++pass) {
        const int color = (first + pass) & 1;
        for (int b = 0; b < b_extent; ++b)
          for (int a = 0; a < a_extent; ++a)
            if (((a + b) & 1) == color) line_solve(o, L, axis, a, b);
      }
    }
  }
}

/* smooth (src/solver_mg.cpp:3541-3589). */
static void smooth(const oracle_t* o, level_t* L, int sweeps, int reverse,
                   int retain) {
  if (L->line_mask == 0) {
    if (L->chebyshev) chebyshev_smooth(o, L, sweeps, retain);
    else point_smooth(o, L, sweeps, reverse, retain);
    return;
  }
  if (reverse) {
    for (int a = 3; a-- > 0;)
      if (L->line_mask & (1 << a)) line_smooth_axis(o, L, a, sweeps, 1);
  } else {
    for (int a = 0; a < 3; ++a)
      if (L->line_mask & (1 << a)) line_smooth_axis(o, L, a, sweeps, 0);
  }
}

/* restrict_residual (src/solver_mg.cpp:3633-3721). */
static void restrict_residual(level_t* F, level_t* C) {
  const int mx = F->coarsen_mask & AXIS_X, my = F->coarsen_mask & AXIS_Y,
            mz = F->coarsen_mask & AXIS_Z;
  const int* cs = C->n;
  const int* fs = F->n;
  for (int k = 0; k < cs[2]; ++k)
    for (int j = 0; j < cs[1]; ++j)
      for (int i = 0; i < cs[0]; ++i) {
        const int xb = mx ? 2 * i : i, yb = my ? 2 * j : j, zb = mz ? 2 * k : k;
        double sum = 0.0;
        for (int dz = 0; dz < (mz ? 2 : 1); ++dz)
          for (int dy = 0; dy < (my ? 2 : 1); ++dy)
            for (int dx = 0; dx < (mx ? 2 : 1); ++dx) {
              const int fx = xb + dx, fy = yb + dy, fz = zb + dz;
              if (fx >= fs[0] || fy >= fs[1] || fz >= fs[2]) continue;
              sum += F->r[idx(fs, fx, fy, fz)];
            }
        C->b[idx(cs, i, j, k)] = sum;
        C->x[idx(cs, i, j, k)] = 0.0;
      }
}

static void interp(int fine, int coarsened, int extent, int* left, int* right,
                   double* weight) {
  if (!coarsened) {
    *left = *right = fine;
    *weight = 0.0;
    return;
  }
  const int parent = fine / 2;
  if ((fine & 1) == 0) {
    *left = parent - 1;
    *right = parent;
    *weight = 0.75;
  } else {
    *left = parent;
    *right = parent + 1;
    *weight = 0.25;
  }
  if (*left < 0) {
    *left = *right = 0;
    *weight = 0.0;
  } else if (*right >= extent) {
    *left = *right = extent - 1;
    *weight = 0.0;
  }
}

/* prolongate_add (src/solver_mg.cpp:3893-3994). */
static void prolongate_add(level_t* F, const level_t* C) {
  const int mx = F->coarsen_mask & AXIS_X, my = F->coarsen_mask & AXIS_Y,
            mz = F->coarsen_mask & AXIS_Z;
  const int* fs = F->n;
  const int* cs = C->n;
  for (int k = 0; k < fs[2]; ++k)
    for (int j = 0; j < fs[1]; ++j)
      for (int i = 0; i < fs[0]; ++i) {
        const size_t c = idx(fs, i, j, k);
        if (F->vol[c] == 0.0) {
          F->x[c] = 0.0;
          continue;
        }
        int xl, xr, yl, yr, zl, zr;
        double xw, yw, zw;
        interp(i, mx, cs[0], &xl, &xr, &xw);
        interp(j, my, cs[1], &yl, &yr, &yw);
        interp(k, mz, cs[2], &zl, &zr, &zw);
        double value = 0.0;
        for (int az = 0; az < (zl == zr ? 1 : 2); ++az) {
          const int gz = az == 0 ? zl : zr;
          const double wz = az == 0 ? 1.0 - zw : zw;
          for (int ay = 0; ay < (yl == yr ? 1 : 2); ++ay) {
            const int gy = ay == 0 ? yl : yr;
            const double wy = ay == 0 ? 1.0 - yw : yw;
            for (int ax = 0; ax < (xl == xr ? 1 : 2); ++ax) {
              const int gx = ax == 0 ? xl : xr;
              const double wx = ax == 0 ? 1.0 - xw : xw;
              value += wx * wy * wz * C->x[idx(cs, gx, gy, gz)];
            }
          }
        }
        F->x[c] += value;
      }
}

/* mg_cycle (src/solver_mg.cpp:4192-4338). */
static void mg_cycle(oracle_t* o, int l, int counter) {
  level_t* L = &o->lv[l];
  if (l + 1 == o->levels) {
    smooth(o, L, o->coarse_sweeps, 0, 0);
    return;
  }
  smooth(o, L, o->pre, 0, 1);
  if (L->line_mask != 0) level_defect(o, L, L->x, L->b, L->r);
  restrict_residual(L, &o->lv[l + 1]);
  mg_cycle(o, l + 1, counter);
  if (counter > 1) mg_cycle(o, l + 1, counter - 1);
  prolongate_add(L, &o->lv[l + 1]);
  smooth(o, L, o->post, 1, 0);
}

/* NativeCartesianMgPlan::apply_impl (src/solver_mg.cpp:4814-5122). */
int hfo_apply_mg(void* handle, const double* residual, double* correction) {
  oracle_t* o = handle;
  level_t* L = &o->lv[0];
  const size_t cells = L->cells;
  for (size_t c = 0; c < cells; ++c) {
    const int act = o->active == NULL || o->active[c] != 0;
    L->x[c] = 0.0;
    L->b[c] = act ? residual[c] : 0.0;
  }
  if (o->diagonal_shortcut) {
    for (size_t c = 0; c < cells; ++c) L->x[c] = L->b[c] / L->diag[c];
  } else {
    mg_cycle(o, 0, o->cycle == 1 ? 2 : 1);
  }
  level_defect(o, L, L->x, L->b, L->r);
  double p0 = 0.0, p1 = 0.0, p2 = 0.0;
  for (size_t c = 0; c < cells; ++c) {
    const int act = o->active == NULL || o->active[c] != 0;
    const double r = act ? residual[c] : 0.0;
    const double az = r - L->r[c];
    p0 += r * r;
    p1 += r * az;
    p2 += az * az;
  }
  if (!isfinite(p0) || !isfinite(p1) || !isfinite(p2)) return 5;
  const double tiny = DBL_EPSILON * p0;
  const double alpha = o->unit_linear ? 1.0 : (p2 > tiny ? p1 / p2 : 0.0);
  for (size_t c = 0; c < cells; ++c) {
    const int act = o->active == NULL || o->active[c] != 0;
    correction[c] = act ? L->x[c] * alpha : 0.0;
  }
  return 0;
}

/* ------------------------------------------------------------------ */
/* Cold-path diagonal incomplete Cholesky (DIC / IC(0))                 */
/* ------------------------------------------------------------------ */
/* Rows of the IBM-decorated operator: identity rows on solid cells; a link
 * to a solid cell or a Neumann boundary face leaves the row's couplings and
 * its coefficient leaves the diagonal (subtracted in face order). */
static void dic_rows(oracle_t* o) {
  const int* n = o->n;
  const size_t cells = o->lv[0].cells;
  for (int k = 0; k < n[2]; ++k)
    for (int j = 0; j < n[1]; ++j)
      for (int i = 0; i < n[0]; ++i) {
        const size_t c = idx(n, i, j, k);
        double* nb = o->dic_nb + 6 * c;
        for (int f = 0; f < 6; ++f) nb[f] = 0.0;
        if (!cell_active(o, i, j, k)) { o->dic_diag[c] = 1.0; continue; }
        double d = o->diag0[c];
        const double face[6] = {o->fx0[fidx_x(n, i, j, k)], o->fx0[fidx_x(n, i + 1, j, k)],
                                o->fy0[fidx_y(n, i, j, k)], o->fy0[fidx_y(n, i, j + 1, k)],
                                o->fz0[fidx_z(n, i, j, k)], o->fz0[fidx_z(n, i, j, k + 1)]};
        const int at[3] = {i, j, k};
        for (int f = 0; f < 6; ++f) {
          const int a = f / 2;
          int q[3] = {i, j, k};
          q[a] += (f & 1) ? 1 : -1;
          if (q[a] < 0 || q[a] >= n[a]) {
            if (o->bc[f] == BC_NEUMANN) d -= face[f];
            continue;
          }
          if (!cell_active(o, q[0], q[1], q[2])) { d -= face[f]; continue; }
          nb[f] = face[f];
          (void)at;
        }
        o->dic_diag[c] = d;
      }
  (void)cells;
}

/* ColdPressureIccg::prepare (src/solver_iccg.hpp:236-256): lexicographic
 * pivots p_i = D_i - sum_axis c^2 / p_(lower neighbour). */
static int dic_prepare(oracle_t* o) {
  const int* n = o->n;
  const size_t stride[3] = {1, (size_t)n[0], (size_t)n[0] * n[1]};
  size_t i = 0;
  for (int z = 0; z < n[2]; ++z)
    for (int y = 0; y < n[1]; ++y)
      for (int x = 0; x < n[0]; ++x, ++i) {
        const int at[3] = {x, y, z};
        double pivot = o->dic_diag[i];
        for (int a = 0; a < 3; ++a) {
          const double lower = o->dic_nb[6 * i + 2 * a];
          if (at[a] > 0) pivot -= lower * lower * o->dic_inv[i - stride[a]];
        }
        if (!(pivot > 0) || !isfinite(pivot)) return 5;
        o->dic_inv[i] = 1 / pivot;
      }
  return 0;
}

/* ColdPressureIccg::apply (src/solver_iccg.hpp:262-284): forward sweep with
 * the lower couplings, backward sweep with the upper ones (the next cell's
 * lower coupling). */
static void dic_apply(const oracle_t* o, const double* in, double* out) {
  const int* n = o->n;
  const size_t sy = (size_t)n[0], sz = sy * n[1];
  size_t i = 0;
  for (int z = 0; z < n[2]; ++z)
    for (int y = 0; y < n[1]; ++y)
      for (int x = 0; x < n[0]; ++x, ++i) {
        double value = in[i];
        if (x > 0) value += o->dic_nb[6 * i + 0] * out[i - 1];
        if (y > 0) value += o->dic_nb[6 * i + 2] * out[i - sy];
        if (z > 0) value += o->dic_nb[6 * i + 4] * out[i - sz];
        out[i] = value * o->dic_inv[i];
      }
  i = o->lv[0].cells;
  for (int z = n[2] - 1; z >= 0; --z)
    for (int y = n[1] - 1; y >= 0; --y)
      for (int x = n[0] - 1; x >= 0; --x) {
        --i;
        double value = 0;
        if (x + 1 < n[0]) value += o->dic_nb[6 * (i + 1) + 0] * out[i + 1];
        if (y + 1 < n[1]) value += o->dic_nb[6 * (i + sy) + 2] * out[i + sy];
        if (z + 1 < n[2]) value += o->dic_nb[6 * (i + sz) + 4] * out[i + sz];
        out[i] += value * o->dic_inv[i];
      }
}

static int apply_pc(oracle_t* o, const double* r, double* z) {
  if (o->pc_kind == 0) return hfo_apply_mg(o, r, z);
  dic_apply(o, r, z);
  return 0;
}

int hfo_apply_preconditioner(void* handle, const double* r, double* z) {
  return apply_pc(handle, r, z);
}

/* ------------------------------------------------------------------ */
/* Exact operator: regular stencil + IBM decoration                    */
/* (src/solver_pressure.cpp:746-811; src/solver_ibm_pressure.cpp:347-385)*/
/* ------------------------------------------------------------------ */
int hfo_apply_operator(void* handle, const double* x, double* y) {
  oracle_t* o = handle;
  const int* n = o->n;
  level_t R;
  memset(&R, 0, sizeof(R));
  R.n[0] = n[0];
  R.n[1] = n[1];
  R.n[2] = n[2];
  R.diag = o->diag0;
  R.fx = o->fx0;
  R.fy = o->fy0;
  R.fz = o->fz0;
  for (int k = 0; k < n[2]; ++k)
    for (int j = 0; j < n[1]; ++j)
      for (int i = 0; i < n[0]; ++i) y[idx(n, i, j, k)] = row_value(o, &R, x, i, j, k);
  if (o->active == NULL) return 0;
  for (size_t c = 0; c < (size_t)n[0] * n[1] * n[2]; ++c)
    if (o->active[c] == 0) y[c] = x[c];
  for (int k = 0; k < n[2]; ++k)
    for (int j = 0; j < n[1]; ++j)
      for (int i = 0; i < n[0]; ++i) {
        const size_t c = idx(n, i, j, k);
        if (o->active[c] == 0) continue;
        const double xf = x[c];
        const int nbr[6][3] = {{i - 1, j, k}, {i + 1, j, k}, {i, j - 1, k},
                               {i, j + 1, k}, {i, j, k - 1}, {i, j, k + 1}};
        const double coef[6] = {o->fx0[fidx_x(n, i, j, k)], o->fx0[fidx_x(n, i + 1, j, k)],
                                o->fy0[fidx_y(n, i, j, k)], o->fy0[fidx_y(n, i, j + 1, k)],
                                o->fz0[fidx_z(n, i, j, k)], o->fz0[fidx_z(n, i, j, k + 1)]};
        for (int f = 0; f < 6; ++f) {
          const int a = nbr[f][0], b = nbr[f][1], cc = nbr[f][2];
          if (a < 0 || b < 0 || cc < 0 || a >= n[0] || b >= n[1] || cc >= n[2]) continue;
          const size_t s = idx(n, a, b, cc);
          if (o->active[s] != 0) continue;
          y[c] += coef[f] * (x[s] - xf);
        }
      }
  return 0;
}

int hfo_apply_level(void* handle, int level, const double* x, double* y) {
  oracle_t* o = handle;
  if (level < 0 || level >= o->levels) return 2;
  const level_t* L = &o->lv[level];
  const int* n = L->n;
  for (int k = 0; k < n[2]; ++k)
    for (int j = 0; j < n[1]; ++j)
      for (int i = 0; i < n[0]; ++i) y[idx(n, i, j, k)] = row_value(o, L, x, i, j, k);
  return 0;
}

/* ------------------------------------------------------------------ */
/* Krylov helpers (src/solver_krylov.cpp:176-204, 650-711)             */
/* ------------------------------------------------------------------ */
static double dot(const double* a, const double* b, size_t n, int* ok) {
  double sum = 0.0, correction = 0.0;
  for (size_t c = 0; c < n; ++c) {
    const double product = a[c] * b[c];
    if (!isfinite(product)) *ok = 0;
    const double next = sum + product;
    if (fabs(sum) >= fabs(product)) correction += (sum - next) + product;
    else correction += (product - next) + sum;
    sum = next;
  }
  return sum + correction;
}

static double norm2(const double* v, size_t n, int* ok) {
  double scale = 0.0;
  for (size_t c = 0; c < n; ++c) {
    if (!isfinite(v[c])) *ok = 0;
    else if (fabs(v[c]) > scale) scale = fabs(v[c]);
  }
  if (scale == 0.0) return 0.0;
  double sum = 0.0, correction = 0.0;
  for (size_t c = 0; c < n; ++c) {
    const double s = v[c] / scale;
    const double sq = s * s;
    const double next = sum + sq;
    if (fabs(sum) >= fabs(sq)) correction += (sum - next) + sq;
    else correction += (sq - next) + sum;
    sum = next;
  }
  sum += correction;
  return scale * sqrt(sum);
}

/* solve_pcg (src/solver_krylov.cpp:1299-1555), including the restart of the
 * search direction after every true-residual verification. */
int hfo_solve(void* handle, const double* rhs, double* x, double rtol,
              double atol, int maxit, int tri, double* out, double* history,
              int hcap) {
  oracle_t* o = handle;
  const size_t n = o->lv[0].cells;
  double* r = o->work[0];
  double* z = o->work[1];
  double* p = o->work[2];
  double* ap = o->work[3];
  int ok = 1;
  long op_applies = 0, pc_applies = 0;
  int it = 0;
  memset(out, 0, 8 * sizeof(double));
  const double bnorm = norm2(rhs, n, &ok);
  if (!ok) { out[3] = TERM_NON_FINITE; return 5; }
  const double tol = atol > rtol * bnorm ? atol : rtol * bnorm;
  out[4] = bnorm;
  out[5] = tol;
  if (bnorm == 0.0) {
    memset(x, 0, n * sizeof(double));
    out[3] = TERM_ZERO_RHS;
    return 0;
  }
#define TRUE_RESIDUAL(dst_norm)                              \
  do {                                                       \
    hfo_apply_operator(o, x, ap);                            \
    ++op_applies;                                            \
    for (size_t c = 0; c < n; ++c) r[c] = 1.0 * rhs[c] + -1.0 * ap[c]; \
    dst_norm = norm2(r, n, &ok);                             \
  } while (0)
  double initial = 0.0, final_true = 0.0;
  TRUE_RESIDUAL(initial);
  final_true = initial;
  out[1] = initial;
  int term = TERM_MAXIMUM;
  int status = 6;
  if (initial <= tol) { term = TERM_CONVERGED; status = 0; goto done; }
  apply_pc(o, r, z);
  ++pc_applies;
  double rho = dot(r, z, n, &ok);
  if (!(rho > 0.0) || !isfinite(rho)) { term = TERM_BREAKDOWN; status = 5; goto done; }
  memcpy(p, z, n * sizeof(double));
  while (it < maxit) {
    hfo_apply_operator(o, p, ap);
    ++op_applies;
    const double denominator = dot(p, ap, n, &ok);
    if (!(denominator > 0.0) || !isfinite(denominator)) { term = TERM_BREAKDOWN; status = 5; goto done; }
    const double alpha = rho / denominator;
    for (size_t c = 0; c < n; ++c) x[c] = x[c] + alpha * p[c];
    for (size_t c = 0; c < n; ++c) r[c] = r[c] + -alpha * ap[c];
    ++it;
    const double recursive = norm2(r, n, &ok);
    if (history && it - 1 < hcap) history[it - 1] = recursive;
    const int verify = recursive <= tol || it % tri == 0 || it == maxit;
    if (verify) {
      TRUE_RESIDUAL(final_true);
      if (final_true <= tol) { term = TERM_CONVERGED; status = 0; goto done; }
      if (it == maxit) { term = TERM_MAXIMUM; status = 6; goto done; }
      apply_pc(o, r, z);
      ++pc_applies;
      rho = dot(r, z, n, &ok);
      if (!(rho > 0.0) || !isfinite(rho)) { term = TERM_BREAKDOWN; status = 5; goto done; }
      memcpy(p, z, n * sizeof(double));
      continue;
    }
    apply_pc(o, r, z);
    ++pc_applies;
    const double rho_next = dot(r, z, n, &ok);
    if (!(rho_next > 0.0) || !isfinite(rho_next)) { term = TERM_BREAKDOWN; status = 5; goto done; }
    const double beta = rho_next / rho;
    for (size_t c = 0; c < n; ++c) p[c] = 1.0 * z[c] + beta * p[c];
    rho = rho_next;
  }
done:
#undef TRUE_RESIDUAL
  out[0] = it;
  out[2] = final_true;
  out[3] = term;
  out[6] = (double)op_applies;
  out[7] = (double)pc_applies;
  return ok ? status : 5;
}

/* ------------------------------------------------------------------ */
/* solve_fgmres (src/solver_krylov.cpp:1557-2650): single-reduction      */
/* Arnoldi on the shifted image w = A z - v (shift 1, :35), one batched */
/* reduction for the projections and |w|^2 (local_multidot, :206-244),  */
/* the Pythagorean norm with its breakdown fallbacks                     */
/* (single_reduction_fgmres_norm, :565-609), Givens rotations, true-     */
/* residual audits of the candidate every true_residual_interval         */
/* iterations and at cycle ends, restarts.  Subspace recycling and the   */
/* convergence audit are inactive, as in the reference harness.          */
/* ------------------------------------------------------------------ */
#define FGMRES_SHIFT 1.0

/* add_scaled_basis (:510-564): dst = dst + s_0 b_0 + s_1 b_1 + ... per cell. */
static int add_scaled_basis(double* dst, double* const* src, const double* s,
                            int count, size_t n) {
  int ok = 1;
  for (size_t c = 0; c < n; ++c) {
    double v = dst[c];
    for (int r = 0; r < count; ++r) v = v + s[r] * src[r][c];
    if (!isfinite(v)) ok = 0;
    dst[c] = v;
  }
  return ok;
}

static int back_substitute(const double* h, const double* g, double* y, int count,
                           int rows) {
  for (int row = count - 1; row >= 0; --row) {
    double value = g[row];
    for (int upper = row + 1; upper < count; ++upper)
      value -= h[(size_t)upper * rows + row] * y[upper];
    const double divisor = h[(size_t)row * rows + row];
    if (divisor == 0.0 || !isfinite(divisor)) return TERM_BREAKDOWN;
    y[row] = value / divisor;
    if (!isfinite(y[row])) return TERM_NON_FINITE;
  }
  return -1;
}

#define RECYCLE_MAX 4

static void recycle_clear(oracle_t* o) {
  o->rc_capture = o->rc_guard_only = o->rc_cycle_active = o->rc_pending = 0;
  o->rc_count = o->rc_oldest = 0;
}

static double* recycle_slot(oracle_t* o, int logical) {
  return o->rc_ring[(o->rc_oldest + logical) % RECYCLE_MAX];
}

/* recycle_capture_cycle_start (src/solver_linear_state.cpp:857-895). */
static void recycle_cycle_start(oracle_t* o, const double* x, size_t n) {
  if (!o->rc_capture) return;
  memcpy(o->rc_snapshot, x, n * sizeof(double));
  o->rc_cycle_active = 1;
}

/* recycle_capture_cycle_publish (:897-1017): correction = x - snapshot;
 * a nonzero one enters the ring, replacing the oldest when it is full. */
static void recycle_publish(oracle_t* o, const double* x, size_t n, long* published) {
  if (!o->rc_capture || !o->rc_cycle_active) return;
  int nonzero = 0;
  for (size_t c = 0; c < n; ++c) {
    const double v = x[c] - o->rc_snapshot[c];
    nonzero = nonzero || v != 0.0;
    o->rc_snapshot[c] = v;
  }
  o->rc_cycle_active = 0;
  if (!nonzero) return;
  ++*published;
  double* slot;
  if (o->rc_count < RECYCLE_MAX) {
    slot = o->rc_ring[(o->rc_oldest + o->rc_count) % RECYCLE_MAX];
    ++o->rc_count;
  } else {
    slot = o->rc_ring[o->rc_oldest];
    o->rc_oldest = (o->rc_oldest + 1) % RECYCLE_MAX;
  }
  memcpy(slot, o->rc_snapshot, n * sizeof(double));
}

int hfo_solve_fgmres(void* handle, const double* rhs, double* x, double rtol,
                     double atol, int maxit, int tri, int restart, int recycle,
                     double* out, double* history, int hcap) {
  oracle_t* o = handle;
  const size_t n = o->lv[0].cells;
  long rc_published = 0, rc_offered = 0, rc_retained = 0, rc_accepted = 0;
  double rc_projected = 0.0;
  if (o->rc_snapshot == NULL) {
    o->rc_snapshot = calloc(n, sizeof(double));
    for (int r = 0; r < RECYCLE_MAX; ++r) {
      o->rc_ring[r] = calloc(n, sizeof(double));
      o->rc_image[r] = calloc(n, sizeof(double));
    }
  }
  /* Session selection as PressureVelocityCoupler makes it
   * (src/solver_piso.cpp:10410-10433). */
  if (recycle == 0) recycle_clear(o);
  else if (recycle == 1) { recycle_clear(o); o->rc_capture = 1; }
  else if (recycle == 2) {
    if (!o->rc_capture || o->rc_cycle_active || o->rc_pending) { out[3] = TERM_BREAKDOWN; return 2; }
    o->rc_capture = 0;
    o->rc_pending = 1;
  } else if (recycle == 3) { recycle_clear(o); o->rc_guard_only = 1; }
  int ok = 1;
  long op_applies = 0, pc_applies = 0;
  int it = 0;
  int term = TERM_MAXIMUM, status = 6;
  memset(out, 0, 13 * sizeof(double));
  if (restart < 1 || restart > 64) { out[3] = TERM_BREAKDOWN; return 2; }
  const int rows = restart + 1;
  double** V = calloc((size_t)rows, sizeof(double*));
  double** Z = calloc((size_t)restart, sizeof(double*));
  double* ax = malloc(n * sizeof(double));
  double* h = calloc((size_t)rows * restart, sizeof(double));
  double* cs = calloc((size_t)restart, sizeof(double));
  double* sn = calloc((size_t)restart, sizeof(double));
  double* g = calloc((size_t)rows, sizeof(double));
  double* y = calloc((size_t)restart, sizeof(double));
  double* scratch = calloc((size_t)rows + 1, sizeof(double));
  double* scales = calloc((size_t)rows, sizeof(double));
  for (int i = 0; i < rows; ++i) V[i] = malloc(n * sizeof(double));
  for (int i = 0; i < restart; ++i) Z[i] = malloc(n * sizeof(double));

  const double bnorm = norm2(rhs, n, &ok);
  double initial = 0.0, final_true = 0.0, recursive = 0.0;
  if (!ok) { term = TERM_NON_FINITE; status = 5; goto done; }
  const double tol = atol > rtol * bnorm ? atol : rtol * bnorm;
  out[4] = bnorm;
  out[5] = tol;
  if (bnorm == 0.0) {
    memset(x, 0, n * sizeof(double));
    term = TERM_ZERO_RHS; status = 0; goto done;
  }
  /* compute_true_residual (:1071-1092): v0 = 1.0 b + -1.0 A x, |v0|. */
#define TRUE_RESIDUAL(dst_norm, sol)                                       \
  do {                                                                     \
    hfo_apply_operator(o, sol, ax);                                        \
    ++op_applies;                                                          \
    for (size_t c = 0; c < n; ++c) V[0][c] = 1.0 * rhs[c] + -1.0 * ax[c];  \
    dst_norm = norm2(V[0], n, &ok);                                        \
  } while (0)
  TRUE_RESIDUAL(initial, x);
  /* reset_to_zero_initial_guess under the recycle guard (:1673-1686). */
  if ((o->rc_capture || o->rc_guard_only) && initial > bnorm) {
    for (size_t c = 0; c < n; ++c) { x[c] = 0.0; V[0][c] = rhs[c]; }
    initial = bnorm;
  }
  final_true = initial;
  recursive = initial;
  if (!ok) { term = TERM_NON_FINITE; status = 5; goto done; }
  if (initial <= tol) { o->rc_pending = 0; term = TERM_CONVERGED; status = 0; goto done; }
  int deferred = 0;
  if (o->rc_pending) {
    /* apply_recycle_projection (src/solver_krylov.cpp:1745-2019): images
     * A d_i, two classical Gram-Schmidt passes against the retained images
     * (directions follow), normalisation, alpha_i = image_i . r, and the
     * candidate x + sum alpha_i d_i accepted if its true residual is lower.
     * The projection's operator applies are not counted as the solve's. */
    o->rc_pending = 0;
    const int offered = o->rc_count;
    rc_offered = offered;
    double* images[RECYCLE_MAX];
    double* dirs[RECYCLE_MAX];
    double pre[RECYCLE_MAX];
    int kept[RECYCLE_MAX];
    double max_pre = 0.0;
    for (int i = 0; i < offered; ++i) {
      dirs[i] = recycle_slot(o, i);
      images[i] = o->rc_image[i];
      hfo_apply_operator(o, dirs[i], images[i]);
      pre[i] = norm2(images[i], n, &ok);
      if (pre[i] > max_pre) max_pre = pre[i];
    }
    int retained = 0;
    if (offered > 0 && max_pre > 0.0 && isfinite(max_pre)) {
      const double threshold = 64.0 * DBL_EPSILON * max_pre;
      for (int i = 0; i < offered; ++i) {
        if (!(pre[i] > threshold)) continue;
        double image_norm = pre[i];
        if (retained != 0) {
          for (int pass = 0; pass < 2; ++pass) {
            double dots[RECYCLE_MAX];
            for (int p = 0; p < retained; ++p) dots[p] = dot(images[kept[p]], images[i], n, &ok);
            for (int p = 0; p < retained; ++p) {
              const double coefficient = dots[p];
              for (size_t c = 0; c < n; ++c)
                images[i][c] = images[i][c] + -coefficient * images[kept[p]][c];
              for (size_t c = 0; c < n; ++c)
                dirs[i][c] = dirs[i][c] + -coefficient * dirs[kept[p]][c];
            }
          }
          image_norm = norm2(images[i], n, &ok);
        }
        if (!(image_norm > threshold) || !isfinite(image_norm)) continue;
        const double inverse = 1.0 / image_norm;
        for (size_t c = 0; c < n; ++c) images[i][c] = inverse * images[i][c];
        for (size_t c = 0; c < n; ++c) dirs[i][c] = inverse * dirs[i][c];
        kept[retained++] = i;
      }
    }
    rc_retained = retained;
    if (retained > 0) {
      double alpha[RECYCLE_MAX];
      for (int p = 0; p < retained; ++p) alpha[p] = dot(images[kept[p]], V[0], n, &ok);
      double* candidate = o->rc_snapshot;
      memcpy(candidate, x, n * sizeof(double));
      for (int p = 0; p < retained; ++p)
        for (size_t c = 0; c < n; ++c)
          candidate[c] = candidate[c] + alpha[p] * dirs[kept[p]][c];
      hfo_apply_operator(o, candidate, ax);
      for (size_t c = 0; c < n; ++c) ax[c] = 1.0 * rhs[c] + -1.0 * ax[c];
      const double candidate_norm = norm2(ax, n, &ok);
      rc_projected = candidate_norm;
      if (isfinite(candidate_norm) && candidate_norm < final_true) {
        memcpy(x, candidate, n * sizeof(double));
        memcpy(V[0], ax, n * sizeof(double));
        final_true = candidate_norm;
        recursive = candidate_norm;
        rc_accepted = 1;
        if (final_true <= tol) { term = TERM_CONVERGED; status = 0; goto done; }
      }
    }
    o->rc_count = 0;
    o->rc_oldest = 0;
  }
  while (it < maxit) {
    recycle_cycle_start(o, x, n);
    const double beta = final_true;
    const double inv_beta = 1.0 / beta;
    for (size_t c = 0; c < n; ++c) V[0][c] = inv_beta * V[0][c];
    for (int i = 0; i < rows; ++i) g[i] = 0.0;
    g[0] = beta;
    int restarted = 0;
    for (int column = 0; column < restart && it < maxit; ++column) {
      double* v = V[column];
      hfo_apply_mg(o, v, Z[column]);
      ++pc_applies;
      hfo_apply_operator(o, Z[column], ax);
      ++op_applies;
      for (size_t c = 0; c < n; ++c) ax[c] = ax[c] + -FGMRES_SHIFT * v[c];
      const int count = column + 1;
      /* local_multidot: Neumaier dots v_i . w and w . w */
      double* column_h = h + (size_t)column * rows;
      for (int i = 0; i <= count; ++i) {
        const double* left = i == count ? ax : V[i];
        column_h[i] = dot(left, ax, n, &ok);
      }
      if (!ok) { term = TERM_NON_FINITE; status = 5; goto done; }
      const double bar_norm = column_h[count];
      for (int r = 0; r < count; ++r) scales[r] = -column_h[r];
      /* single_reduction_fgmres_norm */
      double t = bar_norm;
      for (int r = 0; r < count; ++r) t = t - column_h[r] * column_h[r];
      int unsafe = 0;
      double next_norm;
      if (!isfinite(t)) { term = TERM_NON_FINITE; status = 5; goto done; }
      if (t < 0.0) { unsafe = 1; next_norm = 0.0; }
      else next_norm = sqrt(t);
      if (unsafe && column != 0) {
        /* Discard the column: finish the cycle on the previous columns. */
        ++it;
        const int valid = column;
        const int bs = back_substitute(h, g, y, valid, rows);
        if (bs >= 0) { term = bs; status = 5; goto done; }
        if (!add_scaled_basis(x, Z, y, valid, n)) { term = TERM_NON_FINITE; status = 5; goto done; }
        TRUE_RESIDUAL(final_true, x);
        recycle_publish(o, x, n, &rc_published);
        recursive = final_true;
        if (history && it - 1 < hcap) history[it - 1] = recursive;
        if (final_true <= tol) { term = TERM_CONVERGED; status = 0; goto done; }
        if (it == maxit) { term = TERM_MAXIMUM; status = 6; goto done; }
        memset(h, 0, (size_t)rows * restart * sizeof(double));
        memset(cs, 0, (size_t)restart * sizeof(double));
        memset(sn, 0, (size_t)restart * sizeof(double));
        memset(g, 0, (size_t)rows * sizeof(double));
        memset(y, 0, (size_t)restart * sizeof(double));
        restarted = 1;
        break;
      }
      int explicit_orth = 0;
      if (unsafe || next_norm == 0.0) {
        /* Explicit second orthogonalisation pass, measured stably. */
        add_scaled_basis(ax, V, scales, count, n);
        for (int r = 0; r < count; ++r) y[r] = dot(V[r], ax, n, &ok);
        for (int r = 0; r < count; ++r) {
          column_h[r] += y[r];
          scales[r] = -y[r];
        }
        add_scaled_basis(ax, V, scales, count, n);
        next_norm = norm2(ax, n, &ok);
        if (!ok) { term = TERM_NON_FINITE; status = 5; goto done; }
        explicit_orth = 1;
      }
      column_h[column] += FGMRES_SHIFT;
      column_h[column + 1] = next_norm;
      for (int r = 0; r < column; ++r) {
        double* upper = &h[(size_t)column * rows + r];
        double* lower = &h[(size_t)column * rows + r + 1];
        const double rotated = cs[r] * *upper + sn[r] * *lower;
        *lower = -sn[r] * *upper + cs[r] * *lower;
        *upper = rotated;
      }
      double* diagonal = &h[(size_t)column * rows + column];
      double* subdiagonal = &h[(size_t)column * rows + column + 1];
      const double rotation_norm = hypot(*diagonal, *subdiagonal);
      if (!(rotation_norm > 0.0) || !isfinite(rotation_norm)) {
        term = TERM_BREAKDOWN; status = 5; goto done;
      }
      cs[column] = *diagonal / rotation_norm;
      sn[column] = *subdiagonal / rotation_norm;
      *diagonal = rotation_norm;
      *subdiagonal = 0.0;
      g[column + 1] = -sn[column] * g[column];
      g[column] = cs[column] * g[column];
      recursive = fabs(g[column + 1]);
      ++it;
      if (history && it - 1 < hcap) history[it - 1] = recursive;
      const int happy = next_norm == 0.0;
      const int cycle_end = happy || column + 1 == restart || it == maxit;
      const int verify = happy || (!deferred && recursive <= tol) || it % tri == 0 ||
                         cycle_end;
      if (!cycle_end) {
        if (!explicit_orth) add_scaled_basis(ax, V, scales, count, n);
        const double inv = 1.0 / next_norm;
        for (size_t c = 0; c < n; ++c) V[column + 1][c] = inv * ax[c];
      }
      if (!verify) continue;
      const int bs = back_substitute(h, g, y, count, rows);
      if (bs >= 0) { term = bs; status = 5; goto done; }
      if (!cycle_end) {
        /* Audit the candidate in the unused last basis slot. */
        double* trial = V[restart];
        memcpy(trial, x, n * sizeof(double));
        add_scaled_basis(trial, Z, y, count, n);
        hfo_apply_operator(o, trial, ax);
        ++op_applies;
        for (size_t c = 0; c < n; ++c) ax[c] = 1.0 * rhs[c] + -1.0 * ax[c];
        const double audited = norm2(ax, n, &ok);
        final_true = audited;
        if (audited <= tol) {
          recycle_publish(o, trial, n, &rc_published);
          memcpy(x, trial, n * sizeof(double));
          term = TERM_CONVERGED; status = 0; goto done;
        }
        continue;
      }
      add_scaled_basis(x, Z, y, count, n);
      TRUE_RESIDUAL(final_true, x);
      recycle_publish(o, x, n, &rc_published);
      recursive = final_true;
      if (final_true <= tol) { term = TERM_CONVERGED; status = 0; goto done; }
      if (it == maxit) { term = TERM_MAXIMUM; status = 6; goto done; }
      if (happy) {
        const double guard = 64.0 * DBL_EPSILON * (beta > tol ? beta : tol);
        if (!(final_true + guard < beta)) { term = TERM_BREAKDOWN; status = 5; goto done; }
      }
      restarted = 1;
      break;
    }
    if (!restarted) break;
  }
done:
#undef TRUE_RESIDUAL
  out[0] = it;
  out[1] = initial;
  out[2] = final_true;
  out[3] = term;
  out[6] = (double)op_applies;
  out[7] = (double)pc_applies;
  out[8] = (double)rc_offered;
  out[9] = (double)rc_retained;
  out[10] = (double)rc_accepted;
  out[11] = rc_projected;
  out[12] = (double)rc_published;
  for (int i = 0; i < rows; ++i) free(V[i]);
  for (int i = 0; i < restart; ++i) free(Z[i]);
  free(V); free(Z); free(ax); free(h); free(cs); free(sn); free(g); free(y);
  free(scratch); free(scales);
  (void)recursive;
  return ok ? status : 5;
}

/* ------------------------------------------------------------------ */
/* solve_bicgstab (src/solver_krylov.cpp:2651-3090) with the default      */
/* control (no bounded recurrence, no maximum norm, no best-iterate        */
/* retention): early exit on |s|, restart after every true-residual        */
/* verification that does not converge, rho carried from the fused update. */
/* ------------------------------------------------------------------ */
int hfo_solve_bicgstab(void* handle, const double* rhs, double* x, double rtol,
                       double atol, int maxit, int tri, double* out, double* history,
                       int hcap) {
  oracle_t* o = handle;
  const size_t n = o->lv[0].cells;
  int ok = 1, it = 0, term = TERM_MAXIMUM, status = 6;
  long op_applies = 0, pc_applies = 0;
  memset(out, 0, 8 * sizeof(double));
  double* r = malloc(n * sizeof(double));
  double* rh = malloc(n * sizeof(double));
  double* p = malloc(n * sizeof(double));
  double* sv = malloc(n * sizeof(double));
  double* ph = malloc(n * sizeof(double));
  double* sh = malloc(n * sizeof(double));
  double* v = malloc(n * sizeof(double));
  double* t = malloc(n * sizeof(double));
  double* ax = malloc(n * sizeof(double));
  double initial = 0.0, final_true = 0.0;
  const double bnorm = norm2(rhs, n, &ok);
  if (!ok) { term = TERM_NON_FINITE; status = 5; goto done; }
  const double tol = atol > rtol * bnorm ? atol : rtol * bnorm;
  out[4] = bnorm;
  out[5] = tol;
  if (bnorm == 0.0) { memset(x, 0, n * sizeof(double)); term = TERM_ZERO_RHS; status = 0; goto done; }
#define TRUE_RESIDUAL(dst_norm)                                           \
  do {                                                                    \
    hfo_apply_operator(o, x, ax);                                         \
    ++op_applies;                                                         \
    for (size_t c = 0; c < n; ++c) r[c] = 1.0 * rhs[c] + -1.0 * ax[c];    \
    dst_norm = norm2(r, n, &ok);                                          \
  } while (0)
  TRUE_RESIDUAL(initial);
  final_true = initial;
  if (initial <= tol) { term = TERM_CONVERGED; status = 0; goto done; }
  memcpy(rh, r, n * sizeof(double));
  double rho_prev = 1.0, alpha = 1.0, omega = 1.0;
  int fresh = 1;
  while (it < maxit) {
    const double rho = dot(rh, r, n, &ok);
    if (rho == 0.0 || !isfinite(rho)) { term = TERM_BREAKDOWN; status = 5; goto done; }
    if (fresh) {
      memcpy(p, r, n * sizeof(double));
    } else {
      if (omega == 0.0 || !isfinite(omega)) { term = TERM_BREAKDOWN; status = 5; goto done; }
      const double beta = (rho / rho_prev) * (alpha / omega);
      for (size_t c = 0; c < n; ++c) {
        const double intermediate = 1.0 * p[c] + -omega * v[c];
        p[c] = 1.0 * r[c] + beta * intermediate;
      }
    }
    apply_pc(o, p, ph);
    ++pc_applies;
    hfo_apply_operator(o, ph, v);
    ++op_applies;
    const double denominator = dot(rh, v, n, &ok);
    if (denominator == 0.0 || !isfinite(denominator)) { term = TERM_BREAKDOWN; status = 5; goto done; }
    alpha = rho / denominator;
    for (size_t c = 0; c < n; ++c) sv[c] = 1.0 * r[c] + -alpha * v[c];
    const double s_norm = norm2(sv, n, &ok);
    if (s_norm <= tol) {
      for (size_t c = 0; c < n; ++c) x[c] = x[c] + alpha * ph[c];
      ++it;
      TRUE_RESIDUAL(final_true);
      if (history && it - 1 < hcap) history[it - 1] = final_true;
      if (final_true <= tol) { term = TERM_CONVERGED; status = 0; goto done; }
      if (it == maxit) { term = TERM_MAXIMUM; status = 6; goto done; }
      memcpy(rh, r, n * sizeof(double));
      rho_prev = 1.0; alpha = 1.0; omega = 1.0; fresh = 1;
      continue;
    }
    apply_pc(o, sv, sh);
    ++pc_applies;
    hfo_apply_operator(o, sh, t);
    ++op_applies;
    /* local_dot_pair(t, s): t.s and t.t, Neumaier each */
    const double ts = dot(t, sv, n, &ok);
    const double tt = dot(t, t, n, &ok);
    if (!(tt > 0.0) || !isfinite(ts) || !isfinite(tt)) { term = TERM_BREAKDOWN; status = 5; goto done; }
    omega = ts / tt;
    if (omega == 0.0 || !isfinite(omega)) { term = TERM_BREAKDOWN; status = 5; goto done; }
    for (size_t c = 0; c < n; ++c) {
      const double intermediate = x[c] + alpha * ph[c];
      x[c] = intermediate + omega * sh[c];
      r[c] = 1.0 * sv[c] + -omega * t[c];
    }
    ++it;
    const double recursive = norm2(r, n, &ok);
    if (history && it - 1 < hcap) history[it - 1] = recursive;
    const int verify = recursive <= tol || it % tri == 0 || it == maxit;
    if (verify) {
      TRUE_RESIDUAL(final_true);
      if (final_true <= tol) { term = TERM_CONVERGED; status = 0; goto done; }
      if (it == maxit) { term = TERM_MAXIMUM; status = 6; goto done; }
      memcpy(rh, r, n * sizeof(double));
      rho_prev = 1.0; alpha = 1.0; omega = 1.0; fresh = 1;
      continue;
    }
    rho_prev = rho;
    fresh = 0;
  }
done:
#undef TRUE_RESIDUAL
  out[0] = it;
  out[1] = initial;
  out[2] = final_true;
  out[3] = term;
  out[6] = (double)op_applies;
  out[7] = (double)pc_applies;
  free(r); free(rh); free(p); free(sv); free(ph); free(sh); free(v); free(t); free(ax);
  return ok ? status : 5;
}

/* ------------------------------------------------------------------ */
void* hfo_create(int nx, int ny, int nz, const double* xf, const double* yf,
                 const double* zf, const int* bc, const double* diagonal,
                 const double* fx, const double* fy, const double* fz,
                 const unsigned char* active, const int* options,
                 const double* reals, int* status) {
  *status = 2;
  if (nx <= 0 || ny <= 0 || nz <= 0) return NULL;
  for (int f = 0; f < 6; ++f)
    if (bc[f] != BC_DIRICHLET && bc[f] != BC_NEUMANN) return NULL;
  oracle_t* o = calloc(1, sizeof(oracle_t));
  if (!o) return NULL;
  o->n[0] = nx;
  o->n[1] = ny;
  o->n[2] = nz;
  memcpy(o->bc, bc, sizeof(o->bc));
  const size_t cells = (size_t)nx * ny * nz;
  const size_t nf[3] = {(size_t)(nx + 1) * ny * nz, (size_t)nx * (ny + 1) * nz,
                        (size_t)nx * ny * (nz + 1)};
  const double* src_faces[3] = {xf, yf, zf};
  for (int a = 0; a < 3; ++a) {
    o->faces[a] = malloc((size_t)(o->n[a] + 1) * sizeof(double));
    memcpy(o->faces[a], src_faces[a], (size_t)(o->n[a] + 1) * sizeof(double));
  }
  o->diag0 = malloc(cells * sizeof(double));
  o->fx0 = malloc(nf[0] * sizeof(double));
  o->fy0 = malloc(nf[1] * sizeof(double));
  o->fz0 = malloc(nf[2] * sizeof(double));
  memcpy(o->diag0, diagonal, cells * sizeof(double));
  memcpy(o->fx0, fx, nf[0] * sizeof(double));
  memcpy(o->fy0, fy, nf[1] * sizeof(double));
  memcpy(o->fz0, fz, nf[2] * sizeof(double));
  if (active) {
    o->active = malloc(cells);
    memcpy(o->active, active, cells);
  }
  o->smoother = options[2];
  o->cycle = options[3];
  o->pre = options[4];
  o->post = options[5];
  o->coarse_sweeps = options[6];
  o->unit_linear = options[7];
  o->max_levels = options[8];
  o->min_extent = options[9];
  o->line_order = options[10];
  o->pc_kind = options[11];
  o->cheb_fraction = reals[0];
  o->anisotropy = reals[1];
  o->shortcut_ratio = reals[2];
  for (int w = 0; w < 6; ++w) o->work[w] = calloc(cells, sizeof(double));
  if (build_shapes(o) != 0 || build_coarse(o) != 0) {
    hfo_destroy(o);
    return NULL;
  }
  select_shortcut(o);
  if (o->pc_kind != 0) {
    o->dic_diag = calloc(cells, sizeof(double));
    o->dic_nb = calloc(6 * cells, sizeof(double));
    o->dic_inv = calloc(cells, sizeof(double));
    dic_rows(o);
    if (dic_prepare(o) != 0) {
      hfo_destroy(o);
      *status = 5;
      return NULL;
    }
  }
  *status = 0;
  return o;
}

void hfo_destroy(void* handle) {
  oracle_t* o = handle;
  if (!o) return;
  for (int l = 0; l < o->levels; ++l) {
    level_t* L = &o->lv[l];
    free(L->diag); free(L->vol); free(L->fx); free(L->fy); free(L->fz);
    free(L->x); free(L->b); free(L->r); free(L->t);
  }
  for (int a = 0; a < 3; ++a) free(o->faces[a]);
  for (int w = 0; w < 6; ++w) free(o->work[w]);
  for (int r = 0; r < 4; ++r) { free(o->rc_ring[r]); free(o->rc_image[r]); }
  free(o->dic_diag); free(o->dic_nb); free(o->dic_inv);
  free(o->rc_snapshot);
  free(o->diag0); free(o->fx0); free(o->fy0); free(o->fz0); free(o->active);
  free(o);
}

int hfo_levels(void* handle, int* shapes, int capacity) {
  oracle_t* o = handle;
  for (int l = 0; l < o->levels && l < capacity; ++l) {
    shapes[4 * l + 0] = o->lv[l].n[0];
    shapes[4 * l + 1] = o->lv[l].n[1];
    shapes[4 * l + 2] = o->lv[l].n[2];
    shapes[4 * l + 3] = o->lv[l].line_mask;
  }
  return o->levels;
}

int hfo_level_coefficients(void* handle, int level, double* diagonal,
                           double* face_x, double* face_y, double* face_z,
                           double* volume) {
  oracle_t* o = handle;
  if (level < 0 || level >= o->levels) return 2;
  const level_t* L = &o->lv[level];
  if (diagonal) memcpy(diagonal, L->diag, L->cells * sizeof(double));
  if (face_x) memcpy(face_x, L->fx, L->fxn * sizeof(double));
  if (face_y) memcpy(face_y, L->fy, L->fyn * sizeof(double));
  if (face_z) memcpy(face_z, L->fz, L->fzn * sizeof(double));
  if (volume) memcpy(volume, L->vol, L->cells * sizeof(double));
  return 0;
}
