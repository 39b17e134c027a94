/*
 * hf_pressure_solver.h -- C ABI of the B200 pressure-coupling linear solve.
 *
 * Drop-in for the reference's linear-solver/preconditioner interface on the
 * cell-centred 7-point pressure system  div(beta grad p) = rhs  with IBM-
 * masked cells.  Paths in the citations are relative to versions/v0.4 of the
 * reference.  Every entry point returns an hfps_status whose values are the
 * reference's StatusCode (include/hundun/v04_status.hpp:13-22); nothing
 * throws across this boundary, and a failed solve publishes no solution
 * (src/solver_krylov.cpp:1207-1250).
 *
 * Layout: every cell field is a dense x-fastest array of nx*ny*nz values;
 * face arrays have extents (nx+1,ny,nz), (nx,ny+1,nz), (nx,ny,nz+1), also
 * x-fastest (src/solver_mg.cpp:1456-1466).  A `memory` argument says whether
 * the pointers are host memory (HFPS_HOST) or device memory on the solver's
 * GPU (HFPS_DEVICE).  A handle is bound to one GPU and one CUDA stream and is
 * not thread-safe, matching the reference's one-rank-one-thread contract.
 */
#ifndef HF_PRESSURE_SOLVER_H
#define HF_PRESSURE_SOLVER_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define HFPS_API __attribute__((visibility("default")))
#else
#define HFPS_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* StatusCode (include/hundun/v04_status.hpp:13-22). */
typedef enum hfps_status {
  HFPS_OK = 0,
  HFPS_INVALID_CASE = 1,
  HFPS_INVALID_PLAN = 2,
  HFPS_ALLOCATION_FAILURE = 3,
  HFPS_MPI_FAILURE = 4,
  HFPS_NUMERICAL_FAILURE = 5,
  HFPS_REJECTED_STEP = 6,
  HFPS_IO_FAILURE = 7
} hfps_status;

/* LinearTermination (include/hundun/v04_linear.hpp:77-88). */
typedef enum hfps_termination {
  HFPS_CONVERGED = 0,
  HFPS_ZERO_RHS = 1,
  HFPS_MAXIMUM_ITERATIONS = 2,
  HFPS_BREAKDOWN = 3,
  HFPS_NON_FINITE = 4,
  HFPS_OPERATOR_FAILURE = 5,
  HFPS_PRECONDITIONER_FAILURE = 6,
  HFPS_COLLECTIVE_FAILURE = 7,
  HFPS_TERMINATION_INVALID_PLAN = 8
} hfps_termination;

/* MgBoundaryKind (include/hundun/v04_linear.hpp:100-104).  Periodic is
 * rejected with HFPS_INVALID_PLAN. */
typedef enum hfps_boundary {
  HFPS_DIRICHLET = 0,
  HFPS_NEUMANN = 1,
  HFPS_PERIODIC = 2
} hfps_boundary;

typedef enum hfps_memory { HFPS_HOST = 0, HFPS_DEVICE = 1 } hfps_memory;

/* LinearAlgorithm (include/hundun/v04_case.hpp:21). */
typedef enum hfps_algorithm { HFPS_PCG = 0, HFPS_FGMRES = 1, HFPS_BICGSTAB = 2 } hfps_algorithm;

/* Preconditioner: the multigrid plan, or the cold path's diagonal IC(0)
 * (ColdPressureIccg, src/solver_iccg.hpp:224-293; ColdPressureDilu,
 * src/solver_cold.hpp:484-560, the same factorisation on the symmetric
 * pressure rows), evaluated in the reference's lexicographic order. */
typedef enum hfps_preconditioner {
  HFPS_PRECONDITIONER_MG = 0,
  HFPS_PRECONDITIONER_IC0 = 1
} hfps_preconditioner;

/* FP64: every kernel in FP64.  MIXED: MG hierarchy stored and cycled in
 * FP32 inside an FP64 Krylov/refinement loop; residuals, dot products, norms
 * and the coarsest-grid solve stay FP64. */
typedef enum hfps_precision { HFPS_FP64 = 0, HFPS_MIXED = 1 } hfps_precision;

/* MgHierarchyPolicy (include/hundun/v04_linear.hpp:115-131) plus the
 * correction scaling of NativeCartesianMgSpec (:316-329). */
typedef struct hfps_policy {
  int point_smoother;       /* 0 red-black (omega 0.72), 1 Chebyshev-Jacobi */
  int cycle;                /* 0 V-cycle, 1 F-cycle */
  int pre_sweeps;           /* default 2 */
  int post_sweeps;          /* default 2 */
  int coarse_sweeps;        /* default 24 */
  int maximum_levels;       /* default 32 */
  int minimum_coarse_extent;/* default 3 */
  int unit_linear;          /* 1: correction scale 1 (fixed, PCG);
                               0: residual-minimising (flexible, FGMRES) */
  double chebyshev_lower_spectrum_fraction; /* default 0.3 */
  double anisotropy_threshold;              /* default 4.0 */
  double diagonal_shortcut_maximum_ratio;   /* default 0.0 (off) */
  int preconditioner;                       /* hfps_preconditioner, default MG */
  int null_space;                           /* hfps_null_space, default NONE */
} hfps_policy;

/* MgNullSpace (include/hundun/v04_linear.hpp:104).  CONSTANT, for a system
 * whose operator annihilates constants (every boundary Neumann): the MG
 * application removes the volume-weighted mean from its level-0 rhs, from
 * every restricted coarse rhs and from its result (project_constant,
 * src/solver_mg.cpp:1411-1453, 3708-3716, 4900-4960), and the diagonal
 * shortcut is not taken.  The rhs must be consistent (zero-sum). */
typedef enum hfps_null_space {
  HFPS_NULL_SPACE_NONE = 0,
  HFPS_NULL_SPACE_CONSTANT = 1
} hfps_null_space;

/* Cartesian geometry: face coordinates per axis (n+1 values each),
 * boundary kinds [x_min, x_max, y_min, y_max, z_min, z_max] and an optional
 * host cell activity map (1 fluid, 0 IBM solid; NULL = all fluid). */
typedef struct hfps_geometry {
  int nx, ny, nz;
  const double* x_faces;
  const double* y_faces;
  const double* z_faces;
  int boundary[6];
  const uint8_t* cell_active;
} hfps_geometry;

/* LinearSolveControl (include/hundun/v04_linear.hpp:453-465) plus the
 * algorithm/precision selection. */
typedef struct hfps_control {
  double relative_tolerance;
  double absolute_tolerance;
  uint32_t maximum_iterations;
  uint32_t true_residual_interval;
  uint32_t restart;   /* FGMRES restart length; 0 for PCG */
  int algorithm;      /* hfps_algorithm */
  int precision;      /* hfps_precision */
  int recycle;        /* hfps_recycle (FGMRES only) */
  int norm;           /* hfps_norm */
} hfps_control;

/* How the solve forms the 2-norms of rhs and residuals.  PLAIN (default):
 * sqrt of a fixed-order FP64 sum of squares, fused into the kernel that
 * produces the vector.  SCALED: the reference's global_norm
 * (src/solver_krylov.cpp:650-711): max |v| first, then max * sqrt(sum of
 * (v / max)^2), in two extra passes; used for ||b||, every true residual and
 * the recursive residuals of PCG and BiCGSTAB.  The Arnoldi norms of FGMRES
 * keep their own form (its Pythagorean update with fallbacks). */
typedef enum hfps_norm {
  HFPS_NORM_PLAIN = 0,
  HFPS_NORM_SCALED = 1
} hfps_norm;

/* Subspace recycling across consecutive pressure solves (FGMRES only), as
 * PressureVelocityCoupler selects it per corrector (src/solver_piso.cpp:
 * 10410-10433; SolverWorkspace recycle state, src/solver_linear_state.cpp:
 * 735-1037).  CAPTURE (corrector 1) records the correction of every Arnoldi
 * cycle, up to the 4 latest; PROJECT (corrector 2, same system) starts from
 * the least-squares combination of them when that lowers the true residual
 * (src/solver_krylov.cpp:1745-2019); GUARD only replaces an initial guess
 * whose residual exceeds |b| by zero (also active while capturing). */
typedef enum hfps_recycle {
  HFPS_RECYCLE_NONE = 0,
  HFPS_RECYCLE_CAPTURE = 1,
  HFPS_RECYCLE_PROJECT = 2,
  HFPS_RECYCLE_GUARD = 3
} hfps_recycle;

/* LinearSolveResult subset (include/hundun/v04_linear.hpp:530-579). */
typedef struct hfps_result {
  int status;
  uint32_t detail;
  int termination;
  uint32_t iterations;
  double initial_true_residual;
  double final_true_residual;
  double recursive_residual;
  double rhs_norm;
  double true_residual_limit;
  uint64_t operator_applies;
  uint64_t preconditioner_applies;
  uint32_t history_length;   /* entries written to the history buffer */
  uint32_t levels;           /* MG levels in the hierarchy */
  double seconds;            /* wall time of the solve on the host */
  uint64_t kernel_launches;  /* this library's kernels launched by the call */
  uint32_t recycle_offered;      /* captured corrections offered to the projection */
  uint32_t recycle_retained;     /* kept after the rank test */
  uint32_t recycle_accepted;     /* 1 when the projected start was taken */
  uint32_t recycle_captured;     /* corrections captured by this solve */
  double recycle_projected_residual;
} hfps_result;

typedef struct hfps_solver hfps_solver;

/* Fills `policy` with the MgHierarchyPolicy struct defaults (red-black
 * V(2,2), 24 coarse sweeps, unit_linear). */
HFPS_API void hfps_default_policy(hfps_policy* policy);
/* production_pressure_mg_policy (src/solver_piso_detail.hpp:10-19):
 * Chebyshev pre 1 / post 2, F-cycle, fraction 0.3, diagonal shortcut 0.1. */
HFPS_API void hfps_production_policy(hfps_policy* policy);
HFPS_API void hfps_default_control(hfps_control* control);

/* Builds the level hierarchy and workspaces on the current CUDA device.
 * Replaces NativeCartesianMgPlan::compile + make_mg_workspace_requirements +
 * SolverWorkspace::bind (include/hundun/v04_linear.hpp:945-960, 1046-1064).
 * `stream` is a cudaStream_t on which every later call reads its device
 * inputs and writes its device outputs; the caller orders the producers of
 * HFPS_DEVICE inputs before the call on that stream.  NULL (also what a
 * caller on the legacy default stream passes) makes the solver create and
 * own a blocking stream, which is ordered with the legacy default stream. */
HFPS_API int hfps_create(const hfps_geometry* geometry, const hfps_policy* policy,
                void* stream, hfps_solver** out);

/* Sets the operator: diagonal (cells) and face coefficients (unmasked, as
 * the regular PressureLinearOperator receives them).  Solid cells become
 * identity rows and every fluid/solid face is removed, exactly as
 * IbmPressureOperator::decorate_pressure_action
 * (src/solver_ibm_pressure.cpp:347-385) and copy_finest_coefficients
 * (src/solver_mg.cpp:1469-1570) do; then the coarse levels are aggregated
 * (build_coarse_coefficients, src/solver_mg.cpp:1858-1925).  Replaces
 * NativeCartesianMgPlan::update_coefficients (v04_linear.hpp:955-960). */
HFPS_API int hfps_set_coefficients(hfps_solver* solver, const double* diagonal,
                          const double* face_x, const double* face_y,
                          const double* face_z, int memory);

/* Builds the coefficients from cell beta with face_pressure_coefficient's
 * distance-weighted harmonic rule (src/solver_piso.cpp:1060-1136):
 * interior c = A/(dL/bL + dR/bR), Dirichlet boundary c = A*b/d, Neumann 0;
 * diagonal = sum of faces + storage (storage may be NULL). */
HFPS_API int hfps_set_beta(hfps_solver* solver, const double* beta,
                  const double* storage, int memory);

/* Inputs of the pressure-correction assembly (PressureCorrectionInput,
 * src/solver_pressure.cpp:110-332).  Cell arrays are nx*ny*nz values, flux
 * arrays the face extents; all in the memory the call names. */
typedef struct hfps_assembly {
  int bdf_order;                  /* 1 or 2 */
  double a0, a1, a2;              /* BDF coefficients, a0 > 0 */
  const double* beta;             /* cell beta for face_pressure_coefficient */
  const double* density_trial;    /* rho^*, > 0 */
  const double* density_accepted; /* rho^n, > 0 */
  const double* density_previous; /* rho^{n-1} (BDF2 only; NULL for BDF1) */
  const double* drho_dp;          /* d rho / d p at constant h, Y; > 0 */
  const double* mass_source;      /* NULL = none */
  const double* flux_x;           /* predicted face mass fluxes phi_HbyA */
  const double* flux_y;
  const double* flux_z;
} hfps_assembly;

/* Assembles the pressure-correction system on the device and makes it the
 * solver's operator: face coefficients from beta (face_pressure_coefficient,
 * src/solver_piso.cpp:1060-1136), then per cell, in the reference's order,
 * diag = a0 V drho_dp + sum of the six face coefficients and
 * rhs = -(V (a0 rho + a1 rho_n + a2 rho_{n-1} - S) + outward flux)
 * (assemble_pressure_system_impl, src/solver_pressure.cpp:110-332), then
 * the IBM masking and coarse levels as hfps_set_coefficients.  Writes rhs.
 * Inputs the reference rejects (non-positive densities, derivative, volume
 * or diagonal; negative or non-finite faces; non-finite results) return
 * HFPS_NUMERICAL_FAILURE and change nothing. */
HFPS_API int hfps_assemble(hfps_solver* solver, const hfps_assembly* assembly,
                           double* rhs, int memory);

/* Post-solve flux correction: flux_f += -c_f * (scale * jump_f(correction))
 * on every face, jump = p'_R - p'_L inside, the owner cell's value (negated
 * on a high face) at a Dirichlet boundary face and 0 at a Neumann one
 * (PressureCorrectionBoundaryPlan::mass_flux_response, src/solver_piso.cpp:
 * 1605-1653, as applied over all faces at :7400-7420).  coefficient_* are
 * the pressure face coefficients the caller assembled with; flux_* are
 * updated in place. */
HFPS_API int hfps_correct_flux(hfps_solver* solver, const double* correction,
                               const double* coefficient_x,
                               const double* coefficient_y,
                               const double* coefficient_z,
                               double correction_scale, double* flux_x,
                               double* flux_y, double* flux_z, int memory);

/* solve(rhs, x0, tol) -> x, iterations, residual history.  Replaces
 * solve_pcg / solve_fgmres with NativeCartesianMgPlan as preconditioner
 * (include/hundun/v04_linear.hpp:1070-1088; src/solver_krylov.cpp:1299-1555,
 * 1557-2650).  control->algorithm selects HFPS_PCG (restart 0; needs the
 * unit_linear MG scaling, as solve_pcg needs a fixed SPD preconditioner) or
 * HFPS_FGMRES (restart 1..64; either scaling, the reference's production
 * choice being the residual-minimising one with restart 12).  `solution`
 * holds x0 on entry and x on success; on failure it is left unchanged.
 * `history` (may be NULL) receives the recursive residual norm after every
 * iteration, up to `history_capacity` values. */
HFPS_API int hfps_solve(hfps_solver* solver, const double* rhs, double* solution,
               int memory, const hfps_control* control, hfps_result* result,
               double* history, uint32_t history_capacity);

/* y = A x with the IBM-decorated operator (LinearOperator::apply,
 * include/hundun/v04_linear.hpp:396-405; src/solver_pressure.cpp:969-991). */
HFPS_API int hfps_apply_operator(hfps_solver* solver, const double* x, double* y,
                        int memory);

/* z = M r, one MG preconditioner application (LinearPreconditioner::apply,
 * include/hundun/v04_linear.hpp:418-420; src/solver_mg.cpp:4814-5122). */
HFPS_API int hfps_apply_preconditioner(hfps_solver* solver, const double* r, double* z,
                              int memory, int precision);

/* Adjoint of a converged solve: solves A^T lambda = dL/dp (A is symmetric,
 * so the forward solver is reused) and forms dL/dc_f = -(lambda_i -
 * lambda_j)(p_i - p_j) per interior face (-lambda_i p_i on a Dirichlet
 * boundary face; 0 on Neumann and IBM-removed faces), dL/drhs = lambda.
 * Any of lambda/grad_* may be NULL.  No reference counterpart: the reference
 * has no adjoint path. */
HFPS_API int hfps_adjoint(hfps_solver* solver, const double* solution,
                 const double* dl_dp, double* lambda, double* grad_face_x,
                 double* grad_face_y, double* grad_face_z, int memory,
                 const hfps_control* control, hfps_result* result);

/* Level shapes: writes [nx, ny, nz, line_axis_mask] per level (up to
 * capacity levels) and returns the level count (NativeCartesianMgPlan::level,
 * include/hundun/v04_linear.hpp:968-969). */
HFPS_API int hfps_levels(hfps_solver* solver, int* shapes, int capacity);

/* Copies one level's masked/aggregated coefficients to host arrays (any may
 * be NULL); `volume` receives the fluid volume per cell. */
HFPS_API int hfps_level_coefficients(hfps_solver* solver, int level, double* diagonal,
                            double* face_x, double* face_y, double* face_z,
                            double* volume);

/* Kernel classes timed by hfps_profile_kernel. */
typedef enum hfps_kernel {
  HFPS_KERNEL_OPERATOR = 0,        /* level-0 FP64 stencil y = A x with x.y */
  HFPS_KERNEL_SMOOTH_FP64 = 1,     /* one level-0 smoother pass, FP64 */
  HFPS_KERNEL_SMOOTH_FP32 = 2,     /* one level-0 smoother pass, FP32 */
  HFPS_KERNEL_RESTRICT_FP64 = 3,   /* fused level-0 defect + restriction */
  HFPS_KERNEL_PROLONG_FP64 = 4,    /* level-1 -> level-0 prolongation */
  HFPS_KERNEL_PCG_UPDATE = 5,      /* x += a p, r -= a Ap, |r|^2 */
  HFPS_KERNEL_MG_FP64 = 6,         /* one whole FP64 MG application */
  HFPS_KERNEL_MG_MIXED = 7,        /* one whole FP32 MG application */
  HFPS_KERNEL_RESIDUAL = 8         /* level-0 true residual r = b - A x with |r|^2 */
} hfps_kernel;

/* Launches one kernel class `repetitions` times on the solver's stream
 * between CUDA events, on the solver's current data, and reports the mean
 * device time per launch and the algorithmic HBM bytes one launch must move
 * (each operand read or written once).  Scratch vectors are overwritten; the
 * coefficients are not.  No reference counterpart: the reference's
 * MgApplyProfile (include/hundun/v04_linear.hpp:191-230) times host phases. */
HFPS_API int hfps_profile_kernel(hfps_solver* solver, int kernel,
                                 int repetitions, double* milliseconds,
                                 double* bytes);

/* ---- Allocation-free operator apply ------------------------------------
 * No counterpart in the reference.  Every other entry point works through a
 * solver handle whose workspaces were allocated by hfps_create.  Some callers
 * cannot allocate device memory at the point where they need A x: a step
 * running inside a fixed memory pool or a caching allocator that forbids new
 * device allocations mid-step, or code that must keep a fixed footprint.
 * This entry point serves them.  It works on device arrays the caller
 * already owns, never allocates device or pinned memory, and keeps its
 * reduction scratch in a fixed array inside the library.
 *
 * It computes y = A x and, when x_dot_y is not NULL, x . (A x).  The
 * coefficients are the IBM-masked finest-level ones, laid out as
 * hfps_level_coefficients(solver, 0, ...) returns them: solid cells have an
 * identity row, removed faces are 0.  All arrays are device memory on the
 * current CUDA device; `stream` is a cudaStream_t (NULL: the default stream).
 * The call is asynchronous: y and *x_dot_y are ready when the stream is.
 *
 * The first call on each device does a one-time set-up: it looks up the
 * address of the library's scratch array on that device.  Make that first
 * call before any stream capture begins.  The looked-up address is kept for
 * the life of the process; cudaDeviceReset on a device voids it, so after a
 * reset this entry point must not be called on that device again.  The
 * scratch array is shared by every call on a device, so calls that overlap
 * in time (two streams, two host threads) race and give wrong results:
 * serialise them.
 *
 * Returns HFPS_OK, HFPS_INVALID_CASE when an extent is below 1 or the grid
 * has more than HFPS_NOALLOC_MAX_CELLS cells, or HFPS_INVALID_PLAN for a
 * periodic or unknown boundary kind, a NULL, misaligned or non-device
 * pointer, y overlapping x, x_dot_y inside x or y, or a CUDA runtime
 * error. */
#define HFPS_NOALLOC_MAX_CELLS (1LL << 30)   /* 32-bit face indexing */
#define HFPS_NOALLOC_MAX_BLOCKS 1184         /* reduction partials kept */

typedef struct hfps_operator_view {
  int nx, ny, nz;
  int boundary[6];            /* hfps_boundary per face, x_min..z_max */
  const double* diagonal;     /* nx*ny*nz */
  const double* face_x;       /* (nx+1)*ny*nz */
  const double* face_y;       /* nx*(ny+1)*nz */
  const double* face_z;       /* nx*ny*(nz+1) */
} hfps_operator_view;

HFPS_API int hfps_operator_dot_noalloc(const hfps_operator_view* op,
                                       const double* x, double* y,
                                       double* x_dot_y, void* stream);

/* Sticky error text of the last failing call on this handle.  With a NULL
 * handle: the reason the calling thread's last hfps_create failed. */
HFPS_API const char* hfps_last_error(hfps_solver* solver);

HFPS_API int hfps_destroy(hfps_solver* solver);

#ifdef __cplusplus
}
#endif

#endif /* HF_PRESSURE_SOLVER_H */
