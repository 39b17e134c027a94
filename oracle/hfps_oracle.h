/*
 * CPU restatement of the reference pressure solve (test infrastructure).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline leg use
 * this library, and only as the checker.  It restates, in plain C, the
 * reference's NativeCartesianMgPlan (src/solver_mg.cpp), its level shapes
 * (src/solver_mg_workspace.cpp) and solve_pcg (src/solver_krylov.cpp:
 * 1299-1555) with the same arithmetic order, so that the compiled reference
 * (oracle/_ref) pins it and it in turn pins the CUDA path.
 *
 * Arrays are dense and x-fastest.  Face arrays have extents (nx+1,ny,nz),
 * (nx,ny+1,nz) and (nx,ny,nz+1).
 */
#ifndef HFPS_ORACLE_H
#define HFPS_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* options: [algorithm(0 pcg), restart, smoother(0 red-black,1 chebyshev),
 *           cycle(0 V,1 F), pre, post, coarse_sweeps, scaling(0 residual-
 *           minimising,1 unit_linear), max_levels, min_coarse_extent,
 *           line_order(0 lexicographic as the reference, 1 zebra),
 *           preconditioner(0 MG plan, 1 diagonal IC(0) in the reference's
 *           lexicographic order = ColdPressureIccg / ColdPressureDilu on
 *           symmetric rows)]
 * reals:   [chebyshev_fraction, anisotropy_threshold, diagonal_shortcut] */
void* hfo_create(int nx, int ny, int nz, const double* x_faces,
                 const double* y_faces, const double* z_faces,
                 const int* boundary, const double* diagonal,
                 const double* face_x, const double* face_y,
                 const double* face_z, const unsigned char* active,
                 const int* options, const double* reals, int* status);
void hfo_destroy(void* handle);
int hfo_levels(void* handle, int* shapes, int capacity);
/* Level coefficients after masking/aggregation (diag, x, y, z, volume). */
int hfo_level_coefficients(void* handle, int level, double* diagonal,
                           double* face_x, double* face_y, double* face_z,
                           double* volume);
int hfo_apply_operator(void* handle, const double* x, double* y);
/* One level operator action y = A_l x on level l (level matrices). */
int hfo_apply_level(void* handle, int level, const double* x, double* y);
int hfo_apply_mg(void* handle, const double* r, double* z);
/* outputs: [iterations, initial_true, final_true, termination, rhs_norm,
 *           limit, operator_applies, preconditioner_applies]
 * history[i] = recursive residual norm after iteration i+1. */
int hfo_solve(void* handle, const double* rhs, double* x,
              double relative_tolerance, double absolute_tolerance,
              int maximum_iterations, int true_residual_interval,
              double* outputs, double* history, int history_capacity);

/* z = M r with the session's preconditioner (MG plan or cold-path DIC). */
int hfo_apply_preconditioner(void* handle, const double* r, double* z);
/* solve_bicgstab (src/solver_krylov.cpp:2651-3090), default control; same
 * outputs and history as hfo_solve. */
int hfo_solve_bicgstab(void* handle, const double* rhs, double* x,
                       double relative_tolerance, double absolute_tolerance,
                       int maximum_iterations, int true_residual_interval,
                       double* outputs, double* history, int history_capacity);
/* solve_fgmres (src/solver_krylov.cpp:1557-2650) with the MG plan as the
 * (flexible) preconditioner.  recycle: 0 none, 1 capture cycle corrections
 * for the next solve, 2 project the captured ones, 3 initial-guess guard
 * only.  outputs (13): hfo_solve's eight, then recycle offered, retained,
 * accepted, projected residual, corrections captured by this solve. */
int hfo_solve_fgmres(void* handle, const double* rhs, double* x,
                     double relative_tolerance, double absolute_tolerance,
                     int maximum_iterations, int true_residual_interval,
                     int restart, int recycle, double* outputs,
                     double* history, int history_capacity);

#ifdef __cplusplus
}
#endif
#endif
