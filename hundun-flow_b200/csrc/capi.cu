// extern "C" boundary of the pressure solve (include/hf_pressure_solver.h).
// Nothing throws across it: every failure becomes an hfps_status plus a
// sticky message readable through hfps_last_error.
#include <cstring>
#include <new>
#include <string>

#include "../../include/hf_pressure_solver.h"
#include "solver.hpp"

struct hfps_solver {
  hfps::Solver* impl{};
  std::string error;
};

namespace {

// Reason for the calling thread's last failed hfps_create (no handle exists
// to hold it); hfps_last_error(NULL) returns it.
thread_local std::string create_error;

int finish(hfps_solver* s, hfps::Status st) {
  if (!st && s != nullptr && s->impl != nullptr) s->error = s->impl->last_error();
  return st.code;
}

template <class F>
int guarded(hfps_solver* s, F&& body) {
  if (s == nullptr || s->impl == nullptr) return HFPS_INVALID_PLAN;
  try {
    return finish(s, body(*s->impl));
  } catch (const std::bad_alloc&) {
    s->error = "host allocation failure";
    return HFPS_ALLOCATION_FAILURE;
  } catch (...) {
    s->error = "unexpected host exception";
    return HFPS_INVALID_PLAN;
  }
}

}  // namespace

extern "C" {

void hfps_default_policy(hfps_policy* p) {
  if (p == nullptr) return;
  p->point_smoother = 0;
  p->cycle = 0;
  p->pre_sweeps = 2;
  p->post_sweeps = 2;
  p->coarse_sweeps = 24;
  p->maximum_levels = 32;
  p->minimum_coarse_extent = 3;
  p->unit_linear = 1;
  p->chebyshev_lower_spectrum_fraction = 0.3;
  p->anisotropy_threshold = 4.0;
  p->diagonal_shortcut_maximum_ratio = 0.0;
  p->preconditioner = HFPS_PRECONDITIONER_MG;
  p->null_space = HFPS_NULL_SPACE_NONE;
}

void hfps_production_policy(hfps_policy* p) {
  if (p == nullptr) return;
  hfps_default_policy(p);
  p->point_smoother = 1;
  p->cycle = 1;
  p->pre_sweeps = 1;
  p->post_sweeps = 2;
  p->diagonal_shortcut_maximum_ratio = 0.1;
}

void hfps_default_control(hfps_control* c) {
  if (c == nullptr) return;
  // solver.pressure_linear defaults (include/hundun/v04_case.hpp:314-323)
  // with the PCG algorithm.
  c->relative_tolerance = 1.0e-13;
  c->absolute_tolerance = 1.0e-13;
  c->maximum_iterations = 400;
  c->true_residual_interval = 4;
  c->restart = 0;
  c->algorithm = HFPS_PCG;
  c->precision = HFPS_FP64;
  c->recycle = HFPS_RECYCLE_NONE;
  c->norm = HFPS_NORM_PLAIN;
}

int hfps_create(const hfps_geometry* geometry, const hfps_policy* policy,
                void* stream, hfps_solver** out) {
  create_error.clear();
  if (out == nullptr || geometry == nullptr) {
    create_error = "null geometry or output handle";
    return HFPS_INVALID_PLAN;
  }
  *out = nullptr;
  hfps_policy defaults;
  hfps_default_policy(&defaults);
  try {
    std::string error;
    hfps::Solver* impl = nullptr;
    const hfps::Status st = hfps::Solver::create(
        *geometry, policy != nullptr ? *policy : defaults,
        static_cast<cudaStream_t>(stream), &impl, error);
    if (!st) {
      create_error = error;
      return st.code;
    }
    hfps_solver* handle = new (std::nothrow) hfps_solver();
    if (handle == nullptr) {
      delete impl;
      create_error = "host allocation failure";
      return HFPS_ALLOCATION_FAILURE;
    }
    handle->impl = impl;
    *out = handle;
    return HFPS_OK;
  } catch (const std::bad_alloc&) {
    create_error = "host allocation failure";
    return HFPS_ALLOCATION_FAILURE;
  } catch (...) {
    create_error = "unexpected host exception";
    return HFPS_INVALID_PLAN;
  }
}

int hfps_set_coefficients(hfps_solver* s, const double* diagonal,
                          const double* face_x, const double* face_y,
                          const double* face_z, int memory) {
  return guarded(s, [&](hfps::Solver& v) {
    return v.set_coefficients(diagonal, face_x, face_y, face_z, memory);
  });
}

int hfps_set_beta(hfps_solver* s, const double* beta, const double* storage,
                  int memory) {
  return guarded(s, [&](hfps::Solver& v) { return v.set_beta(beta, storage, memory); });
}

int hfps_assemble(hfps_solver* s, const hfps_assembly* assembly, double* rhs, int memory) {
  if (assembly == nullptr) return HFPS_INVALID_PLAN;
  return guarded(s, [&](hfps::Solver& v) { return v.assemble(*assembly, rhs, memory); });
}

int hfps_correct_flux(hfps_solver* s, const double* correction, const double* coefficient_x,
                      const double* coefficient_y, const double* coefficient_z,
                      double correction_scale, double* flux_x, double* flux_y,
                      double* flux_z, int memory) {
  return guarded(s, [&](hfps::Solver& v) {
    return v.correct_flux(correction, coefficient_x, coefficient_y, coefficient_z,
                          correction_scale, flux_x, flux_y, flux_z, memory);
  });
}

int hfps_solve(hfps_solver* s, const double* rhs, double* solution, int memory,
               const hfps_control* control, hfps_result* result,
               double* history, uint32_t history_capacity) {
  hfps_control defaults;
  hfps_default_control(&defaults);
  hfps_result local{};
  hfps_result* out = result != nullptr ? result : &local;
  return guarded(s, [&](hfps::Solver& v) {
    return v.solve(rhs, solution, memory, control != nullptr ? *control : defaults, *out,
                   history, history_capacity);
  });
}

int hfps_apply_operator(hfps_solver* s, const double* x, double* y,
                        int memory) {
  return guarded(s, [&](hfps::Solver& v) { return v.apply_operator(x, y, memory); });
}

int hfps_apply_preconditioner(hfps_solver* s, const double* r, double* z,
                              int memory, int precision) {
  return guarded(s, [&](hfps::Solver& v) {
    return v.apply_preconditioner(r, z, memory, precision);
  });
}

int hfps_adjoint(hfps_solver* s, const double* solution, const double* dl_dp,
                 double* lambda, double* grad_face_x, double* grad_face_y,
                 double* grad_face_z, int memory, const hfps_control* control,
                 hfps_result* result) {
  hfps_control defaults;
  hfps_default_control(&defaults);
  hfps_result local{};
  hfps_result* out = result != nullptr ? result : &local;
  return guarded(s, [&](hfps::Solver& v) {
    return v.adjoint(solution, dl_dp, lambda, grad_face_x, grad_face_y, grad_face_z,
                     memory, control != nullptr ? *control : defaults, *out);
  });
}

int hfps_levels(hfps_solver* s, int* shapes, int capacity) {
  if (s == nullptr || s->impl == nullptr) return -HFPS_INVALID_PLAN;
  const int count = s->impl->level_count();
  for (int l = 0; l < count && l < capacity && shapes != nullptr; ++l)
    s->impl->level_shape(l, shapes + 4 * l);
  return count;
}

int hfps_level_coefficients(hfps_solver* s, int level, double* diagonal,
                            double* face_x, double* face_y, double* face_z,
                            double* volume) {
  return guarded(s, [&](hfps::Solver& v) {
    return v.level_coefficients(level, diagonal, face_x, face_y, face_z, volume);
  });
}

int hfps_profile_kernel(hfps_solver* s, int kernel, int repetitions,
                        double* milliseconds, double* bytes) {
  return guarded(s, [&](hfps::Solver& v) {
    return v.profile_kernel(kernel, repetitions, milliseconds, bytes);
  });
}

const char* hfps_last_error(hfps_solver* s) {
  if (s == nullptr) return create_error.empty() ? "null solver handle" : create_error.c_str();
  return s->error.c_str();
}

int hfps_destroy(hfps_solver* s) {
  if (s == nullptr) return HFPS_OK;
  delete s->impl;
  delete s;
  return HFPS_OK;
}

}  // extern "C"
