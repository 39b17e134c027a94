// C++ torch extension of the differentiable pressure solve, used for
// gradient checks: a torch::autograd::Function over the C ABI
// (include/hf_pressure_solver.h), the C++ counterpart of
// hfps/autograd.py's PressureSolveFunction.
//
// forward:  diag = storage + the six face coefficients of each cell
//           (src/solver_pressure.cpp:223-226), hfps_set_coefficients,
//           hfps_solve -> p.
// backward: hfps_adjoint on the same operator (A is symmetric): lambda =
//           dL/drhs and dL/dc_f = -(lambda_i - lambda_j)(p_i - p_j) per face;
//           dL/dstorage = -lambda p on fluid cells.  No residual history is
//           kept between the two solves.
// Tensors are CUDA float64 on the solver's device; the solver handle is
// passed as an integer (hfps.PressureSolver's handle).
#include <torch/extension.h>

#include <stdexcept>
#include <string>

#include "hf_pressure_solver.h"

namespace {

using torch::Tensor;
using torch::autograd::AutogradContext;
using torch::autograd::tensor_list;

hfps_solver* as_solver(int64_t handle) { return reinterpret_cast<hfps_solver*>(handle); }

void check(int status, hfps_solver* s, const char* what) {
  if (status != HFPS_OK) {
    const char* reason = hfps_last_error(s);
    throw std::runtime_error(std::string(what) + " failed (status " + std::to_string(status) +
                             "): " + (reason != nullptr ? reason : ""));
  }
}

hfps_control control_of(double rtol, int64_t maxit, int64_t precision) {
  hfps_control c;
  hfps_default_control(&c);
  c.relative_tolerance = rtol;
  c.maximum_iterations = static_cast<uint32_t>(maxit);
  c.precision = static_cast<int>(precision);
  return c;
}

Tensor diagonal(const Tensor& fx, const Tensor& fy, const Tensor& fz, const Tensor& storage,
                int64_t nx, int64_t ny, int64_t nz) {
  const Tensor x = fx.reshape({nz, ny, nx + 1});
  const Tensor y = fy.reshape({nz, ny + 1, nx});
  const Tensor z = fz.reshape({nz + 1, ny, nx});
  using torch::indexing::Slice;
  Tensor d = x.index({Slice(), Slice(), Slice(0, nx)}) + x.index({Slice(), Slice(), Slice(1, nx + 1)}) +
             y.index({Slice(), Slice(0, ny), Slice()}) + y.index({Slice(), Slice(1, ny + 1), Slice()}) +
             z.index({Slice(0, nz), Slice(), Slice()}) + z.index({Slice(1, nz + 1), Slice(), Slice()});
  if (storage.defined() && storage.numel() > 0) d = storage.reshape({nz, ny, nx}) + d;
  return d.reshape({-1}).contiguous();
}

double* data(const Tensor& t) { return t.data_ptr<double>(); }

class PressureSolve : public torch::autograd::Function<PressureSolve> {
 public:
  static Tensor forward(AutogradContext* ctx, int64_t handle, std::vector<int64_t> shape,
                        double rtol, int64_t maxit, int64_t precision, Tensor rhs, Tensor fx,
                        Tensor fy, Tensor fz, Tensor storage, Tensor active) {
    hfps_solver* s = as_solver(handle);
    const int64_t nx = shape[0], ny = shape[1], nz = shape[2];
    const Tensor d = diagonal(fx, fy, fz, storage, nx, ny, nz);
    const Tensor cx = fx.contiguous(), cy = fy.contiguous(), cz = fz.contiguous();
    check(hfps_set_coefficients(s, data(d), data(cx), data(cy), data(cz), HFPS_DEVICE), s,
          "hfps_set_coefficients");
    const Tensor b = rhs.contiguous();
    Tensor p = torch::zeros_like(b);
    const hfps_control c = control_of(rtol, maxit, precision);
    hfps_result r{};
    check(hfps_solve(s, data(b), data(p), HFPS_DEVICE, &c, &r, nullptr, 0), s, "hfps_solve");
    ctx->saved_data["handle"] = handle;
    ctx->saved_data["rtol"] = rtol;
    ctx->saved_data["maxit"] = maxit;
    ctx->saved_data["precision"] = precision;
    ctx->saved_data["has_storage"] = storage.defined() && storage.numel() > 0;
    ctx->save_for_backward({p, active});
    return p;
  }

  static tensor_list backward(AutogradContext* ctx, tensor_list grads) {
    hfps_solver* s = as_solver(ctx->saved_data["handle"].toInt());
    const auto saved = ctx->get_saved_variables();
    const Tensor& p = saved[0];
    const Tensor& active = saved[1];
    const hfps_control c = control_of(ctx->saved_data["rtol"].toDouble(),
                                      ctx->saved_data["maxit"].toInt(),
                                      ctx->saved_data["precision"].toInt());
    const Tensor g = grads[0].contiguous();
    Tensor lam = torch::empty_like(p);
    const auto counts = [&](int axis) {
      int shape[4 * 32];
      const int levels = hfps_levels(s, shape, 32);
      (void)levels;
      const int64_t nx = shape[0], ny = shape[1], nz = shape[2];
      return axis == 0 ? (nx + 1) * ny * nz : (axis == 1 ? nx * (ny + 1) * nz : nx * ny * (nz + 1));
    };
    Tensor gx = torch::empty({counts(0)}, p.options());
    Tensor gy = torch::empty({counts(1)}, p.options());
    Tensor gz = torch::empty({counts(2)}, p.options());
    hfps_result r{};
    check(hfps_adjoint(s, data(p), data(g), data(lam), data(gx), data(gy), data(gz), HFPS_DEVICE,
                       &c, &r),
          s, "hfps_adjoint");
    Tensor g_storage;
    if (ctx->saved_data["has_storage"].toBool()) {
      g_storage = -lam * p;
      if (active.defined() && active.numel() > 0) g_storage = g_storage * active;
    }
    // Gradients for (handle, shape, rtol, maxit, precision, rhs, fx, fy, fz,
    // storage, active).
    return {Tensor(), Tensor(), Tensor(), Tensor(), Tensor(), lam, gx, gy, gz, g_storage, Tensor()};
  }
};

Tensor pressure_solve(int64_t handle, std::vector<int64_t> shape, double rtol, int64_t maxit,
                      int64_t precision, Tensor rhs, Tensor fx, Tensor fy, Tensor fz,
                      Tensor storage, Tensor active) {
  return PressureSolve::apply(handle, shape, rtol, maxit, precision, rhs, fx, fy, fz, storage,
                              active);
}

}  // namespace

PYBIND11_MODULE(TORCH_EXTENSION_NAME, m) {
  m.def("pressure_solve", &pressure_solve,
        "Differentiable pressure solve (forward hfps_solve, backward hfps_adjoint)");
}
