// xfp_solver.hpp -- header-only C++ drop-in for xFluid's VariationalPressureSolver.
//
// Same nine public methods with the same meaning as the reference class
// (xFluid/xFluid/variationalpressure/variational_pressuresolver.h:30-44), so the
// member at xFluid/xFluid/FluidSimulator.h:215
//
//     VariationalPressureSolver _pressureSolver;
//
// becomes
//
//     xfp::VariationalPressureSolver _pressureSolver;
//
// with no other change to FluidSimulator.cpp (the wiring at :216-221 and the
// per-step calls at :505-508 compile as they are).  The grid and field types
// are template parameters of the setters, so this header needs none of the
// reference's headers: any Array3d-like type with sizei()/sizej()/sizek(),
// resize(i,j,k) and element access operator()(int flat) over contiguous
// x-fastest storage works (xFluid/xFluid/array3d.h:89-199).  Material must be
// a one-byte enum with xFluid's values 0 air, 1 fluid, 2 solid
// (xFluid/xFluid/material.h:4-8).
//
// Behaviour that differs from the reference, by design:
//  * solve() always sizes and fills the pressure grid, also when PCG did not
//    converge (it then returns false); the reference leaves the grid unsized
//    (variational_pressuresolver.cpp:80-86) and FluidSimulator applies it anyway.
//  * errors are reported as false plus a message on stderr and last_error(),
//    where the reference prints to cout.
//  * setDensity/setDt/setDx/setDisField are stored but, as in the reference
//    (variational_pressuresolver.cpp:122, scale factor fixed at 1.0), do not
//    change the result.
#pragma once

#include <cstdint>
#include <cstdio>
#include <functional>
#include <string>

#include "xfp.h"

namespace xfp {

class VariationalPressureSolver {
 public:
  // Precision XFP_PREC_F64 reproduces the reference's FP64 operation order.
  explicit VariationalPressureSolver(int precision = XFP_PREC_F64, int device = 0)
      : VariationalPressureSolver(precision, device, XFP_MATRIX_VARIATIONAL) {}
  ~VariationalPressureSolver() {
    if (ctx_) xfp_destroy(ctx_);
  }
  VariationalPressureSolver(const VariationalPressureSolver&) = delete;
  VariationalPressureSolver& operator=(const VariationalPressureSolver&) = delete;

  // ---- the reference's setters (variational_pressuresolver.cpp:11-48) ----
  void setSize(int sizei, int sizej, int sizek) {
    ni_ = sizei;
    nj_ = sizej;
    nk_ = sizek;
  }
  template <class Grid>
  void setVelocityField(Grid* u, Grid* v, Grid* w) {
    u_ = [u] { return static_cast<double*>(&(*u)(0)); };
    v_ = [v] { return static_cast<double*>(&(*v)(0)); };
    w_ = [w] { return static_cast<double*>(&(*w)(0)); };
  }
  template <class MaterialGrid>
  void setMaterial(MaterialGrid* material) {
    static_assert(sizeof((*material)(0)) == 1, "Material must be a one-byte enum");
    mat_ = [material] { return reinterpret_cast<const uint8_t*>(&(*material)(0)); };
  }
  template <class DisField>
  void setDisField(DisField* disfield) { disfield_ = disfield; }
  void setDensity(double density) { density_ = density; }
  void setDt(double dt) { dt_ = dt; }
  void setDx(double dx) { dx_ = dx; }

  // ---- solve / apply (variational_pressuresolver.cpp:50-220) ----
  // stats() and last_error() describe the most recent solve; a solve that
  // cannot start (arguments missing, no CUDA device) leaves stats().status at
  // XFP_ERR_ARGS or XFP_ERR_CUDA.
  template <class Grid>
  bool solve(Grid& pressureGrid) {
    stats_ = xfp_stats{};
    err_.clear();
    if (!ready()) return false;
    pressureGrid.resize(ni_, nj_, nk_);
    const int rc = xfp_solve_f64(ctx_, ni_, nj_, nk_, mat_(), u_(), v_(), w_(), nullptr, nullptr, nullptr,
                                 &pressureGrid(0), &stats_);
    return check(rc);
  }
  template <class Grid>
  bool applyPressure(Grid& pressureGrid) {
    if (!ready()) return false;
    const int rc = xfp_apply_pressure_f64(ctx_, ni_, nj_, nk_, mat_(), nullptr, nullptr, nullptr,
                                          &pressureGrid(0), u_(), v_(), w_());
    return check(rc);
  }

  // ---- the reference's divergence diagnostic (variational_pressuresolver.cpp:526-597) ----
  // _calculate_divergience into div (resized to ni x nj x nk).
  template <class Grid>
  bool calculateDivergence(Grid& div) {
    if (!ready()) return false;
    div.resize(ni_, nj_, nk_);
    return check(xfp_divergence_f64(ctx_, ni_, nj_, nk_, mat_(), u_(), v_(), w_(), &div(0)));
  }

  // ---- the simulator steps either side of the projection ----
  // FluidSimulator::_applyForces (FluidSimulator.cpp:429-499): force*dt on every
  // face next to fluid (an axis with |force*dt| <= 1e-10 is left alone), on the
  // borrowed velocities.
  bool applyForces(const double force[3], double dt) {
    if (!ready()) return false;
    return check(xfp_apply_forces_f64(ctx_, ni_, nj_, nk_, mat_(), u_(), v_(), w_(), force, dt));
  }
  // FluidSimulator::_expolateVelocity (:511-650); the reference passes
  // layers = int(CFL number + 5).
  bool extrapolateVelocity(int layers) {
    if (!ready()) return false;
    return check(xfp_extrapolate_f64(ctx_, ni_, nj_, nk_, mat_(), u_(), v_(), w_(), layers));
  }
  // applyForces, solve, applyPressure and extrapolateVelocity in one call, the
  // force fused into the assembly and apply kernels (timeStep :310-322).
  template <class Grid>
  bool projectStep(Grid& pressureGrid, const double force[3], double dt, int layers) {
    stats_ = xfp_stats{};
    err_.clear();
    if (!ready()) return false;
    pressureGrid.resize(ni_, nj_, nk_);
    return check(xfp_project_step_f64(ctx_, ni_, nj_, nk_, mat_(), u_(), v_(), w_(), nullptr, nullptr, nullptr,
                                      &pressureGrid(0), force, dt, layers, &stats_));
  }

  // ---- extensions ----
  // PCGSolver::set_solver_parameters (pcg_solver.h:234-241).
  void set_solver_parameters(double tol, int max_iter, double omega = 0.97, double min_diag_ratio = 0.25) {
    opt_.tol = tol;
    opt_.max_iter = max_iter;
    opt_.omega = omega;
    opt_.min_diag_ratio = min_diag_ratio;
    if (ctx_) xfp_set_options(ctx_, &opt_);
  }
  const xfp_stats& stats() const { return stats_; }
  const std::string& last_error() const { return err_; }

 protected:
  VariationalPressureSolver(int precision, int device, int matrix) {
    xfp_default_options(&opt_);
    opt_.precision = precision;
    opt_.device = device;
    opt_.matrix = matrix;
  }

 private:
  bool ready() {
    if (!mat_ || !u_ || !v_ || !w_ || ni_ < 1 || nj_ < 1 || nk_ < 1) {
      err_ = "setSize, setMaterial and setVelocityField must be called first";
      stats_.status = XFP_ERR_ARGS;
      std::fprintf(stderr, "xfp: %s\n", err_.c_str());
      return false;
    }
    if (!ctx_ && xfp_create(&ctx_, &opt_) != XFP_OK) {
      ctx_ = nullptr;
      err_ = "xfp_create failed (no CUDA device?)";
      stats_.status = XFP_ERR_CUDA;
      std::fprintf(stderr, "xfp: %s\n", err_.c_str());
      return false;
    }
    return true;
  }
  bool check(int rc) {
    if (rc == XFP_OK) return true;
    err_ = rc == XFP_NOT_CONVERGED ? "PCG did not converge" : xfp_last_error(ctx_);
    std::fprintf(stderr, "xfp: %s\n", err_.c_str());
    return false;
  }

  xfp_options opt_{};
  xfp_ctx* ctx_ = nullptr;
  xfp_stats stats_{};
  std::string err_;
  int ni_ = 0, nj_ = 0, nk_ = 0;
  std::function<double*()> u_, v_, w_;
  std::function<const uint8_t*()> mat_;
  void* disfield_ = nullptr;
  double density_ = 0.0, dt_ = 0.0, dx_ = 0.0;
};

// xFluid's NormalPressureSolver (xFluid/xFluid/pressuresolver.h:9-25): the same
// nine methods over the classic Poisson matrix (pressuresolver.cpp:220-347) and
// its applyPressure (:109-212), for a simulator built with the member at
// FluidSimulator.h:216 (NormalPressureSolver _pressureSolver;).
class NormalPressureSolver : public VariationalPressureSolver {
 public:
  explicit NormalPressureSolver(int precision = XFP_PREC_F64, int device = 0)
      : VariationalPressureSolver(precision, device, XFP_MATRIX_NORMAL) {}
};

}  // namespace xfp
