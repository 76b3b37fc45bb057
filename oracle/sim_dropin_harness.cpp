// sim_dropin_harness.cpp -- TEST INFRASTRUCTURE ONLY (part of the oracle).
//
// Steps xFluid's own FluidSimulator, compiled from the reference sources by
// oracle/build_sim.sh with ONE declaration changed in a temporary copy of
// FluidSimulator.h: the pressure-solver member at FluidSimulator.h:215,
//
//     VariationalPressureSolver _pressureSolver;
// becomes
//     xfp::VariationalPressureSolver _pressureSolver;
//
// (include/xfp_solver.hpp, backed by libxfp.so on the GPU).  FluidSimulator.cpp
// compiles as it is (beyond the :179 g++ fix every build of it needs), so its
// own wiring at :216-221 and its own _solvePressure at :501-509 drive the
// library.  A step follows FluidSimulator::timeStep (:265-335) without the mesh
// output, as oracle/sim_harness.cpp does for the stock build, so a test can
// run both builds side by side from the same seed and compare them step by
// step.
//
// Private members are reached by mapping private/protected to public around
// the header; std::cout is muted around every call.

#include <climits>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <iostream>
#include <sstream>
#include <string>

#define private public
#define protected public
#include "FluidSimulator.h"
#undef private
#undef protected

namespace {

struct MuteCout {
  std::streambuf* saved;
  std::ostringstream sink;
  MuteCout() : saved(std::cout.rdbuf(sink.rdbuf())) {}
  ~MuteCout() { std::cout.rdbuf(saved); }
};

struct Sim {
  FluidSimulator fs;
  double dt = 0.0;
  explicit Sim(int n) : fs(n, n, n) {}
};

template <typename T>
void dump(Array3d<T>& a, T* dst) {
  for (int k = 0; k < a.sizek(); ++k)
    for (int j = 0; j < a.sizej(); ++j)
      for (int i = 0; i < a.sizei(); ++i)
        dst[(size_t)k * a.sizei() * a.sizej() + (size_t)j * a.sizei() + i] = a(i, j, k);
}

}  // namespace

extern "C" {

// The member's type as compiled into this build (a check that the swap took).
const char* xfsd_solver_type() { return "xfp::VariationalPressureSolver"; }

// An n^3 dam break with cell width 1/n: fluid box (0,0,0)-(0.4,0.5,1),
// gravity (0,g,0), CFL number cfl; the library solver at tol/maxit (its
// set_solver_parameters, the counterpart of pcg_solver.h:234-241).  The
// caller seeds rand() before this call: init's particle jitter draws from it.
void* xfsd_create_dam(int n, double cfl, double gravity, double tol, int maxit) {
  MuteCout mute;
  Sim* s = new Sim(n);
  s->fs.setCellWidth(1.0 / n);
  s->fs.addConstantForce(0.0, gravity, 0.0);
  s->fs._CFLnumber = cfl;
  s->fs._pressureSolver.set_solver_parameters(tol, maxit);
  s->fs.addCubicFluid(Vec3d(0.0, 0.0, 0.0), Vec3d(0.4, 0.5, 1.0));
  s->fs.init();
  return s;
}

void xfsd_destroy(void* h) { delete static_cast<Sim*>(h); }

// Everything before the projection (timeStep :274-310); returns dt and writes
// the snapshot the projection will see.
double xfsd_begin_step(void* h, double max_dt, uint8_t* mat, double* u, double* v, double* w) {
  MuteCout mute;
  Sim* s = static_cast<Sim*>(h);
  FluidSimulator& f = s->fs;
  const double maxv = f._maxVelocity();
  double dt = maxv == 0.0 ? f._maxStepTime : f._CFLnumber * f._dx / maxv;
  dt = dt < f._maxStepTime ? dt : f._maxStepTime;
  dt = dt < max_dt ? dt : max_dt;
  s->dt = dt;
  f._dis_field.updateFeild();
  f._dis_field.updateSurfaceInfo(f._material);
  f._updateMaterial();
  f._saveVelocity();
  f._applyForces(dt);
  for (int k = 0; k < f._material.sizek(); ++k)
    for (int j = 0; j < f._material.sizej(); ++j)
      for (int i = 0; i < f._material.sizei(); ++i)
        mat[(size_t)k * f._ni * f._nj + (size_t)j * f._ni + i] = static_cast<uint8_t>(f._material(i, j, k));
  dump(f._u, u);
  dump(f._v, v);
  dump(f._w, w);
  return dt;
}

// The simulator's own _solvePressure (FluidSimulator.cpp:501-509), which now
// calls the library class.  Writes the projected velocities; returns the
// solve's status as the library reported it (0 OK, 1 not converged, < 0
// error) and its iteration count.
int xfsd_project(void* h, double* u, double* v, double* w, int* iters) {
  MuteCout mute;
  Sim* s = static_cast<Sim*>(h);
  FluidSimulator& f = s->fs;
  f._solvePressure(s->dt);
  const xfp_stats& st = f._pressureSolver.stats();
  if (iters) *iters = st.iterations;
  dump(f._u, u);
  dump(f._v, v);
  dump(f._w, w);
  return st.status;
}

void xfsd_end_step(void* h) {
  MuteCout mute;
  Sim* s = static_cast<Sim*>(h);
  s->fs._expolateVelocity();
  s->fs._advectParticles(s->dt);
}

long long xfsd_particle_count(void* h) { return (long long)static_cast<Sim*>(h)->fs._particles.size(); }

void xfsd_particles(void* h, double* P) {
  const FluidSimulator& f = static_cast<Sim*>(h)->fs;
  for (size_t q = 0; q < f._particles.size(); ++q) {
    const Particle& a = f._particles[q];
    const double x[6] = {a.p.x, a.p.y, a.p.z, a.v.x, a.v.y, a.v.z};
    for (int e = 0; e < 6; ++e) P[6 * q + e] = x[e];
  }
}

}  // extern "C"
