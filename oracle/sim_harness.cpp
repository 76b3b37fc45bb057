// sim_harness.cpp -- TEST INFRASTRUCTURE ONLY (part of the oracle).
//
// Drives xFluid's own FluidSimulator (compiled from the reference sources by
// oracle/build_sim.sh) one time step at a time, stopping just before the
// pressure projection so a test can hand the very same (material, u, v, w)
// snapshot to the CUDA path and compare.  The simulator then continues with
// its own projection, so every step's snapshot is the reference's.
//
// A step follows FluidSimulator::timeStep (xFluid/xFluid/FluidSimulator.cpp:
// 265-335) with the mesh output left out:
//   xfsim_begin_step  dt as frameStep picks it (:228-253, capped at max_dt),
//                     distance field + surface + material update (:274-277),
//                     _saveVelocity (:286), _applyForces (:310)
//   xfsim_project     _solvePressure (:501-509): setDt, solve, applyPressure
//   xfsim_end_step    _expolateVelocity (:322), _advectParticles (:328)
// Scenes: FluidSimulator(n,n,n), setCellWidth(1/n), gravity (0,g,0)
// (:142-150), fluid from addCubicFluid (:123-140) and addSpereFluid (:98-121),
// then init (:186-222: solid border, 8 jittered particles per fluid cell,
// :168-184 and :347-370).  xfsim_create_dam builds the dam break of the plain
// CPU-runnable configuration: fluid box (0,0,0)-(0.4,0.5,1).
//
// Private members (CFL number, pressure solver, grids) are reached by mapping
// private/protected to public around the reference header.  std::cout is muted
// around every call (the reference prints timings each step).

#include <climits>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

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
  int iters = 0;
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

// An n^3 simulator with cell width 1/n (unit cube); add fluid, then init.
void* xfsim_create(int n, double cfl, double gravity, double tol, int maxit) {
  MuteCout mute;
  Sim* s = new Sim(n);
  s->fs.setCellWidth(1.0 / n);
  s->fs.addConstantForce(0.0, gravity, 0.0);
  s->fs._CFLnumber = cfl;
  s->fs._pressureSolver.solver.set_solver_parameters(tol, maxit);
  return s;
}
// addCubicFluid (FluidSimulator.cpp:123-140): cells whose centre lies in the box
void xfsim_add_box(void* h, double x0, double y0, double z0, double x1, double y1, double z1) {
  static_cast<Sim*>(h)->fs.addCubicFluid(Vec3d(x0, y0, z0), Vec3d(x1, y1, z1));
}
// addSpereFluid (FluidSimulator.cpp:98-121)
void xfsim_add_sphere(void* h, double cx, double cy, double cz, double r) {
  static_cast<Sim*>(h)->fs.addSpereFluid(cx, cy, cz, r);
}
// init (FluidSimulator.cpp:186-222): solid border, particles, distance field, solver wiring
void xfsim_init(void* h) {
  MuteCout mute;
  Sim* s = static_cast<Sim*>(h);
  s->fs.init();
  // init() does not touch the PCG parameters set at creation
}
// The dam break: fluid box (0,0,0)-(0.4,0.5,1).
void* xfsim_create_dam(int n, double cfl, double gravity, double tol, int maxit) {
  void* h = xfsim_create(n, cfl, gravity, tol, maxit);
  xfsim_add_box(h, 0.0, 0.0, 0.0, 0.4, 0.5, 1.0);
  xfsim_init(h);
  return h;
}

void xfsim_destroy(void* h) { delete static_cast<Sim*>(h); }

// Everything before the projection; writes the snapshot the projection sees.
double xfsim_begin_step(void* h, double max_dt, uint8_t* mat, double* u, double* v, double* w) {
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

// The reference's own projection of the snapshot; writes its pressure (when
// the solve succeeded) and the projected velocities.  Returns 1 on success.
int xfsim_project(void* h, double* p, double* u, double* v, double* w, int* iters) {
  MuteCout mute;
  Sim* s = static_cast<Sim*>(h);
  FluidSimulator& f = s->fs;
  // iterations: the same PCG rerun on the same system (solve() does not report them)
  if (iters) {
    SparseMatrix<double> A;
    std::vector<double> b;
    f._pressureSolver._calculate_coefficient(A, b);
    std::vector<double> x(b.size(), 0.0);
    double res = 0.0;
    int it = 0;
    PCGSolver<double> pcg;
    pcg.set_solver_parameters(f._pressureSolver.solver.tolerance_factor, f._pressureSolver.solver.max_iterations);
    pcg.solve(A, b, x, res, it);
    *iters = it;
  }
  Array3d<double> pressure;
  f._pressureSolver.setDt(s->dt);
  const bool ok = f._pressureSolver.solve(pressure);
  f._pressureSolver.applyPressure(pressure);
  if (ok && p) dump(pressure, p);
  dump(f._u, u);
  dump(f._v, v);
  dump(f._w, w);
  return ok ? 1 : 0;
}

void xfsim_end_step(void* h) {
  MuteCout mute;
  Sim* s = static_cast<Sim*>(h);
  s->fs._expolateVelocity();
  s->fs._advectParticles(s->dt);
}

int xfsim_fluid_cells(void* h) { return static_cast<Sim*>(h)->fs._countFluidCell(); }

// The simulator's current material and face velocities (no stepping).
void xfsim_fields(void* h, uint8_t* mat, double* u, double* v, double* w) {
  FluidSimulator& f = static_cast<Sim*>(h)->fs;
  for (int k = 0; k < f._material.sizek(); ++k)
    for (int j = 0; j < f._material.sizej(); ++j)
      for (int i = 0; i < f._material.sizei(); ++i)
        mat[(size_t)k * f._ni * f._nj + (size_t)j * f._ni + i] = static_cast<uint8_t>(f._material(i, j, k));
  dump(f._u, u);
  dump(f._v, v);
  dump(f._w, w);
}

long long xfsim_particle_count(void* h) { return (long long)static_cast<Sim*>(h)->fs._particles.size(); }

// The simulator's particles as (p, v) rows of 6 doubles.
void xfsim_particles(void* h, double* P) {
  const FluidSimulator& f = static_cast<Sim*>(h)->fs;
  for (size_t q = 0; q < f._particles.size(); ++q) {
    const Particle& a = f._particles[q];
    const double x[6] = {a.p.x, a.p.y, a.p.z, a.v.x, a.v.y, a.v.z};
    for (int e = 0; e < 6; ++e) P[6 * q + e] = x[e];
  }
}

// The two steps either side of the projection on given arrays, through a
// simulator of the grid's size (FluidSimulator(ni,nj,nk) only sizes its grids,
// FluidSimulator.cpp:26-31): material and faces are filled in, the step runs,
// the faces are read back.
namespace {
struct Fields {
  FluidSimulator fs;
  Fields(int ni, int nj, int nk, const uint8_t* mat, const double* u, const double* v, const double* w)
      : fs(ni, nj, nk) {
    for (int k = 0; k < nk; ++k)
      for (int j = 0; j < nj; ++j)
        for (int i = 0; i < ni; ++i)
          fs._material(i, j, k) = static_cast<Material>(mat[(size_t)k * ni * nj + (size_t)j * ni + i]);
    fill(fs._u, u);
    fill(fs._v, v);
    fill(fs._w, w);
  }
  static void fill(Array3d<double>& a, const double* src) {
    for (int k = 0; k < a.sizek(); ++k)
      for (int j = 0; j < a.sizej(); ++j)
        for (int i = 0; i < a.sizei(); ++i)
          a(i, j, k) = src[(size_t)k * a.sizei() * a.sizej() + (size_t)j * a.sizei() + i];
  }
  void out(double* u, double* v, double* w) {
    dump(fs._u, u);
    dump(fs._v, v);
    dump(fs._w, w);
  }
};
}  // namespace

// _applyForces (FluidSimulator.cpp:429-499) with one constant force (fx,fy,fz).
void xfsim_apply_forces(int ni, int nj, int nk, const uint8_t* mat, double* u, double* v, double* w,
                        double fx, double fy, double fz, double dt) {
  MuteCout mute;
  Fields f(ni, nj, nk, mat, u, v, w);
  f.fs._forces.clear();
  f.fs.addConstantForce(Vec3d(fx, fy, fz));
  f.fs._applyForces(dt);
  f.out(u, v, w);
}

// _expolateVelocity(layers, axis) for axes 0, 1, 2 (FluidSimulator.cpp:516-518, 521-650).
void xfsim_extrapolate(int ni, int nj, int nk, const uint8_t* mat, double* u, double* v, double* w, int layers) {
  MuteCout mute;
  Fields f(ni, nj, nk, mat, u, v, w);
  for (int axis = 0; axis < 3; ++axis) f.fs._expolateVelocity(layers, axis);
  f.out(u, v, w);
}

namespace {
void set_particles(FluidSimulator& fs, long long n, const double* P) {
  fs._particles.clear();
  for (long long q = 0; q < n; ++q)
    fs._particles.push_back(Particle(Vec3d(P[6 * q], P[6 * q + 1], P[6 * q + 2]),
                                     Vec3d(P[6 * q + 3], P[6 * q + 4], P[6 * q + 5])));
}
void get_particles(const FluidSimulator& fs, double* P) {
  for (size_t q = 0; q < fs._particles.size(); ++q) {
    const Particle& a = fs._particles[q];
    const double x[6] = {a.p.x, a.p.y, a.p.z, a.v.x, a.v.y, a.v.z};
    for (int e = 0; e < 6; ++e) P[6 * q + e] = x[e];
  }
}
}  // namespace

// _advectParticles(dt) (FluidSimulator.cpp:652-728): FLIP/PIC update from
// (u,v,w) and the saved (us,vs,ws), RK4 advection with solid collisions, then
// the reference's own particle-to-grid transfer into (uo,vo,wo).  No fluid
// sources (_applyFluidSource is then a no-op).
void xfsim_advect_particles(int ni, int nj, int nk, double dx, const uint8_t* mat, const double* u, const double* v,
                            const double* w, const double* us, const double* vs, const double* ws, double ratio,
                            double dt, long long n, double* parts, double* uo, double* vo, double* wo) {
  MuteCout mute;
  Fields f(ni, nj, nk, mat, us, vs, ws);
  f.fs._dx = dx;
  f.fs._usaved = f.fs._u;
  f.fs._vsaved = f.fs._v;
  f.fs._wsaved = f.fs._w;
  Fields::fill(f.fs._u, u);
  Fields::fill(f.fs._v, v);
  Fields::fill(f.fs._w, w);
  f.fs._ratioFLIP = ratio;
  f.fs._fluidSources.clear();
  set_particles(f.fs, n, parts);
  f.fs._advectParticles(dt);
  get_particles(f.fs, parts);
  f.out(uo, vo, wo);
}

// _updateVelocityByParticles (FluidSimulator.cpp:909-1085) on given particles.
void xfsim_p2g(int ni, int nj, int nk, double dx, long long n, const double* parts, double* u, double* v, double* w) {
  MuteCout mute;
  std::vector<uint8_t> mat((size_t)ni * nj * nk, 0);
  Fields f(ni, nj, nk, mat.data(), u, v, w);
  f.fs._dx = dx;
  set_particles(f.fs, n, parts);
  f.fs._updateVelocityByParticles();
  f.out(u, v, w);
}

// The material update of timeStep (FluidSimulator.cpp:274-276):
// DirectedDistanceField::updateFeild and updateSurfaceInfo(material) with the
// field set up as init does (:207-213, with the given subdivision, radius and
// threshold), then _updateMaterial.  Writes phi, the material after
// updateSurfaceInfo (ms) and after _updateMaterial (mf).
void xfsim_material(int ni, int nj, int nk, double dx, int subdiv, double radius, double threshold, long long n,
                    const double* parts, const uint8_t* mat, double* phi, uint8_t* ms, uint8_t* mf) {
  MuteCout mute;
  std::vector<double> zu((size_t)(ni + 1) * nj * nk), zv((size_t)ni * (nj + 1) * nk), zw((size_t)ni * nj * (nk + 1));
  Fields f(ni, nj, nk, mat, zu.data(), zv.data(), zw.data());
  f.fs._dx = dx;
  set_particles(f.fs, n, parts);
  DirectedDistanceField& d = f.fs._dis_field;
  d.setSize(ni, nj, nk);
  d.setParticleVector(&f.fs._particles);
  d.setSubDivisionLevel(subdiv);
  d.setParticleRadius(radius);
  d.setDx(dx);
  d.setThreshold(threshold);
  d.initField();
  d.updateFeild();
  d.updateSurfaceInfo(f.fs._material);
  dump(d._phi, phi);
  auto dump_mat = [&](uint8_t* dst) {
    for (int k = 0; k < nk; ++k)
      for (int j = 0; j < nj; ++j)
        for (int i = 0; i < ni; ++i)
          dst[(size_t)k * ni * nj + (size_t)j * ni + i] = static_cast<uint8_t>(f.fs._material(i, j, k));
  };
  dump_mat(ms);
  f.fs._updateMaterial();
  dump_mat(mf);
}

}  // extern "C"
