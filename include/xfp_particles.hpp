// xfp_particles.hpp -- header-only C++ drop-in for the particle steps of
// xFluid's FluidSimulator around the pressure projection
// (xFluid/xFluid/FluidSimulator.cpp, directeddistancefield.cpp):
//
//   advectParticles            FluidSimulator::_advectParticles steps a-b  :652-723
//   updateVelocityByParticles  FluidSimulator::_updateVelocityByParticles  :909-1085
//   updateMaterial             FluidSimulator::_updateMaterial             :402-427
//   updateField                DirectedDistanceField::updateFeild          :122-165
//                              (+ updateSurfaceInfo's material, :167-215)
//
// In FluidSimulator.cpp, with a member `xfp::ParticleSteps _gpuParticles;`:
//
//   _dis_field.updateFeild(); _dis_field.updateSurfaceInfo(_material);   (:274-275)
//     -> _gpuParticles.updateField(_particles, _dis_field._phi, &_material, _dx,
//                                  _subDivisionLevel, _particleRadius * 3.0, _threshold);
//   _updateMaterial();                                                   (:276)
//     -> _gpuParticles.updateMaterial(_particles, _material, _dx);
//   _advectParticles(dt) steps a-b, then _updateVelocityByParticles()    (:328)
//     -> _gpuParticles.advectParticles(_particles, _material, _u, _v, _w,
//                                      _usaved, _vsaved, _wsaved, _dx, dt, _ratioFLIP);
//        _gpuParticles.updateVelocityByParticles(_particles, _u, _v, _w, _dx);
//
// The particle container needs data() and size() over elements laid out as
// struct Particle {Vec3d p; Vec3d v;} (particle.h:5-15): six doubles.  Grids are
// any Array3d-like type with sizei()/sizej()/sizek() and operator()(int flat)
// over contiguous x-fastest storage (array3d.h:89-199); Material is a one-byte
// enum with xFluid's values (material.h:4-8).  The grid sizes come from the
// arrays: material (ni,nj,nk), u (ni+1,nj,nk), v (ni,nj+1,nk), w (ni,nj,nk+1).
//
// Results: advection and the material update are bit-identical to the
// reference; the face transfer and phi sum the same contributions in another
// order (equal to FP64 rounding).  A particle whose collision point lies in a
// cell outside the grid stays in place (the reference reads the material out
// of bounds there).  Errors: false, a message on stderr and last_error().
#pragma once

#include <cstdint>
#include <cstdio>
#include <string>

#include "xfp.h"

namespace xfp {

class ParticleSteps {
 public:
  explicit ParticleSteps(int device = 0) {
    xfp_default_options(&opt_);
    opt_.device = device;
  }
  ~ParticleSteps() {
    if (ctx_) xfp_destroy(ctx_);
  }
  ParticleSteps(const ParticleSteps&) = delete;
  ParticleSteps& operator=(const ParticleSteps&) = delete;

  // _advectParticles steps a-b: FLIP/PIC update from (u,v,w) and the faces
  // saved before the forces, RK4 over dt, solid collisions.
  template <class Particles, class MatGrid, class Grid>
  bool advectParticles(Particles& particles, MatGrid& material, Grid& u, Grid& v, Grid& w, Grid& u_saved,
                       Grid& v_saved, Grid& w_saved, double dx, double dt, double ratioFLIP) {
    if (!ready() || !sizes(material, &u, &v, &w) || !faces_like(u, u_saved) || !faces_like(v, v_saved) ||
        !faces_like(w, w_saved))
      return false;
    return check(xfp_advect_particles_f64(ctx_, ni_, nj_, nk_, dx, mat(material), &u(0), &v(0), &w(0),
                                          &u_saved(0), &v_saved(0), &w_saved(0), ratioFLIP, dt,
                                          count(particles), parts(particles)));
  }

  // _updateVelocityByParticles: every face of u, v, w from the particles.
  template <class Particles, class Grid>
  bool updateVelocityByParticles(const Particles& particles, Grid& u, Grid& v, Grid& w, double dx) {
    if (!ready()) return false;
    ni_ = u.sizei() - 1;
    nj_ = u.sizej();
    nk_ = u.sizek();
    if (!faces_ok(u, v, w)) return false;
    return check(xfp_particles_to_grid_f64(ctx_, ni_, nj_, nk_, dx, count(particles), parts(particles), &u(0),
                                           &v(0), &w(0)));
  }

  // _updateMaterial: non-solid cells become air, cells holding a particle fluid.
  template <class Particles, class MatGrid>
  bool updateMaterial(const Particles& particles, MatGrid& material, double dx) {
    if (!ready()) return false;
    cells(material);
    return check(xfp_update_material(ctx_, ni_, nj_, nk_, dx, count(particles), parts(particles),
                                     reinterpret_cast<uint8_t*>(&material(0))));
  }

  // DirectedDistanceField::updateFeild into phi ((ni*subdiv+1) x (nj*subdiv+1)
  // x (nk*subdiv+1) vertices), then, when material is given, the material part
  // of updateSurfaceInfo.
  template <class Particles, class Field, class MatGrid>
  bool updateField(const Particles& particles, Field& phi, MatGrid* material, double dx, int subdiv, double radius,
                   double threshold) {
    if (!ready()) return false;
    if (subdiv < 1) return fail("subdivision level must be >= 1");
    ni_ = (phi.sizei() - 1) / subdiv;
    nj_ = (phi.sizej() - 1) / subdiv;
    nk_ = (phi.sizek() - 1) / subdiv;
    if (ni_ * subdiv + 1 != phi.sizei() || nj_ * subdiv + 1 != phi.sizej() || nk_ * subdiv + 1 != phi.sizek())
      return fail("phi must have n*subdiv+1 vertices per axis");
    if (material && (material->sizei() != ni_ || material->sizej() != nj_ || material->sizek() != nk_))
      return fail("material does not match phi's grid");
    return check(xfp_distance_field_f64(ctx_, ni_, nj_, nk_, dx, subdiv, radius, threshold, count(particles),
                                        parts(particles), &phi(0),
                                        material ? reinterpret_cast<uint8_t*>(&(*material)(0)) : nullptr));
  }

  const std::string& last_error() const { return err_; }

 private:
  template <class Particles>
  static long long count(const Particles& p) {
    static_assert(sizeof(*p.data()) == sizeof(xfp_particle), "a particle must be six doubles: Vec3d p, v");
    return (long long)p.size();
  }
  template <class Particles>
  static xfp_particle* parts(Particles& p) {
    return reinterpret_cast<xfp_particle*>(p.data());
  }
  template <class Particles>
  static const xfp_particle* parts(const Particles& p) {
    return reinterpret_cast<const xfp_particle*>(p.data());
  }
  template <class MatGrid>
  static const uint8_t* mat(MatGrid& m) {
    static_assert(sizeof(m(0)) == 1, "Material must be a one-byte enum");
    return reinterpret_cast<const uint8_t*>(&m(0));
  }
  template <class MatGrid>
  void cells(MatGrid& m) {
    ni_ = m.sizei();
    nj_ = m.sizej();
    nk_ = m.sizek();
  }
  template <class MatGrid, class Grid>
  bool sizes(MatGrid& m, Grid* u, Grid* v, Grid* w) {
    cells(m);
    return faces_ok(*u, *v, *w);
  }
  template <class Grid>
  bool faces_ok(Grid& u, Grid& v, Grid& w) {
    if (u.sizei() != ni_ + 1 || u.sizej() != nj_ || u.sizek() != nk_ || v.sizei() != ni_ || v.sizej() != nj_ + 1 ||
        v.sizek() != nk_ || w.sizei() != ni_ || w.sizej() != nj_ || w.sizek() != nk_ + 1)
      return fail("face grids must be (ni+1,nj,nk), (ni,nj+1,nk), (ni,nj,nk+1)");
    return true;
  }
  template <class Grid>
  bool faces_like(Grid& a, Grid& b) {
    if (a.sizei() != b.sizei() || a.sizej() != b.sizej() || a.sizek() != b.sizek())
      return fail("saved faces must match the current faces");
    return true;
  }
  bool ready() {
    if (!ctx_ && xfp_create(&ctx_, &opt_) != XFP_OK) {
      ctx_ = nullptr;
      return fail("xfp_create failed (no CUDA device?)");
    }
    return true;
  }
  bool fail(const char* msg) {
    err_ = msg;
    std::fprintf(stderr, "xfp: %s\n", msg);
    return false;
  }
  bool check(int rc) {
    if (rc == XFP_OK) return true;
    err_ = xfp_last_error(ctx_);
    std::fprintf(stderr, "xfp: %s\n", err_.c_str());
    return false;
  }

  xfp_options opt_{};
  xfp_ctx* ctx_ = nullptr;
  std::string err_;
  int ni_ = 0, nj_ = 0, nk_ = 0;
};

}  // namespace xfp
