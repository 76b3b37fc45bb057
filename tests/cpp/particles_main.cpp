// Drives xfp::ParticleSteps (include/xfp_particles.hpp) with xFluid's own
// types: a std::vector of struct Particle {Vec3d p; Vec3d v;} and grids with
// Array3d's access pattern, in the order FluidSimulator::timeStep calls the
// steps (FluidSimulator.cpp:274-276, :328).
//
//   particles_main DIR ni nj nk n dx dt ratio subdiv radius threshold
// reads DIR/{mat.u8, u.f64, v.f64, w.f64, us.f64, vs.f64, ws.f64, parts.f64}
// and writes DIR/{phi.f64, mat_surface.u8, mat_final.u8, parts_out.f64,
// u_out.f64, v_out.f64, w_out.f64}.  Exit status: 0 done, 3 a step returned
// false (message on stderr), 2 usage or I/O error.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "xfp_particles.hpp"

enum class Material : char { air = 0, fluid = 1, solid = 2 };

struct Vec3d {
  double x, y, z;
};
struct Particle {
  Vec3d p;
  Vec3d v;
};

template <class T>
class Grid {
 public:
  Grid(int i = 0, int j = 0, int k = 0) { resize(i, j, k); }
  void resize(int i, int j, int k) {
    ni_ = i; nj_ = j; nk_ = k;
    v_.resize((size_t)i * j * k);
  }
  T& operator()(int flat) { return v_[flat]; }
  int sizei() const { return ni_; }
  int sizej() const { return nj_; }
  int sizek() const { return nk_; }
  std::vector<T>& data() { return v_; }

 private:
  int ni_ = 0, nj_ = 0, nk_ = 0;
  std::vector<T> v_;
};

template <class V>
static bool io(const std::string& path, V& v, bool write) {
  FILE* f = std::fopen(path.c_str(), write ? "wb" : "rb");
  if (!f) return false;
  const size_t bytes = v.size() * sizeof(v[0]);
  const size_t n = write ? std::fwrite(v.data(), 1, bytes, f) : std::fread(v.data(), 1, bytes, f);
  std::fclose(f);
  return n == bytes;
}

int main(int argc, char** argv) {
  if (argc != 12) {
    std::fprintf(stderr, "usage: particles_main DIR ni nj nk n dx dt ratio subdiv radius threshold\n");
    return 2;
  }
  const std::string d = std::string(argv[1]) + "/";
  const int ni = std::atoi(argv[2]), nj = std::atoi(argv[3]), nk = std::atoi(argv[4]);
  const long long n = std::atoll(argv[5]);
  const double dx = std::atof(argv[6]), dt = std::atof(argv[7]), ratio = std::atof(argv[8]);
  const int subdiv = std::atoi(argv[9]);
  const double radius = std::atof(argv[10]), threshold = std::atof(argv[11]);

  Grid<Material> material(ni, nj, nk);
  Grid<double> u(ni + 1, nj, nk), v(ni, nj + 1, nk), w(ni, nj, nk + 1);
  Grid<double> us(ni + 1, nj, nk), vs(ni, nj + 1, nk), ws(ni, nj, nk + 1);
  Grid<double> phi(ni * subdiv + 1, nj * subdiv + 1, nk * subdiv + 1);
  std::vector<Particle> particles((size_t)n);
  if (!io(d + "mat.u8", material.data(), false) || !io(d + "u.f64", u.data(), false) ||
      !io(d + "v.f64", v.data(), false) || !io(d + "w.f64", w.data(), false) || !io(d + "us.f64", us.data(), false) ||
      !io(d + "vs.f64", vs.data(), false) || !io(d + "ws.f64", ws.data(), false) ||
      !io(d + "parts.f64", particles, false))
    return 2;

  xfp::ParticleSteps steps;
  // timeStep :274-276
  if (!steps.updateField(particles, phi, &material, dx, subdiv, radius, threshold)) return 3;
  std::vector<Material> surface = material.data();
  if (!steps.updateMaterial(particles, material, dx)) return 3;
  // :328
  if (!steps.advectParticles(particles, material, u, v, w, us, vs, ws, dx, dt, ratio)) return 3;
  if (!steps.updateVelocityByParticles(particles, u, v, w, dx)) return 3;

  if (!io(d + "phi.f64", phi.data(), true) || !io(d + "mat_surface.u8", surface, true) ||
      !io(d + "mat_final.u8", material.data(), true) || !io(d + "parts_out.f64", particles, true) ||
      !io(d + "u_out.f64", u.data(), true) || !io(d + "v_out.f64", v.data(), true) ||
      !io(d + "w_out.f64", w.data(), true))
    return 2;
  return 0;
}
