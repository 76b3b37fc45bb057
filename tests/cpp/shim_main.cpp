// Drives xfp::VariationalPressureSolver (include/xfp_solver.hpp) the way
// xFluid's FluidSimulator does (FluidSimulator.cpp:216-221 wiring, :505-508
// per step), on a grid type with Array3d's interface.
//
//   shim_main DIR ni nj nk
// reads DIR/{mat.u8,u.f64,v.f64,w.f64}, runs setDt -> solve -> applyPressure
// then the divergence diagnostic of the projected velocities, and writes
// DIR/{p.f64,u_out.f64,v_out.f64,w_out.f64,div.f64}.  Exit status: 0 solved
// and applied, 3 solve() returned false (message on stderr), 2 I/O error.
#include <cstdio>
#include <string>
#include <vector>

#include "xfp_solver.hpp"

enum class Material : char { air = 0, fluid = 1, solid = 2 };

// Minimal grid with the reference Array3d's access pattern (x fastest).
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

template <class T>
static bool read_into(const std::string& path, Grid<T>& g) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) return false;
  const size_t n = std::fread(g.data().data(), sizeof(T), g.data().size(), f);
  std::fclose(f);
  return n == g.data().size();
}
template <class T>
static bool write_from(const std::string& path, Grid<T>& g) {
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) return false;
  const size_t n = std::fwrite(g.data().data(), sizeof(T), g.data().size(), f);
  std::fclose(f);
  return n == g.data().size();
}

int main(int argc, char** argv) {
  if (argc != 5) {
    std::fprintf(stderr, "usage: shim_main DIR ni nj nk\n");
    return 2;
  }
  const std::string dir = argv[1];
  const int ni = std::atoi(argv[2]), nj = std::atoi(argv[3]), nk = std::atoi(argv[4]);
  Grid<Material> mat(ni, nj, nk);
  Grid<double> u(ni + 1, nj, nk), v(ni, nj + 1, nk), w(ni, nj, nk + 1);
  if (!read_into(dir + "/mat.u8", mat) || !read_into(dir + "/u.f64", u) || !read_into(dir + "/v.f64", v) ||
      !read_into(dir + "/w.f64", w)) {
    std::fprintf(stderr, "cannot read inputs from %s\n", dir.c_str());
    return 2;
  }
  xfp::VariationalPressureSolver solver;
  int disfield = 0;
  solver.setDensity(1000.0);
  solver.setDisField(&disfield);
  solver.setDx(1.0 / ni);
  solver.setMaterial(&mat);
  solver.setSize(ni, nj, nk);
  solver.setVelocityField(&u, &v, &w);

  Grid<double> pressure;
  solver.setDt(1.0 / 30.0);
  if (!solver.solve(pressure)) return 3;
  if (!solver.applyPressure(pressure)) return 3;
  std::printf("iterations %d rows %lld\n", solver.stats().iterations, solver.stats().rows);
  // the reference's divergence diagnostic of the projected velocities
  Grid<double> div;
  if (!solver.calculateDivergence(div)) return 3;
  if (!write_from(dir + "/p.f64", pressure) || !write_from(dir + "/u_out.f64", u) ||
      !write_from(dir + "/v_out.f64", v) || !write_from(dir + "/w_out.f64", w) || !write_from(dir + "/div.f64", div))
    return 2;
  return 0;
}
