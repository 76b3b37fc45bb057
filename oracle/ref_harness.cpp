// ref_harness.cpp -- TEST INFRASTRUCTURE ONLY (part of the oracle).
//
// Binds xFluid's own variational pressure solver, compiled unmodified from the
// reference sources by oracle/build_ref.sh, behind a small C ABI so the tests
// can run the reference on the same seeded inputs as the CUDA path.  Nothing in
// the product links or loads this file.
//
// What each entry point drives (reference paths, relative to the xFluid source
// directory xFluid/xFluid/):
//   xfref_solve      VariationalPressureSolver::solve        variationalpressure/variational_pressuresolver.cpp:50-118
//   xfref_apply      VariationalPressureSolver::applyPressure variationalpressure/variational_pressuresolver.cpp:120-220
//   xfref_assemble   VariationalPressureSolver::_calculate_coefficient  :231-327
//   xfref_factor     factor_modified_incomplete_cholesky0    variationalpressure/pcg_solver.h:85-186
//   xfref_precond    solve_lower + solve_lower_transpose_in_place  pcg_solver.h:192-220
//   xfref_divergence VariationalPressureSolver::_calculate_divergience :526-597
//   xfref_normal_*   NormalPressureSolver (pressuresolver.cpp): solve :50-106,
//                    applyPressure :109-212, _calculate_coefficient :220-347
//
// The solver's members are private; standard headers are included first and the
// reference header is then included with private/protected mapped to public so
// the harness can set the PCG tolerance (pcg_solver.h:234) and call the
// assembly routine directly.  The reference prints to std::cout on every solve
// (variational_pressuresolver.cpp:74-75,113); the harness mutes std::cout
// around each call.

#include <chrono>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <iostream>
#include <map>
#include <sstream>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#define private public
#define protected public
#include "variationalpressure/variational_pressuresolver.h"
#include "pressuresolver.h"
#undef private
#undef protected

namespace {

struct MuteCout {
  std::streambuf* saved;
  std::ostringstream sink;
  MuteCout() : saved(std::cout.rdbuf(sink.rdbuf())) {}
  ~MuteCout() { std::cout.rdbuf(saved); }
};

struct Scene {
  int ni, nj, nk;
  Array3d<Material> mat;
  Array3d<double> u, v, w;
  Scene(int ni_, int nj_, int nk_, const uint8_t* m, const double* uu,
        const double* vv, const double* ww)
      : ni(ni_), nj(nj_), nk(nk_), mat(ni_, nj_, nk_), u(ni_ + 1, nj_, nk_),
        v(ni_, nj_ + 1, nk_), w(ni_, nj_, nk_ + 1) {
    for (int k = 0; k < nk; ++k)
      for (int j = 0; j < nj; ++j)
        for (int i = 0; i < ni; ++i)
          mat(i, j, k) = static_cast<Material>(m[(size_t)k * ni * nj + (size_t)j * ni + i]);
    fill(u, uu);
    fill(v, vv);
    fill(w, ww);
  }
  static void fill(Array3d<double>& a, const double* src) {
    if (!src) { a.fill(0.0); return; }
    for (int k = 0; k < a.sizek(); ++k)
      for (int j = 0; j < a.sizej(); ++j)
        for (int i = 0; i < a.sizei(); ++i)
          a(i, j, k) = src[(size_t)k * a.sizei() * a.sizej() + (size_t)j * a.sizei() + i];
  }
  static void dump(Array3d<double>& a, double* dst) {
    for (int k = 0; k < a.sizek(); ++k)
      for (int j = 0; j < a.sizej(); ++j)
        for (int i = 0; i < a.sizei(); ++i)
          dst[(size_t)k * a.sizei() * a.sizej() + (size_t)j * a.sizei() + i] = a(i, j, k);
  }
  template <typename Solver>
  void wire(Solver& s) {
    s.setSize(ni, nj, nk);
    s.setMaterial(&mat);
    s.setVelocityField(&u, &v, &w);
    s.setDensity(1.0);
    s.setDx(1.0);
    s.setDt(1.0);
    s.setDisField(nullptr);
  }
};

// A(c, c-off) for the 7-point structure, 0 when the entry does not exist.
double entry(const SparseMatrix<double>& A, unsigned row, long col) {
  if (col < 0) return 0.0;
  return A(row, (unsigned)col);
}

}  // namespace

extern "C" {

// Full reference solve: assembly + MIC(0)-PCG at (tol, maxit).  Writes the
// pressure grid (ni*nj*nk) only when the reference reports success, exactly as
// the reference does.  Returns 1 on success, 0 on failure.
int xfref_solve(int ni, int nj, int nk, const uint8_t* mat, const double* u,
                const double* v, const double* w, double tol, int maxit,
                double* p_out, int* iters_out, double* resid_out) {
  MuteCout mute;
  Scene sc(ni, nj, nk, mat, u, v, w);
  VariationalPressureSolver s;
  sc.wire(s);
  s.solver.set_solver_parameters(tol, maxit);
  Array3d<double> p;
  bool ok = s.solve(p);
  // solve() does not expose iterations/residual; rerun the PCG on the same
  // system to read them (deterministic, identical result).
  SparseMatrix<double> A;
  std::vector<double> b;
  s._calculate_coefficient(A, b);
  std::vector<double> x(b.size(), 0.0);
  double res = 0.0;
  int it = 0;
  PCGSolver<double> pcg;
  pcg.set_solver_parameters(tol, maxit);
  pcg.solve(A, b, x, res, it);
  if (iters_out) *iters_out = it;
  if (resid_out) *resid_out = res;
  if (ok && p_out) Scene::dump(p, p_out);
  return ok ? 1 : 0;
}

// One reference projection exactly as FluidSimulator::_solvePressure runs it
// (xFluid/xFluid/FluidSimulator.cpp:501-509): solve() then applyPressure() on
// the same grids.  Used to time the reference CPU path; (u,v,w) are updated in
// place and the pressure grid is written when the solve succeeds.
int xfref_project(int ni, int nj, int nk, const uint8_t* mat, double* u,
                  double* v, double* w, double tol, int maxit, double* p_out) {
  MuteCout mute;
  Scene sc(ni, nj, nk, mat, u, v, w);
  VariationalPressureSolver s;
  sc.wire(s);
  s.solver.set_solver_parameters(tol, maxit);
  Array3d<double> p;
  bool ok = s.solve(p);
  if (!ok) p.resize(ni, nj, nk);  // the reference leaves p unsized here (UB); keep it defined
  s.applyPressure(p);
  if (p_out) Scene::dump(p, p_out);
  Scene::dump(sc.u, u);
  Scene::dump(sc.v, v);
  Scene::dump(sc.w, w);
  return ok ? 1 : 0;
}

// Reference applyPressure on (u,v,w) in place, given a pressure grid.
// OpenMP threads the reference's parallel loops use (applyPressure's loop over
// i, variational_pressuresolver.cpp:134); returns the count in effect before
// (1 when the build has no OpenMP).
int xfref_set_threads(int n) {
#ifdef _OPENMP
  const int before = omp_get_max_threads();
  if (n > 0) omp_set_num_threads(n);
  return before;
#else
  (void)n;
  return 1;
#endif
}

// applyPressure alone (:120-220) on `threads` threads: the solver is wired once
// and the call repeated `reps` times after one untimed call; returns the mean
// seconds per call (u, v, w are updated in place each time).
double xfref_time_apply(int ni, int nj, int nk, const uint8_t* mat, const double* p, double* u, double* v, double* w,
                        int threads, int reps) {
  MuteCout mute;
  const int before = xfref_set_threads(threads);
  Scene sc(ni, nj, nk, mat, u, v, w);
  VariationalPressureSolver s;
  sc.wire(s);
  Array3d<double> pg(ni, nj, nk);
  Scene::fill(pg, p);
  s.applyPressure(pg);
  const auto t0 = std::chrono::steady_clock::now();
  for (int r = 0; r < reps; ++r) s.applyPressure(pg);
  const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  xfref_set_threads(before);
  return sec / (reps > 0 ? reps : 1);
}

void xfref_apply(int ni, int nj, int nk, const uint8_t* mat, const double* p,
                 double* u, double* v, double* w) {
  MuteCout mute;
  Scene sc(ni, nj, nk, mat, u, v, w);
  VariationalPressureSolver s;
  sc.wire(s);
  Array3d<double> pg(ni, nj, nk);
  Scene::fill(pg, p);
  s.applyPressure(pg);
  Scene::dump(sc.u, u);
  Scene::dump(sc.v, v);
  Scene::dump(sc.w, w);
}

// Reference assembly.  Outputs dense per-cell arrays: diag = A(c,c),
// ax = A(c,c-1), ay = A(c,c-ni), az = A(c,c-ni*nj), b.  Returns the largest
// row length seen (7 for a 7-point pattern).
int xfref_assemble(int ni, int nj, int nk, const uint8_t* mat, const double* u,
                   const double* v, const double* w, double* diag, double* ax,
                   double* ay, double* az, double* b_out) {
  MuteCout mute;
  Scene sc(ni, nj, nk, mat, u, v, w);
  VariationalPressureSolver s;
  sc.wire(s);
  SparseMatrix<double> A;
  std::vector<double> b;
  s._calculate_coefficient(A, b);
  const long n = (long)ni * nj * nk, nn = (long)ni * nj;
  int maxrow = 0;
  for (long c = 0; c < n; ++c) {
    if ((int)A.index[c].size() > maxrow) maxrow = (int)A.index[c].size();
    diag[c] = A(c, c);
    ax[c] = entry(A, c, c - 1);
    ay[c] = entry(A, c, c - ni);
    az[c] = entry(A, c, c - nn);
    b_out[c] = b[c];
  }
  return maxrow;
}

// Reference MIC(0) factor of the assembled system.  Outputs invdiag and the
// strictly-lower factor entries keyed by the higher cell: lx[c] = L(c,c-1),
// ly[c] = L(c,c-ni), lz[c] = L(c,c-ni*nj).
void xfref_factor(int ni, int nj, int nk, const uint8_t* mat, const double* u,
                  const double* v, const double* w, double* invdiag, double* lx,
                  double* ly, double* lz) {
  MuteCout mute;
  Scene sc(ni, nj, nk, mat, u, v, w);
  VariationalPressureSolver s;
  sc.wire(s);
  SparseMatrix<double> A;
  std::vector<double> b;
  s._calculate_coefficient(A, b);
  SparseColumnLowerFactor<double> f;
  factor_modified_incomplete_cholesky0(A, f);
  const long n = (long)ni * nj * nk, nn = (long)ni * nj;
  for (long c = 0; c < n; ++c) { lx[c] = ly[c] = lz[c] = 0.0; invdiag[c] = f.invdiag[c]; }
  for (long col = 0; col < n; ++col) {
    for (unsigned p = f.colstart[col]; p < f.colstart[col + 1]; ++p) {
      long row = f.rowindex[p];
      long d = row - col;
      if (d == 1) lx[row] = f.value[p];
      else if (d == ni) ly[row] = f.value[p];
      else if (d == nn) lz[row] = f.value[p];
    }
  }
}

// Reference preconditioner application z = (L L^T)^{-1} r on the assembled
// system of the given scene.
void xfref_precond(int ni, int nj, int nk, const uint8_t* mat, const double* u,
                   const double* v, const double* w, const double* r, double* z) {
  MuteCout mute;
  Scene sc(ni, nj, nk, mat, u, v, w);
  VariationalPressureSolver s;
  sc.wire(s);
  SparseMatrix<double> A;
  std::vector<double> b;
  s._calculate_coefficient(A, b);
  SparseColumnLowerFactor<double> f;
  factor_modified_incomplete_cholesky0(A, f);
  const size_t n = (size_t)ni * nj * nk;
  std::vector<double> rr(r, r + n), zz(n, 0.0);
  solve_lower(f, rr, zz);
  solve_lower_transpose_in_place(f, zz);
  std::memcpy(z, zz.data(), n * sizeof(double));
}

// Reference divergence diagnostic (unit weights, solid faces skipped).
void xfref_divergence(int ni, int nj, int nk, const uint8_t* mat, const double* u,
                      const double* v, const double* w, double* div) {
  MuteCout mute;
  Scene sc(ni, nj, nk, mat, u, v, w);
  VariationalPressureSolver s;
  sc.wire(s);
  std::vector<double> d;
  s._calculate_divergience(d);
  std::memcpy(div, d.data(), d.size() * sizeof(double));
}

// ---- NormalPressureSolver (pressuresolver.cpp), the classic Poisson matrix ----

// Its assembly, as dense per-cell arrays (the layout of xfref_assemble).
int xfref_normal_assemble(int ni, int nj, int nk, const uint8_t* mat, const double* u,
                          const double* v, const double* w, double* diag, double* ax,
                          double* ay, double* az, double* b_out) {
  MuteCout mute;
  Scene sc(ni, nj, nk, mat, u, v, w);
  NormalPressureSolver s;
  sc.wire(s);
  SparseMatrix<double> A;
  std::vector<double> b;
  s._calculate_coefficient(A, b);
  const long n = (long)ni * nj * nk, nn = (long)ni * nj;
  int maxrow = 0;
  for (long c = 0; c < n; ++c) {
    if ((int)A.index[c].size() > maxrow) maxrow = (int)A.index[c].size();
    diag[c] = A(c, c);
    ax[c] = entry(A, c, c - 1);
    ay[c] = entry(A, c, c - ni);
    az[c] = entry(A, c, c - nn);
    b_out[c] = b[c];
  }
  return maxrow;
}

// Its solve at (tol, maxit); pressure written when it reports success.
// Iterations and residual from the same PCG rerun on the same system.
int xfref_normal_solve(int ni, int nj, int nk, const uint8_t* mat, const double* u,
                       const double* v, const double* w, double tol, int maxit,
                       double* p_out, int* iters_out, double* resid_out) {
  MuteCout mute;
  Scene sc(ni, nj, nk, mat, u, v, w);
  NormalPressureSolver s;
  sc.wire(s);
  s.solver.set_solver_parameters(tol, maxit);
  Array3d<double> p;
  bool ok = s.solve(p);
  SparseMatrix<double> A;
  std::vector<double> b;
  s._calculate_coefficient(A, b);
  std::vector<double> x(b.size(), 0.0);
  double res = 0.0;
  int it = 0;
  PCGSolver<double> pcg;
  pcg.set_solver_parameters(tol, maxit);
  pcg.solve(A, b, x, res, it);
  if (iters_out) *iters_out = it;
  if (resid_out) *resid_out = res;
  if (ok && p_out) Scene::dump(p, p_out);
  return ok ? 1 : 0;
}

// Its applyPressure on (u,v,w) in place, given a pressure grid.
void xfref_normal_apply(int ni, int nj, int nk, const uint8_t* mat, const double* p,
                        double* u, double* v, double* w) {
  MuteCout mute;
  Scene sc(ni, nj, nk, mat, u, v, w);
  NormalPressureSolver s;
  sc.wire(s);
  Array3d<double> pg(ni, nj, nk);
  Scene::fill(pg, p);
  s.applyPressure(pg);
  Scene::dump(sc.u, u);
  Scene::dump(sc.v, v);
  Scene::dump(sc.w, w);
}

}  // extern "C"
