/* xfp_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU FP64 restatement of xFluid's variational pressure projection, used by the
 * tests and by bench.py's CPU-baseline leg as the checker.  The product (the
 * CUDA library) never links or calls this file.
 *
 * Parity pin: tests/test_oracle.py checks every routine here against the
 * reference itself (oracle/_ref/libxfref.so, built from the reference sources
 * by oracle/build_ref.sh) and against the committed golden vectors in
 * tests/golden/, which that same reference build produced.  In reference mode
 * (no face weights) assembly, factor, preconditioner, SpMV, PCG and
 * applyPressure are bit-identical to the reference, because every loop below
 * performs the same floating-point operations in the same order (built with
 * -ffp-contract=off, like the reference build).
 *
 * Reference paths are relative to xFluid/xFluid/ in the xFluid checkout.
 *
 * Layout: xFluid's Array3d, flat index k*ni*nj + j*ni + i (array3d.h:143-146).
 * Faces: u (ni+1,nj,nk), v (ni,nj+1,nk), w (ni,nj,nk+1) (FluidSimulator.h:177-181).
 * Material: 0 air, 1 fluid, 2 solid (material.h:4-8).
 *
 * The normal solver (pressuresolver.cpp, the classic Poisson matrix and its
 * applyPressure) is restated at the end of the file, pinned the same way.
 *
 * Generalisation beyond the reference (fractional mode): optional per-face
 * open fractions wu/wv/ww in [0,1] multiply every face's contribution.  NULL
 * weights give exactly the reference's matrix.  A neighbour outside the grid is
 * a closed face that contributes nothing (the reference reads out of bounds
 * there and relies on a solid border ring, FluidSimulator.cpp:64-96).
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define AIR 0
#define FLUID 1
#define SOLID 2

typedef struct {
  int ni, nj, nk;
  size_t nn, n;
} grid_t;

static grid_t mkgrid(int ni, int nj, int nk) {
  grid_t g;
  g.ni = ni; g.nj = nj; g.nk = nk;
  g.nn = (size_t)ni * nj;
  g.n = g.nn * nk;
  return g;
}

static inline size_t cidx(const grid_t* g, int i, int j, int k) {
  return (size_t)k * g->nn + (size_t)j * g->ni + i;
}
static inline size_t uidx(const grid_t* g, int i, int j, int k) {
  return ((size_t)k * g->nj + j) * (size_t)(g->ni + 1) + i;
}
static inline size_t vidx(const grid_t* g, int i, int j, int k) {
  return ((size_t)k * (g->nj + 1) + j) * (size_t)g->ni + i;
}
static inline size_t widx(const grid_t* g, int i, int j, int k) {
  return ((size_t)k * g->nj + j) * (size_t)g->ni + i;
}
static inline int inrange(const grid_t* g, int i, int j, int k) {
  return i >= 0 && j >= 0 && k >= 0 && i < g->ni && j < g->nj && k < g->nk;
}

/* Face between cell (i,j,k) and its neighbour n in xFluid's neighbour order
 * +i,-i,+j,-j,+k,-k (xfluidutil.cpp:33-41).  Returns the face value, its weight,
 * vsign (+1 when the neighbour is on the low side, -1 on the high side,
 * variational_pressuresolver.cpp:258-288) and the neighbour coordinates. */
typedef struct {
  int di, dj, dk;
} off3;
static const off3 NEI[6] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};

static void face_of(const grid_t* g, int i, int j, int k, int nb, const double* u,
                    const double* v, const double* w, const double* wu,
                    const double* wv, const double* ww, double* uf, double* mf,
                    double* vsign) {
  int di = NEI[nb].di, dj = NEI[nb].dj, dk = NEI[nb].dk;
  int hi = (di + dj + dk) > 0;
  int fi = i + (di > 0), fj = j + (dj > 0), fk = k + (dk > 0);
  size_t f;
  *vsign = hi ? -1.0 : 1.0;
  if (di) {
    f = uidx(g, fi, fj, fk); *uf = u[f]; *mf = wu ? wu[f] : 1.0;
  } else if (dj) {
    f = vidx(g, fi, fj, fk); *uf = v[f]; *mf = wv ? wv[f] : 1.0;
  } else {
    f = widx(g, fi, fj, fk); *uf = w[f]; *mf = ww ? ww[f] : 1.0;
  }
}

/* Assembly, gather form of VariationalPressureSolver::_calculate_coefficient
 * (variational_pressuresolver.cpp:231-327).
 *  fluid c, neighbour n across face f (weight m):
 *    n fluid: A(c,c)+=m, A(c,n)=-m,     b(c)+=vsign*u*m        (:294-301)
 *    n air:   A(c,c)+=2m,               b(c)+=vsign*u*m        (:302-308)
 *    n solid: A(c,c)+=0.5m, A(c,n)=-0.5m, b(c)+=vsign*u*0.5*m   (:309-316)
 *  solid s with fluid neighbour f (the reference adds these from f's loop,
 *  :318-320, so s receives them in the loop order i-major/j/k-minor, i.e. from
 *  neighbours -x,-y,-z,+z,+y,+x):
 *    A(s,s)+=0.5m, A(s,f)=-0.5m, b(s)+= -vsign_f*u*0.5*m
 *  Off-diagonals are stored keyed by the higher cell: ax[c]=A(c,c-1),
 *  ay[c]=A(c,c-ni), az[c]=A(c,c-ni*nj). */
void xo_assemble(int ni, int nj, int nk, const uint8_t* mat, const double* u,
                 const double* v, const double* w, const double* wu,
                 const double* wv, const double* ww, double* diag, double* ax,
                 double* ay, double* az, double* b) {
  grid_t g = mkgrid(ni, nj, nk);
  /* neighbour visiting order for a solid cell: -x,-y,-z,+z,+y,+x */
  static const int SOLID_ORDER[6] = {1, 3, 5, 4, 2, 0};
  for (int k = 0; k < nk; ++k)
    for (int j = 0; j < nj; ++j)
      for (int i = 0; i < ni; ++i) {
        size_t c = cidx(&g, i, j, k);
        double d = 0.0, bb = 0.0, ox = 0.0, oy = 0.0, oz = 0.0;
        uint8_t m = mat[c];
        if (m == FLUID) {
          for (int nb = 0; nb < 6; ++nb) {
            int a = i + NEI[nb].di, bj = j + NEI[nb].dj, ck = k + NEI[nb].dk;
            if (!inrange(&g, a, bj, ck)) continue;
            double uf, mf, vs;
            face_of(&g, i, j, k, nb, u, v, w, wu, wv, ww, &uf, &mf, &vs);
            uint8_t mn = mat[cidx(&g, a, bj, ck)];
            double off = 0.0;
            if (mn == FLUID) {
              d += 1.0 * mf;
              off = -1.0 * mf;
              bb += (vs * uf) * mf;
            } else if (mn == AIR) {
              d += 2.0 * mf;
              bb += (vs * uf) * mf;
            } else {
              d += 0.5 * mf;
              off = -0.5 * mf;
              bb += ((vs * uf) * 0.5) * mf;
            }
            if (nb == 1) ox = off;
            else if (nb == 3) oy = off;
            else if (nb == 5) oz = off;
          }
        } else if (m == SOLID) {
          for (int t = 0; t < 6; ++t) {
            int nb = SOLID_ORDER[t];
            int a = i + NEI[nb].di, bj = j + NEI[nb].dj, ck = k + NEI[nb].dk;
            if (!inrange(&g, a, bj, ck)) continue;
            if (mat[cidx(&g, a, bj, ck)] != FLUID) continue;
            double uf, mf, vs;
            face_of(&g, i, j, k, nb, u, v, w, wu, wv, ww, &uf, &mf, &vs);
            /* from the fluid cell's side vsign flips: -vsign_f = vs here */
            d += 0.5 * mf;
            double off = -0.5 * mf;
            bb += ((vs * uf) * 0.5) * mf;
            if (nb == 1) ox = off;
            else if (nb == 3) oy = off;
            else if (nb == 5) oz = off;
          }
        }
        diag[c] = d; ax[c] = ox; ay[c] = oy; az[c] = oz; b[c] = bb;
      }
}

/* SpMV z = A s in the order of multiply(FixedSparseMatrix) (sparse_matrix.h:264-276):
 * row entries in ascending column order c-nn, c-ni, c-1, c, c+1, c+ni, c+nn,
 * accumulated from 0, absent entries skipped. */
void xo_spmv(int ni, int nj, int nk, const double* diag, const double* ax,
             const double* ay, const double* az, const double* s, double* z) {
  grid_t g = mkgrid(ni, nj, nk);
  for (size_t c = 0; c < g.n; ++c) {
    double acc = 0.0;
    if (c >= g.nn && az[c] != 0.0) acc += az[c] * s[c - g.nn];
    if (c >= (size_t)ni && ay[c] != 0.0) acc += ay[c] * s[c - ni];
    if (c >= 1 && ax[c] != 0.0) acc += ax[c] * s[c - 1];
    if (diag[c] != 0.0) acc += diag[c] * s[c];
    if (c + 1 < g.n && ax[c + 1] != 0.0) acc += ax[c + 1] * s[c + 1];
    if (c + ni < g.n && ay[c + ni] != 0.0) acc += ay[c + ni] * s[c + ni];
    if (c + g.nn < g.n && az[c + g.nn] != 0.0) acc += az[c + g.nn] * s[c + g.nn];
    z[c] = acc;
  }
}

/* Modified incomplete Cholesky(0), factor_modified_incomplete_cholesky0
 * (pcg_solver.h:85-186), specialised to the 7-point pattern.  Column n's
 * strictly-lower entries are its upper neighbours n+1, n+ni, n+nn (when coupled);
 * none of them is in another's pattern, so every off-column product is dropped
 * fill and goes to `missing`.  Cell c therefore receives, in column order
 * (c-nn, then c-ni, then c-1), d -= L*L then d -= omega*L*missing, and its pivot
 * falls back to adiag when d < ratio*adiag (:126-131).  Outputs invdiag and
 * lx[c]=L(c,c-1), ly[c]=L(c,c-ni), lz[c]=L(c,c-nn). */
void xo_factor(int ni, int nj, int nk, const double* diag, const double* ax,
               const double* ay, const double* az, double omega, double ratio,
               double* inv, double* lx, double* ly, double* lz) {
  grid_t g = mkgrid(ni, nj, nk);
  const size_t step[3] = {g.nn, (size_t)ni, 1};   /* column order z, y, x */
  for (size_t c = 0; c < g.n; ++c) {
    lx[c] = ly[c] = lz[c] = 0.0;
    inv[c] = 0.0;
    double ad = diag[c];
    if (ad == 0.0) continue;
    double d = ad;
    const double acoef[3] = {az[c], ay[c], ax[c]};
    for (int t = 0; t < 3; ++t) {
      if (acoef[t] == 0.0 || c < step[t]) continue;
      size_t n = c - step[t];
      double invn = inv[n];
      double L = acoef[t] * invn;
      /* column n's entries in ascending row order: n+1, n+ni, n+nn */
      double up[3];
      up[0] = (n + 1 < g.n) ? ax[n + 1] : 0.0;
      up[1] = (n + ni < g.n) ? ay[n + ni] : 0.0;
      up[2] = (n + g.nn < g.n) ? az[n + g.nn] : 0.0;
      int self = 2 - t; /* which of n's upper entries is c itself */
      double missing = 0.0;
      for (int q = 0; q < 3; ++q) {
        if (q == self || up[q] == 0.0) continue;
        missing += up[q] * invn;
      }
      d -= L * L;
      d -= omega * L * missing;
      if (t == 0) lz[c] = L;
      else if (t == 1) ly[c] = L;
      else lx[c] = L;
    }
    if (d < ratio * ad)
      inv[c] = 1 / sqrt(ad);
    else
      inv[c] = 1 / sqrt(d);
  }
}

/* z = (L L^T)^{-1} r: solve_lower (column scatter, pcg_solver.h:192-204) then
 * solve_lower_transpose_in_place (pcg_solver.h:207-220). */
void xo_precond(int ni, int nj, int nk, const double* inv, const double* lx,
                const double* ly, const double* lz, const double* r, double* z) {
  grid_t g = mkgrid(ni, nj, nk);
  memcpy(z, r, g.n * sizeof(double));
  for (size_t c = 0; c < g.n; ++c) {
    z[c] *= inv[c];
    if (c + 1 < g.n && lx[c + 1] != 0.0) z[c + 1] -= lx[c + 1] * z[c];
    if (c + ni < g.n && ly[c + ni] != 0.0) z[c + ni] -= ly[c + ni] * z[c];
    if (c + g.nn < g.n && lz[c + g.nn] != 0.0) z[c + g.nn] -= lz[c + g.nn] * z[c];
  }
  size_t c = g.n;
  do {
    --c;
    if (c + 1 < g.n && lx[c + 1] != 0.0) z[c] -= lx[c + 1] * z[c + 1];
    if (c + ni < g.n && ly[c + ni] != 0.0) z[c] -= ly[c + ni] * z[c + ni];
    if (c + g.nn < g.n && lz[c + g.nn] != 0.0) z[c] -= lz[c + g.nn] * z[c + g.nn];
    z[c] *= inv[c];
  } while (c != 0);
}

/* The two halves of xo_precond separately: y = L^{-1} r, z = L^{-T} y. */
void xo_forward(int ni, int nj, int nk, const double* inv, const double* lx,
                const double* ly, const double* lz, const double* r, double* y) {
  grid_t g = mkgrid(ni, nj, nk);
  memcpy(y, r, g.n * sizeof(double));
  for (size_t c = 0; c < g.n; ++c) {
    y[c] *= inv[c];
    if (c + 1 < g.n && lx[c + 1] != 0.0) y[c + 1] -= lx[c + 1] * y[c];
    if (c + ni < g.n && ly[c + ni] != 0.0) y[c + ni] -= ly[c + ni] * y[c];
    if (c + g.nn < g.n && lz[c + g.nn] != 0.0) y[c + g.nn] -= lz[c + g.nn] * y[c];
  }
}
void xo_backward(int ni, int nj, int nk, const double* inv, const double* lx,
                 const double* ly, const double* lz, const double* y, double* z) {
  grid_t g = mkgrid(ni, nj, nk);
  memcpy(z, y, g.n * sizeof(double));
  size_t c = g.n;
  do {
    --c;
    if (c + 1 < g.n && lx[c + 1] != 0.0) z[c] -= lx[c + 1] * z[c + 1];
    if (c + ni < g.n && ly[c + ni] != 0.0) z[c] -= ly[c + ni] * z[c + ni];
    if (c + g.nn < g.n && lz[c + g.nn] != 0.0) z[c] -= lz[c + g.nn] * z[c + g.nn];
    z[c] *= inv[c];
  } while (c != 0);
}

/* BLAS::dot / abs_max / add_scaled (blas_wrapper.h:12-51): sequential loops. */
static double dot(size_t n, const double* x, const double* y) {
  double s = 0;
  for (size_t i = 0; i < n; ++i) s += x[i] * y[i];
  return s;
}
static double absmax(size_t n, const double* x) {
  double m = 0;
  size_t mi = 0;
  for (size_t i = 0; i < n; ++i)
    if (fabs(x[i]) > m) { m = fabs(x[i]); mi = i; }
  return n ? fabs(x[mi]) : 0.0;
}
static void add_scaled(size_t n, double a, const double* x, double* y) {
  for (size_t i = 0; i < n; ++i) y[i] += a * x[i];
}

/* PCGSolver<double>::solve (pcg_solver.h:243-285) on the assembled system.
 * Returns 1 on convergence (|r|_inf <= tol*|b|_inf), 0 otherwise; x holds the
 * last iterate either way. */
int xo_pcg(int ni, int nj, int nk, const double* diag, const double* ax,
           const double* ay, const double* az, const double* b, double tol,
           int maxit, double omega, double ratio, double* x, int* iters_out,
           double* resid_out) {
  grid_t g = mkgrid(ni, nj, nk);
  size_t n = g.n;
  if (tol < 1e-30) tol = 1e-30; /* set_solver_parameters, :237 */
  double *r = malloc(n * sizeof(double)), *z = malloc(n * sizeof(double)),
         *s = malloc(n * sizeof(double)), *inv = malloc(n * sizeof(double)),
         *lx = malloc(n * sizeof(double)), *ly = malloc(n * sizeof(double)),
         *lz = malloc(n * sizeof(double));
  int ok = 0, it = 0;
  memset(x, 0, n * sizeof(double));
  memcpy(r, b, n * sizeof(double));
  double res = absmax(n, r);
  if (res == 0) { ok = 1; it = 0; goto done; }
  double tolabs = tol * res;
  xo_factor(ni, nj, nk, diag, ax, ay, az, omega, ratio, inv, lx, ly, lz);
  xo_precond(ni, nj, nk, inv, lx, ly, lz, r, z);
  double rho = dot(n, z, r);
  if (rho == 0 || rho != rho) { ok = 0; it = 0; goto done; }
  memcpy(s, z, n * sizeof(double));
  for (it = 0; it < maxit; ++it) {
    xo_spmv(ni, nj, nk, diag, ax, ay, az, s, z);
    double alpha = rho / dot(n, s, z);
    add_scaled(n, alpha, s, x);
    add_scaled(n, -alpha, z, r);
    res = absmax(n, r);
    if (res <= tolabs) { ok = 1; ++it; goto done; }
    xo_precond(ni, nj, nk, inv, lx, ly, lz, r, z);
    double rho_new = dot(n, z, r);
    double beta = rho_new / rho;
    add_scaled(n, beta, s, z); /* z = z + beta*s, then s <-> z (:280) */
    double* t = s; s = z; z = t;
    rho = rho_new;
  }
done:
  if (iters_out) *iters_out = it;
  if (resid_out) *resid_out = res;
  free(r); free(z); free(s); free(inv); free(lx); free(ly); free(lz);
  return ok;
}

/* applyPressure (variational_pressuresolver.cpp:120-220) for one face with
 * left cell l and right cell r (out of range counts as solid, :151-152).
 * Returns 1 and the pressure difference p2-p1 when the face is updated. */
static int face_dp(const grid_t* g, const uint8_t* mat, const double* p, int il,
                   int jl, int kl, int ir, int jr, int kr, double* dp) {
  int inl = inrange(g, il, jl, kl), inr = inrange(g, ir, jr, kr);
  uint8_t ml = inl ? mat[cidx(g, il, jl, kl)] : SOLID;
  uint8_t mr = inr ? mat[cidx(g, ir, jr, kr)] : SOLID;
  double p1, p2;
  if (ml != FLUID && mr != FLUID) return 0;
  if (ml == FLUID && mr == FLUID) {
    p2 = p[cidx(g, ir, jr, kr)];
    p1 = p[cidx(g, il, jl, kl)];
  } else if (ml == FLUID) {
    p1 = p[cidx(g, il, jl, kl)];
    if (mr == SOLID) {
      if (!inr) return 0; /* closed grid boundary: no unknown behind it */
      p2 = p[cidx(g, ir, jr, kr)];
    } else {
      p2 = -p1;
    }
  } else {
    p2 = p[cidx(g, ir, jr, kr)];
    if (ml == SOLID) {
      if (!inl) return 0;
      p1 = p[cidx(g, il, jl, kl)];
    } else {
      p1 = -p2;
    }
  }
  *dp = p2 - p1;
  return 1;
}

/* u -= 1.0*(p2-p1) on every face touching fluid (factor 1.0, :122).  A face
 * with zero open fraction is closed and left unchanged. */
void xo_apply(int ni, int nj, int nk, const uint8_t* mat, const double* wu,
              const double* wv, const double* ww, const double* p, double* u,
              double* v, double* w) {
  grid_t g = mkgrid(ni, nj, nk);
  const double factor = 1.0;
  for (int k = 0; k < nk; ++k)
    for (int j = 0; j < nj; ++j)
      for (int i = 0; i <= ni; ++i) {
        double dp; size_t f = uidx(&g, i, j, k);
        if (wu && wu[f] == 0.0) continue;
        if (face_dp(&g, mat, p, i - 1, j, k, i, j, k, &dp)) u[f] = u[f] - factor * dp;
      }
  for (int k = 0; k < nk; ++k)
    for (int j = 0; j <= nj; ++j)
      for (int i = 0; i < ni; ++i) {
        double dp; size_t f = vidx(&g, i, j, k);
        if (wv && wv[f] == 0.0) continue;
        if (face_dp(&g, mat, p, i, j - 1, k, i, j, k, &dp)) v[f] = v[f] - factor * dp;
      }
  for (int k = 0; k <= nk; ++k)
    for (int j = 0; j < nj; ++j)
      for (int i = 0; i < ni; ++i) {
        double dp; size_t f = widx(&g, i, j, k);
        if (ww && ww[f] == 0.0) continue;
        if (face_dp(&g, mat, p, i, j, k - 1, i, j, k, &dp)) w[f] = w[f] - factor * dp;
      }
}

/* Adjoint of xo_apply's pressure term: q = G^T gbar, where apply computes
 * u_out = u - G p.  q[c] = sum over updated faces of d(p2-p1)/dp[c] * gbar[f]. */
void xo_apply_T(int ni, int nj, int nk, const uint8_t* mat, const double* wu,
                const double* wv, const double* ww, const double* gu,
                const double* gv, const double* gw, double* q) {
  grid_t g = mkgrid(ni, nj, nk);
  memset(q, 0, g.n * sizeof(double));
  for (int axis = 0; axis < 3; ++axis) {
    int si = ni + (axis == 0), sj = nj + (axis == 1), sk = nk + (axis == 2);
    for (int k = 0; k < sk; ++k)
      for (int j = 0; j < sj; ++j)
        for (int i = 0; i < si; ++i) {
          size_t f; const double* wt; const double* gb;
          if (axis == 0) { f = uidx(&g, i, j, k); wt = wu; gb = gu; }
          else if (axis == 1) { f = vidx(&g, i, j, k); wt = wv; gb = gv; }
          else { f = widx(&g, i, j, k); wt = ww; gb = gw; }
          if (wt && wt[f] == 0.0) continue;
          int il = i - (axis == 0), jl = j - (axis == 1), kl = k - (axis == 2);
          int inl = inrange(&g, il, jl, kl), inr = inrange(&g, i, j, k);
          uint8_t ml = inl ? mat[cidx(&g, il, jl, kl)] : SOLID;
          uint8_t mr = inr ? mat[cidx(&g, i, j, k)] : SOLID;
          if (ml != FLUID && mr != FLUID) continue;
          double gf = gb[f];
          /* dp = p2 - p1; u_out = u - dp  ->  dp's coefficients on p */
          if (ml == FLUID && mr == FLUID) {
            q[cidx(&g, i, j, k)] += gf; q[cidx(&g, il, jl, kl)] -= gf;
          } else if (ml == FLUID) {
            if (mr == SOLID) {
              if (!inr) continue;
              q[cidx(&g, i, j, k)] += gf; q[cidx(&g, il, jl, kl)] -= gf;
            } else {
              q[cidx(&g, il, jl, kl)] -= 2.0 * gf;
            }
          } else {
            if (ml == SOLID) {
              if (!inl) continue;
              q[cidx(&g, i, j, k)] += gf; q[cidx(&g, il, jl, kl)] -= gf;
            } else {
              q[cidx(&g, i, j, k)] += 2.0 * gf;
            }
          }
        }
  }
}

/* Adjoint of the right-hand side assembly: (u,v,w)-shaped D^T lam, where
 * xo_assemble computes b = D u (same coefficients: vsign*m for fluid and air
 * neighbours, vsign*0.5*m for solid ones, and the mirrored solid-cell rows). */
void xo_rhs_T(int ni, int nj, int nk, const uint8_t* mat, const double* wu,
              const double* wv, const double* ww, const double* lam, double* gu,
              double* gv, double* gw) {
  grid_t g = mkgrid(ni, nj, nk);
  memset(gu, 0, (size_t)(ni + 1) * nj * nk * sizeof(double));
  memset(gv, 0, (size_t)ni * (nj + 1) * nk * sizeof(double));
  memset(gw, 0, (size_t)ni * nj * (nk + 1) * sizeof(double));
  for (int k = 0; k < nk; ++k)
    for (int j = 0; j < nj; ++j)
      for (int i = 0; i < ni; ++i) {
        size_t c = cidx(&g, i, j, k);
        uint8_t m = mat[c];
        if (m != FLUID && m != SOLID) continue;
        for (int nb = 0; nb < 6; ++nb) {
          int a = i + NEI[nb].di, bj = j + NEI[nb].dj, ck = k + NEI[nb].dk;
          if (!inrange(&g, a, bj, ck)) continue;
          uint8_t mn = mat[cidx(&g, a, bj, ck)];
          double coef;
          if (m == FLUID) coef = (mn == SOLID) ? 0.5 : 1.0;
          else if (mn == FLUID) coef = 0.5;
          else continue;
          int di = NEI[nb].di, dj = NEI[nb].dj, dk = NEI[nb].dk;
          double vs = (di + dj + dk) > 0 ? -1.0 : 1.0;
          int fi = i + (di > 0), fj = j + (dj > 0), fk = k + (dk > 0);
          if (di) { size_t f = uidx(&g, fi, fj, fk); gu[f] += vs * coef * (wu ? wu[f] : 1.0) * lam[c]; }
          else if (dj) { size_t f = vidx(&g, fi, fj, fk); gv[f] += vs * coef * (wv ? wv[f] : 1.0) * lam[c]; }
          else { size_t f = widx(&g, fi, fj, fk); gw[f] += vs * coef * (ww ? ww[f] : 1.0) * lam[c]; }
        }
      }
}

/* The reference's divergence diagnostic (_calculate_divergience,
 * variational_pressuresolver.cpp:526-597): per fluid cell, unit-weight sum of
 * u(low)-u(high) over faces whose neighbour is not solid (out of range counts
 * as solid). */
void xo_divergence_ref(int ni, int nj, int nk, const uint8_t* mat, const double* u,
                       const double* v, const double* w, double* div) {
  grid_t g = mkgrid(ni, nj, nk);
  memset(div, 0, g.n * sizeof(double));
#define MATOR(a, b, c) (inrange(&g, a, b, c) ? mat[cidx(&g, a, b, c)] : SOLID)
  for (int i = 0; i < ni; ++i)
    for (int j = 0; j < nj; ++j)
      for (int k = 0; k < nk; ++k) {
        size_t c = cidx(&g, i, j, k);
        if (mat[c] != FLUID) continue;
        if (MATOR(i - 1, j, k) != SOLID) div[c] += u[uidx(&g, i, j, k)];
        if (MATOR(i + 1, j, k) != SOLID) div[c] -= u[uidx(&g, i + 1, j, k)];
        if (MATOR(i, j - 1, k) != SOLID) div[c] += v[vidx(&g, i, j, k)];
        if (MATOR(i, j + 1, k) != SOLID) div[c] -= v[vidx(&g, i, j + 1, k)];
        if (MATOR(i, j, k - 1) != SOLID) div[c] += w[widx(&g, i, j, k)];
        if (MATOR(i, j, k + 1) != SOLID) div[c] -= w[widx(&g, i, j, k + 1)];
      }
#undef MATOR
}

/* Full projection in reference order: assemble, PCG, pressure for every cell
 * (null rows 0), then applyPressure.  Returns the PCG status. */
int xo_project(int ni, int nj, int nk, const uint8_t* mat, double* u, double* v,
               double* w, const double* wu, const double* wv, const double* ww,
               double tol, int maxit, double* p, int* iters, double* resid) {
  grid_t g = mkgrid(ni, nj, nk);
  size_t n = g.n;
  double *d = malloc(n * sizeof(double)), *ax = malloc(n * sizeof(double)),
         *ay = malloc(n * sizeof(double)), *az = malloc(n * sizeof(double)),
         *b = malloc(n * sizeof(double));
  xo_assemble(ni, nj, nk, mat, u, v, w, wu, wv, ww, d, ax, ay, az, b);
  int ok = xo_pcg(ni, nj, nk, d, ax, ay, az, b, tol, maxit, 0.97, 0.25, p, iters, resid);
  xo_apply(ni, nj, nk, mat, wu, wv, ww, p, u, v, w);
  free(d); free(ax); free(ay); free(az); free(b);
  return ok;
}

/* ---- NormalPressureSolver (pressuresolver.cpp): the classic Poisson matrix ----
 * Assembly, _calculate_coefficient (:220-347).  Fluid rows only: A(c,c) is the
 * number of in-range neighbours that are not solid, A(c,n) = -1 for each fluid
 * neighbour n.  b(c) gathers the faces towards non-solid neighbours (out of
 * range counts as solid, :288-339) in the order low-x face added, high-x face
 * subtracted, then y, then z.  Each entry is written once, so the visiting
 * order of the matrix loop does not matter; b's order does. */
void xo_assemble_normal(int ni, int nj, int nk, const uint8_t* mat, const double* u,
                        const double* v, const double* w, double* diag, double* ax,
                        double* ay, double* az, double* b) {
  grid_t g = mkgrid(ni, nj, nk);
  static const int B_ORDER[6] = {1, 0, 3, 2, 5, 4}; /* -x,+x,-y,+y,-z,+z */
  for (int k = 0; k < nk; ++k)
    for (int j = 0; j < nj; ++j)
      for (int i = 0; i < ni; ++i) {
        size_t c = cidx(&g, i, j, k);
        double bb = 0.0, ox = 0.0, oy = 0.0, oz = 0.0;
        int count = 0;
        if (mat[c] == FLUID) {
          for (int t = 0; t < 6; ++t) {
            int nb = B_ORDER[t];
            int a = i + NEI[nb].di, bj = j + NEI[nb].dj, ck = k + NEI[nb].dk;
            if (!inrange(&g, a, bj, ck)) continue;
            uint8_t mn = mat[cidx(&g, a, bj, ck)];
            if (mn == SOLID) continue;
            double uf, mf, vs;
            face_of(&g, i, j, k, nb, u, v, w, NULL, NULL, NULL, &uf, &mf, &vs);
            ++count;
            bb += vs * uf; /* +u on the low face, -u on the high face */
            double off = mn == FLUID ? -1.0 : 0.0;
            if (nb == 1) ox = off;
            else if (nb == 3) oy = off;
            else if (nb == 5) oz = off;
          }
        }
        diag[c] = (double)count; ax[c] = ox; ay[c] = oy; az[c] = oz; b[c] = bb;
      }
}

/* applyPressure (:109-212), factor 1.0, for the face between cells l and r
 * (out of range counts as solid, :141-142): both fluid p2-p1; fluid|solid
 * takes p2 = p1 + u, solid|fluid p1 = p2 - u; an air side is 0. */
static int face_dp_normal(const grid_t* g, const uint8_t* mat, const double* p, int il, int jl,
                          int kl, int ir, int jr, int kr, double uf, double* dp) {
  int inl = inrange(g, il, jl, kl), inr = inrange(g, ir, jr, kr);
  uint8_t ml = inl ? mat[cidx(g, il, jl, kl)] : SOLID;
  uint8_t mr = inr ? mat[cidx(g, ir, jr, kr)] : SOLID;
  const double factor = 1.0;
  double p1, p2;
  if (ml != FLUID && mr != FLUID) return 0;
  if (ml == FLUID && mr == FLUID) {
    p2 = p[cidx(g, ir, jr, kr)];
    p1 = p[cidx(g, il, jl, kl)];
  } else if (ml == FLUID) {
    p1 = p[cidx(g, il, jl, kl)];
    p2 = mr == SOLID ? p1 + uf / factor : 0.0;
  } else {
    p2 = p[cidx(g, ir, jr, kr)];
    p1 = ml == SOLID ? p2 - uf / factor : 0.0;
  }
  *dp = p2 - p1;
  return 1;
}

void xo_apply_normal(int ni, int nj, int nk, const uint8_t* mat, const double* p, double* u,
                     double* v, double* w) {
  grid_t g = mkgrid(ni, nj, nk);
  const double factor = 1.0;
  double dp;
  for (int k = 0; k < nk; ++k)
    for (int j = 0; j < nj; ++j)
      for (int i = 0; i <= ni; ++i) {
        size_t f = uidx(&g, i, j, k);
        if (face_dp_normal(&g, mat, p, i - 1, j, k, i, j, k, u[f], &dp)) u[f] = u[f] - factor * dp;
      }
  for (int k = 0; k < nk; ++k)
    for (int j = 0; j <= nj; ++j)
      for (int i = 0; i < ni; ++i) {
        size_t f = vidx(&g, i, j, k);
        if (face_dp_normal(&g, mat, p, i, j - 1, k, i, j, k, v[f], &dp)) v[f] = v[f] - factor * dp;
      }
  for (int k = 0; k <= nk; ++k)
    for (int j = 0; j < nj; ++j)
      for (int i = 0; i < ni; ++i) {
        size_t f = widx(&g, i, j, k);
        if (face_dp_normal(&g, mat, p, i, j, k - 1, i, j, k, w[f], &dp)) w[f] = w[f] - factor * dp;
      }
}

/* NormalPressureSolver::solve (:50-106) + applyPressure on the same grids. */
int xo_project_normal(int ni, int nj, int nk, const uint8_t* mat, double* u, double* v, double* w,
                      double tol, int maxit, double* p, int* iters, double* resid) {
  grid_t g = mkgrid(ni, nj, nk);
  size_t n = g.n;
  double *d = malloc(n * sizeof(double)), *ax = malloc(n * sizeof(double)),
         *ay = malloc(n * sizeof(double)), *az = malloc(n * sizeof(double)),
         *b = malloc(n * sizeof(double));
  xo_assemble_normal(ni, nj, nk, mat, u, v, w, d, ax, ay, az, b);
  int ok = xo_pcg(ni, nj, nk, d, ax, ay, az, b, tol, maxit, 0.97, 0.25, p, iters, resid);
  xo_apply_normal(ni, nj, nk, mat, p, u, v, w);
  free(d); free(ax); free(ay); free(az); free(b);
  return ok;
}

/* ---- The simulator steps either side of the projection (FluidSimulator.cpp) ---- */

/* _applyForces (:429-499): dv = (sum of forces) * dt per axis; every face with
 * an in-range fluid cell on either side gets +dv; an axis with |dv| <= 1e-10
 * is skipped. */
void xo_apply_forces(int ni, int nj, int nk, const uint8_t* mat, double* u, double* v, double* w,
                     double fx, double fy, double fz, double dt) {
  grid_t g = mkgrid(ni, nj, nk);
  double dv[3] = {fx * dt, fy * dt, fz * dt};
  double* f[3] = {u, v, w};
  for (int a = 0; a < 3; ++a) {
    if (!(dv[a] > 1e-10 || dv[a] < -1e-10)) continue;
    int si = ni + (a == 0), sj = nj + (a == 1), sk = nk + (a == 2);
    for (int k = 0; k < sk; ++k)
      for (int j = 0; j < sj; ++j)
        for (int i = 0; i < si; ++i) {
          int il = i - (a == 0), jl = j - (a == 1), kl = k - (a == 2);
          int fr = inrange(&g, i, j, k) && mat[cidx(&g, i, j, k)] == FLUID;
          int fl = inrange(&g, il, jl, kl) && mat[cidx(&g, il, jl, kl)] == FLUID;
          if (fr || fl) {
            size_t q = ((size_t)k * sj + j) * si + i;
            f[a][q] += dv[a];
          }
        }
  }
}

/* _expolateVelocity(layers, axis) (:521-650) on one face grid (si,sj,sk):
 * marker 0 on the faces of fluid cells, -1 elsewhere; layer 1 = unmarked
 * faces with a layer-0 neighbour; then for each layer in turn every face of it
 * takes the average of its neighbours in the layer before (neighbour order
 * +i,-i,+j,-j,+k,-k) and hands its unmarked neighbours to the next layer. */
static void extrapolate_axis(const grid_t* g, const uint8_t* mat, int a, double* f, int layers) {
  int si = g->ni + (a == 0), sj = g->nj + (a == 1), sk = g->nk + (a == 2);
  size_t n = (size_t)si * sj * sk;
  int* mk = malloc(n * sizeof(int));
  size_t* cur = malloc(n * sizeof(size_t));
  size_t* nxt = malloc(n * sizeof(size_t));
  size_t ncur = 0, nnxt;
  for (size_t q = 0; q < n; ++q) mk[q] = -1;
  for (int k = 0; k < g->nk; ++k)
    for (int j = 0; j < g->nj; ++j)
      for (int i = 0; i < g->ni; ++i)
        if (mat[cidx(g, i, j, k)] == FLUID) {
          mk[((size_t)k * sj + j) * si + i] = 0;
          mk[((size_t)(k + (a == 2)) * sj + (j + (a == 1))) * si + (i + (a == 0))] = 0;
        }
#define NB(i, j, k, nb, ii, jj, kk) \
  (ii = (i) + NEI[nb].di, jj = (j) + NEI[nb].dj, kk = (k) + NEI[nb].dk, \
   ii >= 0 && jj >= 0 && kk >= 0 && ii < si && jj < sj && kk < sk)
  for (int k = 0; k < sk; ++k)
    for (int j = 0; j < sj; ++j)
      for (int i = 0; i < si; ++i) {
        size_t q = ((size_t)k * sj + j) * si + i;
        if (mk[q] != -1) continue;
        for (int nb = 0; nb < 6; ++nb) {
          int ii, jj, kk;
          if (NB(i, j, k, nb, ii, jj, kk) && mk[((size_t)kk * sj + jj) * si + ii] == 0) {
            cur[ncur++] = q;
            mk[q] = 1;
            break;
          }
        }
      }
  for (int L = 1; L <= layers; ++L) {
    nnxt = 0;
    for (size_t t = 0; t < ncur; ++t) {
      size_t q = cur[t];
      int i = (int)(q % si), j = (int)((q / si) % sj), k = (int)(q / ((size_t)si * sj));
      double sum = 0.0;
      int count = 0;
      for (int nb = 0; nb < 6; ++nb) {
        int ii, jj, kk;
        if (NB(i, j, k, nb, ii, jj, kk) && mk[((size_t)kk * sj + jj) * si + ii] == L - 1) {
          sum += f[((size_t)kk * sj + jj) * si + ii];
          count += 1;
        }
      }
      if (count == 0) continue;
      f[q] = sum / (double)count;
      for (int nb = 0; nb < 6; ++nb) {
        int ii, jj, kk;
        if (NB(i, j, k, nb, ii, jj, kk)) {
          size_t p = ((size_t)kk * sj + jj) * si + ii;
          if (mk[p] == -1) {
            nxt[nnxt++] = p;
            mk[p] = L + 1;
          }
        }
      }
    }
    size_t* tmp = cur; cur = nxt; nxt = tmp;
    ncur = nnxt;
  }
#undef NB
  free(mk); free(cur); free(nxt);
}

void xo_extrapolate(int ni, int nj, int nk, const uint8_t* mat, double* u, double* v, double* w, int layers) {
  grid_t g = mkgrid(ni, nj, nk);
  extrapolate_axis(&g, mat, 0, u, layers);
  extrapolate_axis(&g, mat, 1, v, layers);
  extrapolate_axis(&g, mat, 2, w, layers);
}
