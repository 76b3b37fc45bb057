/* xfp_particles_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU FP64 restatement of the particle steps around xFluid's projection, used
 * by the tests as the checker.  The product (the CUDA library) never links or
 * calls this file.
 *
 *   xo_advect_particles  FluidSimulator::_advectParticles steps a and b
 *                        (FluidSimulator.cpp:652-723): FLIP/PIC velocity
 *                        update from the grid, RK4 advection (:895-906 with
 *                        _getVelocity :730-893), solid collision
 *                        (collision.cpp:293-393 line-voxel walk, :396-440
 *                        ray/AABB)
 *   xo_p2g               FluidSimulator::_updateVelocityByParticles (:909-1085)
 *   xo_update_material   FluidSimulator::_updateMaterial (:402-427)
 *   xo_distance_field    DirectedDistanceField::updateFeild (:122-165) and the
 *                        material part of updateSurfaceInfo (:167-215)
 *                        (directeddistancefield.cpp)
 *
 * Reference paths are relative to xFluid/xFluid/ in the xFluid checkout.
 * Every loop performs the reference's floating-point operations in its order
 * (built with -ffp-contract=off), so the results are bit-identical to the
 * reference's own build; tests/test_particles.py pins that against golden
 * vectors the reference produced (tests/golden/make_golden.py) and, where
 * oracle/_ref is built, against the reference on further seeded inputs.
 *
 * Particles are xFluid's struct Particle {Vec3d p; Vec3d v;} (particle.h:5-15):
 * six doubles per particle, p then v.
 *
 * Where the reference reads outside an array or can loop without end, this
 * restatement (and the CUDA path) defines the result instead:
 *   - _getVelocity's unclamped index along a face's own axis reads face n+1
 *     when the position is exactly on the far wall (p.x == dx*ni): the pair is
 *     taken as (n-1, n) with weight 1 on face n, the wall's own value;
 *   - the resolved collision position's cell is read without a range check
 *     (:714): outside the grid the particle stays where it was, as for solid;
 *   - the voxel walk (collision.cpp:353-391) has no iteration bound (its
 *     assertion is commented out): it stops after as many steps as the
 *     segment's cells differ along the three axes, reporting no voxel.
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
  double x, y, z;
} vec3;

static inline vec3 v3(double x, double y, double z) {
  vec3 r = {x, y, z};
  return r;
}
static inline vec3 vadd(vec3 a, vec3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline vec3 vsub(vec3 a, vec3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline vec3 vmul(vec3 a, double s) { return v3(a.x * s, a.y * s, a.z * s); }
static inline double vdot(vec3 a, vec3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

/* XFluid::pos2Index (xfluidutil.cpp:3-6): truncation toward zero */
static inline void pos2index(vec3 p, double dx, int* i, int* j, int* k) {
  *i = (int)(p.x / dx);
  *j = (int)(p.y / dx);
  *k = (int)(p.z / dx);
}

/* XFluid::trilinearInterpolate (xfluidutil.cpp:55-67) */
static double trilinear(const double* p, double x, double y, double z) {
  double v0 = (1.0 - x) * p[0] + x * p[1];
  double v1 = (1.0 - x) * p[2] + x * p[3];
  double v2 = (1.0 - x) * p[4] + x * p[5];
  double v3_ = (1.0 - x) * p[6] + x * p[7];
  v0 = (1.0 - y) * v0 + y * v1;
  v1 = (1.0 - y) * v2 + y * v3_;
  return (1.0 - z) * v0 + z * v1;
}

/* One face component of _getVelocity (FluidSimulator.cpp:829-892): `a` is the
 * face axis; the grid has extents (si,sj,sk) = cells + e_a. */
static double sample_axis(const double* f, int ni, int nj, int nk, int a, vec3 p, double dx) {
  const double invdx = 1.0 / dx;
  const int si = ni + (a == 0), sj = nj + (a == 1);
  double c[3];
  c[0] = a == 0 ? p.x * invdx : (p.x - 0.5 * dx) * invdx;
  c[1] = a == 1 ? p.y * invdx : (p.y - 0.5 * dx) * invdx;
  c[2] = a == 2 ? p.z * invdx : (p.z - 0.5 * dx) * invdx;
  const int n[3] = {ni, nj, nk};
  int id[3];
  for (int q = 0; q < 3; ++q) {
    if (q == a) {
      id[q] = (int)c[q];
      if (id[q] > n[q] - 1) id[q] = n[q] - 1; /* the far-wall read, defined */
    } else {
      id[q] = c[q] < 0.0 ? 0 : (int)c[q];
      id[q] = id[q] > (n[q] - 2) ? (n[q] - 2) : id[q];
    }
  }
  const int i = id[0], j = id[1], k = id[2];
  const double x = c[0] - i, y = c[1] - j, z = c[2] - k;
#define F(ii, jj, kk) f[(size_t)(kk) * si * sj + (size_t)(jj) * si + (ii)]
  const double t[8] = {F(i, j, k),         F(i + 1, j, k),         F(i, j + 1, k),         F(i + 1, j + 1, k),
                       F(i, j, k + 1),     F(i + 1, j, k + 1),     F(i, j + 1, k + 1),     F(i + 1, j + 1, k + 1)};
#undef F
  return trilinear(t, x, y, z);
}

/* FluidSimulator::_getVelocity (:730-893) with _isInRange (:337-340) */
static vec3 get_velocity(const double* u, const double* v, const double* w, int ni, int nj, int nk, double dx, vec3 p) {
  if (!((p.x >= 0.0) && (p.y >= 0.0) && (p.z >= 0.0) && (p.x <= dx * ni) && (p.y <= dx * nj) && (p.z <= dx * nk)))
    return v3(0.0, 0.0, 0.0);
  return v3(sample_axis(u, ni, nj, nk, 0, p, dx), sample_axis(v, ni, nj, nk, 1, p, dx),
            sample_axis(w, ni, nj, nk, 2, p, dx));
}

static inline int mat_in(int ni, int nj, int nk, int i, int j, int k) {
  return i >= 0 && j >= 0 && k >= 0 && i < ni && j < nj && k < nk;
}
#define MAT(i, j, k) mat[(size_t)(k) * ni * nj + (size_t)(j) * ni + (i)]

/* Collision::getLineSegmentVoxelIntersection (collision.cpp:293-393) */
static int segment_voxel(vec3 p0, vec3 p1, double dx, const uint8_t* mat, int ni, int nj, int nk, int* vox) {
  const double invdx = 1.0 / dx;
  p0 = vmul(p0, invdx);
  p1 = vmul(p1, invdx);
  const int gx0 = (int)floor(p0.x), gy0 = (int)floor(p0.y), gz0 = (int)floor(p0.z);
  const int gx1 = (int)floor(p1.x), gy1 = (int)floor(p1.y), gz1 = (int)floor(p1.z);
  const int sx = gx1 > gx0 ? 1 : gx1 < gx0 ? -1 : 0;
  const int sy = gy1 > gy0 ? 1 : gy1 < gy0 ? -1 : 0;
  const int sz = gz1 > gz0 ? 1 : gz1 < gz0 ? -1 : 0;
  int gx = gx0, gy = gy0, gz = gz0;
  const double gxp = gx0 + (gx1 > gx0 ? 1 : 0);
  const double gyp = gy0 + (gy1 > gy0 ? 1 : 0);
  const double gzp = gz0 + (gz1 > gz0 ? 1 : 0);
  const double vx = p1.x == p0.x ? 1 : p1.x - p0.x;
  const double vy = p1.y == p0.y ? 1 : p1.y - p0.y;
  const double vz = p1.z == p0.z ? 1 : p1.z - p0.z;
  const double vxvy = vx * vy, vxvz = vx * vz, vyvz = vy * vz;
  double errx = (gxp - p0.x) * vyvz;
  double erry = (gyp - p0.y) * vxvz;
  double errz = (gzp - p0.z) * vxvy;
  const double derrx = sx * vyvz, derry = sy * vxvz, derrz = sz * vxvy;
  const long long limit = (long long)abs(gx1 - gx0) + abs(gy1 - gy0) + abs(gz1 - gz0);
  for (long long it = 0;; ++it) {
    if (mat_in(ni, nj, nk, gx, gy, gz) && MAT(gx, gy, gz) == SOLID) {
      vox[0] = gx;
      vox[1] = gy;
      vox[2] = gz;
      return 1;
    }
    if (gx == gx1 && gy == gy1 && gz == gz1) break;
    if (it >= limit) break; /* the defined bound (see the header) */
    const double xr = fabs(errx), yr = fabs(erry), zr = fabs(errz);
    if (sx != 0 && (sy == 0 || xr < yr) && (sz == 0 || xr < zr)) {
      gx += sx;
      errx += derrx;
    } else if (sy != 0 && (sz == 0 || yr < zr)) {
      gy += sy;
      erry += derry;
    } else if (sz != 0) {
      gz += sz;
      errz += derrz;
    }
  }
  return 0;
}

/* Collision::rayIntersectsAABB (collision.cpp:396-440); the third small-
 * component test reads dir.x, as the reference does. */
static int ray_aabb(vec3 p0, vec3 dir, vec3 bmin, vec3 bmax, vec3* hit) {
  const double eps = 1e-10;
  if (fabs(dir.x) < eps) dir.x = dir.x < 0 ? -eps : eps;
  if (fabs(dir.y) < eps) dir.y = dir.y < 0 ? -eps : eps;
  if (fabs(dir.x) < eps) dir.z = dir.z < 0 ? -eps : eps;
  const vec3 inv = v3(1.0 / dir.x, 1.0 / dir.y, 1.0 / dir.z);
  double t1 = (bmin.x - p0.x) * inv.x, t2 = (bmax.x - p0.x) * inv.x;
  double tmin = fmin(t1, t2), tmax = fmax(t1, t2);
  t1 = (bmin.y - p0.y) * inv.y;
  t2 = (bmax.y - p0.y) * inv.y;
  tmin = fmax(tmin, fmin(t1, t2));
  tmax = fmin(tmax, fmax(t1, t2));
  t1 = (bmin.z - p0.z) * inv.z;
  t2 = (bmax.z - p0.z) * inv.z;
  tmin = fmax(tmin, fmin(t1, t2));
  tmax = fmin(tmax, fmax(t1, t2));
  if (tmax > fmax(tmin, 0.0)) {
    *hit = vadd(p0, vmul(dir, tmin));
    return 1;
  }
  return 0;
}

/* FluidSimulator::_advectParticles steps a and b (:652-723).  The reference
 * splits the particles into 6 chunks of n/6 (integer division) and leaves the
 * last n mod 6 particles untouched; this does the same.  us/vs/ws are the
 * velocities saved before the forces (_saveVelocity, :1095-1100).
 * status (optional, per particle): 0 advected, 1 moved to the collision
 * point, 2 collision point in a cell outside the grid (the reference reads out
 * of bounds there; kept in place here), 3 left in place by the collision test,
 * 4 beyond the six chunks (untouched). */
void xo_advect_particles(int ni, int nj, int nk, double dx, const uint8_t* mat, const double* u, const double* v,
                         const double* w, const double* us, const double* vs, const double* ws, double ratio, double dt,
                         long long n, double* parts, int* status) {
  const long long nper = n / 6;
  const long long m = nper * 6;
  if (status)
    for (long long q = 0; q < n; ++q) status[q] = q < m ? 0 : 4;
  for (long long q = 0; q < m; ++q) {
    double* P = parts + 6 * q;
    const vec3 p = v3(P[0], P[1], P[2]);
    /* a. FLIP/PIC blend (:667-678) */
    const vec3 vnew = get_velocity(u, v, w, ni, nj, nk, dx, p);
    const vec3 vold = get_velocity(us, vs, ws, ni, nj, nk, dx, p);
    const vec3 vflip = vsub(vadd(v3(P[3], P[4], P[5]), vnew), vold);
    const vec3 vb = vadd(vmul(vnew, 1.0 - ratio), vmul(vflip, ratio));
    P[3] = vb.x;
    P[4] = vb.y;
    P[5] = vb.z;
  }
  for (long long q = 0; q < m; ++q) {
    double* P = parts + 6 * q;
    const vec3 cur = v3(P[0], P[1], P[2]);
    /* b. RK4 (:895-906) */
    const vec3 k1 = get_velocity(u, v, w, ni, nj, nk, dx, cur);
    const vec3 k2 = get_velocity(u, v, w, ni, nj, nk, dx, vadd(cur, vmul(k1, 0.5 * dt)));
    const vec3 k3 = get_velocity(u, v, w, ni, nj, nk, dx, vadd(cur, vmul(k2, 0.5 * dt)));
    const vec3 k4 = get_velocity(u, v, w, ni, nj, nk, dx, vadd(cur, vmul(k3, dt)));
    const vec3 np = vadd(cur, vmul(vadd(vadd(vadd(k1, vmul(k2, 2.0)), vmul(k3, 2.0)), k4), dt / 6.0));
    int gi, gj, gk;
    pos2index(np, dx, &gi, &gj, &gk);
    if (mat_in(ni, nj, nk, gi, gj, gk) && MAT(gi, gj, gk) != SOLID) {
      P[0] = np.x;
      P[1] = np.y;
      P[2] = np.z;
      continue;
    }
    /* into a solid (:691-721) */
    int vox[3];
    if (status) status[q] = 3;
    if (!segment_voxel(cur, np, dx, mat, ni, nj, nk, vox)) continue;
    const vec3 d = vsub(np, cur);
    const double l = sqrt(d.x * d.x + d.y * d.y + d.z * d.z);
    const vec3 ray = v3(d.x / l, d.y / l, d.z / l);
    const vec3 bmin = v3((vox[0] + 0.5) * dx, (vox[1] + 0.5) * dx, (vox[2] + 0.5) * dx);
    const vec3 bmax = vadd(bmin, v3(dx, dx, dx));
    vec3 hit;
    if (!ray_aabb(cur, ray, bmin, bmax, &hit)) continue;
    const vec3 res = vsub(hit, vmul(ray, (double)(float)(0.05 * dx)));
    int ri, rj, rk;
    pos2index(res, dx, &ri, &rj, &rk);
    if (mat_in(ni, nj, nk, ri, rj, rk) && MAT(ri, rj, rk) != SOLID) {
      P[0] = res.x;
      P[1] = res.y;
      P[2] = res.z;
      if (status) status[q] = 1;
    } else if (status && !mat_in(ni, nj, nk, ri, rj, rk)) {
      status[q] = 2;
    }
  }
}

/* FluidSimulator::_updateVelocityByParticles (:909-1085), one face axis at a
 * time, particles in index order; face grid of axis a has extents cells+e_a. */
void xo_p2g(int ni, int nj, int nk, double dx, long long n, const double* parts, double* u, double* v, double* w) {
  const double r = 1.5 * dx, r2 = r * r;
  const double c0 = (4.0 / 9.0) * (1.0 / (r2 * r2 * r2));
  const double c1 = (17.0 / 9.0) * (1.0 / (r2 * r2));
  const double c2 = (22.0 / 9.0) * (1.0 / (r2));
  double* out[3] = {u, v, w};
  for (int a = 0; a < 3; ++a) {
    const int si = ni + (a == 0), sj = nj + (a == 1), sk = nk + (a == 2);
    const size_t nf = (size_t)si * sj * sk;
    double* wt = (double*)calloc(nf, sizeof(double));
    double* val = (double*)calloc(nf, sizeof(double));
    for (long long q = 0; q < n; ++q) {
      const double* P = parts + 6 * q;
      const vec3 p = vadd(v3(P[0], P[1], P[2]), v3(a == 0 ? 0.5 * dx : 0.0, a == 1 ? 0.5 * dx : 0.0,
                                                   a == 2 ? 0.5 * dx : 0.0));
      const double vel = P[3 + a];
      int i0, j0, k0, i1, j1, k1;
      pos2index(vadd(v3(-r, -r, -r), p), dx, &i0, &j0, &k0); /* getBoundingGrid (xfluidutil.cpp:23-31) */
      pos2index(vadd(p, v3(r, r, r)), dx, &i1, &j1, &k1);
      for (int i = i0; i <= i1; ++i)
        for (int j = j0; j <= j1; ++j)
          for (int k = k0; k <= k1; ++k) {
            if (!(i >= 0 && j >= 0 && k >= 0 && i < si && j < sj && k < sk)) continue;
            const vec3 cr = vsub(p, v3((i + 0.5) * dx, (j + 0.5) * dx, (k + 0.5) * dx));
            const double rs = vdot(cr, cr);
            const double cw = rs < r2 ? 1.0 - c0 * rs * rs * rs + c1 * rs * rs - c2 * rs : 0.0;
            const size_t id = (size_t)k * si * sj + (size_t)j * si + i;
            wt[id] += cw;
            val[id] += vel * cw;
          }
    }
    for (size_t id = 0; id < nf; ++id) out[a][id] = wt[id] > 0.0000001 ? val[id] / wt[id] : 0.0;
    free(wt);
    free(val);
  }
}

/* FluidSimulator::_updateMaterial (:402-427) */
void xo_update_material(int ni, int nj, int nk, double dx, long long n, const double* parts, uint8_t* mat) {
  const size_t nc = (size_t)ni * nj * nk;
  for (size_t c = 0; c < nc; ++c)
    if (mat[c] != SOLID) mat[c] = AIR;
  for (long long q = 0; q < n; ++q) {
    int i, j, k;
    pos2index(v3(parts[6 * q], parts[6 * q + 1], parts[6 * q + 2]), dx, &i, &j, &k);
    if (mat_in(ni, nj, nk, i, j, k) && MAT(i, j, k) != SOLID) MAT(i, j, k) = FLUID;
  }
}

/* DirectedDistanceField::updateFeild (directeddistancefield.cpp:122-165) with
 * _addParticleWeightParallel (:275-302) and _weight (:245-255): six partial
 * fields over chunks of n/6+1 particles, summed in chunk order.  phi has
 * extents (ni*s+1, nj*s+1, nk*s+1).  Then, when mat is given, the material
 * part of updateSurfaceInfo (:167-215) with _isCellSurface (:304-327) and
 * _centerPhi (:329-344). */
void xo_distance_field(int ni, int nj, int nk, double dx, int s, double radius, double threshold, long long n,
                       const double* parts, double* phi, uint8_t* mat) {
  const int pi_ = ni * s + 1, pj = nj * s + 1, pk = nk * s + 1;
  const size_t np = (size_t)pi_ * pj * pk;
  const double sq = radius * radius;
  const double c0 = (4.0 / 9.0) * (1.0 / (sq * sq * sq));
  const double c1 = (17.0 / 9.0) * (1.0 / (sq * sq));
  const double c2 = (22.0 / 9.0) * (1.0 / (sq));
  const double subdx = dx / (double)s;
  const long long nper = n / 6 + 1;
  double* part = (double*)malloc(np * sizeof(double));
  for (size_t q = 0; q < np; ++q) phi[q] = 0.0;
  for (int t = 0; t < 6; ++t) {
    for (size_t q = 0; q < np; ++q) part[q] = 0.0;
    const long long a = t * nper;
    long long b = a + nper;
    b = b > n ? n : b;
    for (long long q = a; q < b; ++q) {
      const vec3 p = v3(parts[6 * q], parts[6 * q + 1], parts[6 * q + 2]);
      int i0, j0, k0, i1, j1, k1;
      pos2index(vadd(v3(-radius, -radius, -radius), p), dx, &i0, &j0, &k0);
      pos2index(vadd(p, v3(radius, radius, radius)), dx, &i1, &j1, &k1);
      i0 *= s; j0 *= s; k0 *= s;
      i1 = (i1 + 1) * s; j1 = (j1 + 1) * s; k1 = (k1 + 1) * s;
      for (int i = i0; i <= i1; ++i)
        for (int j = j0; j <= j1; ++j)
          for (int k = k0; k <= k1; ++k) {
            if (!(i >= 0 && j >= 0 && k >= 0 && i < pi_ && j < pj && k < pk)) continue;
            const vec3 gp = v3((i + 0.5) * subdx, (j + 0.5) * subdx, (k + 0.5) * subdx);
            const double rs = vdot(vsub(gp, p), vsub(gp, p));
            part[(size_t)k * pi_ * pj + (size_t)j * pi_ + i] +=
                rs < sq ? 1.0 - c0 * rs * rs * rs + c1 * rs * rs - c2 * rs : 0.0;
          }
    }
    for (size_t q = 0; q < np; ++q) phi[q] += part[q];
  }
  free(part);
  if (!mat) return;
#define PHI(i, j, k) phi[(size_t)(k) * pi_ * pj + (size_t)(j) * pi_ + (i)]
  for (int k = 0; k < nk; ++k)
    for (int j = 0; j < nj; ++j)
      for (int i = 0; i < ni; ++i) {
        const int si = i * s, sj = j * s, sk = k * s;
        int in = 0, out = 0;
        for (int a = si; a <= si + s; ++a)
          for (int b = sj; b <= sj + s; ++b)
            for (int c = sk; c <= sk + s; ++c) {
              if (PHI(a, b, c) >= threshold) in = 1;
              else out = 1;
            }
        double val;
        if (in && out) {
          if (s % 2 == 0) {
            val = PHI(si + s / 2, sj + s / 2, sk + s / 2);
          } else {
            val = 0.0;
            for (int a = si; a <= si + s; a += s)
              for (int b = sj; b <= sj + s; b += s)
                for (int c = sk; c <= sk + s; c += s) val += PHI(a, b, c);
            val = val / 8.0;
          }
        } else {
          val = PHI(si, sj, sk);
        }
        if (MAT(i, j, k) != SOLID) MAT(i, j, k) = val >= threshold ? FLUID : AIR;
      }
#undef PHI
}
#undef MAT
