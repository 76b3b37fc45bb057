// xfp_particles.cu -- the particle steps either side of the projection
// (xFluid/xFluid/FluidSimulator.cpp, directeddistancefield.cpp):
//
//   xfp_advect_particles_f64   _advectParticles steps a-b        :652-723
//                              FLIP/PIC update (_getVelocity :730-893), RK4
//                              (:895-906), solid collision (collision.cpp:
//                              293-393 voxel walk, :396-440 ray/AABB)
//   xfp_particles_to_grid_f64  _updateVelocityByParticles        :909-1085
//   xfp_update_material        _updateMaterial                   :402-427
//   xfp_distance_field_f64     DirectedDistanceField::updateFeild :122-165
//                              + updateSurfaceInfo's material     :167-215
//
// Particles are xFluid's struct Particle {Vec3d p; Vec3d v;}: six doubles.
//
// Advection and the material update are per-particle work, done one thread
// per particle with every FP64 operation rounded as the reference rounds it
// (__dadd_rn and friends, no contraction): bit-identical results.
//
// The two transfers (particle -> face weights, particle -> distance field) are
// sums over particles.  The reference scatters particle by particle; here each
// output gathers.  Particles are binned by the low corner of their own bounding
// box (per face axis for the transfer, per cell for the field), clamped at 0,
// with a stable radix sort, so a bin's particles are in index order.  An output
// at index i is covered only by boxes with gmin <= i <= gmax, so it scans the
// bins [i - maxspan, i] per axis (maxspan = the widest box, reduced from the
// boxes themselves) and keeps the particles whose box holds it: exactly the
// reference's set of contributions, no atomics, and a fixed summation order.
// That order is not the reference's particle order, so these sums agree with
// the reference to FP64 rounding rather than bit for bit.
//
// Where the reference reads outside an array or can loop without end, a result
// is defined instead: a far-wall face read (x == ni) takes the wall face; a
// collision point in a cell outside the grid leaves the particle in place; the
// voxel walk stops after the segment's Manhattan cell distance.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <string>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "xfp_context.h"

namespace xfp {
namespace {

constexpr uint8_t P_AIR = 0, P_FLUID = 1, P_SOLID = 2;

struct V3 {
  double x, y, z;
};
__device__ __forceinline__ V3 v3(double x, double y, double z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 vadd(V3 a, V3 b) { return v3(add_rn(a.x, b.x), add_rn(a.y, b.y), add_rn(a.z, b.z)); }
__device__ __forceinline__ V3 vsub(V3 a, V3 b) { return v3(sub_rn(a.x, b.x), sub_rn(a.y, b.y), sub_rn(a.z, b.z)); }
__device__ __forceinline__ V3 vmul(V3 a, double s) { return v3(mul_rn(a.x, s), mul_rn(a.y, s), mul_rn(a.z, s)); }
__device__ __forceinline__ double vdot(V3 a, V3 b) {
  return add_rn(add_rn(mul_rn(a.x, b.x), mul_rn(a.y, b.y)), mul_rn(a.z, b.z));
}

// C's (int) conversion of a double that is in int range (truncation toward
// zero); values outside it (and NaN) are clamped first so the conversion is
// defined -- only boxes far outside the grid are affected, which cover nothing
__device__ __forceinline__ int trunc_i(double x) {
  if (!(x > -1.0e9)) return -1000000000;
  if (x > 1.0e9) return 1000000000;
  return __double2int_rz(x);
}
__device__ __forceinline__ int floor_i(double x) { return trunc_i(floor(x)); }

// XFluid::trilinearInterpolate (xfluidutil.cpp:55-67)
__device__ double trilinear(const double* t, double x, double y, double z) {
  const double ox = sub_rn(1.0, x), oy = sub_rn(1.0, y), oz = sub_rn(1.0, z);
  double v0 = add_rn(mul_rn(ox, t[0]), mul_rn(x, t[1]));
  double v1 = add_rn(mul_rn(ox, t[2]), mul_rn(x, t[3]));
  const double v2 = add_rn(mul_rn(ox, t[4]), mul_rn(x, t[5]));
  const double v3_ = add_rn(mul_rn(ox, t[6]), mul_rn(x, t[7]));
  v0 = add_rn(mul_rn(oy, v0), mul_rn(y, v1));
  v1 = add_rn(mul_rn(oy, v2), mul_rn(y, v3_));
  return add_rn(mul_rn(oz, v0), mul_rn(z, v1));
}

struct PGrid {
  int ni, nj, nk;
  double dx;
};

// One face component of _getVelocity (FluidSimulator.cpp:829-892); `a` is
// the face axis, the face grid has extents cells + e_a.
__device__ double sample_axis(const double* __restrict__ f, const PGrid& G, int a, V3 p) {
  const double invdx = div_rn(1.0, G.dx);
  const double h = mul_rn(0.5, G.dx);
  const int si = G.ni + (a == 0), sj = G.nj + (a == 1);
  double c[3];
  c[0] = a == 0 ? mul_rn(p.x, invdx) : mul_rn(sub_rn(p.x, h), invdx);
  c[1] = a == 1 ? mul_rn(p.y, invdx) : mul_rn(sub_rn(p.y, h), invdx);
  c[2] = a == 2 ? mul_rn(p.z, invdx) : mul_rn(sub_rn(p.z, h), invdx);
  const int n[3] = {G.ni, G.nj, G.nk};
  int id[3];
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    if (q == a) {
      id[q] = trunc_i(c[q]);
      id[q] = min(max(id[q], 0), n[q] - 1);   // far-wall read defined; in range p gives >= 0
    } else {
      id[q] = c[q] < 0.0 ? 0 : trunc_i(c[q]);
      id[q] = id[q] > n[q] - 2 ? n[q] - 2 : id[q];
    }
  }
  const int i = id[0], j = id[1], k = id[2];
  const double x = sub_rn(c[0], (double)i), y = sub_rn(c[1], (double)j), z = sub_rn(c[2], (double)k);
  auto F = [&](int ii, int jj, int kk) { return __ldg(&f[(size_t)kk * si * sj + (size_t)jj * si + ii]); };
  const double t[8] = {F(i, j, k),     F(i + 1, j, k),     F(i, j + 1, k),     F(i + 1, j + 1, k),
                       F(i, j, k + 1), F(i + 1, j, k + 1), F(i, j + 1, k + 1), F(i + 1, j + 1, k + 1)};
  return trilinear(t, x, y, z);
}

// _getVelocity (:730-893) with _isInRange (:337-340)
__device__ V3 get_velocity(const double* u, const double* v, const double* w, const PGrid& G, V3 p) {
  if (!((p.x >= 0.0) && (p.y >= 0.0) && (p.z >= 0.0) && (p.x <= mul_rn(G.dx, (double)G.ni)) &&
        (p.y <= mul_rn(G.dx, (double)G.nj)) && (p.z <= mul_rn(G.dx, (double)G.nk))))
    return v3(0.0, 0.0, 0.0);
  return v3(sample_axis(u, G, 0, p), sample_axis(v, G, 1, p), sample_axis(w, G, 2, p));
}

__device__ __forceinline__ bool in_grid(const PGrid& G, int i, int j, int k) {
  return i >= 0 && j >= 0 && k >= 0 && i < G.ni && j < G.nj && k < G.nk;
}
__device__ __forceinline__ uint8_t mat_at(const uint8_t* m, const PGrid& G, int i, int j, int k) {
  return m[(size_t)k * G.ni * G.nj + (size_t)j * G.ni + i];
}

// XFluid::pos2Index (xfluidutil.cpp:3-6)
__device__ __forceinline__ void pos2index(V3 p, double dx, int* i, int* j, int* k) {
  *i = trunc_i(div_rn(p.x, dx));
  *j = trunc_i(div_rn(p.y, dx));
  *k = trunc_i(div_rn(p.z, dx));
}

// Collision::getLineSegmentVoxelIntersection (collision.cpp:293-393), with
// the walk bounded by the segment's Manhattan cell distance
__device__ bool segment_voxel(V3 p0, V3 p1, const PGrid& G, const uint8_t* mat, int* vox) {
  const double invdx = div_rn(1.0, G.dx);
  p0 = vmul(p0, invdx);
  p1 = vmul(p1, invdx);
  const int gx0 = floor_i(p0.x), gy0 = floor_i(p0.y), gz0 = floor_i(p0.z);
  const int gx1 = floor_i(p1.x), gy1 = floor_i(p1.y), gz1 = floor_i(p1.z);
  const int sx = gx1 > gx0 ? 1 : gx1 < gx0 ? -1 : 0;
  const int sy = gy1 > gy0 ? 1 : gy1 < gy0 ? -1 : 0;
  const int sz = gz1 > gz0 ? 1 : gz1 < gz0 ? -1 : 0;
  int gx = gx0, gy = gy0, gz = gz0;
  const double gxp = (double)(gx0 + (gx1 > gx0 ? 1 : 0));
  const double gyp = (double)(gy0 + (gy1 > gy0 ? 1 : 0));
  const double gzp = (double)(gz0 + (gz1 > gz0 ? 1 : 0));
  const double vx = p1.x == p0.x ? 1.0 : sub_rn(p1.x, p0.x);
  const double vy = p1.y == p0.y ? 1.0 : sub_rn(p1.y, p0.y);
  const double vz = p1.z == p0.z ? 1.0 : sub_rn(p1.z, p0.z);
  const double vxvy = mul_rn(vx, vy), vxvz = mul_rn(vx, vz), vyvz = mul_rn(vy, vz);
  double errx = mul_rn(sub_rn(gxp, p0.x), vyvz);
  double erry = mul_rn(sub_rn(gyp, p0.y), vxvz);
  double errz = mul_rn(sub_rn(gzp, p0.z), vxvy);
  const double derrx = mul_rn((double)sx, vyvz), derry = mul_rn((double)sy, vxvz), derrz = mul_rn((double)sz, vxvy);
  const long long limit = (long long)abs(gx1 - gx0) + abs(gy1 - gy0) + abs(gz1 - gz0);
  for (long long it = 0;; ++it) {
    if (in_grid(G, gx, gy, gz) && mat_at(mat, G, gx, gy, gz) == P_SOLID) {
      vox[0] = gx;
      vox[1] = gy;
      vox[2] = gz;
      return true;
    }
    if ((gx == gx1 && gy == gy1 && gz == gz1) || it >= limit) break;
    const double xr = fabs(errx), yr = fabs(erry), zr = fabs(errz);
    if (sx != 0 && (sy == 0 || xr < yr) && (sz == 0 || xr < zr)) {
      gx += sx;
      errx = add_rn(errx, derrx);
    } else if (sy != 0 && (sz == 0 || yr < zr)) {
      gy += sy;
      erry = add_rn(erry, derry);
    } else if (sz != 0) {
      gz += sz;
      errz = add_rn(errz, derrz);
    }
  }
  return false;
}

// Collision::rayIntersectsAABB (collision.cpp:396-440), with its third
// small-component test on dir.x kept as it is
__device__ bool ray_aabb(V3 p0, V3 dir, V3 bmin, V3 bmax, V3* hit) {
  const double eps = 1e-10;
  if (fabs(dir.x) < eps) dir.x = dir.x < 0 ? -eps : eps;
  if (fabs(dir.y) < eps) dir.y = dir.y < 0 ? -eps : eps;
  if (fabs(dir.x) < eps) dir.z = dir.z < 0 ? -eps : eps;
  const V3 inv = v3(div_rn(1.0, dir.x), div_rn(1.0, dir.y), div_rn(1.0, dir.z));
  double t1 = mul_rn(sub_rn(bmin.x, p0.x), inv.x), t2 = mul_rn(sub_rn(bmax.x, p0.x), inv.x);
  double tmin = fmin(t1, t2), tmax = fmax(t1, t2);
  t1 = mul_rn(sub_rn(bmin.y, p0.y), inv.y);
  t2 = mul_rn(sub_rn(bmax.y, p0.y), inv.y);
  tmin = fmax(tmin, fmin(t1, t2));
  tmax = fmin(tmax, fmax(t1, t2));
  t1 = mul_rn(sub_rn(bmin.z, p0.z), inv.z);
  t2 = mul_rn(sub_rn(bmax.z, p0.z), inv.z);
  tmin = fmax(tmin, fmin(t1, t2));
  tmax = fmin(tmax, fmax(t1, t2));
  if (tmax > fmax(tmin, 0.0)) {
    *hit = vadd(p0, vmul(dir, tmin));
    return true;
  }
  return false;
}

// _advectParticles steps a and b (:652-723) for particles [0, m), m = 6*(n/6)
// (the reference's six chunks of n/6 leave the rest untouched).
__global__ void advect_particles_kernel(PGrid G, const uint8_t* __restrict__ mat, const double* __restrict__ u,
                                        const double* __restrict__ v, const double* __restrict__ w,
                                        const double* __restrict__ us, const double* __restrict__ vs,
                                        const double* __restrict__ ws, double ratio, double dt, long long m,
                                        double* __restrict__ parts) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < m; q += (long long)gridDim.x * blockDim.x) {
    double* P = parts + 6 * q;
    const V3 cur = v3(P[0], P[1], P[2]);
    // a. FLIP/PIC blend (:667-678)
    const V3 vnew = get_velocity(u, v, w, G, cur);
    const V3 vold = get_velocity(us, vs, ws, G, cur);
    const V3 vflip = vsub(vadd(v3(P[3], P[4], P[5]), vnew), vold);
    const V3 vb = vadd(vmul(vnew, sub_rn(1.0, ratio)), vmul(vflip, ratio));
    P[3] = vb.x;
    P[4] = vb.y;
    P[5] = vb.z;
    // b. RK4 (:895-906)
    const double hdt = mul_rn(0.5, dt);
    const V3 k1 = get_velocity(u, v, w, G, cur);
    const V3 k2 = get_velocity(u, v, w, G, vadd(cur, vmul(k1, hdt)));
    const V3 k3 = get_velocity(u, v, w, G, vadd(cur, vmul(k2, hdt)));
    const V3 k4 = get_velocity(u, v, w, G, vadd(cur, vmul(k3, dt)));
    const V3 np = vadd(cur, vmul(vadd(vadd(vadd(k1, vmul(k2, 2.0)), vmul(k3, 2.0)), k4), div_rn(dt, 6.0)));
    int gi, gj, gk;
    pos2index(np, G.dx, &gi, &gj, &gk);
    if (in_grid(G, gi, gj, gk) && mat_at(mat, G, gi, gj, gk) != P_SOLID) {
      P[0] = np.x;
      P[1] = np.y;
      P[2] = np.z;
      continue;
    }
    // into a solid (:691-721)
    int vox[3];
    if (!segment_voxel(cur, np, G, mat, vox)) continue;
    const V3 d = vsub(np, cur);
    const double l = __dsqrt_rn(vdot(d, d));
    const V3 ray = v3(div_rn(d.x, l), div_rn(d.y, l), div_rn(d.z, l));
    const V3 bmin = v3(mul_rn(add_rn((double)vox[0], 0.5), G.dx), mul_rn(add_rn((double)vox[1], 0.5), G.dx),
                       mul_rn(add_rn((double)vox[2], 0.5), G.dx));
    const V3 bmax = vadd(bmin, v3(G.dx, G.dx, G.dx));
    V3 hit;
    if (!ray_aabb(cur, ray, bmin, bmax, &hit)) continue;
    const V3 res = vsub(hit, vmul(ray, (double)__double2float_rn(mul_rn(0.05, G.dx))));
    int ri, rj, rk;
    pos2index(res, G.dx, &ri, &rj, &rk);
    if (in_grid(G, ri, rj, rk) && mat_at(mat, G, ri, rj, rk) != P_SOLID) {
      P[0] = res.x;
      P[1] = res.y;
      P[2] = res.z;
    }
  }
}

// ---------------------------------------------------------------- binning
// Bounding box of a particle over an output grid (getBoundingGrid,
// xfluidutil.cpp:23-31, on the position shifted by `sh`): per axis the first
// and last covered index, cell units scaled to output units by `s`:
//   lo = gmin*s, hi = (gmax+1)*s - (s == 1 ? 1 : 0)
// (s == 1: the face transfer, lo..hi = gmin..gmax; s > 1: field vertices).
struct BoxSpec {
  double r;      // box half-width
  double sh[3];  // position shift (0.5 dx on the face axis for the transfer)
  int s;         // output units per cell
  int ext[3];    // output grid extents
};

__device__ __forceinline__ void particle_box(const double* P, const BoxSpec& B, double dx, int lo[3], int hi[3],
                                             V3* ps) {
  const V3 p = vadd(v3(P[0], P[1], P[2]), v3(B.sh[0], B.sh[1], B.sh[2]));
  *ps = p;
  int a0, a1, a2, b0, b1, b2;
  pos2index(vadd(v3(-B.r, -B.r, -B.r), p), dx, &a0, &a1, &a2);
  pos2index(vadd(p, v3(B.r, B.r, B.r)), dx, &b0, &b1, &b2);
  const int g0[3] = {a0, a1, a2}, g1[3] = {b0, b1, b2};
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    if (B.s == 1) {
      lo[q] = g0[q];
      hi[q] = g1[q];
    } else {
      lo[q] = (int)max(min((long long)g0[q] * B.s, (long long)INT_MAX / 2), (long long)INT_MIN / 2);
      hi[q] = (int)max(min(((long long)g1[q] + 1) * B.s, (long long)INT_MAX / 2), (long long)INT_MIN / 2);
    }
  }
}

// Key = bin of the box's low corner (clamped at 0, in cells), or nbins for
// a box that covers no output; the widest box (in bins) goes to maxspan[q].
__global__ void box_key_kernel(const double* __restrict__ parts, long long n, BoxSpec B, double dx, int nb0, int nb1,
                               int nb2, long long nbins, unsigned* __restrict__ key, int* __restrict__ idx, int* __restrict__ box,
                               double* __restrict__ pos, int* __restrict__ maxspan) {
  int span[3] = {0, 0, 0};
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    int lo[3], hi[3];
    V3 p;
    particle_box(parts + 6 * q, B, dx, lo, hi, &p);
    bool hits = true;
    int bc[3];
    const int nb[3] = {nb0, nb1, nb2};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      hits = hits && hi[a] >= 0 && lo[a] <= B.ext[a] - 1;
      // bin = cell of the low corner; for vertices lo = gmin*s, so lo / s
      bc[a] = min(max(lo[a], 0) / B.s, nb[a] - 1);
    }
    key[q] = hits ? (unsigned)(((long long)bc[2] * nb1 + bc[1]) * nb0 + bc[0]) : (unsigned)nbins;
    idx[q] = (int)q;
    if (hits) {
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        // bins an output at index t must scan: [floor(t/s) - span, floor(t/s)]
        const int sp = (min(hi[a], B.ext[a] - 1) / B.s) - bc[a];
        span[a] = max(span[a], sp);
      }
    }
    int* bx = box + 6 * q;
    bx[0] = lo[0]; bx[1] = hi[0]; bx[2] = lo[1]; bx[3] = hi[1]; bx[4] = lo[2]; bx[5] = hi[2];
    pos[3 * q] = p.x;
    pos[3 * q + 1] = p.y;
    pos[3 * q + 2] = p.z;
  }
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    int s = span[a];
    for (int o = 16; o > 0; o >>= 1) s = max(s, __shfl_xor_sync(0xffffffffu, s, o));
    if ((threadIdx.x & 31) == 0) atomicMax(&maxspan[a], s);
  }
}

__global__ void bin_count_kernel(const unsigned* __restrict__ key, long long n, long long nbins,
                                 int* __restrict__ count) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    if ((long long)key[q] < nbins) atomicAdd(&count[key[q]], 1);
}

// sorted copies: box, shifted position and the carried value (velocity
// component for the transfer, unused for the field)
__global__ void bin_gather_kernel(const int* __restrict__ sidx, long long n, const int* __restrict__ box,
                                  const double* __restrict__ pos, const double* __restrict__ parts, int vcomp,
                                  int4* __restrict__ sbox_xy, int2* __restrict__ sbox_z,
                                  double2* __restrict__ spos) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int o = sidx[q];
    const int* b = box + 6 * (size_t)o;
    sbox_xy[q] = make_int4(b[0], b[1], b[2], b[3]);
    sbox_z[q] = make_int2(b[4], b[5]);
    spos[2 * q] = make_double2(pos[3 * (size_t)o], pos[3 * (size_t)o + 1]);
    spos[2 * q + 1] = make_double2(pos[3 * (size_t)o + 2], vcomp >= 0 ? parts[6 * (size_t)o + 3 + vcomp] : 0.0);
  }
}

// weight polynomial (FluidSimulator.cpp:918-931, directeddistancefield.cpp:245-255)
struct Poly {
  double r2, c0, c1, c2;
};
__device__ __forceinline__ double poly_w(const Poly& W, double rs) {
  if (!(rs < W.r2)) return 0.0;
  const double a = mul_rn(mul_rn(mul_rn(W.c0, rs), rs), rs);
  const double b = mul_rn(mul_rn(W.c1, rs), rs);
  return sub_rn(add_rn(sub_rn(1.0, a), b), mul_rn(W.c2, rs));
}

// One output per thread: sum of the covering particles' weights (and
// weighted values) over the bins [t/s - span, t/s] per axis, rows of bins
// contiguous along x.  Transfer: out = value/weight where weight > 1e-7, else 0
// (:1010-1027).  Field: out = weight sum.
template <bool FIELD>
__global__ void gather_kernel(int e0, int e1, int e2, int s, double unit, int nb0, int nb1, int nb2, int sp0, int sp1,
                              int sp2, const int* __restrict__ start, const int4* __restrict__ sbox_xy,
                              const int2* __restrict__ sbox_z, const double2* __restrict__ spos, Poly W,
                              double* __restrict__ out) {
  const long long total = (long long)e0 * e1 * e2;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % e0), j = (int)((t / e0) % e1), k = (int)(t / ((long long)e0 * e1));
    // output position: idx2Pos (xfluidutil.cpp:13-16) at this grid's spacing
    const V3 g = v3(mul_rn(add_rn((double)i, 0.5), unit), mul_rn(add_rn((double)j, 0.5), unit),
                    mul_rn(add_rn((double)k, 0.5), unit));
    const int bi = min(i / s, nb0 - 1), bj = min(j / s, nb1 - 1), bk = min(k / s, nb2 - 1);
    const int i0 = max(bi - sp0, 0), j0 = max(bj - sp1, 0), k0 = max(bk - sp2, 0);
    double wsum = 0.0, vsum = 0.0;
    for (int ck = k0; ck <= bk; ++ck)
      for (int cj = j0; cj <= bj; ++cj) {
        const long long row = ((long long)ck * nb1 + cj) * nb0;
        const int qa = __ldg(&start[row + i0]), qb = __ldg(&start[row + bi + 1]);
        for (int q = qa; q < qb; ++q) {
          const int4 bxy = __ldg(&sbox_xy[q]);
          const int2 bz = __ldg(&sbox_z[q]);
          if (i < bxy.x || i > bxy.y || j < bxy.z || j > bxy.w || k < bz.x || k > bz.y) continue;
          const double2 pxy = __ldg(&spos[2 * (size_t)q]), pzv = __ldg(&spos[2 * (size_t)q + 1]);
          const V3 p = v3(pxy.x, pxy.y, pzv.x);
          // transfer: curR = p - idx2Pos (:960); field: gp - p (:296)
          const V3 d = FIELD ? vsub(g, p) : vsub(p, g);
          const double cw = poly_w(W, vdot(d, d));
          wsum = add_rn(wsum, cw);
          if (!FIELD) vsum = add_rn(vsum, mul_rn(pzv.y, cw));
        }
      }
    if (FIELD) out[t] = wsum;
    else out[t] = wsum > 0.0000001 ? div_rn(vsum, wsum) : 0.0;
  }
}

// _updateMaterial (:402-427)
__global__ void material_reset_kernel(uint8_t* __restrict__ mat, long long nc) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < nc; c += (long long)gridDim.x * blockDim.x)
    if (mat[c] != P_SOLID) mat[c] = P_AIR;
}
__global__ void material_mark_kernel(PGrid G, const double* __restrict__ parts, long long n, uint8_t* __restrict__ mat) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    pos2index(v3(parts[6 * q], parts[6 * q + 1], parts[6 * q + 2]), G.dx, &i, &j, &k);
    if (in_grid(G, i, j, k)) {
      uint8_t* c = &mat[(size_t)k * G.ni * G.nj + (size_t)j * G.ni + i];
      if (*c != P_SOLID) *c = P_FLUID;   // every writer stores the same value
    }
  }
}

// updateSurfaceInfo's material part (directeddistancefield.cpp:167-215) with
// _isCellSurface (:304-327) and _centerPhi (:329-344)
__global__ void classify_kernel(PGrid G, int s, double thr, const double* __restrict__ phi, uint8_t* __restrict__ mat) {
  const int pi = G.ni * s + 1, pj = G.nj * s + 1;
  const long long nc = (long long)G.ni * G.nj * G.nk;
  auto PHI = [&](int a, int b, int c) { return __ldg(&phi[(size_t)c * pi * pj + (size_t)b * pi + a]); };
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < nc; c += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(c % G.ni), j = (int)((c / G.ni) % G.nj), k = (int)(c / ((long long)G.ni * G.nj));
    if (mat[c] == P_SOLID) continue;
    const int si = i * s, sj = j * s, sk = k * s;
    bool in = false, out = false;
    for (int a = si; a <= si + s; ++a)
      for (int b = sj; b <= sj + s; ++b)
        for (int cc = sk; cc <= sk + s; ++cc) {
          if (PHI(a, b, cc) >= thr) in = true;
          else out = true;
        }
    double val;
    if (in && out) {
      if (s % 2 == 0) {
        val = PHI(si + s / 2, sj + s / 2, sk + s / 2);
      } else {
        val = 0.0;
        for (int a = si; a <= si + s; a += s)
          for (int b = sj; b <= sj + s; b += s)
            for (int cc = sk; cc <= sk + s; cc += s) val = add_rn(val, PHI(a, b, cc));
        val = div_rn(val, 8.0);
      }
    } else {
      val = PHI(si, sj, sk);
    }
    mat[c] = val >= thr ? P_FLUID : P_AIR;
  }
}

unsigned pgrid(long long n) { return (unsigned)std::max<long long>(1, std::min<long long>((n + 255) / 256, 148LL * 16)); }

}  // namespace
}  // namespace xfp

namespace xfp_host {
using namespace xfp;

namespace {

constexpr long long kMaxParticles = 1LL << 31;

int check_particle_args(xfp_ctx* ctx, int ni, int nj, int nk, double dx, long long n, const void* parts) {
  if (!ctx) return XFP_ERR_ARGS;
  if (ni < 2 || nj < 2 || nk < 2) return fail(ctx, XFP_ERR_ARGS, "grid must be at least 2 cells on every axis");
  if ((long long)ni * nj * nk >= (1LL << 31) / 8)
    return fail(ctx, XFP_ERR_ARGS, "grid too large for the particle steps");
  if (!(dx > 0.0) || !std::isfinite(dx)) return fail(ctx, XFP_ERR_ARGS, "dx must be positive and finite");
  if (n < 0 || n >= kMaxParticles) return fail(ctx, XFP_ERR_ARGS, "particle count out of range");
  if (n > 0 && !parts) return fail(ctx, XFP_ERR_ARGS, "particles are NULL");
  return XFP_OK;
}

// Bins the particles by their box over an output grid and gathers every
// output (see the file comment).  `out` is on the device.
template <bool FIELD>
int bin_and_gather(xfp_ctx* ctx, const double* dparts, long long n, const BoxSpec& B, double dx, double unit,
                   int vcomp, const Poly& W, double* out) {
  cudaStream_t st = ctx->stream;
  const int nb0 = (B.ext[0] + B.s - 1) / B.s, nb1 = (B.ext[1] + B.s - 1) / B.s, nb2 = (B.ext[2] + B.s - 1) / B.s;
  const long long nbins = (long long)nb0 * nb1 * nb2;
  const long long total = (long long)B.ext[0] * B.ext[1] * B.ext[2];
  const size_t nn = (size_t)std::max<long long>(n, 1);
  XFP_CUDA(ctx, ctx->part_key.ensure(nn * 2 * sizeof(unsigned)));
  XFP_CUDA(ctx, ctx->part_idx.ensure(nn * 2 * sizeof(int)));
  XFP_CUDA(ctx, ctx->part_box.ensure(nn * 6 * sizeof(int)));
  XFP_CUDA(ctx, ctx->part_pos.ensure(nn * 3 * sizeof(double)));
  XFP_CUDA(ctx, ctx->part_sbox.ensure(nn * (sizeof(int4) + sizeof(int2))));
  XFP_CUDA(ctx, ctx->part_spos.ensure(nn * 2 * sizeof(double2)));
  XFP_CUDA(ctx, ctx->part_start.ensure((size_t)(nbins + 2) * sizeof(int) * 2 + 16));
  unsigned* key = ctx->part_key.as<unsigned>();
  unsigned* key2 = key + nn;
  int* idx = ctx->part_idx.as<int>();
  int* idx2 = idx + nn;
  int* box = ctx->part_box.as<int>();
  double* pos = ctx->part_pos.as<double>();
  // sorted copies for the gather: box as int4 (x, y) + int2 (z), position and
  // carried value as two double2 -- four vector loads per candidate
  int4* sbox_xy = ctx->part_sbox.as<int4>();
  int2* sbox_z = reinterpret_cast<int2*>(sbox_xy + nn);
  double2* spos = ctx->part_spos.as<double2>();
  int* count = ctx->part_start.as<int>();
  int* start = count + (nbins + 2);
  XFP_CUDA(ctx, ctx->part_span.ensure(4 * sizeof(int)));
  int* dspan = ctx->part_span.as<int>();
  // counts and starts zeroed (with no particles the starts stay zero)
  XFP_CUDA(ctx, cudaMemsetAsync(count, 0, (size_t)(nbins + 2) * 2 * sizeof(int), st));
  XFP_CUDA(ctx, cudaMemsetAsync(dspan, 0, 4 * sizeof(int), st));
  if (n > 0) {
    ++g_kernel_launches;
    box_key_kernel<<<pgrid(n), 256, 0, st>>>(dparts, n, B, dx, nb0, nb1, nb2, nbins, key, idx, box, pos,
                                               dspan);
    XFP_CUDA(ctx, cudaGetLastError());
    // stable sort by bin (keys < nbins, no-cover key = nbins): a bin's
    // particles stay in index order
    int end_bit = 1;
    while (end_bit < 32 && (1LL << end_bit) <= nbins) ++end_bit;
    size_t tmp = 0, tmp2 = 0;
    XFP_CUDA(ctx, cub::DeviceRadixSort::SortPairs(nullptr, tmp, key, key2, idx, idx2, (int)n, 0, end_bit, st));
    XFP_CUDA(ctx, cub::DeviceScan::ExclusiveSum(nullptr, tmp2, count, start, (int)(nbins + 1), st));
    XFP_CUDA(ctx, ctx->part_tmp.ensure(std::max(tmp, tmp2)));
    tmp = ctx->part_tmp.cap;
    XFP_CUDA(ctx, cub::DeviceRadixSort::SortPairs(ctx->part_tmp.p, tmp, key, key2, idx, idx2, (int)n, 0, end_bit,
                                                  st));
    g_kernel_launches += 4;
    ++g_kernel_launches;
    bin_count_kernel<<<pgrid(n), 256, 0, st>>>(key, n, nbins, count);
    XFP_CUDA(ctx, cudaGetLastError());
    tmp2 = ctx->part_tmp.cap;
    XFP_CUDA(ctx, cub::DeviceScan::ExclusiveSum(ctx->part_tmp.p, tmp2, count, start, (int)(nbins + 1), st));
    g_kernel_launches += 2;
    ++g_kernel_launches;
    bin_gather_kernel<<<pgrid(n), 256, 0, st>>>(idx2, n, box, pos, dparts, vcomp, sbox_xy, sbox_z, spos);
    XFP_CUDA(ctx, cudaGetLastError());
  }
  int span[4] = {0, 0, 0, 0};
  XFP_CUDA(ctx, cudaMemcpyAsync(span, dspan, 4 * sizeof(int), cudaMemcpyDeviceToHost, st));
  XFP_CUDA(ctx, cudaStreamSynchronize(st));
  ++g_kernel_launches;
  gather_kernel<FIELD><<<pgrid(total), 256, 0, st>>>(B.ext[0], B.ext[1], B.ext[2], B.s, unit, nb0, nb1, nb2, span[0],
                                                     span[1], span[2], start, sbox_xy, sbox_z, spos, W, out);
  XFP_CUDA(ctx, cudaGetLastError());
  return XFP_OK;
}

Poly make_poly(double r) {
  const double r2 = r * r;
  Poly W;
  W.r2 = r2;
  W.c0 = (4.0 / 9.0) * (1.0 / (r2 * r2 * r2));
  W.c1 = (17.0 / 9.0) * (1.0 / (r2 * r2));
  W.c2 = (22.0 / 9.0) * (1.0 / (r2));
  return W;
}

// stage the particles (host mode) or use them in place
int stage_particles(xfp_ctx* ctx, const xfp_particle* parts, long long n, const double** dev) {
  return stage_in<double>(ctx, ctx->part_io, reinterpret_cast<const double*>(parts), (size_t)n * 6, dev);
}

}  // namespace

int advect_particles_impl(xfp_ctx* ctx, int ni, int nj, int nk, double dx, const uint8_t* mat, const double* u,
                          const double* v, const double* w, const double* us, const double* vs, const double* ws,
                          double ratio, double dt, long long n, xfp_particle* parts) {
  int rc = check_particle_args(ctx, ni, nj, nk, dx, n, parts);
  if (rc) return rc;
  if (!mat || !u || !v || !w || !us || !vs || !ws) return fail(ctx, XFP_ERR_ARGS, "NULL array");
  if (!std::isfinite(dt) || !std::isfinite(ratio)) return fail(ctx, XFP_ERR_ARGS, "dt and ratio must be finite");
  XFP_CUDA(ctx, cudaSetDevice(ctx->device));
  const uint8_t* dmat;
  const double *du_, *dv, *dw, *dus, *dvs, *dws, *dp;
  if ((rc = stage_in(ctx, ctx->io_mat, mat, ncells(ni, nj, nk), &dmat))) return rc;
  if ((rc = stage_in<double>(ctx, ctx->io_u, u, nu(ni, nj, nk), &du_))) return rc;
  if ((rc = stage_in<double>(ctx, ctx->io_v, v, nv(ni, nj, nk), &dv))) return rc;
  if ((rc = stage_in<double>(ctx, ctx->io_w, w, nw_(ni, nj, nk), &dw))) return rc;
  if ((rc = stage_in<double>(ctx, ctx->io_gu, us, nu(ni, nj, nk), &dus))) return rc;
  if ((rc = stage_in<double>(ctx, ctx->io_gv, vs, nv(ni, nj, nk), &dvs))) return rc;
  if ((rc = stage_in<double>(ctx, ctx->io_gw, ws, nw_(ni, nj, nk), &dws))) return rc;
  if ((rc = stage_particles(ctx, parts, n, &dp))) return rc;
  const long long m = (n / 6) * 6;
  if (m > 0) {
    ++g_kernel_launches;
    advect_particles_kernel<<<pgrid(m), 128, 0, ctx->stream>>>(PGrid{ni, nj, nk, dx}, dmat, du_, dv, dw, dus, dvs,
                                                               dws, ratio, dt, m, const_cast<double*>(dp));
    XFP_CUDA(ctx, cudaGetLastError());
  }
  if (!ctx->opt.device_pointers && n > 0)
    XFP_CUDA(ctx, cudaMemcpyAsync(parts, dp, (size_t)n * 6 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  XFP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return XFP_OK;
}

int particles_to_grid_impl(xfp_ctx* ctx, int ni, int nj, int nk, double dx, long long n, const xfp_particle* parts,
                           double* u, double* v, double* w) {
  int rc = check_particle_args(ctx, ni, nj, nk, dx, n, parts);
  if (rc) return rc;
  if (!u || !v || !w) return fail(ctx, XFP_ERR_ARGS, "NULL array");
  XFP_CUDA(ctx, cudaSetDevice(ctx->device));
  const double* dp;
  if ((rc = stage_particles(ctx, parts, n, &dp))) return rc;
  double* out[3] = {u, v, w};
  DevBuf* io[3] = {&ctx->io_u, &ctx->io_v, &ctx->io_w};
  const Poly W = make_poly(1.5 * dx);
  for (int a = 0; a < 3; ++a) {
    BoxSpec B;
    B.r = 1.5 * dx;
    for (int q = 0; q < 3; ++q) B.sh[q] = q == a ? 0.5 * dx : 0.0;
    B.s = 1;
    B.ext[0] = ni + (a == 0);
    B.ext[1] = nj + (a == 1);
    B.ext[2] = nk + (a == 2);
    const size_t nf = (size_t)B.ext[0] * B.ext[1] * B.ext[2];
    double* dout = out[a];
    if (!ctx->opt.device_pointers) {
      XFP_CUDA(ctx, io[a]->ensure(nf * sizeof(double)));
      dout = io[a]->as<double>();
    }
    if ((rc = bin_and_gather<false>(ctx, dp, n, B, dx, dx, a, W, dout))) return rc;
    if (!ctx->opt.device_pointers)
      XFP_CUDA(ctx, cudaMemcpyAsync(out[a], dout, nf * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  }
  XFP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return XFP_OK;
}

int update_material_impl(xfp_ctx* ctx, int ni, int nj, int nk, double dx, long long n, const xfp_particle* parts,
                         uint8_t* mat) {
  int rc = check_particle_args(ctx, ni, nj, nk, dx, n, parts);
  if (rc) return rc;
  if (!mat) return fail(ctx, XFP_ERR_ARGS, "material is NULL");
  XFP_CUDA(ctx, cudaSetDevice(ctx->device));
  const double* dp;
  const uint8_t* dmat;
  if ((rc = stage_in(ctx, ctx->io_mat, mat, ncells(ni, nj, nk), &dmat))) return rc;
  if ((rc = stage_particles(ctx, parts, n, &dp))) return rc;
  uint8_t* m = const_cast<uint8_t*>(dmat);
  const long long nc = (long long)ni * nj * nk;
  ++g_kernel_launches;
  material_reset_kernel<<<pgrid(nc), 256, 0, ctx->stream>>>(m, nc);
  if (n > 0) {
    ++g_kernel_launches;
    material_mark_kernel<<<pgrid(n), 256, 0, ctx->stream>>>(PGrid{ni, nj, nk, dx}, dp, n, m);
  }
  XFP_CUDA(ctx, cudaGetLastError());
  if (!ctx->opt.device_pointers)
    XFP_CUDA(ctx, cudaMemcpyAsync(mat, m, (size_t)nc, cudaMemcpyDeviceToHost, ctx->stream));
  XFP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return XFP_OK;
}

int distance_field_impl(xfp_ctx* ctx, int ni, int nj, int nk, double dx, int subdiv, double radius, double threshold,
                        long long n, const xfp_particle* parts, double* phi, uint8_t* mat) {
  int rc = check_particle_args(ctx, ni, nj, nk, dx, n, parts);
  if (rc) return rc;
  if (subdiv < 1 || subdiv > 8) return fail(ctx, XFP_ERR_ARGS, "subdivision level must be in [1, 8]");
  if (!(radius > 0.0) || !std::isfinite(radius) || radius > 64.0 * dx)
    return fail(ctx, XFP_ERR_ARGS, "radius must be in (0, 64 dx]");
  if (!std::isfinite(threshold)) return fail(ctx, XFP_ERR_ARGS, "threshold must be finite");
  if (!phi && !mat) return fail(ctx, XFP_ERR_ARGS, "phi and material are both NULL");
  const long long pts = ((long long)ni * subdiv + 1) * ((long long)nj * subdiv + 1) * ((long long)nk * subdiv + 1);
  if (pts >= (1LL << 31)) return fail(ctx, XFP_ERR_ARGS, "subdivided grid too large");
  XFP_CUDA(ctx, cudaSetDevice(ctx->device));
  const double* dp;
  if ((rc = stage_particles(ctx, parts, n, &dp))) return rc;
  double* dphi = phi;
  if (!ctx->opt.device_pointers || !phi) {
    XFP_CUDA(ctx, ctx->phi_io.ensure((size_t)pts * sizeof(double)));
    dphi = ctx->phi_io.as<double>();
  }
  BoxSpec B;
  B.r = radius;
  B.sh[0] = B.sh[1] = B.sh[2] = 0.0;
  B.s = subdiv;
  B.ext[0] = ni * subdiv + 1;
  B.ext[1] = nj * subdiv + 1;
  B.ext[2] = nk * subdiv + 1;
  if ((rc = bin_and_gather<true>(ctx, dp, n, B, dx, dx / (double)subdiv, -1, make_poly(radius), dphi))) return rc;
  if (mat) {
    const uint8_t* dmat;
    if ((rc = stage_in(ctx, ctx->io_mat, mat, ncells(ni, nj, nk), &dmat))) return rc;
    const long long nc = (long long)ni * nj * nk;
    ++g_kernel_launches;
    classify_kernel<<<pgrid(nc), 256, 0, ctx->stream>>>(PGrid{ni, nj, nk, dx}, subdiv, threshold, dphi,
                                                        const_cast<uint8_t*>(dmat));
    XFP_CUDA(ctx, cudaGetLastError());
    if (!ctx->opt.device_pointers)
      XFP_CUDA(ctx, cudaMemcpyAsync(mat, dmat, (size_t)nc, cudaMemcpyDeviceToHost, ctx->stream));
  }
  if (phi && dphi != phi)
    XFP_CUDA(ctx, cudaMemcpyAsync(phi, dphi, (size_t)pts * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  XFP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return XFP_OK;
}

// FluidSimulator::_maxVelocity (FluidSimulator.cpp:387-400): the largest
// v.v over the particles, v.v formed as x*x + y*y + z*z left to right with
// every product and sum rounded (Vec3::operator*, array3d.h:33-36), then its
// square root.  The max is exact in any order: each block's maximum goes to
// one 64-bit word by atomicMax on the bit pattern (non-negative doubles order
// like their bits); NaN speeds propagate as the largest pattern.
__global__ void max_speed_kernel(const double* __restrict__ p, long long n, unsigned long long* __restrict__ out) {
  unsigned long long m = 0ull;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const double vx = p[6 * q + 3], vy = p[6 * q + 4], vz = p[6 * q + 5];
    const double vv = __dadd_rn(__dadd_rn(__dmul_rn(vx, vx), __dmul_rn(vy, vy)), __dmul_rn(vz, vz));
    const unsigned long long b = (unsigned long long)__double_as_longlong(vv);
    m = b > m ? b : m;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long t = __shfl_xor_sync(0xffffffffu, m, o);
    m = t > m ? t : m;
  }
  if ((threadIdx.x & 31) == 0 && m != 0ull) atomicMax(out, m);
}

int max_speed_impl(xfp_ctx* ctx, long long n, const xfp_particle* parts, double* max_speed) {
  if (!ctx) return XFP_ERR_ARGS;
  if (!max_speed) return fail(ctx, XFP_ERR_ARGS, "max_speed is NULL");
  if (n < 0 || (n > 0 && !parts)) return fail(ctx, XFP_ERR_ARGS, "bad particle arguments");
  XFP_CUDA(ctx, cudaSetDevice(ctx->device));
  *max_speed = 0.0;
  if (n == 0) return XFP_OK;
  const double* dp;
  int rc;
  if ((rc = stage_particles(ctx, parts, n, &dp))) return rc;
  XFP_CUDA(ctx, ctx->part_tmp.ensure(std::max<size_t>(ctx->part_tmp.cap, 64)));
  unsigned long long* word = reinterpret_cast<unsigned long long*>(ctx->part_tmp.p);
  XFP_CUDA(ctx, cudaMemsetAsync(word, 0, sizeof(unsigned long long), ctx->stream));
  ++g_kernel_launches;
  max_speed_kernel<<<pgrid(n), 256, 0, ctx->stream>>>(dp, n, word);
  XFP_CUDA(ctx, cudaGetLastError());
  unsigned long long h = 0ull;
  XFP_CUDA(ctx, cudaMemcpyAsync(&h, word, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
  XFP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  double vv;
  std::memcpy(&vv, &h, sizeof(vv));
  *max_speed = std::sqrt(vv);
  return XFP_OK;
}

}  // namespace xfp_host

using namespace xfp_host;

extern "C" {

int xfp_advect_particles_f64(xfp_ctx* ctx, int ni, int nj, int nk, double dx, const uint8_t* material, const double* u,
                             const double* v, const double* w, const double* u_saved, const double* v_saved,
                             const double* w_saved, double ratio_flip, double dt, long long n,
                             xfp_particle* particles) {
  return advect_particles_impl(ctx, ni, nj, nk, dx, material, u, v, w, u_saved, v_saved, w_saved, ratio_flip, dt, n,
                               particles);
}

int xfp_particles_to_grid_f64(xfp_ctx* ctx, int ni, int nj, int nk, double dx, long long n,
                              const xfp_particle* particles, double* u, double* v, double* w) {
  return particles_to_grid_impl(ctx, ni, nj, nk, dx, n, particles, u, v, w);
}

int xfp_max_speed_f64(xfp_ctx* ctx, long long n, const xfp_particle* particles, double* max_speed) {
  return max_speed_impl(ctx, n, particles, max_speed);
}

int xfp_update_material(xfp_ctx* ctx, int ni, int nj, int nk, double dx, long long n, const xfp_particle* particles,
                        uint8_t* material) {
  return update_material_impl(ctx, ni, nj, nk, dx, n, particles, material);
}

int xfp_distance_field_f64(xfp_ctx* ctx, int ni, int nj, int nk, double dx, int subdiv, double radius,
                           double threshold, long long n, const xfp_particle* particles, double* phi,
                           uint8_t* material) {
  return distance_field_impl(ctx, ni, nj, nk, dx, subdiv, radius, threshold, n, particles, phi, material);
}

}  // extern "C"
