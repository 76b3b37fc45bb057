// xfp_advect.cu -- semi-Lagrangian self-advection of the MAC velocity and its
// exact adjoint, for differentiable rollouts (advect -> project, repeated).
//
// xFluid moves velocity with particles (FluidSimulator.cpp:652-1085); these
// kernels are this library's own differentiable step, defined as follows
// (positions in cell units, cell (i,j,k) centred at (i+.5, j+.5, k+.5)):
//   faces    u(i,j,k) at (i, j+.5, k+.5), v at (i+.5, j, k+.5), w at (i+.5, j+.5, k)
//   sample   G(p): trilinear in G's node lattice, each lattice coordinate
//            clamped to [0, n-1] (derivative 0 where clamped)
//   velocity vel(x) = (u(x), v(x), w(x)) sampled at a face position x
//   advect   out_G[f] = G(x_f - c * vel(x_f)),  c = dt / dx
// The adjoint is the transpose of the Jacobian of that map, with both terms:
// the interpolation weights at the departure point, and the dependence of the
// departure point on vel(x_f) through the sampled gradient of G.  Adjoint
// contributions are scattered with FP64 (or FP32) atomics.
#include <cmath>

#include "xfp_common.cuh"
#include "xfp_context.h"
#include "xfp_kernels.h"

namespace xfp {
namespace {

// Component lattice: node (a,b,c) at (a+ox, b+oy, c+oz), extents (na,nb,nc).
struct Lat {
  int na, nb, nc;
  float ox, oy, oz;
};
__device__ __forceinline__ Lat lat_of(int comp, int ni, int nj, int nk) {
  if (comp == 0) return {ni + 1, nj, nk, 0.f, .5f, .5f};
  if (comp == 1) return {ni, nj + 1, nk, .5f, 0.f, .5f};
  return {ni, nj, nk + 1, .5f, .5f, 0.f};
}

// One axis of the clamped linear stencil: lower node, weight of the upper
// node, and whether the coordinate was inside (derivative defined).
template <typename T>
__device__ __forceinline__ void axis(T x, float o, int n, int& a0, int& a1, T& t, bool& inside) {
  T f = x - (T)o;
  inside = f > T(0) && f < (T)(n - 1);
  f = f < T(0) ? T(0) : (f > (T)(n - 1) ? (T)(n - 1) : f);
  int a = (int)floor((double)f);
  if (a > n - 2) a = n - 2;
  if (a < 0) a = 0;
  a0 = a;
  a1 = n > 1 ? a + 1 : a;
  t = n > 1 ? f - (T)a : T(0);
}

template <typename T>
struct Stencil {
  size_t idx[8];
  T w[8];
  T dw[3][8];   // d weight / d position (x, y, z); 0 on a clamped axis
};

template <typename T>
__device__ __forceinline__ void stencil(const Lat& L, T x, T y, T z, Stencil<T>& s) {
  int a0, a1, b0, b1, c0, c1;
  T ta, tb, tc;
  bool ia, ib, ic;
  axis(x, L.ox, L.na, a0, a1, ta, ia);
  axis(y, L.oy, L.nb, b0, b1, tb, ib);
  axis(z, L.oz, L.nc, c0, c1, tc, ic);
  const T wa[2] = {T(1) - ta, ta}, wb[2] = {T(1) - tb, tb}, wc[2] = {T(1) - tc, tc};
  const T da[2] = {ia ? T(-1) : T(0), ia ? T(1) : T(0)};
  const T db[2] = {ib ? T(-1) : T(0), ib ? T(1) : T(0)};
  const T dc[2] = {ic ? T(-1) : T(0), ic ? T(1) : T(0)};
  const int A[2] = {a0, a1}, B[2] = {b0, b1}, Cc[2] = {c0, c1};
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const int qa = q & 1, qb = (q >> 1) & 1, qc = q >> 2;
    s.idx[q] = ((size_t)Cc[qc] * L.nb + B[qb]) * L.na + A[qa];
    s.w[q] = wa[qa] * wb[qb] * wc[qc];
    s.dw[0][q] = da[qa] * wb[qb] * wc[qc];
    s.dw[1][q] = wa[qa] * db[qb] * wc[qc];
    s.dw[2][q] = wa[qa] * wb[qb] * dc[qc];
  }
}

template <typename T>
__device__ __forceinline__ T gather(const T* __restrict__ G, const Stencil<T>& s) {
  T v = T(0);
#pragma unroll
  for (int q = 0; q < 8; ++q) v += s.w[q] * G[s.idx[q]];
  return v;
}

// Face f of component comp: its lattice coordinates and position.
__device__ __forceinline__ bool face_of(long long f, int ni, int nj, int nk, int& comp, float& x, float& y,
                                        float& z, long long& local) {
  const long long nu = (long long)(ni + 1) * nj * nk, nv = (long long)ni * (nj + 1) * nk,
                  nw = (long long)ni * nj * (nk + 1);
  if (f < nu) comp = 0, local = f;
  else if (f < nu + nv) comp = 1, local = f - nu;
  else if (f < nu + nv + nw) comp = 2, local = f - nu - nv;
  else return false;
  const Lat L = lat_of(comp, ni, nj, nk);
  const int a = (int)(local % L.na);
  const long long bc = local / L.na;
  const int b = (int)(bc % L.nb), c = (int)(bc / L.nb);
  x = a + L.ox; y = b + L.oy; z = c + L.oz;
  return true;
}

template <typename T>
__global__ void advect_kernel(const T* __restrict__ u, const T* __restrict__ v, const T* __restrict__ w,
                              T* __restrict__ ou, T* __restrict__ ov, T* __restrict__ ow, int ni, int nj, int nk,
                              T c) {
  const long long total = (long long)(ni + 1) * nj * nk + (long long)ni * (nj + 1) * nk + (long long)ni * nj * (nk + 1);
  const T* G[3] = {u, v, w};
  T* O[3] = {ou, ov, ow};
  for (long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x; f < total;
       f += (long long)gridDim.x * blockDim.x) {
    int comp;
    float xf, yf, zf;
    long long local;
    face_of(f, ni, nj, nk, comp, xf, yf, zf, local);
    const T x = xf, y = yf, z = zf;
    T vel[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      Stencil<T> s;
      stencil(lat_of(d, ni, nj, nk), x, y, z, s);
      vel[d] = gather(G[d], s);
    }
    Stencil<T> s;
    stencil(lat_of(comp, ni, nj, nk), x - c * vel[0], y - c * vel[1], z - c * vel[2], s);
    O[comp][local] = gather(G[comp], s);
  }
}

template <typename T>
__global__ void advect_adjoint_kernel(const T* __restrict__ u, const T* __restrict__ v, const T* __restrict__ w,
                                      const T* __restrict__ gu, const T* __restrict__ gv, const T* __restrict__ gw,
                                      T* __restrict__ du, T* __restrict__ dv, T* __restrict__ dw, int ni, int nj,
                                      int nk, T c) {
  const long long total = (long long)(ni + 1) * nj * nk + (long long)ni * (nj + 1) * nk + (long long)ni * nj * (nk + 1);
  const T* G[3] = {u, v, w};
  const T* Gb[3] = {gu, gv, gw};
  T* D[3] = {du, dv, dw};
  for (long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x; f < total;
       f += (long long)gridDim.x * blockDim.x) {
    int comp;
    float xf, yf, zf;
    long long local;
    face_of(f, ni, nj, nk, comp, xf, yf, zf, local);
    const T g = Gb[comp][local];
    if (g == T(0)) continue;
    const T x = xf, y = yf, z = zf;
    Stencil<T> sv[3];
    T vel[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      stencil(lat_of(d, ni, nj, nk), x, y, z, sv[d]);
      vel[d] = gather(G[d], sv[d]);
    }
    Stencil<T> s;
    stencil(lat_of(comp, ni, nj, nk), x - c * vel[0], y - c * vel[1], z - c * vel[2], s);
    // interpolation weights at the departure point
    T grad[3] = {T(0), T(0), T(0)};
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      atomicAdd(&D[comp][s.idx[q]], s.w[q] * g);
      const T gv_ = G[comp][s.idx[q]];
      grad[0] += s.dw[0][q] * gv_;
      grad[1] += s.dw[1][q] * gv_;
      grad[2] += s.dw[2][q] * gv_;
    }
    // departure point p = x - c vel(x): d out / d vel_d = -c * dG/dp_d
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const T pv = -c * grad[d] * g;
      if (pv == T(0)) continue;
#pragma unroll
      for (int q = 0; q < 8; ++q)
        if (sv[d].w[q] != T(0)) atomicAdd(&D[d][sv[d].idx[q]], sv[d].w[q] * pv);
    }
  }
}

// Loss = sum of squared face velocities whose (unit-cube) position lies in
// the box; grad = 2 * value there, 0 elsewhere.  loss accumulates atomically.
template <typename T>
__global__ void box_loss_kernel(const T* __restrict__ u, const T* __restrict__ v, const T* __restrict__ w,
                                T* __restrict__ gu, T* __restrict__ gv, T* __restrict__ gw, int ni, int nj, int nk,
                                double x0, double x1, double y0, double y1, double z0, double z1,
                                double* __restrict__ loss) {
  const long long total = (long long)(ni + 1) * nj * nk + (long long)ni * (nj + 1) * nk + (long long)ni * nj * (nk + 1);
  const T* G[3] = {u, v, w};
  T* D[3] = {gu, gv, gw};
  double acc = 0.0;
  for (long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x; f < total;
       f += (long long)gridDim.x * blockDim.x) {
    int comp;
    float xf, yf, zf;
    long long local;
    face_of(f, ni, nj, nk, comp, xf, yf, zf, local);
    const double X = xf / (double)ni, Y = yf / (double)nj, Z = zf / (double)nk;
    const bool in = X >= x0 && X <= x1 && Y >= y0 && Y <= y1 && Z >= z0 && Z <= z1;
    const T val = G[comp][local];
    if (in) acc += (double)val * (double)val;
    if (D[comp]) D[comp][local] = in ? T(2) * val : T(0);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(XFP_FULL, acc, o);
  if ((threadIdx.x & 31) == 0 && acc != 0.0) atomicAdd(loss, acc);
}

long long faces_total(int ni, int nj, int nk) {
  return (long long)(ni + 1) * nj * nk + (long long)ni * (nj + 1) * nk + (long long)ni * nj * (nk + 1);
}
unsigned grid_for(long long n) { return (unsigned)std::min<long long>((n + 255) / 256, 148LL * 16); }

}  // namespace

template <typename T>
cudaError_t advect(const T* u, const T* v, const T* w, T* ou, T* ov, T* ow, int ni, int nj, int nk, T c,
                   cudaStream_t st) {
  ++g_kernel_launches;
  advect_kernel<T><<<grid_for(faces_total(ni, nj, nk)), 256, 0, st>>>(u, v, w, ou, ov, ow, ni, nj, nk, c);
  return cudaGetLastError();
}
template <typename T>
cudaError_t advect_adjoint(const T* u, const T* v, const T* w, const T* gu, const T* gv, const T* gw, T* du,
                           T* dv, T* dw, int ni, int nj, int nk, T c, cudaStream_t st) {
  const size_t fu = (size_t)(ni + 1) * nj * nk, fv = (size_t)ni * (nj + 1) * nk, fw = (size_t)ni * nj * (nk + 1);
  cudaError_t e;
  if ((e = cudaMemsetAsync(du, 0, fu * sizeof(T), st))) return e;
  if ((e = cudaMemsetAsync(dv, 0, fv * sizeof(T), st))) return e;
  if ((e = cudaMemsetAsync(dw, 0, fw * sizeof(T), st))) return e;
  ++g_kernel_launches;
  advect_adjoint_kernel<T><<<grid_for(faces_total(ni, nj, nk)), 256, 0, st>>>(u, v, w, gu, gv, gw, du, dv, dw, ni,
                                                                              nj, nk, c);
  return cudaGetLastError();
}
template <typename T>
cudaError_t box_loss(const T* u, const T* v, const T* w, T* gu, T* gv, T* gw, int ni, int nj, int nk,
                     const double box[6], double* loss, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(loss, 0, sizeof(double), st);
  if (e) return e;
  ++g_kernel_launches;
  box_loss_kernel<T><<<grid_for(faces_total(ni, nj, nk)), 256, 0, st>>>(u, v, w, gu, gv, gw, ni, nj, nk, box[0],
                                                                        box[1], box[2], box[3], box[4], box[5], loss);
  return cudaGetLastError();
}

template cudaError_t advect<double>(const double*, const double*, const double*, double*, double*, double*, int,
                                    int, int, double, cudaStream_t);
template cudaError_t advect<float>(const float*, const float*, const float*, float*, float*, float*, int, int, int,
                                   float, cudaStream_t);
template cudaError_t advect_adjoint<double>(const double*, const double*, const double*, const double*,
                                            const double*, const double*, double*, double*, double*, int, int, int,
                                            double, cudaStream_t);
template cudaError_t advect_adjoint<float>(const float*, const float*, const float*, const float*, const float*,
                                           const float*, float*, float*, float*, int, int, int, float, cudaStream_t);
template cudaError_t box_loss<double>(const double*, const double*, const double*, double*, double*, double*, int,
                                      int, int, const double*, double*, cudaStream_t);
template cudaError_t box_loss<float>(const float*, const float*, const float*, float*, float*, float*, int, int,
                                     int, const double*, double*, cudaStream_t);

}  // namespace xfp

// ---------------------------------------------------------------- C ABI
namespace {

using xfp_host::fail;

int check_adv(xfp_ctx* ctx, int ni, int nj, int nk, std::initializer_list<const void*> ptrs) {
  if (!ctx) return XFP_ERR_ARGS;
  if (ni < 1 || nj < 1 || nk < 1) return fail(ctx, XFP_ERR_ARGS, "grid sizes must be >= 1");
  if ((long long)(ni + 1) * (nj + 1) * (nk + 1) >= (1LL << 31)) return fail(ctx, XFP_ERR_ARGS, "grid too large");
  if (!ctx->opt.device_pointers)
    return fail(ctx, XFP_ERR_ARGS, "advection entry points take device arrays: set options.device_pointers");
  for (const void* p : ptrs)
    if (!p) return fail(ctx, XFP_ERR_ARGS, "array argument is NULL");
  if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, XFP_ERR_CUDA, "cudaSetDevice failed");
  return XFP_OK;
}

template <typename T>
int advect_impl(xfp_ctx* ctx, int ni, int nj, int nk, const T* u, const T* v, const T* w, T* ou, T* ov, T* ow,
                double c) {
  int rc = check_adv(ctx, ni, nj, nk, {u, v, w, ou, ov, ow});
  if (rc) return rc;
  XFP_CUDA(ctx, (xfp::advect<T>(u, v, w, ou, ov, ow, ni, nj, nk, (T)c, ctx->stream)));
  XFP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return XFP_OK;
}
template <typename T>
int advect_bwd_impl(xfp_ctx* ctx, int ni, int nj, int nk, const T* u, const T* v, const T* w, const T* gu,
                    const T* gv, const T* gw, T* du, T* dv, T* dw, double c) {
  int rc = check_adv(ctx, ni, nj, nk, {u, v, w, gu, gv, gw, du, dv, dw});
  if (rc) return rc;
  XFP_CUDA(ctx, (xfp::advect_adjoint<T>(u, v, w, gu, gv, gw, du, dv, dw, ni, nj, nk, (T)c, ctx->stream)));
  XFP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return XFP_OK;
}
template <typename T>
int box_loss_impl(xfp_ctx* ctx, int ni, int nj, int nk, const T* u, const T* v, const T* w, const double* box,
                  double* loss, T* gu, T* gv, T* gw) {
  int rc = check_adv(ctx, ni, nj, nk, {u, v, w, box, loss});
  if (rc) return rc;
  if ((gu == nullptr) != (gv == nullptr) || (gu == nullptr) != (gw == nullptr))
    return fail(ctx, XFP_ERR_ARGS, "gradient outputs: pass all three or none");
  XFP_CUDA(ctx, ctx->partials.ensure(xfp_host::NBLK_MAX * sizeof(double)));
  double* dl = ctx->partials.as<double>();
  XFP_CUDA(ctx, (xfp::box_loss<T>(u, v, w, gu, gv, gw, ni, nj, nk, box, dl, ctx->stream)));
  XFP_CUDA(ctx, cudaMemcpyAsync(loss, dl, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  XFP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return XFP_OK;
}

}  // namespace

extern "C" {
int xfp_advect_f64(xfp_ctx* ctx, int ni, int nj, int nk, const double* u, const double* v, const double* w,
                   double* ou, double* ov, double* ow, double dt_over_dx) {
  return advect_impl<double>(ctx, ni, nj, nk, u, v, w, ou, ov, ow, dt_over_dx);
}
int xfp_advect_f32(xfp_ctx* ctx, int ni, int nj, int nk, const float* u, const float* v, const float* w,
                   float* ou, float* ov, float* ow, double dt_over_dx) {
  return advect_impl<float>(ctx, ni, nj, nk, u, v, w, ou, ov, ow, dt_over_dx);
}
int xfp_advect_backward_f64(xfp_ctx* ctx, int ni, int nj, int nk, const double* u, const double* v,
                            const double* w, const double* gu, const double* gv, const double* gw, double* du,
                            double* dv, double* dw, double dt_over_dx) {
  return advect_bwd_impl<double>(ctx, ni, nj, nk, u, v, w, gu, gv, gw, du, dv, dw, dt_over_dx);
}
int xfp_advect_backward_f32(xfp_ctx* ctx, int ni, int nj, int nk, const float* u, const float* v, const float* w,
                            const float* gu, const float* gv, const float* gw, float* du, float* dv, float* dw,
                            double dt_over_dx) {
  return advect_bwd_impl<float>(ctx, ni, nj, nk, u, v, w, gu, gv, gw, du, dv, dw, dt_over_dx);
}
int xfp_box_loss_f64(xfp_ctx* ctx, int ni, int nj, int nk, const double* u, const double* v, const double* w,
                     const double* box, double* loss, double* gu, double* gv, double* gw) {
  return box_loss_impl<double>(ctx, ni, nj, nk, u, v, w, box, loss, gu, gv, gw);
}
int xfp_box_loss_f32(xfp_ctx* ctx, int ni, int nj, int nk, const float* u, const float* v, const float* w,
                     const double* box, double* loss, float* gu, float* gv, float* gw) {
  return box_loss_impl<float>(ctx, ni, nj, nk, u, v, w, box, loss, gu, gv, gw);
}
}
