// xfp_ops.cu -- assembly, pressure update, adjoint pieces and the PCG vector
// kernels of libxfp, over the line-compacted layout (xfp_common.cuh).
//
// Reference (paths relative to xFluid/xFluid/):
//   assembly        variationalpressure/variational_pressuresolver.cpp:231-327
//   applyPressure   variationalpressure/variational_pressuresolver.cpp:120-220
//   SpMV            variationalpressure/sparse_matrix.h:264-276
//   PCG loop        variationalpressure/pcg_solver.h:243-285
//   dot/axpy/absmax variationalpressure/blas_wrapper.h:12-51
#include <algorithm>
#include <type_traits>

#include "xfp_common.cuh"
#include "xfp_kernels.h"

namespace xfp {

long long g_kernel_launches = 0;

__device__ __forceinline__ size_t uix(int ni, int nj, int i, int j, int k) {
  return ((size_t)k * nj + j) * (size_t)(ni + 1) + i;
}
__device__ __forceinline__ size_t vix(int ni, int nj, int i, int j, int k) {
  return ((size_t)k * (nj + 1) + j) * (size_t)ni + i;
}
__device__ __forceinline__ size_t wix(int ni, int nj, int i, int j, int k) {
  return ((size_t)k * nj + j) * (size_t)ni + i;
}

// ---------------------------------------------------------------------------
// Assembly: one warp per x-line, lanes over the line's stored span.
//  fluid c, neighbour n across face f (weight m), order +i,-i,+j,-j,+k,-k
//  (xfluidutil.cpp:33-41):
//    n fluid: A(c,c)+=m,    A(c,n)=-m,    b(c)+=vsign*u*m      (:294-301)
//    n air:   A(c,c)+=2m,                 b(c)+=vsign*u*m      (:302-308)
//    n solid: A(c,c)+=0.5m, A(c,n)=-0.5m, b(c)+=vsign*u*0.5*m  (:309-316)
//  solid s: rows added from its fluid neighbours' loops (:318-320) in the
//  loop order i-major, j, k-minor, i.e. neighbours -x,-y,-z,+z,+y,+x.
// ---------------------------------------------------------------------------
template <typename FT, typename AT>
__global__ void assemble_kernel(const uint8_t* __restrict__ mat, const FT* __restrict__ u,
                                const FT* __restrict__ v, const FT* __restrict__ w,
                                const FT* __restrict__ wu, const FT* __restrict__ wv,
                                const FT* __restrict__ ww, int ni, int nj, int nk,
                                const Line* __restrict__ lines, AT* __restrict__ diag,
                                AT* __restrict__ ax, AT* __restrict__ ay, AT* __restrict__ az,
                                AT* __restrict__ b, int matrix, Force3 frc, float* __restrict__ d32,
                                float* __restrict__ x32, float* __restrict__ y32, float* __restrict__ z32) {
  const int lane = threadIdx.x & 31;
  const long long nlines = (long long)nj * nk;
  const size_t nn = (size_t)ni * nj;
  for (long long line = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); line < nlines;
       line += (long long)gridDim.x * (blockDim.x >> 5)) {
    const Line L = lines[line];
    if (L.len == 0) continue;
    const int j = (int)(line % nj), k = (int)(line / nj);
    for (int q = lane; q < L.len; q += 32) {
      const int i = L.lo + q;
      const size_t c = (size_t)k * nn + (size_t)j * ni + i;
      const size_t o = (size_t)L.off + q;
      AT d = AT(0), bb = AT(0), ox = AT(0), oy = AT(0), oz = AT(0);
      const uint8_t m = (i >= 0 && i < ni) ? mat[c] : MAT_AIR;
      if (m == MAT_FLUID || m == MAT_SOLID) {
        // neighbour (di,dj,dk), face value, weight, vsign
        auto face = [&](int nb, AT& uf, AT& mf, AT& vs, int& ii, int& jj, int& kk) -> bool {
          const int di = nb == 0 ? 1 : nb == 1 ? -1 : 0;
          const int dj = nb == 2 ? 1 : nb == 3 ? -1 : 0;
          const int dk = nb == 4 ? 1 : nb == 5 ? -1 : 0;
          ii = i + di; jj = j + dj; kk = k + dk;
          if (ii < 0 || jj < 0 || kk < 0 || ii >= ni || jj >= nj || kk >= nk) return false;
          vs = (di + dj + dk) > 0 ? AT(-1) : AT(1);
          const int fi = i + (di > 0), fj = j + (dj > 0), fk = k + (dk > 0);
          // every face read here borders a fluid cell, so a body force applies
          // to all of them (added in the I/O type, before the conversion)
          if (di) {
            const size_t f = uix(ni, nj, fi, fj, fk);
            uf = (AT)(frc.axis_on(0) ? add_rn(u[f], (FT)frc.d[0]) : u[f]); mf = wu ? (AT)wu[f] : AT(1);
          } else if (dj) {
            const size_t f = vix(ni, nj, fi, fj, fk);
            uf = (AT)(frc.axis_on(1) ? add_rn(v[f], (FT)frc.d[1]) : v[f]); mf = wv ? (AT)wv[f] : AT(1);
          } else {
            const size_t f = wix(ni, nj, fi, fj, fk);
            uf = (AT)(frc.axis_on(2) ? add_rn(w[f], (FT)frc.d[2]) : w[f]); mf = ww ? (AT)ww[f] : AT(1);
          }
          return true;
        };
        if (matrix == XFP_MATRIX_NORMAL) {
          // NormalPressureSolver::_calculate_coefficient (pressuresolver.cpp:220-347):
          // fluid rows only; diagonal = in-range non-solid neighbours, -1 to
          // each fluid neighbour; b gathers the faces towards non-solid
          // neighbours (out of range counts as solid) in the order u low, u
          // high, v low, v high, w low, w high, the low face added and the
          // high face subtracted.
          if (m == MAT_FLUID) {
            int count = 0;
            const int order[6] = {1, 0, 3, 2, 5, 4};
#pragma unroll
            for (int t = 0; t < 6; ++t) {
              const int nb = order[t];
              AT uf, mf, vs;
              int ii, jj, kk;
              if (!face(nb, uf, mf, vs, ii, jj, kk)) continue;
              const uint8_t mn = mat[(size_t)kk * nn + (size_t)jj * ni + ii];
              if (mn == MAT_SOLID) continue;
              ++count;
              bb = add_rn(bb, mul_rn(vs, uf));
              const AT off = mn == MAT_FLUID ? AT(-1) : AT(0);
              if (nb == 1) ox = off;
              if (nb == 3) oy = off;
              if (nb == 5) oz = off;
            }
            d = AT(count);
          }
        } else if (m == MAT_FLUID) {
#pragma unroll
          for (int nb = 0; nb < 6; ++nb) {
            AT uf, mf, vs;
            int ii, jj, kk;
            if (!face(nb, uf, mf, vs, ii, jj, kk)) continue;
            const uint8_t mn = mat[(size_t)kk * nn + (size_t)jj * ni + ii];
            AT off = AT(0);
            if (mn == MAT_FLUID) {
              d = add_rn(d, mul_rn(AT(1), mf));
              off = mul_rn(AT(-1), mf);
              bb = add_rn(bb, mul_rn(mul_rn(vs, uf), mf));
            } else if (mn == MAT_AIR) {
              d = add_rn(d, mul_rn(AT(2), mf));
              bb = add_rn(bb, mul_rn(mul_rn(vs, uf), mf));
            } else {
              d = add_rn(d, mul_rn(AT(0.5), mf));
              off = mul_rn(AT(-0.5), mf);
              bb = add_rn(bb, mul_rn(mul_rn(mul_rn(vs, uf), AT(0.5)), mf));
            }
            if (nb == 1) ox = off;
            if (nb == 3) oy = off;
            if (nb == 5) oz = off;
          }
        } else {
          const int order[6] = {1, 3, 5, 4, 2, 0};
#pragma unroll
          for (int t = 0; t < 6; ++t) {
            const int nb = order[t];
            AT uf, mf, vs;
            int ii, jj, kk;
            if (!face(nb, uf, mf, vs, ii, jj, kk)) continue;
            if (mat[(size_t)kk * nn + (size_t)jj * ni + ii] != MAT_FLUID) continue;
            d = add_rn(d, mul_rn(AT(0.5), mf));
            const AT off = mul_rn(AT(-0.5), mf);
            bb = add_rn(bb, mul_rn(mul_rn(mul_rn(vs, uf), AT(0.5)), mf));
            if (nb == 1) ox = off;
            if (nb == 3) oy = off;
            if (nb == 5) oz = off;
          }
        }
      }
      diag[o] = d; ax[o] = ox; ay[o] = oy; az[o] = oz; b[o] = bb;
      // the mixed form's FP32 stencil, written by the assembly itself
      if (d32 != nullptr) {
        d32[o] = (float)d; x32[o] = (float)ox; y32[o] = (float)oy; z32[o] = (float)oz;
      }
    }
  }
}

template <typename FT, typename AT>
cudaError_t assemble(const uint8_t* mat, const FT* u, const FT* v, const FT* w, const FT* wu,
                     const FT* wv, const FT* ww, int ni, int nj, int nk, const Line* lines,
                     AT* diag, AT* ax, AT* ay, AT* az, AT* b, cudaStream_t st, int matrix, Force3 frc,
                     float* const A32[4]) {
  const long long nlines = (long long)nj * nk;
  long long blocks = (nlines + 7) / 8;
  if (blocks > 65535 * 8) blocks = 65535 * 8;
  ++g_kernel_launches;
  assemble_kernel<FT, AT><<<(unsigned)blocks, 256, 0, st>>>(
      mat, u, v, w, wu, wv, ww, ni, nj, nk, lines, diag, ax, ay, az, b, matrix, frc, A32 ? A32[0] : nullptr,
      A32 ? A32[1] : nullptr, A32 ? A32[2] : nullptr, A32 ? A32[3] : nullptr);
  return cudaGetLastError();
}
template cudaError_t assemble<double, double>(const uint8_t*, const double*, const double*,
                                              const double*, const double*, const double*,
                                              const double*, int, int, int, const Line*, double*,
                                              double*, double*, double*, double*, cudaStream_t, int, Force3, float* const*);
template cudaError_t assemble<float, float>(const uint8_t*, const float*, const float*, const float*,
                                            const float*, const float*, const float*, int, int, int,
                                            const Line*, float*, float*, float*, float*, float*,
                                            cudaStream_t, int, Force3, float* const*);
template cudaError_t assemble<float, double>(const uint8_t*, const float*, const float*,
                                             const float*, const float*, const float*, const float*,
                                             int, int, int, const Line*, double*, double*, double*,
                                             double*, double*, cudaStream_t, int, Force3, float* const*);
template cudaError_t assemble<double, float>(const uint8_t*, const double*, const double*,
                                             const double*, const double*, const double*,
                                             const double*, int, int, int, const Line*, float*,
                                             float*, float*, float*, float*, cudaStream_t, int, Force3, float* const*);

// ---------------------------------------------------------------------------
// Compact -> dense pressure grid: every cell written, 0 outside unknowns
// (variational_pressuresolver.cpp:86-101 copies every cell of the solution).
// ---------------------------------------------------------------------------
template <typename T>
__global__ void scatter_dense_kernel(const T* __restrict__ x, const Line* __restrict__ lines, int ni,
                                     int nj, int nk, T* __restrict__ dense) {
  const size_t n = (size_t)ni * nj * nk;
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(c % ni);
    const size_t line = c / ni;
    const Line L = lines[line];
    T val = T(0);
    if ((unsigned)(i - L.lo) < (unsigned)L.len) val = x[(size_t)L.off + (i - L.lo)];
    dense[c] = val;
  }
}
template <typename T>
cudaError_t scatter_dense(const T* x, const Line* lines, int ni, int nj, int nk, T* dense,
                          cudaStream_t st) {
  size_t n = (size_t)ni * nj * nk;
  unsigned blocks = (unsigned)std::min<size_t>((n + 255) / 256, 148 * 32);
  ++g_kernel_launches;
  scatter_dense_kernel<T><<<blocks, 256, 0, st>>>(x, lines, ni, nj, nk, dense);
  return cudaGetLastError();
}
template cudaError_t scatter_dense<double>(const double*, const Line*, int, int, int, double*, cudaStream_t);
template cudaError_t scatter_dense<float>(const float*, const Line*, int, int, int, float*, cudaStream_t);

// Dense -> compact (cells of every stored span; padding cells get 0).
template <typename T>
__global__ void gather_compact_kernel(const T* __restrict__ dense, const Line* __restrict__ lines, int ni,
                                      int nj, int nk, T* __restrict__ x) {
  const int lane = threadIdx.x & 31;
  const long long nlines = (long long)nj * nk;
  for (long long line = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); line < nlines;
       line += (long long)gridDim.x * (blockDim.x >> 5)) {
    const Line L = lines[line];
    for (int q = lane; q < L.len; q += 32) {
      const int i = L.lo + q;
      x[(size_t)L.off + q] = (i >= 0 && i < ni) ? dense[(size_t)line * ni + i] : T(0);
    }
  }
}
template <typename T>
cudaError_t gather_compact(const T* dense, const Line* lines, int ni, int nj, int nk, T* x,
                           cudaStream_t st) {
  const long long nlines = (long long)nj * nk;
  long long blocks = std::min<long long>((nlines + 7) / 8, 65535LL * 8);
  ++g_kernel_launches;
  gather_compact_kernel<T><<<(unsigned)blocks, 256, 0, st>>>(dense, lines, ni, nj, nk, x);
  return cudaGetLastError();
}
template cudaError_t gather_compact<double>(const double*, const Line*, int, int, int, double*, cudaStream_t);
template cudaError_t gather_compact<float>(const float*, const Line*, int, int, int, float*, cudaStream_t);

// ---------------------------------------------------------------------------
// applyPressure: per face, left/right cells (out of range counts as solid,
// :151-152); fluid|fluid and fluid|solid use both pressures, fluid|air uses the
// ghost -p (:161-198); u -= 1.0*(p2-p1) (:200).  Faces with weight 0 are closed.
// ---------------------------------------------------------------------------
template <typename PT>
__device__ __forceinline__ bool face_dp(const uint8_t* mat, const PT* p, int ni, int nj, int nk,
                                        int il, int jl, int kl, int ir, int jr, int kr, PT& dp) {
  const size_t nn = (size_t)ni * nj;
  const bool inl = il >= 0 && jl >= 0 && kl >= 0 && il < ni && jl < nj && kl < nk;
  const bool inr = ir >= 0 && jr >= 0 && kr >= 0 && ir < ni && jr < nj && kr < nk;
  const size_t cl = inl ? (size_t)kl * nn + (size_t)jl * ni + il : 0;
  const size_t cr = inr ? (size_t)kr * nn + (size_t)jr * ni + ir : 0;
  const uint8_t ml = inl ? mat[cl] : MAT_SOLID;
  const uint8_t mr = inr ? mat[cr] : MAT_SOLID;
  if (ml != MAT_FLUID && mr != MAT_FLUID) return false;
  PT p1, p2;
  if (ml == MAT_FLUID && mr == MAT_FLUID) {
    p2 = p[cr]; p1 = p[cl];
  } else if (ml == MAT_FLUID) {
    p1 = p[cl];
    if (mr == MAT_SOLID) {
      if (!inr) return false;
      p2 = p[cr];
    } else {
      p2 = -p1;
    }
  } else {
    p2 = p[cr];
    if (ml == MAT_SOLID) {
      if (!inl) return false;
      p1 = p[cl];
    } else {
      p1 = -p2;
    }
  }
  dp = sub_rn(p2, p1);
  return true;
}

// NormalPressureSolver::applyPressure (pressuresolver.cpp:109-212) for one face
// with left cell l and right cell r (out of range counts as solid), factor 1:
// fluid|solid takes p2 = p1 + f, solid|fluid p1 = p2 - f, a fluid|air face
// takes 0 for the air side.  Returns false where no side is fluid.
template <typename PT>
__device__ __forceinline__ bool face_dp_normal(const uint8_t* __restrict__ mat, const PT* __restrict__ p, int ni,
                                               int nj, int nk, int il, int jl, int kl, int ir, int jr, int kr, PT fv,
                                               PT& dp) {
  const size_t nn = (size_t)ni * nj;
  const bool inl = il >= 0 && jl >= 0 && kl >= 0 && il < ni && jl < nj && kl < nk;
  const bool inr = ir >= 0 && jr >= 0 && kr >= 0 && ir < ni && jr < nj && kr < nk;
  const size_t cl = inl ? (size_t)kl * nn + (size_t)jl * ni + il : 0;
  const size_t cr = inr ? (size_t)kr * nn + (size_t)jr * ni + ir : 0;
  const uint8_t ml = inl ? mat[cl] : MAT_SOLID;
  const uint8_t mr = inr ? mat[cr] : MAT_SOLID;
  if (ml != MAT_FLUID && mr != MAT_FLUID) return false;
  PT p1, p2;
  if (ml == MAT_FLUID && mr == MAT_FLUID) {
    p2 = p[cr]; p1 = p[cl];
  } else if (ml == MAT_FLUID) {
    p1 = p[cl];
    p2 = mr == MAT_SOLID ? add_rn(p1, fv) : PT(0);
  } else {
    p2 = p[cr];
    p1 = ml == MAT_SOLID ? sub_rn(p2, fv) : PT(0);
  }
  dp = sub_rn(p2, p1);
  return true;
}

template <typename FT, typename PT>
__global__ void apply_kernel(const uint8_t* __restrict__ mat, const FT* __restrict__ wt,
                             const PT* __restrict__ p, int ni, int nj, int nk, int axis,
                             FT* __restrict__ f, int matrix, Force3 frc) {
  const int si = ni + (axis == 0), sj = nj + (axis == 1), sk = nk + (axis == 2);
  const size_t n = (size_t)si * sj * sk;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(idx % si);
    const int j = (int)((idx / si) % sj);
    const int k = (int)(idx / ((size_t)si * sj));
    // a body force first moves every face that borders fluid (_applyForces),
    // then the pressure update uses the moved value
    FT fv = f[idx];
    bool changed = false;
    if (frc.axis_on(axis)) {
      const int il = i - (axis == 0), jl = j - (axis == 1), kl = k - (axis == 2);
      const size_t nn = (size_t)ni * nj;
      const bool fl = il >= 0 && jl >= 0 && kl >= 0 && mat[(size_t)kl * nn + (size_t)jl * ni + il] == MAT_FLUID;
      const bool fr = i < ni && j < nj && k < nk && mat[(size_t)k * nn + (size_t)j * ni + i] == MAT_FLUID;
      if (fl || fr) {
        fv = add_rn(fv, (FT)frc.d[axis]);
        changed = true;
      }
    }
    PT dp;
    if (matrix == XFP_MATRIX_NORMAL) {
      if (face_dp_normal(mat, p, ni, nj, nk, i - (axis == 0), j - (axis == 1), k - (axis == 2), i, j, k,
                         (PT)fv, dp)) {
        fv = sub_rn(fv, (FT)mul_rn(PT(1), dp));
        changed = true;
      }
    } else if (!(wt && wt[idx] == FT(0)) &&
               face_dp(mat, p, ni, nj, nk, i - (axis == 0), j - (axis == 1), k - (axis == 2), i, j, k, dp)) {
      fv = sub_rn(fv, (FT)mul_rn(PT(1), dp));
      changed = true;
    }
    if (changed) f[idx] = fv;
  }
}
template <typename FT, typename PT>
cudaError_t apply_pressure(const uint8_t* mat, const FT* wu, const FT* wv, const FT* ww,
                           const PT* p, int ni, int nj, int nk, FT* u, FT* v, FT* w,
                           cudaStream_t st, int matrix, Force3 frc) {
  for (int axis = 0; axis < 3; ++axis) {
    size_t n = (size_t)(ni + (axis == 0)) * (nj + (axis == 1)) * (nk + (axis == 2));
    unsigned blocks = (unsigned)std::min<size_t>((n + 255) / 256, 148 * 32);
    ++g_kernel_launches;
    apply_kernel<FT, PT><<<blocks, 256, 0, st>>>(mat, axis == 0 ? wu : axis == 1 ? wv : ww, p, ni, nj, nk,
                                                axis, axis == 0 ? u : axis == 1 ? v : w, matrix, frc);
  }
  return cudaGetLastError();
}
template cudaError_t apply_pressure<double, double>(const uint8_t*, const double*, const double*,
                                                    const double*, const double*, int, int, int,
                                                    double*, double*, double*, cudaStream_t, int, Force3);
template cudaError_t apply_pressure<float, float>(const uint8_t*, const float*, const float*,
                                                  const float*, const float*, int, int, int, float*,
                                                  float*, float*, cudaStream_t, int, Force3);

// ---------------------------------------------------------------------------
// Adjoint of the pressure update: q = G^T g, where applyPressure computes
// u_out = u - G p (dp = p2 - p1 per updated face).  Gather per unknown cell.
// ---------------------------------------------------------------------------
template <typename FT, typename PT>
__global__ void apply_T_kernel(const uint8_t* __restrict__ mat, const FT* __restrict__ wu,
                               const FT* __restrict__ wv, const FT* __restrict__ ww,
                               const FT* __restrict__ gu, const FT* __restrict__ gv,
                               const FT* __restrict__ gw, int ni, int nj, int nk,
                               const Line* __restrict__ lines, PT* __restrict__ q) {
  const int lane = threadIdx.x & 31;
  const long long nlines = (long long)nj * nk;
  const size_t nn = (size_t)ni * nj;
  for (long long line = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); line < nlines;
       line += (long long)gridDim.x * (blockDim.x >> 5)) {
    const Line L = lines[line];
    if (L.len == 0) continue;
    const int j = (int)(line % nj), k = (int)(line / nj);
    for (int qq = lane; qq < L.len; qq += 32) {
      const int i = L.lo + qq;
      PT acc = PT(0);
      if (i >= 0 && i < ni) {
        const uint8_t mc = mat[(size_t)k * nn + (size_t)j * ni + i];
        if (mc == MAT_FLUID || mc == MAT_SOLID) {
          // faces: low/high per axis; c is the right cell of its low face and
          // the left cell of its high face
          for (int axis = 0; axis < 3; ++axis) {
            for (int side = 0; side < 2; ++side) {
              const int di = axis == 0, dj = axis == 1, dk = axis == 2;
              // face index (fi,fj,fk) and the other cell
              const int fi = i + (side ? di : 0), fj = j + (side ? dj : 0), fk = k + (side ? dk : 0);
              const int oi = side ? i + di : i - di, oj = side ? j + dj : j - dj, ok = side ? k + dk : k - dk;
              size_t f;
              const FT* wt;
              const FT* gb;
              if (axis == 0) { f = uix(ni, nj, fi, fj, fk); wt = wu; gb = gu; }
              else if (axis == 1) { f = vix(ni, nj, fi, fj, fk); wt = wv; gb = gv; }
              else { f = wix(ni, nj, fi, fj, fk); wt = ww; gb = gw; }
              if (wt && wt[f] == FT(0)) continue;
              const bool ino = oi >= 0 && oj >= 0 && ok >= 0 && oi < ni && oj < nj && ok < nk;
              const uint8_t mo = ino ? mat[(size_t)ok * nn + (size_t)oj * ni + oi] : MAT_SOLID;
              // c is 'r' when side==0 (low face), 'l' when side==1
              const uint8_t ml = side ? mc : mo, mr = side ? mo : mc;
              if (ml != MAT_FLUID && mr != MAT_FLUID) continue;
              const PT g = (PT)gb[f];
              PT coef = PT(0);
              if (ml == MAT_FLUID && mr == MAT_FLUID) {
                coef = side ? PT(-1) : PT(1);
              } else if (ml == MAT_FLUID) {  // right is solid or air
                if (mr == MAT_SOLID) {
                  if (!ino && !side) continue;
                  if (side && !ino) continue;
                  coef = side ? PT(-1) : PT(1);
                } else {
                  coef = side ? PT(-2) : PT(0);
                }
              } else {  // left is solid or air, right is fluid
                if (ml == MAT_SOLID) {
                  if (!ino) continue;
                  coef = side ? PT(-1) : PT(1);
                } else {
                  coef = side ? PT(0) : PT(2);
                }
              }
              acc += coef * g;
            }
          }
        }
      }
      q[(size_t)L.off + qq] = acc;
    }
  }
}
template <typename FT, typename PT>
cudaError_t apply_pressure_T(const uint8_t* mat, const FT* wu, const FT* wv, const FT* ww,
                             const FT* gu, const FT* gv, const FT* gw, int ni, int nj, int nk,
                             const Line* lines, PT* q, cudaStream_t st) {
  const long long nlines = (long long)nj * nk;
  long long blocks = std::min<long long>((nlines + 7) / 8, 65535LL * 8);
  apply_T_kernel<FT, PT><<<(unsigned)blocks, 256, 0, st>>>(mat, wu, wv, ww, gu, gv, gw, ni, nj, nk, lines, q);
  return cudaGetLastError();
}
template cudaError_t apply_pressure_T<double, double>(const uint8_t*, const double*, const double*,
                                                      const double*, const double*, const double*,
                                                      const double*, int, int, int, const Line*,
                                                      double*, cudaStream_t);
template cudaError_t apply_pressure_T<float, float>(const uint8_t*, const float*, const float*,
                                                    const float*, const float*, const float*,
                                                    const float*, int, int, int, const Line*,
                                                    float*, cudaStream_t);
template cudaError_t apply_pressure_T<double, float>(const uint8_t*, const double*, const double*,
                                                     const double*, const double*, const double*,
                                                     const double*, int, int, int, const Line*,
                                                     float*, cudaStream_t);
template cudaError_t apply_pressure_T<float, double>(const uint8_t*, const float*, const float*,
                                                     const float*, const float*, const float*,
                                                     const float*, int, int, int, const Line*,
                                                     double*, cudaStream_t);

// ---------------------------------------------------------------------------
// Adjoint of the right-hand side: d = g - D^T lam per face, D the assembly's
// b = D u (coefficients vsign*m, halved next to solid; solid rows mirrored).
// lam is the dense cell grid.
// ---------------------------------------------------------------------------
template <typename FT, typename PT>
__global__ void rhs_T_kernel(const uint8_t* __restrict__ mat, const FT* __restrict__ wt,
                             const PT* __restrict__ lam, int ni, int nj, int nk, int axis,
                             const FT* __restrict__ g, FT* __restrict__ out) {
  const int si = ni + (axis == 0), sj = nj + (axis == 1), sk = nk + (axis == 2);
  const size_t n = (size_t)si * sj * sk;
  const size_t nn = (size_t)ni * nj;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(idx % si);
    const int j = (int)((idx / si) % sj);
    const int k = (int)(idx / ((size_t)si * sj));
    const int il = i - (axis == 0), jl = j - (axis == 1), kl = k - (axis == 2);
    const bool inl = il >= 0 && jl >= 0 && kl >= 0;
    const bool inr = i < ni && j < nj && k < nk;
    PT acc = PT(0);
    if (inl && inr) {
      const size_t cl = (size_t)kl * nn + (size_t)jl * ni + il, cr = (size_t)k * nn + (size_t)j * ni + i;
      const uint8_t ml = mat[cl], mr = mat[cr];
      const PT m = wt ? (PT)wt[idx] : PT(1);
      // from the left cell: this is its high face, vsign = -1
      if (ml == MAT_FLUID) acc += -(mr == MAT_SOLID ? PT(0.5) : PT(1)) * m * lam[cl];
      else if (ml == MAT_SOLID && mr == MAT_FLUID) acc += -PT(0.5) * m * lam[cl];
      // from the right cell: its low face, vsign = +1
      if (mr == MAT_FLUID) acc += (ml == MAT_SOLID ? PT(0.5) : PT(1)) * m * lam[cr];
      else if (mr == MAT_SOLID && ml == MAT_FLUID) acc += PT(0.5) * m * lam[cr];
    }
    out[idx] = (FT)((PT)g[idx] - acc);
  }
}
template <typename FT, typename PT>
cudaError_t rhs_T(const uint8_t* mat, const FT* wu, const FT* wv, const FT* ww, const PT* lam,
                  const Line* lines, int ni, int nj, int nk, const FT* gu, const FT* gv,
                  const FT* gw, FT* du, FT* dv, FT* dw, cudaStream_t st) {
  (void)lines;
  for (int axis = 0; axis < 3; ++axis) {
    size_t n = (size_t)(ni + (axis == 0)) * (nj + (axis == 1)) * (nk + (axis == 2));
    unsigned blocks = (unsigned)std::min<size_t>((n + 255) / 256, 148 * 32);
    rhs_T_kernel<FT, PT><<<blocks, 256, 0, st>>>(mat, axis == 0 ? wu : axis == 1 ? wv : ww, lam, ni, nj, nk,
                                                axis, axis == 0 ? gu : axis == 1 ? gv : gw,
                                                axis == 0 ? du : axis == 1 ? dv : dw);
  }
  return cudaGetLastError();
}
template cudaError_t rhs_T<double, double>(const uint8_t*, const double*, const double*, const double*,
                                           const double*, const Line*, int, int, int, const double*,
                                           const double*, const double*, double*, double*, double*,
                                           cudaStream_t);
template cudaError_t rhs_T<float, float>(const uint8_t*, const float*, const float*, const float*,
                                         const float*, const Line*, int, int, int, const float*,
                                         const float*, const float*, float*, float*, float*,
                                         cudaStream_t);
template cudaError_t rhs_T<float, double>(const uint8_t*, const float*, const float*, const float*,
                                          const double*, const Line*, int, int, int, const float*,
                                          const float*, const float*, float*, float*, float*,
                                          cudaStream_t);

// ---------------------------------------------------------------------------
// Block reduction helpers.  Every reduction is deterministic: fixed per-thread
// order, fixed tree, per-block partials summed in block order by the last
// block (last-block-done counter in PcgScalars::red_count).
// ---------------------------------------------------------------------------
template <typename DT>
__device__ __forceinline__ DT block_sum(DT v, DT* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = add_rn(v, __shfl_xor_sync(XFP_FULL, v, o));
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = v;
  __syncthreads();
  DT t = DT(0);
  if (threadIdx.x == 0)
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) t = add_rn(t, sh[q]);
  __syncthreads();
  return t;  // valid in thread 0
}
__device__ __forceinline__ double block_max(double v, double* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(XFP_FULL, v, o));
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) t = fmax(t, sh[q]);
  __syncthreads();
  return t;
}
// The last block's max over the nblk per-block partials, read by all its
// threads (partial b by thread b mod blockDim, then the block tree).  A max is
// exact in any order, so this equals the sequential max bit for bit; it replaces
// one thread walking every partial (up to NBLK_MAX dependent L2 reads).  Call
// from every thread of the block; the result is valid in thread 0.
__device__ __forceinline__ double partials_max(const double* partials, unsigned nblk, double* sh) {
  double m = 0.0;
  for (unsigned b = threadIdx.x; b < nblk; b += blockDim.x) m = fmax(m, ((volatile const double*)partials)[b]);
  return block_max(m, sh);
}

// Returns true, in every thread of the block, in the last of nblk blocks to
// finish (a batch runs one such group of blocks per scene, each with its own
// counter).
__device__ __forceinline__ bool last_block(PcgScalars* sc, unsigned nblk) {
  __shared__ bool s_last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    unsigned t = atomicAdd(&sc->red_count, 1u);
    s_last = (t == nblk - 1);
  }
  __syncthreads();
  return s_last;
}

// Batch of scenes in one launch: block b belongs to the scene whose range of
// blocks [start, start + count) holds it; the scene's blocks then run exactly
// the decomposition a single-scene launch of `count` blocks would.
// kind: which block range of the scene a block belongs to (0 cell-based
// kernels, 1 line-based kernels, 2 the SpMV's 4-cell groups).
__device__ __forceinline__ int batch_scene_of(const BatchSeg* __restrict__ segs, int nseg, int kind) {
  __shared__ int s_seg;
  if (threadIdx.x == 0) {
    int lo = 0, hi = nseg - 1;
    const int b = (int)blockIdx.x;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      const int start = kind == 1 ? segs[mid].blk_lines_start
                                  : kind == 2 ? segs[mid].blk_groups_start : segs[mid].blk_cells_start;
      if (start <= b) lo = mid; else hi = mid - 1;
    }
    s_seg = lo;
  }
  __syncthreads();
  return s_seg;
}

// The last block's sum over the nblk per-block partials: partial b goes to
// thread b mod blockDim, each thread adds its share in increasing b, then the
// block tree.  The order depends only on nblk and blockDim, so the result is
// deterministic (and the same for a batch scene as for its single launch).
// Call from every thread of the block; the result is valid in thread 0.
template <typename DT>
__device__ __forceinline__ DT partials_sum(const DT* partials, unsigned nblk, DT* sh) {
  DT t = DT(0);
  for (unsigned b = threadIdx.x; b < nblk; b += blockDim.x) t = add_rn(t, ((volatile const DT*)partials)[b]);
  return block_sum(t, sh);
}

// ---------------------------------------------------------------------------
// z = A s (7-point, row order of sparse_matrix.h:264-276: columns c-nn, c-ni,
// c-1, c, c+1, c+ni, c+nn; absent entries skipped) fused with the partial dot
// s.z.  mode 0: alpha = rho / (s.z) (pcg_solver.h:269); mode 1: no dot.
//
// One thread per aligned group of 4 stored cells.  Lines start at multiples
// of 4 and hold multiples of 4 cells, so a group never straddles two lines:
// the thread reads its line once (group_line), loads s and the four
// coefficient arrays as 16-byte vectors (two for FP64), takes its x
// neighbours from the vectors (plus one cell either side), and finds its y/z
// neighbours through the four neighbouring lines' records (shared by every
// group of the line, so L1 hits).  Per cell the products are added in the
// reference's column order, so the FP64 result is the reference's.
// ---------------------------------------------------------------------------
template <typename VT, typename AT, typename DT>
__device__ __forceinline__ void spmv_dot_body(
    unsigned bid, unsigned nblk, const AT* __restrict__ diag, const AT* __restrict__ ax,
    const AT* __restrict__ ay, const AT* __restrict__ az, const VT* __restrict__ s, VT* __restrict__ z,
    const Line* __restrict__ lines, const int* __restrict__ group_line, int nj, int nk, long long base, long long M,
    PcgScalars* sc, DT* __restrict__ partials, int mode) {
  static_assert(std::is_same<VT, AT>::value, "the vector and coefficient types agree");
  __shared__ DT sh[32];
  if (sc && *(volatile int*)&sc->done) return;
  DT acc = DT(0);
  const long long G = M >> 2;
  for (long long q = (long long)bid * blockDim.x + threadIdx.x; q < G; q += (long long)nblk * blockDim.x) {
    const long long c = base + 4 * q;
    const int line = group_line[(base >> 2) + q];
    const Line L = lines[line];
    const int i0 = L.lo + (int)(c - L.off);
    const int j = line % nj, k = line / nj;
    VT sv[4], dv[4], xv[4], yv[4], zv[4];
    ldg(sv, s + c);
    ldg(dv, diag + c);
    ldg(xv, ax + c);
    ldg(yv, ay + c);
    ldg(zv, az + c);
    // one cell either side of the group (when the line has it)
    const VT sl = c > L.off ? s[c - 1] : VT(0);
    const bool right = c + 4 < (long long)L.off + L.len;
    const VT sr = right ? s[c + 4] : VT(0);
    const VT xr = right ? ax[c + 4] : VT(0);
    const Line Z = {0, 0, 0, 0};
    const Line Lym = j > 0 ? lines[line - 1] : Z;
    const Line Lyp = j + 1 < nj ? lines[line + 1] : Z;
    const Line Lzm = k > 0 ? lines[line - nj] : Z;
    const Line Lzp = k + 1 < nk ? lines[line + nj] : Z;
    VT out[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int i = i0 + e;
      VT a = VT(0);
      // a nonzero lower coefficient means the neighbour is an unknown, stored in its line
      if (zv[e] != VT(0)) a = add_rn(a, mul_rn(zv[e], s[(size_t)Lzm.off + (i - Lzm.lo)]));
      if (yv[e] != VT(0)) a = add_rn(a, mul_rn(yv[e], s[(size_t)Lym.off + (i - Lym.lo)]));
      if (xv[e] != VT(0)) a = add_rn(a, mul_rn(xv[e], e == 0 ? sl : sv[e == 0 ? 0 : e - 1]));
      if (dv[e] != VT(0)) a = add_rn(a, mul_rn(dv[e], sv[e]));
      const VT cx = e < 3 ? xv[e < 3 ? e + 1 : 3] : xr;
      if (cx != VT(0)) a = add_rn(a, mul_rn(cx, e < 3 ? sv[e < 3 ? e + 1 : 3] : sr));
      if ((unsigned)(i - Lyp.lo) < (unsigned)Lyp.len) {
        const size_t n = (size_t)Lyp.off + (i - Lyp.lo);
        const VT cy = ay[n];
        if (cy != VT(0)) a = add_rn(a, mul_rn(cy, s[n]));
      }
      if ((unsigned)(i - Lzp.lo) < (unsigned)Lzp.len) {
        const size_t n = (size_t)Lzp.off + (i - Lzp.lo);
        const VT cz = az[n];
        if (cz != VT(0)) a = add_rn(a, mul_rn(cz, s[n]));
      }
      out[e] = a;
      if (mode == 0) acc = add_rn(acc, mul_rn((DT)sv[e], (DT)a));
    }
    stg(z + c, out);
  }
  if (mode != 0) return;
  DT t = block_sum(acc, sh);
  if (threadIdx.x == 0) partials[bid] = t;
  if (!last_block(sc, nblk)) return;   // uniform over the block
  const DT tot = partials_sum(partials, nblk, sh);
  if (threadIdx.x == 0) {
    if (std::is_same<DT, float>::value)
      sc->alpha = (double)__fdiv_rn((float)sc->rho, (float)tot);
    else
      sc->alpha = __ddiv_rn(sc->rho, (double)tot);
    sc->red_count = 0;
  }
}
// Blocks of the SpMV for M stored cells (one thread per 4-cell group); a batch
// gives each scene the same count, so its reduction order is the single one's.
long long spmv_block_count(long long M, int nblk_max) {
  const long long b = ((M >> 2) + 255) / 256;
  return b < 1 ? 1 : (b < nblk_max ? b : nblk_max);
}
template <typename VT, typename AT, typename DT>
__global__ void __launch_bounds__(256) spmv_dot_kernel(
    const AT* __restrict__ diag, const AT* __restrict__ ax, const AT* __restrict__ ay,
    const AT* __restrict__ az, const VT* __restrict__ s, VT* __restrict__ z,
    const Line* __restrict__ lines, const int* __restrict__ group_line, int nj, int nk, long long M, PcgScalars* sc,
    DT* __restrict__ partials, int mode) {
  spmv_dot_body<VT, AT, DT>(blockIdx.x, gridDim.x, diag, ax, ay, az, s, z, lines, group_line, nj, nk, 0, M, sc,
                            partials, mode);
}
template <typename VT, typename AT, typename DT>
__global__ void __launch_bounds__(256) batch_spmv_dot_kernel(
    const BatchSeg* __restrict__ segs, int nseg, const AT* __restrict__ diag, const AT* __restrict__ ax,
    const AT* __restrict__ ay, const AT* __restrict__ az, const VT* __restrict__ s, VT* __restrict__ z,
    const int* __restrict__ group_line, PcgScalars* sc, int mode) {
  const int q = batch_scene_of(segs, nseg, 2);
  const BatchSeg& S = segs[q];
  spmv_dot_body<VT, AT, DT>(blockIdx.x - S.blk_groups_start, S.blk_groups, diag, ax, ay, az, s, z, S.lines,
                            group_line, S.nj, S.nk, S.base, S.M, sc + q, reinterpret_cast<DT*>(S.partials), mode);
}
template <typename VT, typename AT, typename DT>
cudaError_t spmv_dot(const AT* diag, const AT* ax, const AT* ay, const AT* az, const VT* s, VT* z,
                     const Line* lines, const int* group_line, int nj, int nk, long long M, PcgScalars* sc,
                     DT* partials, int nblk_max, int mode, cudaStream_t st) {
  const int blocks = (int)spmv_block_count(M, nblk_max);
  ++g_kernel_launches;
  spmv_dot_kernel<VT, AT, DT><<<blocks, 256, 0, st>>>(diag, ax, ay, az, s, z, lines, group_line, nj, nk, M, sc,
                                                     partials, mode);
  return cudaGetLastError();
}
template cudaError_t spmv_dot<double, double, double>(const double*, const double*, const double*,
                                                      const double*, const double*, double*, const Line*,
                                                      const int*, int, int, long long, PcgScalars*, double*, int,
                                                      int, cudaStream_t);
template cudaError_t spmv_dot<float, float, float>(const float*, const float*, const float*, const float*,
                                                   const float*, float*, const Line*, const int*, int, int,
                                                   long long, PcgScalars*, float*, int, int, cudaStream_t);
template cudaError_t spmv_dot<float, float, double>(const float*, const float*, const float*, const float*,
                                                    const float*, float*, const Line*, const int*, int, int,
                                                    long long, PcgScalars*, double*, int, int, cudaStream_t);

// ---------------------------------------------------------------------------
// x += alpha s ; r += (-alpha) z ; |r|_inf  (pcg_solver.h:270-276).  The last
// block decides convergence: |r|_inf <= tol*|b|_inf, or the iteration cap.
// ---------------------------------------------------------------------------
//
// One thread per aligned 4-cell group, with 16-byte vector accesses (two for
// FP64).  With a sweep layout the group's four cells sit at four consecutive
// sweep-layout elements (consecutive forward steps, aligned to a group of 4),
// so r goes there with one vector store at perm[c].
template <typename VT>
__device__ __forceinline__ void update_xr_body(unsigned bid, unsigned nblk, VT* __restrict__ x,
                                               VT* __restrict__ r, const VT* __restrict__ s,
                                               const VT* __restrict__ z, long long M, PcgScalars* sc,
                                               double* __restrict__ partials, VT* __restrict__ rsw = nullptr,
                                               const int* __restrict__ perm = nullptr) {
  __shared__ double sh[32];
  if (*(volatile int*)&sc->done) return;
  const VT alpha = (VT)sc->alpha;
  const VT nalpha = -alpha;
  double m = 0.0;
  const long long G = M >> 2;
  const long long stride = (long long)nblk * blockDim.x;
  // two groups in flight per thread: the next group's loads are issued before
  // the current group's arithmetic and stores (two buffers, no copies)
  struct Buf {
    VT x[4], r[4], s[4], z[4];
    int p;
  };
  auto load = [&](Buf& B, long long q) {
    const long long c = 4 * q;
    ldg(B.x, x + c);
    ldg(B.r, r + c);
    ldg(B.s, s + c);
    ldg(B.z, z + c);
    B.p = rsw != nullptr ? perm[c] : 0;
  };
  auto finish = [&](Buf& B, long long q) {
    const long long c = 4 * q;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      B.x[e] = add_rn(B.x[e], mul_rn(alpha, B.s[e]));
      B.r[e] = add_rn(B.r[e], mul_rn(nalpha, B.z[e]));
      m = fmax(m, (double)fabs(B.r[e]));
    }
    stg(x + c, B.x);
    stg(r + c, B.r);
    if (rsw != nullptr) stg(rsw + B.p, B.r);
  };
  Buf A, B;
  long long q = (long long)bid * blockDim.x + threadIdx.x;
  if (q < G) load(A, q);
  for (; q < G; q += 2 * stride) {
    const bool nb = q + stride < G;
    if (nb) load(B, q + stride);
    finish(A, q);
    if (!nb) break;
    if (q + 2 * stride < G) load(A, q + 2 * stride);
    finish(B, q + stride);
  }
  double t = block_max(m, sh);
  if (threadIdx.x == 0) partials[bid] = t;
  if (!last_block(sc, nblk)) return;   // uniform over the block
  const double tot = partials_max(partials, nblk, sh);
  if (threadIdx.x == 0) {
    sc->res = tot;
    sc->iters += 1;
    if (tot <= sc->tolabs) {
      sc->done = 1;
      sc->status = 0;
    } else if (sc->iters >= sc->maxit) {
      sc->done = 1;
      sc->status = 1;
    }
    sc->red_count = 0;
  }
}
template <typename VT>
__global__ void __launch_bounds__(256) update_xr_kernel(VT* __restrict__ x, VT* __restrict__ r,
                                                        const VT* __restrict__ s,
                                                        const VT* __restrict__ z, long long M,
                                                        PcgScalars* sc, double* __restrict__ partials,
                                                        VT* __restrict__ rsw, const int* __restrict__ perm) {
  update_xr_body<VT>(blockIdx.x, gridDim.x, x, r, s, z, M, sc, partials, rsw, perm);
}
template <typename VT>
__global__ void __launch_bounds__(256) batch_update_xr_kernel(const BatchSeg* __restrict__ segs, int nseg,
                                                              VT* __restrict__ x, VT* __restrict__ r,
                                                              const VT* __restrict__ s, const VT* __restrict__ z,
                                                              PcgScalars* sc, VT* __restrict__ rsw,
                                                              const int* __restrict__ perm) {
  const int q = batch_scene_of(segs, nseg, 0);
  const BatchSeg& S = segs[q];
  update_xr_body<VT>(blockIdx.x - S.blk_cells_start, S.blk_cells, x + S.base, r + S.base, s + S.base,
                     z + S.base, S.M, sc + q, S.partials, rsw, perm ? perm + S.base : nullptr);
}
template <typename VT, typename DT>
cudaError_t update_xr(VT* x, VT* r, const VT* s, const VT* z, long long M, PcgScalars* sc,
                      double* partials, int nblk_max, cudaStream_t st, VT* rsw, const int* perm) {
  // 4-cell groups over at most nblk_max blocks
  int blocks = (int)std::min<long long>((M / 4 + 255) / 256, (long long)nblk_max);
  if (blocks < 1) blocks = 1;
  ++g_kernel_launches;
  update_xr_kernel<VT><<<blocks, 256, 0, st>>>(x, r, s, z, M, sc, partials, rsw, perm);
  return cudaGetLastError();
}
template cudaError_t update_xr<double, double>(double*, double*, const double*, const double*, long long,
                                               PcgScalars*, double*, int, cudaStream_t, double*, const int*);
template cudaError_t update_xr<float, float>(float*, float*, const float*, const float*, long long,
                                             PcgScalars*, double*, int, cudaStream_t, float*, const int*);
template cudaError_t update_xr<float, double>(float*, float*, const float*, const float*, long long,
                                              PcgScalars*, double*, int, cudaStream_t, float*, const int*);

// s = z + beta s  (add_scaled(beta, s, z) then swap, pcg_solver.h:280); one
// thread per aligned 4-cell group, z read from the sweep layout at perm[c]
// (four consecutive elements) when there is one.
template <typename VT>
__device__ __forceinline__ void update_s_body(unsigned bid, unsigned nblk, VT* __restrict__ s,
                                              const VT* __restrict__ z, long long M, PcgScalars* sc,
                                              const VT* __restrict__ zsw = nullptr,
                                              const int* __restrict__ perm = nullptr) {
  if (*(volatile int*)&sc->done) return;
  const VT beta = (VT)sc->beta;
  const long long G = M >> 2;
  const long long stride = (long long)nblk * blockDim.x;
  // two groups in flight per thread (as in update_xr_body)
  struct Buf {
    VT s[4], z[4];
  };
  auto load = [&](Buf& B, long long q) {
    const long long c = 4 * q;
    ldg(B.s, s + c);
    ldg(B.z, zsw != nullptr ? zsw + perm[c] : z + c);
  };
  auto finish = [&](Buf& B, long long q) {
#pragma unroll
    for (int e = 0; e < 4; ++e) B.s[e] = add_rn(B.z[e], mul_rn(beta, B.s[e]));
    stg(s + 4 * q, B.s);
  };
  Buf A, B;
  long long q = (long long)bid * blockDim.x + threadIdx.x;
  if (q < G) load(A, q);
  for (; q < G; q += 2 * stride) {
    const bool nb = q + stride < G;
    if (nb) load(B, q + stride);
    finish(A, q);
    if (!nb) break;
    if (q + 2 * stride < G) load(A, q + 2 * stride);
    finish(B, q + stride);
  }
}
template <typename VT>
__global__ void update_s_kernel(VT* __restrict__ s, const VT* __restrict__ z, long long M,
                                PcgScalars* sc, const VT* __restrict__ zsw, const int* __restrict__ perm) {
  update_s_body<VT>(blockIdx.x, gridDim.x, s, z, M, sc, zsw, perm);
}
template <typename VT>
__global__ void batch_update_s_kernel(const BatchSeg* __restrict__ segs, int nseg, VT* __restrict__ s,
                                      const VT* __restrict__ z, PcgScalars* sc, const VT* __restrict__ zsw,
                                      const int* __restrict__ perm) {
  const int q = batch_scene_of(segs, nseg, 0);
  const BatchSeg& S = segs[q];
  update_s_body<VT>(blockIdx.x - S.blk_cells_start, S.blk_cells, s + S.base, z + S.base, S.M, sc + q, zsw,
                    perm ? perm + S.base : nullptr);
}
template <typename VT>
cudaError_t update_s(VT* s, const VT* z, long long M, PcgScalars* sc, cudaStream_t st, const VT* zsw,
                     const int* perm, int nblk_max) {
  // 4-cell groups over at most nblk_max blocks (one thread per group measured
  // slower at 256^3: more blocks, fewer groups per thread)
  int blocks = (int)std::min<long long>((M / 4 + 255) / 256, (long long)nblk_max);
  if (blocks < 1) blocks = 1;
  ++g_kernel_launches;
  update_s_kernel<VT><<<blocks, 256, 0, st>>>(s, z, M, sc, zsw, perm);
  return cudaGetLastError();
}
template cudaError_t update_s<double>(double*, const double*, long long, PcgScalars*, cudaStream_t, const double*,
                                      const int*, int);
template cudaError_t update_s<float>(float*, const float*, long long, PcgScalars*, cudaStream_t, const float*,
                                     const int*, int);

// |b|_inf, tolerance and loop state at the start of a solve (pcg_solver.h:247-254).
template <typename VT>
__device__ __forceinline__ void absmax_init_body(unsigned bid, unsigned nblk, const VT* __restrict__ b,
                                                 long long M, PcgScalars* sc, double* __restrict__ partials,
                                                 double tol, int maxit) {
  __shared__ double sh[32];
  double m = 0.0;
  for (long long c = (long long)bid * blockDim.x + threadIdx.x; c < M; c += (long long)nblk * blockDim.x)
    m = fmax(m, (double)fabs(b[c]));
  double t = block_max(m, sh);
  if (threadIdx.x == 0) partials[bid] = t;
  if (!last_block(sc, nblk)) return;   // uniform over the block
  const double tot = partials_max(partials, nblk, sh);
  if (threadIdx.x == 0) {
    sc->bnorm = tot;
    sc->res = tot;
    sc->tolabs = tol * tot;
    sc->iters = 0;
    sc->maxit = maxit;
    sc->status = 0;
    sc->done = (tot == 0.0 || maxit <= 0) ? 1 : 0;
    if (tot != 0.0 && maxit <= 0) sc->status = 1;
    sc->red_count = 0;
  }
}
template <typename VT>
__global__ void absmax_init_kernel(const VT* __restrict__ b, long long M, PcgScalars* sc,
                                   double* __restrict__ partials, double tol, int maxit) {
  absmax_init_body<VT>(blockIdx.x, gridDim.x, b, M, sc, partials, tol, maxit);
}
template <typename VT>
__global__ void batch_absmax_init_kernel(const BatchSeg* __restrict__ segs, int nseg, const VT* __restrict__ b,
                                         PcgScalars* sc, double tol, int maxit, const double* __restrict__ tols,
                                         const int* __restrict__ maxits) {
  const int q = batch_scene_of(segs, nseg, 0);
  const BatchSeg& S = segs[q];
  absmax_init_body<VT>(blockIdx.x - S.blk_cells_start, S.blk_cells, b + S.base, S.M, sc + q, S.partials,
                       tols ? tols[q] : tol, maxits ? maxits[q] : maxit);
}
template <typename VT>
cudaError_t absmax_init(const VT* b, long long M, PcgScalars* sc, double* partials, int nblk_max,
                        double tol, int maxit, cudaStream_t st) {
  int blocks = (int)std::min<long long>((M + 255) / 256, (long long)nblk_max);
  if (blocks < 1) blocks = 1;
  ++g_kernel_launches;
  absmax_init_kernel<VT><<<blocks, 256, 0, st>>>(b, M, sc, partials, tol, maxit);
  return cudaGetLastError();
}
template cudaError_t absmax_init<double>(const double*, long long, PcgScalars*, double*, int, double, int,
                                         cudaStream_t);
template cudaError_t absmax_init<float>(const float*, long long, PcgScalars*, double*, int, double, int,
                                        cudaStream_t);

template <typename A, typename B>
__global__ void convert_kernel(const A* __restrict__ in, B* __restrict__ out, long long n) {
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x)
    out[c] = (B)in[c];
}
template <typename A, typename B>
cudaError_t convert(const A* in, B* out, long long n, cudaStream_t st) {
  int blocks = (int)std::min<long long>((n + 255) / 256, 148LL * 16);
  if (blocks < 1) blocks = 1;
  ++g_kernel_launches;
  convert_kernel<A, B><<<blocks, 256, 0, st>>>(in, out, n);
  return cudaGetLastError();
}
template cudaError_t convert<double, float>(const double*, float*, long long, cudaStream_t);
template cudaError_t convert<float, double>(const float*, double*, long long, cudaStream_t);

template <typename T>
cudaError_t copy_vec(const T* in, T* out, long long n, cudaStream_t st) {
  return cudaMemcpyAsync(out, in, n * sizeof(T), cudaMemcpyDeviceToDevice, st);
}
template cudaError_t copy_vec<double>(const double*, double*, long long, cudaStream_t);
template cudaError_t copy_vec<float>(const float*, float*, long long, cudaStream_t);

// ---------------------------------------------------------------------------
// Mixed precision: FP64 residual r = b - A x with |r|_inf (into sc->res), on
// the FP64 copy of A; and x64 += e32 after each FP32 inner solve.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void residual64_body(
    unsigned bid, unsigned nblk, const double* __restrict__ diag, const double* __restrict__ ax,
    const double* __restrict__ ay, const double* __restrict__ az, const double* __restrict__ b,
    const double* __restrict__ x, double* __restrict__ r, const Line* __restrict__ lines, int ni, int nj,
    int nk, PcgScalars* sc, double* __restrict__ partials) {
  __shared__ double sh[32];
  const int lane = threadIdx.x & 31;
  const long long nlines = (long long)nj * nk;
  double m = 0.0;
  for (long long line = (long long)bid * (blockDim.x >> 5) + (threadIdx.x >> 5); line < nlines;
       line += (long long)nblk * (blockDim.x >> 5)) {
    const Line L = lines[line];
    if (L.len == 0) continue;
    const int j = (int)(line % nj), k = (int)(line / nj);
    Line Lym = {0, 0, 0, 0}, Lyp = {0, 0, 0, 0}, Lzm = {0, 0, 0, 0}, Lzp = {0, 0, 0, 0};
    if (j > 0) Lym = lines[line - 1];
    if (j + 1 < nj) Lyp = lines[line + 1];
    if (k > 0) Lzm = lines[line - nj];
    if (k + 1 < nk) Lzp = lines[line + nj];
    for (int q = lane; q < L.len; q += 32) {
      const int i = L.lo + q;
      const size_t c = (size_t)L.off + q;
      double a = 0.0;
      if (az[c] != 0.0) a += az[c] * x[(size_t)Lzm.off + (i - Lzm.lo)];
      if (ay[c] != 0.0) a += ay[c] * x[(size_t)Lym.off + (i - Lym.lo)];
      if (ax[c] != 0.0) a += ax[c] * x[c - 1];
      a += diag[c] * x[c];
      if (q + 1 < L.len && ax[c + 1] != 0.0) a += ax[c + 1] * x[c + 1];
      if ((unsigned)(i - Lyp.lo) < (unsigned)Lyp.len) {
        const size_t n = (size_t)Lyp.off + (i - Lyp.lo);
        if (ay[n] != 0.0) a += ay[n] * x[n];
      }
      if ((unsigned)(i - Lzp.lo) < (unsigned)Lzp.len) {
        const size_t n = (size_t)Lzp.off + (i - Lzp.lo);
        if (az[n] != 0.0) a += az[n] * x[n];
      }
      const double rv = b[c] - a;
      r[c] = rv;
      m = fmax(m, fabs(rv));
    }
  }
  double t = block_max(m, sh);
  if (threadIdx.x == 0) partials[bid] = t;
  if (!last_block(sc, nblk)) return;   // uniform over the block
  const double tot = partials_max(partials, nblk, sh);
  if (threadIdx.x == 0) {
    sc->res = tot;
    sc->red_count = 0;
  }
}
__global__ void __launch_bounds__(256) residual64_kernel(
    const double* __restrict__ diag, const double* __restrict__ ax, const double* __restrict__ ay,
    const double* __restrict__ az, const double* __restrict__ b, const double* __restrict__ x,
    double* __restrict__ r, const Line* __restrict__ lines, int ni, int nj, int nk, PcgScalars* sc,
    double* __restrict__ partials) {
  residual64_body(blockIdx.x, gridDim.x, diag, ax, ay, az, b, x, r, lines, ni, nj, nk, sc, partials);
}
__global__ void __launch_bounds__(256) batch_residual64_kernel(
    const BatchSeg* __restrict__ segs, int nseg, const double* __restrict__ diag, const double* __restrict__ ax,
    const double* __restrict__ ay, const double* __restrict__ az, const double* __restrict__ b,
    const double* __restrict__ x, double* __restrict__ r, PcgScalars* sc) {
  const int q = batch_scene_of(segs, nseg, 1);
  const BatchSeg& S = segs[q];
  residual64_body(blockIdx.x - S.blk_lines_start, S.blk_lines, diag, ax, ay, az, b, x, r, S.lines, S.ni, S.nj,
                  S.nk, sc + q, S.partials);
}
cudaError_t batch_residual64(const BatchSeg* segs, int nseg, int blocks, const double* diag, const double* ax,
                             const double* ay, const double* az, const double* b, const double* x, double* r,
                             PcgScalars* sc, cudaStream_t st) {
  ++g_kernel_launches;
  batch_residual64_kernel<<<blocks, 256, 0, st>>>(segs, nseg, diag, ax, ay, az, b, x, r, sc);
  return cudaGetLastError();
}
cudaError_t residual64(const double* diag, const double* ax, const double* ay, const double* az,
                       const double* b, const double* x, double* r, const Line* lines, int ni,
                       int nj, int nk, long long M, PcgScalars* sc, double* partials,
                       int nblk_max, cudaStream_t st) {
  (void)M;
  const long long nlines = (long long)nj * nk;
  int blocks = (int)std::min<long long>((nlines + 7) / 8, (long long)nblk_max);
  ++g_kernel_launches;
  residual64_kernel<<<blocks, 256, 0, st>>>(diag, ax, ay, az, b, x, r, lines, ni, nj, nk, sc, partials);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Batch launchers and the per-scene reductions of a batch.
// ---------------------------------------------------------------------------
template <typename VT, typename AT, typename DT>
cudaError_t batch_spmv_dot(const BatchSeg* segs, int nseg, int blocks, const AT* diag, const AT* ax,
                           const AT* ay, const AT* az, const VT* s, VT* z, const int* group_line, PcgScalars* sc,
                           int mode, cudaStream_t st) {
  ++g_kernel_launches;
  batch_spmv_dot_kernel<VT, AT, DT><<<blocks, 256, 0, st>>>(segs, nseg, diag, ax, ay, az, s, z, group_line, sc,
                                                           mode);
  return cudaGetLastError();
}
template cudaError_t batch_spmv_dot<double, double, double>(const BatchSeg*, int, int, const double*,
                                                            const double*, const double*, const double*,
                                                            const double*, double*, const int*, PcgScalars*, int,
                                                            cudaStream_t);
template cudaError_t batch_spmv_dot<float, float, float>(const BatchSeg*, int, int, const float*, const float*,
                                                         const float*, const float*, const float*, float*,
                                                         const int*, PcgScalars*, int, cudaStream_t);
template cudaError_t batch_spmv_dot<float, float, double>(const BatchSeg*, int, int, const float*, const float*,
                                                          const float*, const float*, const float*, float*,
                                                          const int*, PcgScalars*, int, cudaStream_t);

// cell_line[c] = the line (index in its scene's table) that stores cell c;
// group_line[c / 4] the same for every aligned 4-cell group (lines start at
// multiples of 4 and hold multiples of 4 cells).
__global__ void cell_line_kernel(const Line* __restrict__ lines, long long nlines, int* __restrict__ cell_line,
                                 int* __restrict__ group_line) {
  const int lane = threadIdx.x & 31;
  for (long long line = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); line < nlines;
       line += (long long)gridDim.x * (blockDim.x >> 5)) {
    const Line L = lines[line];
    for (int q = lane; q < L.len; q += 32) cell_line[(size_t)L.off + q] = (int)line;
    for (int q = lane; q < (L.len >> 2); q += 32) group_line[((size_t)L.off >> 2) + q] = (int)line;
  }
}
cudaError_t build_cell_line(const Line* lines, long long nlines, int* cell_line, int* group_line, cudaStream_t st) {
  if (nlines <= 0) return cudaSuccess;
  ++g_kernel_launches;
  cell_line_kernel<<<(unsigned)std::min<long long>((nlines + 7) / 8, 65535LL * 8), 256, 0, st>>>(lines, nlines,
                                                                                              cell_line, group_line);
  return cudaGetLastError();
}

template <typename VT>
cudaError_t batch_update_xr(const BatchSeg* segs, int nseg, int blocks, VT* x, VT* r, const VT* s,
                            const VT* z, PcgScalars* sc, cudaStream_t st, VT* rsw, const int* perm) {
  ++g_kernel_launches;
  batch_update_xr_kernel<VT><<<blocks, 256, 0, st>>>(segs, nseg, x, r, s, z, sc, rsw, perm);
  return cudaGetLastError();
}
template cudaError_t batch_update_xr<double>(const BatchSeg*, int, int, double*, double*, const double*,
                                             const double*, PcgScalars*, cudaStream_t, double*, const int*);
template cudaError_t batch_update_xr<float>(const BatchSeg*, int, int, float*, float*, const float*,
                                            const float*, PcgScalars*, cudaStream_t, float*, const int*);

template <typename VT>
cudaError_t batch_update_s(const BatchSeg* segs, int nseg, int blocks, VT* s, const VT* z, PcgScalars* sc,
                           cudaStream_t st, const VT* zsw, const int* perm) {
  ++g_kernel_launches;
  batch_update_s_kernel<VT><<<blocks, 256, 0, st>>>(segs, nseg, s, z, sc, zsw, perm);
  return cudaGetLastError();
}
template cudaError_t batch_update_s<double>(const BatchSeg*, int, int, double*, const double*, PcgScalars*,
                                            cudaStream_t, const double*, const int*);
template cudaError_t batch_update_s<float>(const BatchSeg*, int, int, float*, const float*, PcgScalars*,
                                           cudaStream_t, const float*, const int*);

template <typename VT>
cudaError_t batch_absmax_init(const BatchSeg* segs, int nseg, int blocks, const VT* b, PcgScalars* sc,
                              double tol, int maxit, const double* tols, const int* maxits, cudaStream_t st) {
  ++g_kernel_launches;
  batch_absmax_init_kernel<VT><<<blocks, 256, 0, st>>>(segs, nseg, b, sc, tol, maxit, tols, maxits);
  return cudaGetLastError();
}
template cudaError_t batch_absmax_init<double>(const BatchSeg*, int, int, const double*, PcgScalars*, double,
                                               int, const double*, const int*, cudaStream_t);
template cudaError_t batch_absmax_init<float>(const BatchSeg*, int, int, const float*, PcgScalars*, double, int,
                                              const double*, const int*, cudaStream_t);

// One block per scene: z.r from the scene's per-line partials with line_sum,
// the same order the single-scene backward sweep's last CTA uses.
template <typename DT>
__global__ void __launch_bounds__(256) batch_bwd_reduce_kernel(const BatchSeg* __restrict__ segs,
                                                               const double* __restrict__ lpart, PcgScalars* sc,
                                                               int mode) {
  __shared__ double s[256];
  const int q = blockIdx.x;
  PcgScalars* S = sc + q;
  if (*(volatile int*)&S->done) return;
  const BatchSeg& G = segs[q];
  const double rho_new = line_sum<std::is_same<DT, float>::value>(lpart + G.line_base, (long long)G.nj * G.nk, s);
  if (threadIdx.x != 0) return;
  if (mode == 0) {
    S->rho = rho_new;
    if (rho_new == 0.0 || rho_new != rho_new) { S->status = -5; S->done = 1; }
  } else {
    S->beta = std::is_same<DT, float>::value ? (double)__fdiv_rn((float)rho_new, (float)S->rho)
                                             : __ddiv_rn(rho_new, S->rho);
    S->rho = rho_new;
  }
}
template <typename DT>
cudaError_t batch_bwd_reduce(const BatchSeg* segs, int nseg, const double* line_partials, PcgScalars* sc, int mode,
                             cudaStream_t st) {
  ++g_kernel_launches;
  batch_bwd_reduce_kernel<DT><<<nseg, 256, 0, st>>>(segs, line_partials, sc, mode);
  return cudaGetLastError();
}
template cudaError_t batch_bwd_reduce<double>(const BatchSeg*, int, const double*, PcgScalars*, int, cudaStream_t);
template cudaError_t batch_bwd_reduce<float>(const BatchSeg*, int, const double*, PcgScalars*, int, cudaStream_t);

__global__ void offset_lines_kernel(Line* __restrict__ lines, long long nlines, long long base) {
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < nlines;
       q += (long long)gridDim.x * blockDim.x)
    lines[q].off += (int)base;
}
cudaError_t offset_lines(Line* lines, long long nlines, long long base, cudaStream_t st) {
  if (base == 0 || nlines <= 0) return cudaSuccess;
  ++g_kernel_launches;
  offset_lines_kernel<<<(unsigned)std::min<long long>((nlines + 255) / 256, 148LL * 8), 256, 0, st>>>(lines, nlines,
                                                                                                   base);
  return cudaGetLastError();
}

__global__ void refine_update_kernel(double* __restrict__ x64, const float* __restrict__ e32, long long M) {
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < M; c += (long long)gridDim.x * blockDim.x)
    x64[c] += (double)e32[c];
}
cudaError_t refine_update(double* x64, const float* e32, long long M, cudaStream_t st) {
  int blocks = (int)std::min<long long>((M + 255) / 256, 148LL * 16);
  if (blocks < 1) blocks = 1;
  ++g_kernel_launches;
  refine_update_kernel<<<blocks, 256, 0, st>>>(x64, e32, M);
  return cudaGetLastError();
}

}  // namespace xfp
