// xfp_steps.cu -- the simulator steps either side of the projection, on the
// device: the constant body force before it and the velocity extrapolation
// after it (xFluid/xFluid/FluidSimulator.cpp).
//
//   apply_forces  FluidSimulator::_applyForces              :429-499
//   extrapolate   FluidSimulator::_expolateVelocity(layers) :511-650
//
// The extrapolation is a breadth-first walk over the face grid of each axis,
// layer by layer.  A face of layer L takes the average of its neighbours of
// layer L-1, in the reference's neighbour order (+i,-i,+j,-j,+k,-k,
// xfluidutil.cpp:33-41), and the unmarked neighbours of layer L become layer
// L+1.  No face reads a value written in its own layer and a face's layer does
// not depend on the order a layer is visited in, so each layer is one
// data-parallel pass and the FP64 result is bit-identical to the sequential
// reference.  Bandwidth-bound stencil work: grid-stride loops over the faces.
#include <algorithm>

#include "xfp_common.cuh"
#include "xfp_kernels.h"

namespace xfp {
namespace {

__device__ __forceinline__ bool fluid_at(const uint8_t* __restrict__ mat, int ni, int nj, int nk, int i, int j, int k) {
  return i >= 0 && j >= 0 && k >= 0 && i < ni && j < nj && k < nk &&
         mat[(size_t)k * ni * nj + (size_t)j * ni + i] == MAT_FLUID;
}

// a face of `axis` at (i,j,k) lies between cells (i,j,k) and (i,j,k) - e_axis
__device__ __forceinline__ bool borders_fluid(const uint8_t* __restrict__ mat, int ni, int nj, int nk, int axis, int i,
                                              int j, int k) {
  return fluid_at(mat, ni, nj, nk, i, j, k) ||
         fluid_at(mat, ni, nj, nk, i - (axis == 0), j - (axis == 1), k - (axis == 2));
}

template <typename FT>
__global__ void forces_kernel(const uint8_t* __restrict__ mat, int ni, int nj, int nk, int axis, FT* __restrict__ f,
                              FT dv) {
  const int si = ni + (axis == 0), sj = nj + (axis == 1), sk = nk + (axis == 2);
  const size_t n = (size_t)si * sj * sk;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(idx % si), j = (int)((idx / si) % sj), k = (int)(idx / ((size_t)si * sj));
    if (borders_fluid(mat, ni, nj, nk, axis, i, j, k)) f[idx] = add_rn(f[idx], dv);
  }
}

// layer 0: the faces of fluid cells (:547-560)
__global__ void xmark_init_kernel(const uint8_t* __restrict__ mat, int ni, int nj, int nk, int axis,
                                  short* __restrict__ mk) {
  const int si = ni + (axis == 0), sj = nj + (axis == 1), sk = nk + (axis == 2);
  const size_t n = (size_t)si * sj * sk;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(idx % si), j = (int)((idx / si) % sj), k = (int)(idx / ((size_t)si * sj));
    mk[idx] = borders_fluid(mat, ni, nj, nk, axis, i, j, k) ? 0 : -1;
  }
}

// One layer: faces of layer L (L >= 1) take the average of their layer-(L-1)
// neighbours (:599-625); unmarked faces next to layer L become layer L+1
// (:628-637; with L = 0 this is the first layer, :565-590).
template <typename FT>
__global__ void xlayer_kernel(short* __restrict__ mk, FT* __restrict__ f, int si, int sj, int sk, int L) {
  const size_t n = (size_t)si * sj * sk;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(idx % si), j = (int)((idx / si) % sj), k = (int)(idx / ((size_t)si * sj));
    const short m = mk[idx];
    if (m != -1 && !(L >= 1 && m == L)) continue;
    FT sum = FT(0);
    int count = 0;
    bool next = false;
#pragma unroll
    for (int nb = 0; nb < 6; ++nb) {
      const int a = i + (nb == 0) - (nb == 1), b = j + (nb == 2) - (nb == 3), c = k + (nb == 4) - (nb == 5);
      if (a < 0 || b < 0 || c < 0 || a >= si || b >= sj || c >= sk) continue;
      const size_t q = (size_t)c * si * sj + (size_t)b * si + a;
      const short mq = mk[q];
      if (m == L && mq == L - 1) {
        sum = add_rn(sum, f[q]);
        ++count;
      }
      if (m == -1 && mq == L) next = true;
    }
    if (m == L && count > 0) f[idx] = div_rn(sum, FT(count));
    if (m == -1 && next) mk[idx] = (short)(L + 1);
  }
}

// VariationalPressureSolver::_calculate_divergience
// (variationalpressure/variational_pressuresolver.cpp:526-597): per fluid cell
// the sum of +u(low face) - u(high face) over the axes, a face counted only when
// the cell across it is not solid (outside the grid counts as solid); 0 for
// other cells.  Six additions from 0 in the reference's order.
template <typename FT>
__global__ void divergence_kernel(const uint8_t* __restrict__ mat, int ni, int nj, int nk, const FT* __restrict__ u,
                                  const FT* __restrict__ v, const FT* __restrict__ w, FT* __restrict__ div) {
  const size_t n = (size_t)ni * nj * nk;
  auto solid_at = [&](int i, int j, int k) {
    return !(i >= 0 && j >= 0 && k >= 0 && i < ni && j < nj && k < nk) ||
           mat[(size_t)k * ni * nj + (size_t)j * ni + i] == MAT_SOLID;
  };
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(c % ni), j = (int)((c / ni) % nj), k = (int)(c / ((size_t)ni * nj));
    FT d = FT(0);
    if (mat[c] == MAT_FLUID) {
      const size_t uu = (size_t)k * (ni + 1) * nj + (size_t)j * (ni + 1) + i;
      const size_t vv = (size_t)k * ni * (nj + 1) + (size_t)j * ni + i;
      const size_t ww = c;
      if (!solid_at(i - 1, j, k)) d = add_rn(d, u[uu]);
      if (!solid_at(i + 1, j, k)) d = sub_rn(d, u[uu + 1]);
      if (!solid_at(i, j - 1, k)) d = add_rn(d, v[vv]);
      if (!solid_at(i, j + 1, k)) d = sub_rn(d, v[vv + ni]);
      if (!solid_at(i, j, k - 1)) d = add_rn(d, w[ww]);
      if (!solid_at(i, j, k + 1)) d = sub_rn(d, w[ww + (size_t)ni * nj]);
    }
    div[c] = d;
  }
}

unsigned grid_for(size_t n) { return (unsigned)std::min<size_t>((n + 255) / 256, 148 * 32); }

}  // namespace

template <typename FT>
cudaError_t divergence(const uint8_t* mat, int ni, int nj, int nk, const FT* u, const FT* v, const FT* w, FT* div,
                       cudaStream_t st) {
  ++g_kernel_launches;
  divergence_kernel<FT><<<grid_for((size_t)ni * nj * nk), 256, 0, st>>>(mat, ni, nj, nk, u, v, w, div);
  return cudaGetLastError();
}
template cudaError_t divergence<double>(const uint8_t*, int, int, int, const double*, const double*, const double*,
                                        double*, cudaStream_t);
template cudaError_t divergence<float>(const uint8_t*, int, int, int, const float*, const float*, const float*, float*,
                                       cudaStream_t);

template <typename FT>
cudaError_t apply_forces(const uint8_t* mat, int ni, int nj, int nk, FT* u, FT* v, FT* w, Force3 frc,
                         cudaStream_t st) {
  FT* f[3] = {u, v, w};
  for (int axis = 0; axis < 3; ++axis) {
    if (!frc.axis_on(axis)) continue;
    const size_t n = (size_t)(ni + (axis == 0)) * (nj + (axis == 1)) * (nk + (axis == 2));
    ++g_kernel_launches;
    forces_kernel<FT><<<grid_for(n), 256, 0, st>>>(mat, ni, nj, nk, axis, f[axis], (FT)frc.d[axis]);
  }
  return cudaGetLastError();
}

template <typename FT>
cudaError_t extrapolate(const uint8_t* mat, int ni, int nj, int nk, FT* u, FT* v, FT* w, int layers,
                        short* marker, cudaStream_t st) {
  FT* f[3] = {u, v, w};
  for (int axis = 0; axis < 3; ++axis) {
    const int si = ni + (axis == 0), sj = nj + (axis == 1), sk = nk + (axis == 2);
    const size_t n = (size_t)si * sj * sk;
    ++g_kernel_launches;
    xmark_init_kernel<<<grid_for(n), 256, 0, st>>>(mat, ni, nj, nk, axis, marker);
    for (int L = 0; L <= layers; ++L) {
      ++g_kernel_launches;
      xlayer_kernel<FT><<<grid_for(n), 256, 0, st>>>(marker, f[axis], si, sj, sk, L);
    }
  }
  return cudaGetLastError();
}

template cudaError_t apply_forces<double>(const uint8_t*, int, int, int, double*, double*, double*, Force3,
                                          cudaStream_t);
template cudaError_t apply_forces<float>(const uint8_t*, int, int, int, float*, float*, float*, Force3, cudaStream_t);
template cudaError_t extrapolate<double>(const uint8_t*, int, int, int, double*, double*, double*, int, short*,
                                         cudaStream_t);
template cudaError_t extrapolate<float>(const uint8_t*, int, int, int, float*, float*, float*, int, short*,
                                        cudaStream_t);

}  // namespace xfp
