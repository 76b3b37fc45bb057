// xfp_hostio.cu -- host-pointer mode, sparse face transfer.
//
// A projection reads the face velocities of fluid cells only (the assembly:
// divergence and weights of fluid cells, variational_pressuresolver.cpp:
// 245-321) and changes only faces with a fluid side (applyPressure, :161-200;
// the body force of _applyForces, FluidSimulator.cpp:430-470, moves the same
// faces).  When the caller's velocity arrays are page-locked host memory that
// the device can address in place, only those faces cross PCIe: each face row
// (the faces along i at one (j, k)) copies the span between the first and the
// last face that borders a fluid cell, read straight from host memory before
// the solve and written straight back after the apply.  Faces outside the
// spans are neither read nor written, so the caller's values there stay as
// they were, which is what the reference leaves there too.
#include <algorithm>
#include <climits>

#include "xfp_common.cuh"
#include "xfp_kernels.h"

namespace xfp {

// Fluid span of every x-line: {first fluid i, last fluid i + 1}, {0, 0} when
// the line has none.  One warp per line.
__global__ void fluid_span_kernel(const uint8_t* __restrict__ mat, int ni, int nj, int nk,
                                  int2* __restrict__ span) {
  const int lane = threadIdx.x & 31;
  const long long line = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (line >= (long long)nj * nk) return;
  const uint8_t* row = mat + line * ni;
  int lo = INT_MAX, hi = -1;
  for (int i = lane; i < ni; i += 32) {
    if (row[i] == MAT_FLUID) {
      lo = min(lo, i);
      hi = max(hi, i);
    }
  }
  lo = __reduce_min_sync(XFP_FULL, lo);
  hi = __reduce_max_sync(XFP_FULL, hi);
  if (lane == 0) span[line] = hi >= 0 ? make_int2(lo, hi + 1) : make_int2(0, 0);
}

// Face row r of `axis` -> the span of its faces that border a fluid cell.
// u (nk, nj, ni+1): row k*nj + j borders line (j, k): faces lo .. hi (cells
// lo-1 | lo up to hi | hi+1).  v (nk, nj+1, ni): row k*(nj+1) + j borders lines
// (j-1, k) and (j, k).  w (nk+1, nj, ni): row k*nj + j borders lines (j, k-1)
// and (j, k).
__device__ __forceinline__ int2 face_row_span(const int2* __restrict__ span, int ni, int nj, int nk, int axis,
                                              long long r) {
  auto join = [](int2 a, int2 b) -> int2 {
    if (a.y <= a.x) return b;
    if (b.y <= b.x) return a;
    return make_int2(min(a.x, b.x), max(a.y, b.y));
  };
  if (axis == 0) {
    const int2 s = span[r];
    return s.y > s.x ? make_int2(s.x, s.y + 1) : s;
  }
  if (axis == 1) {
    const int j = (int)(r % (nj + 1)), k = (int)(r / (nj + 1));
    int2 s = make_int2(0, 0);
    if (j > 0) s = join(s, span[(long long)k * nj + j - 1]);
    if (j < nj) s = join(s, span[(long long)k * nj + j]);
    return s;
  }
  const int j = (int)(r % nj), k = (int)(r / nj);
  int2 s = make_int2(0, 0);
  if (k > 0) s = join(s, span[(long long)(k - 1) * nj + j]);
  if (k < nk) s = join(s, span[(long long)k * nj + j]);
  return s;
}

// Copies the fluid-bordering span of every face row of `axis` from src to dst
// (the same element indices), one warp per row, and adds the bytes copied to
// *bytes (one atomic per block).
template <typename T>
__global__ void face_rows_copy_kernel(const int2* __restrict__ span, int ni, int nj, int nk, int axis,
                                      const T* __restrict__ src, T* __restrict__ dst,
                                      unsigned long long* __restrict__ bytes) {
  __shared__ unsigned long long blk;
  if (threadIdx.x == 0) blk = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int len = ni + (axis == 0);
  const long long nrows = (long long)(nj + (axis == 1)) * (nk + (axis == 2));
  const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
  unsigned long long mine = 0;
  for (long long r = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < nrows; r += warps) {
    const int2 s = face_row_span(span, ni, nj, nk, axis, r);
    if (s.y <= s.x) continue;
    const size_t base = (size_t)r * len;
    // four loads in flight per lane before the stores
    int i = s.x + lane;
    for (; i + 96 < s.y; i += 128) {
      const T a = src[base + i], b = src[base + i + 32], c = src[base + i + 64], d = src[base + i + 96];
      dst[base + i] = a;
      dst[base + i + 32] = b;
      dst[base + i + 64] = c;
      dst[base + i + 96] = d;
    }
    for (; i < s.y; i += 32) dst[base + i] = src[base + i];
    mine += (unsigned long long)(s.y - s.x) * sizeof(T);
  }
  if (lane == 0 && mine) atomicAdd(&blk, mine);
  __syncthreads();
  if (threadIdx.x == 0 && blk) atomicAdd(bytes, blk);
}

cudaError_t fluid_spans(const uint8_t* mat, int ni, int nj, int nk, int2* span, cudaStream_t st) {
  const long long nlines = (long long)nj * nk;
  if (nlines == 0) return cudaSuccess;
  ++g_kernel_launches;
  fluid_span_kernel<<<(unsigned)((nlines + 7) / 8), 256, 0, st>>>(mat, ni, nj, nk, span);
  return cudaGetLastError();
}

template <typename T>
cudaError_t face_rows_copy(const int2* span, int ni, int nj, int nk, const T* const src[3], T* const dst[3],
                           unsigned long long* bytes, cudaStream_t st) {
  for (int axis = 0; axis < 3; ++axis) {
    const long long nrows = (long long)(nj + (axis == 1)) * (nk + (axis == 2));
    const unsigned blocks = (unsigned)std::min<long long>((nrows + 7) / 8, 148 * 16);
    ++g_kernel_launches;
    face_rows_copy_kernel<T><<<blocks, 256, 0, st>>>(span, ni, nj, nk, axis, src[axis], dst[axis], bytes);
  }
  return cudaGetLastError();
}
template cudaError_t face_rows_copy<float>(const int2*, int, int, int, const float* const[3], float* const[3],
                                          unsigned long long*, cudaStream_t);
template cudaError_t face_rows_copy<double>(const int2*, int, int, int, const double* const[3], double* const[3],
                                           unsigned long long*, cudaStream_t);

}  // namespace xfp
