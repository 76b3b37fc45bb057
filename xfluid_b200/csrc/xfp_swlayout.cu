// xfp_swlayout.cu -- the sweep layout: tile table and permutation between the
// line layout and the sweep-ordered copies the triangular solves stream
// (SwTile in xfp_common.cuh describes the order).
#include <algorithm>
#include <climits>

#include "xfp_common.cuh"
#include "xfp_kernels.h"

namespace xfp {
namespace {

// One warp per tile: the forward step span of its lines, exactly as the solve
// kernel derives it (min/max of lo+j+k and lo+len-1+j+k over lines with cells).
__global__ void sw_tiles_kernel(const Line* __restrict__ lines, const int* __restrict__ tiles, int ntiles, int nj,
                                int nk, int nw, int NJt, SwTile* __restrict__ swt, int* __restrict__ tile_pos) {
  const int t = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (t >= ntiles) return;
  const int packed = tiles[t];
  const int J = packed & 0xffff, K = packed >> 16;
  const int j = J * 32 + lane;
  int lo = INT_MAX, hi = INT_MIN;
  for (int w = 0; w < nw; ++w) {
    const int k = K * nw + w;
    if (j < nj && k < nk) {
      const Line L = lines[(size_t)k * nj + j];
      if (L.len > 0) {
        lo = min(lo, L.lo + j + k);
        hi = max(hi, L.lo + L.len - 1 + j + k);
      }
    }
  }
  lo = __reduce_min_sync(XFP_FULL, lo);
  hi = __reduce_max_sync(XFP_FULL, hi);
  if (lane == 0) {
    SwTile s;
    s.off = 0;
    s.g0 = lo == INT_MAX ? 0 : (lo >> 2);
    s.ng = lo == INT_MAX ? 0 : (hi >> 2) - (lo >> 2) + 1;
    swt[t] = s;
    tile_pos[K * NJt + J] = t;
  }
}

// Batch form of sw_tiles_kernel: tile t belongs to scene tile_scene[t], whose
// line table and sizes come from its BatchSeg.
__global__ void sw_tiles_batch_kernel(const int* __restrict__ tiles, const int* __restrict__ tile_scene,
                                      const BatchSeg* __restrict__ segs, int ntiles, int nw, SwTile* __restrict__ swt) {
  const int t = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (t >= ntiles) return;
  const BatchSeg& S = segs[tile_scene[t]];
  const int packed = tiles[t];
  const int J = packed & 0xffff, K = packed >> 16;
  const int j = J * 32 + lane;
  int lo = INT_MAX, hi = INT_MIN;
  for (int w = 0; w < nw; ++w) {
    const int k = K * nw + w;
    if (j < S.nj && k < S.nk) {
      const Line L = S.lines[(size_t)k * S.nj + j];
      if (L.len > 0) {
        lo = min(lo, L.lo + j + k);
        hi = max(hi, L.lo + L.len - 1 + j + k);
      }
    }
  }
  lo = __reduce_min_sync(XFP_FULL, lo);
  hi = __reduce_max_sync(XFP_FULL, hi);
  if (lane == 0) {
    SwTile s;
    s.off = 0;
    s.g0 = lo == INT_MAX ? 0 : (lo >> 2);
    s.ng = lo == INT_MAX ? 0 : (hi >> 2) - (lo >> 2) + 1;
    swt[t] = s;
  }
}

// perm[c] = sweep-layout element of stored cell cell_base + c (line offsets
// in `lines` count from cell 0 of the compact arrays)
__global__ void sw_perm_kernel(const int* __restrict__ cell_line, const Line* __restrict__ lines, int nj, int nw,
                               int NJt, const int* __restrict__ tile_pos, const SwTile* __restrict__ swt, long long M,
                               long long cell_base, int* __restrict__ perm) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < M; c += (long long)gridDim.x * blockDim.x) {
    const int l = cell_line[c];
    const int j = l % nj, k = l / nj;
    const Line L = lines[l];
    const int tau = L.lo + (int)(cell_base + c - L.off) + j + k;
    const SwTile S = swt[tile_pos[(k / nw) * NJt + (j >> 5)]];
    perm[c] = (int)(S.off + ((long long)(k % nw) * S.ng + ((tau >> 2) - S.g0)) * 128 + (j & 31) * 4 + (tau & 3));
  }
}

template <typename T>
__global__ void sw_permute_kernel(T* __restrict__ line, T* __restrict__ sw, const int* __restrict__ perm, long long M,
                                  int dir) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < M; c += (long long)gridDim.x * blockDim.x) {
    if (dir == 0) sw[perm[c]] = line[c];
    else line[c] = sw[perm[c]];
  }
}

}  // namespace

cudaError_t sw_tiles_build(const Line* lines, const int* tiles, int ntiles, int nj, int nk, int nw, int NJt,
                           SwTile* swt, int* tile_pos, cudaStream_t st) {
  if (ntiles <= 0) return cudaSuccess;
  ++g_kernel_launches;
  sw_tiles_kernel<<<(ntiles + 7) / 8, 256, 0, st>>>(lines, tiles, ntiles, nj, nk, nw, NJt, swt, tile_pos);
  return cudaGetLastError();
}

cudaError_t sw_perm_build(const int* cell_line, const Line* lines, int nj, int nw, int NJt, const int* tile_pos,
                          const SwTile* swt, long long M, int* perm, cudaStream_t st, long long cell_base) {
  if (M <= 0) return cudaSuccess;
  ++g_kernel_launches;
  const long long blocks = std::min<long long>((M + 255) / 256, 148LL * 16);
  sw_perm_kernel<<<(unsigned)blocks, 256, 0, st>>>(cell_line, lines, nj, nw, NJt, tile_pos, swt, M, cell_base, perm);
  return cudaGetLastError();
}

cudaError_t sw_tiles_build_batch(const int* tiles, const int* tile_scene, const BatchSeg* segs, int ntiles, int nw,
                                 SwTile* swt, cudaStream_t st) {
  if (ntiles <= 0) return cudaSuccess;
  ++g_kernel_launches;
  sw_tiles_batch_kernel<<<(ntiles + 7) / 8, 256, 0, st>>>(tiles, tile_scene, segs, ntiles, nw, swt);
  return cudaGetLastError();
}

template <typename T>
cudaError_t sw_permute(T* line, T* sw, const int* perm, long long M, int dir, cudaStream_t st) {
  if (M <= 0) return cudaSuccess;
  ++g_kernel_launches;
  const long long blocks = std::min<long long>((M + 255) / 256, 148LL * 16);
  sw_permute_kernel<T><<<(unsigned)blocks, 256, 0, st>>>(line, sw, perm, M, dir);
  return cudaGetLastError();
}
template cudaError_t sw_permute<float>(float*, float*, const int*, long long, int, cudaStream_t);
template cudaError_t sw_permute<double>(double*, double*, const int*, long long, int, cudaStream_t);

}  // namespace xfp
