// xfp_layout.cu -- line-compacted storage layout for one material grid.
//
// Unknown rows are xFluid's: fluid cells and solid cells with a fluid
// neighbour (variational_pressuresolver.cpp:245-321: only fluid cells assemble,
// and each solid neighbour of a fluid cell receives a row).  Every (j,k) x-line
// stores its active span, rounded out to whole groups of XFP_ALIGN cells that
// are aligned to the wavefront (see xfp_common.cuh).
#include <climits>

#include "xfp_common.cuh"
#include "xfp_kernels.h"

namespace xfp {

__device__ __forceinline__ bool is_unknown(const uint8_t* mat, int ni, int nj, int nk, int i, int j,
                                           int k) {
  const size_t nn = (size_t)ni * nj;
  const size_t c = (size_t)k * nn + (size_t)j * ni + i;
  const uint8_t m = mat[c];
  if (m == MAT_FLUID) return true;
  if (m != MAT_SOLID) return false;
  if (i > 0 && mat[c - 1] == MAT_FLUID) return true;
  if (i + 1 < ni && mat[c + 1] == MAT_FLUID) return true;
  if (j > 0 && mat[c - ni] == MAT_FLUID) return true;
  if (j + 1 < nj && mat[c + ni] == MAT_FLUID) return true;
  if (k > 0 && mat[c - nn] == MAT_FLUID) return true;
  if (k + 1 < nk && mat[c + nn] == MAT_FLUID) return true;
  return false;
}

// One warp per x-line: span of unknowns and their count.
__global__ void line_span_kernel(const uint8_t* __restrict__ mat, int ni, int nj, int nk,
                                 Line* __restrict__ lines, int* __restrict__ lens) {
  const int lane = threadIdx.x & 31;
  const long long line = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (line >= (long long)nj * nk) return;
  const int j = (int)(line % nj), k = (int)(line / nj);
  int lo = INT_MAX, hi = -1, cnt = 0;
  for (int i = lane; i < ni; i += 32) {
    if (is_unknown(mat, ni, nj, nk, i, j, k)) {
      lo = min(lo, i);
      hi = max(hi, i);
      ++cnt;
    }
  }
  lo = __reduce_min_sync(XFP_FULL, lo);
  hi = __reduce_max_sync(XFP_FULL, hi);
  cnt = __reduce_add_sync(XFP_FULL, cnt);
  if (lane == 0) {
    Line L = {0, 0, 0, 0};
    if (cnt > 0) {
      // first stored cell S <= lo with S + j + k = 0 (mod XFP_ALIGN): cell i
      // then sits at an address = i + j + k (mod XFP_ALIGN); S may be < 0
      L.lo = lo - ((lo + j + k) & (XFP_ALIGN - 1));
      L.len = ((hi + 1 - L.lo) + XFP_ALIGN - 1) & ~(XFP_ALIGN - 1);
      L.nrows = cnt;
    }
    lines[line] = L;
    lens[line] = L.len;
  }
}

// Single-CTA exclusive scan of line lengths -> offsets; totals into counters.
__global__ void line_scan_kernel(Line* __restrict__ lines, const int* __restrict__ lens,
                                 long long nlines, long long* __restrict__ counters) {
  __shared__ long long s_sum[1024];
  __shared__ long long s_carry;
  __shared__ long long s_rows, s_lines;
  const int t = threadIdx.x, nt = blockDim.x;
  if (t == 0) { s_carry = 0; s_rows = 0; s_lines = 0; }
  __syncthreads();
  long long rows = 0, act = 0;
  for (long long base = 0; base < nlines; base += (long long)nt * 8) {
    long long v[8];
    long long local = 0;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      long long idx = base + (long long)t * 8 + q;
      v[q] = idx < nlines ? lens[idx] : 0;
      local += v[q];
    }
    s_sum[t] = local;
    __syncthreads();
    for (int o = 1; o < nt; o <<= 1) {
      long long add = t >= o ? s_sum[t - o] : 0;
      __syncthreads();
      s_sum[t] += add;
      __syncthreads();
    }
    long long run = s_carry + s_sum[t] - local;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      long long idx = base + (long long)t * 8 + q;
      if (idx < nlines) {
        lines[idx].off = (int)run;
        rows += lines[idx].nrows;
        act += v[q] > 0;
      }
      run += v[q];
    }
    __syncthreads();
    if (t == nt - 1) s_carry += s_sum[t];
    __syncthreads();
  }
  atomicAdd((unsigned long long*)&s_rows, (unsigned long long)rows);
  atomicAdd((unsigned long long*)&s_lines, (unsigned long long)act);
  __syncthreads();
  if (t == 0) {
    counters[0] = s_carry;
    counters[1] = s_rows;
    counters[2] = s_lines;
  }
}

// Tile activity: a tile is a 32 (j) x tile_k (k) block of lines.
__global__ void tile_active_kernel(const Line* __restrict__ lines, int nj, int nk, int tile_k,
                                   int NJt, int NKt, unsigned char* __restrict__ act) {
  const int t = blockIdx.x;
  const int J = t % NJt, K = t / NJt;
  int any = 0;
  for (int q = threadIdx.x; q < 32 * tile_k; q += blockDim.x) {
    const int j = J * 32 + (q & 31), k = K * tile_k + (q >> 5);
    if (j < nj && k < nk && lines[(size_t)k * nj + j].len > 0) any = 1;
  }
  any = __syncthreads_or(any);
  if (threadIdx.x == 0) act[t] = (unsigned char)any;
}

// Active tiles in topological order of the lower sweep: (J+K) ascending, then J.
__global__ void tile_order_kernel(const unsigned char* __restrict__ act, int NJt, int NKt,
                                  int* __restrict__ tiles, long long* __restrict__ counters) {
  if (threadIdx.x != 0) return;
  int n = 0;
  for (int dsum = 0; dsum <= NJt + NKt - 2; ++dsum) {
    const int jlo = max(0, dsum - (NKt - 1)), jhi = min(dsum, NJt - 1);
    for (int J = jlo; J <= jhi; ++J) {
      const int K = dsum - J;
      if (act[(size_t)K * NJt + J]) tiles[n++] = J | (K << 16);
    }
  }
  counters[3] = n;
}

cudaError_t layout_build(const uint8_t* mat, int ni, int nj, int nk, int tile_k, LayoutDev L,
                         cudaStream_t st) {
  const long long nlines = (long long)nj * nk;
  const int wpb = 8;
  ++g_kernel_launches;
  line_span_kernel<<<(unsigned)((nlines + wpb - 1) / wpb), wpb * 32, 0, st>>>(mat, ni, nj, nk, L.lines,
                                                                              L.line_len_scan);
  ++g_kernel_launches;
  line_scan_kernel<<<1, 1024, 0, st>>>(L.lines, L.line_len_scan, nlines, L.counters);
  const int NJt = (nj + 31) / 32, NKt = (nk + tile_k - 1) / tile_k;
  ++g_kernel_launches;
  tile_active_kernel<<<NJt * NKt, 256, 0, st>>>(L.lines, nj, nk, tile_k, NJt, NKt, L.tile_active);
  ++g_kernel_launches;
  tile_order_kernel<<<1, 32, 0, st>>>(L.tile_active, NJt, NKt, L.tiles, L.counters);
  return cudaGetLastError();
}

}  // namespace xfp
