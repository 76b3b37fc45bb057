// xfp_common.cuh -- shared device helpers and layout structures for libxfp.
//
// Storage layout ("line-compacted"): the grid is cut into x-lines, one per
// (j,k).  Each line that holds an unknown stores the cells [lo, lo+len)
// contiguously at offset `off` in every per-cell array: lo is the first
// unknown moved down by 0..3 cells so that lo + j + k = 0 (mod XFP_ALIGN), len
// is rounded up to a multiple of XFP_ALIGN, and off is a multiple of
// XFP_ALIGN.  Cell (i,j,k) therefore sits at an address = i + j + k (mod
// XFP_ALIGN): every cell of one wavefront hyperplane i+j+k = t has the same
// position inside its aligned group of XFP_ALIGN cells, which is what lets
// the triangular-solve sweeps move whole groups with one vector access.  lo
// may be negative and lo+len may pass ni; cells inside a span that are not
// unknowns (air, uncoupled solid, outside the grid) are padding: zero
// coefficients, zero vectors, null rows.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#define XFP_ALIGN 4
#define XFP_FULL 0xffffffffu
#ifndef XFP_MATRIX_NORMAL   // the same values as include/xfp.h
#define XFP_MATRIX_VARIATIONAL 0
#define XFP_MATRIX_NORMAL 1
#endif

namespace xfp {

enum : uint8_t { MAT_AIR = 0, MAT_FLUID = 1, MAT_SOLID = 2 };

// Per-line record: off (start in compact arrays), lo (first stored i), len
// (stored cells, 0 = line has no unknown), nrows (unknowns on the line).
struct __align__(16) Line {
  int off, lo, len, nrows;
};

// Constant body-force velocity increment (force * dt per axis), added to every
// face that borders a fluid cell, as xFluid's FluidSimulator::_applyForces does
// (FluidSimulator.cpp:429-499): an axis whose |dv| is not above 1e-10 is left
// alone.  on = 0: no force.
struct Force3 {
  double d[3] = {0.0, 0.0, 0.0};
  int on = 0;
  __host__ __device__ bool axis_on(int a) const { return on && (d[a] > 1e-10 || d[a] < -1e-10); }
};

// Sweep-ordered copy ("sweep layout") of the arrays the triangular solves
// stream.  For every active tile, compute warp (k) and group g of 4 forward
// wavefront steps (steps 4g..4g+3) it holds a block of 32 lanes x 4 cells:
// element [off + (w*ng + g - g0)*128 + lane*4 + e] is the cell of line
// (j0+lane, k0+w) at forward step 4g+e, or zero where that line has no cell.
// A warp's group access is then 512 contiguous bytes (4-byte values) instead
// of 32 scattered 16-byte pieces.  g0/ng: the tile's first group and group
// count (its step span, both sweep directions); off: its first element.
struct __align__(16) SwTile {
  long long off;
  int g0, ng;
};

// Control block of the persistent sweep kernels (one per context).
struct SweepCtl {
  unsigned int gen;        // launch generation; stamped words carry it in their high half
  unsigned int finished;   // CTAs finished in the current launch
  unsigned int err;        // nonzero: a bounded wait ran out (XFP_ERR_TIMEOUT)
  unsigned int err_where;  // which wait ran out first (diagnostics)
  int err_tile, err_tau, err_thread, err_op;
  unsigned long long err_word;   // the word the failed wait last saw
  unsigned int err_expect, err_pad;
};

// One scene of a batch: its grid, its slice [base, base+M) of the compact
// arrays, its line table (offsets already global) and the blocks the vector
// kernels give it (line-based and cell-based grids, consecutive per scene).
struct BatchSeg {
  int ni, nj, nk;
  int blk_lines, blk_lines_start;   // line-based kernels (residual)
  int blk_cells, blk_cells_start;   // cell-based kernels (updates, norms)
  int blk_groups, blk_groups_start; // the SpMV (one thread per 4-cell group)
  int tile_base;                    // first slot of this scene's (K, J) -> tile map
  long long base, M;
  const Line* lines;
  double* partials;                 // this scene's reduction slots
  long long line_base;              // first line of this scene in the batch's line table
};

// z.r from one partial per x-line, in an order that depends only on the
// number of lines (never on the sweep's tile shape): 256 contiguous chunks,
// each summed in line order, then a fixed pairwise tree.  Called by every
// thread of a block of at least 256 threads; the sum is returned to all.
template <bool F32>
__device__ __forceinline__ double line_sum(const double* __restrict__ part, long long n, double* s) {
  const int t = threadIdx.x;
  if (t < 256) {
    const long long C = (n + 255) / 256, a = (long long)t * C, b = a + C < n ? a + C : n;
    double acc = 0.0;
    float accf = 0.f;
    for (long long q = a; q < b; ++q) {
      const double v = ((volatile const double*)part)[q];
      if (F32) accf = __fadd_rn(accf, (float)v); else acc = __dadd_rn(acc, v);
    }
    s[t] = F32 ? (double)accf : acc;
  }
  __syncthreads();
  for (int h = 128; h > 0; h >>= 1) {
    if (t < h) s[t] = F32 ? (double)__fadd_rn((float)s[t], (float)s[t + h]) : __dadd_rn(s[t], s[t + h]);
    __syncthreads();
  }
  const double r = s[0];
  __syncthreads();
  return r;
}

// Scalars of one PCG solve, resident on the device.
struct PcgScalars {
  double rho, alpha, beta, res, tolabs, bnorm, dot_tmp;
  int done, iters, status, maxit;
  unsigned int red_count;  // last-block-done counter of the reductions
  unsigned int pad;
};

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ double ld_relaxed(const double* p) {
  double v;
  asm volatile("ld.relaxed.gpu.global.f64 %0, [%1];" : "=d"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ float ld_relaxed(const float* p) {
  float v;
  asm volatile("ld.relaxed.gpu.global.f32 %0, [%1];" : "=f"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned int ld_volatile_u32(const unsigned int* p) {
  return *(const volatile unsigned int*)p;
}

// Rounded arithmetic without contraction: the FP64 path follows xFluid's
// operation order exactly, so no multiply-add may be fused.
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double div_rn(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float div_rn(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double rsqrt_ref(double x) { return __ddiv_rn(1.0, __dsqrt_rn(x)); }
__device__ __forceinline__ float rsqrt_ref(float x) { return __fdiv_rn(1.0f, __fsqrt_rn(x)); }

// One group of XFP_ALIGN (4) consecutive cells of an array, from/to a
// group-aligned index: one 16-byte access (FP32) or two (FP64).  Groups of 8
// with 32-byte accesses were measured too in the sweeps: faster on long full
// lines, slower on the 256^3 blob scene (more padding steps, more registers).
__device__ __forceinline__ void ldg(float (&v)[4], const float* p) {
  const float4 t = *reinterpret_cast<const float4*>(p);
  v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
}
__device__ __forceinline__ void ldg(double (&v)[4], const double* p) {
  const double2 a = reinterpret_cast<const double2*>(p)[0], b = reinterpret_cast<const double2*>(p)[1];
  v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
__device__ __forceinline__ void stg(float* p, const float (&v)[4]) {
  *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void stg(double* p, const double (&v)[4]) {
  reinterpret_cast<double2*>(p)[0] = make_double2(v[0], v[1]);
  reinterpret_cast<double2*>(p)[1] = make_double2(v[2], v[3]);
}
template <typename T>
__device__ __forceinline__ T shfl_up(T v, int d) { return __shfl_up_sync(XFP_FULL, v, d); }
template <typename T>
__device__ __forceinline__ T shfl_down(T v, int d) { return __shfl_down_sync(XFP_FULL, v, d); }

}  // namespace xfp
