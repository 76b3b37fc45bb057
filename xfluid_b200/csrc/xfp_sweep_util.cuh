// xfp_sweep_util.cuh -- device helpers shared by the wavefront kernels
// (factorisation in xfp_sweep.cu, triangular solves in xfp_solve.cu):
// payload <-> 32-bit word conversion, stamped 64-bit hand-off words, grouped
// 4-cell loads/stores and bounded waits with error reporting.
#pragma once

#include <climits>
#include <type_traits>

#include "xfp_common.cuh"
#include "xfp_kernels.h"

namespace xfp {

constexpr int INF_T = INT_MAX;

template <typename T>
struct Pair {
  T a, b;
};

// ---- payload <-> 32-bit words ----
template <typename T>
struct Words {
  static constexpr int P = sizeof(T) / 4;
};
template <typename T>
__device__ __forceinline__ void to_words(const T& v, uint32_t* w) {
  union {
    T v;
    uint32_t w[sizeof(T) / 4];
  } u;
  u.v = v;
#pragma unroll
  for (int p = 0; p < (int)(sizeof(T) / 4); ++p) w[p] = u.w[p];
}
template <typename T>
__device__ __forceinline__ T from_words(const uint32_t* w) {
  union {
    T v;
    uint32_t w[sizeof(T) / 4];
  } u;
#pragma unroll
  for (int p = 0; p < (int)(sizeof(T) / 4); ++p) u.w[p] = w[p];
  return u.v;
}
template <typename T>
__device__ __forceinline__ T shfl_up_any(const T& v) {
  uint32_t w[sizeof(T) / 4];
  to_words(v, w);
#pragma unroll
  for (int p = 0; p < (int)(sizeof(T) / 4); ++p) w[p] = __shfl_up_sync(XFP_FULL, w[p], 1);
  return from_words<T>(w);
}
template <typename T>
__device__ __forceinline__ T shfl_down_any(const T& v) {
  uint32_t w[sizeof(T) / 4];
  to_words(v, w);
#pragma unroll
  for (int p = 0; p < (int)(sizeof(T) / 4); ++p) w[p] = __shfl_down_sync(XFP_FULL, w[p], 1);
  return from_words<T>(w);
}

__device__ __forceinline__ unsigned long long stamped(uint32_t stamp, uint32_t word) {
  return ((unsigned long long)stamp << 32) | word;
}
__device__ __forceinline__ unsigned long long ld_vol64(const unsigned long long* p) {
  return *(const volatile unsigned long long*)p;
}
__device__ __forceinline__ void st_vol64(unsigned long long* p, unsigned long long v) {
  *(volatile unsigned long long*)p = v;
}
__device__ __forceinline__ unsigned long long ld_gpu64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ void st_gpu64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v));
}


struct Spin {
  long long n = 0;
  __device__ __forceinline__ bool step(const SweepCtl* ctl, long long limit) {
    ++n;
    if (n > 256) __nanosleep(n > 8192 ? 256 : 20);
    if ((n & 255) == 0 && ld_volatile_u32(&ctl->err)) return false;
    return n < limit;
  }
};

// Records the first wait that ran out (site, tile, step, thread) and raises
// the error flag every other wait checks.
__device__ __forceinline__ void raise_timeout(SweepCtl* ctl, unsigned where, int tile = -1, int tau = -1,
                                              int op = -1, unsigned long long seen = 0, unsigned expect = 0) {
  if (atomicCAS(&ctl->err, 0u, 1u) == 0u) {
    ctl->err_word = seen;
    ctl->err_expect = expect;
    ctl->err_where = where;
    ctl->err_tile = tile;
    ctl->err_tau = tau;
    ctl->err_thread = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    ctl->err_op = op;
  }
}

// Poll a stamped shared-memory payload until every word carries `stamp`.
__device__ __forceinline__ void trace_wait(const SweepGrid& g, int site, int step) {
  if (g.trace && !ld_volatile_u32(&g.ctl->err)) {
    int* t = g.trace + ((size_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 4;
    *(volatile int*)&t[0] = site;
    *(volatile int*)&t[1] = step;
    *(volatile int*)&t[3] = (int)(threadIdx.x & 31);
  }
}
template <typename T>
__device__ __forceinline__ T poll_smem(const unsigned long long* base, int stride, uint32_t stamp,
                                       const SweepGrid& g, unsigned where) {
  constexpr int P = Words<T>::P;
  uint32_t w[P];
#pragma unroll
  for (int p = 0; p < P; ++p) {
    unsigned long long v = ld_vol64(base + (size_t)p * stride);
    if ((uint32_t)(v >> 32) != stamp) {
      trace_wait(g, (int)where, (int)(stamp & 0xfffff));
      Spin sp;
      do {
        if (!sp.step(g.ctl, g.spin_limit)) { raise_timeout(g.ctl, where, -1, (int)(stamp & 0xfffff), -1, v, stamp); break; }
        v = ld_vol64(base + (size_t)p * stride);
      } while ((uint32_t)(v >> 32) != stamp);
      trace_wait(g, 0, (int)(stamp & 0xfffff));
    }
    w[p] = (uint32_t)v;
  }
  return from_words<T>(w);
}

}  // namespace xfp
