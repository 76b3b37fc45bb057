// xfp_noalloc.cu -- xfp_rhs_inf_noalloc_f64: |b|_inf of the pressure system's
// right-hand side, computed without allocating any device memory.
//
// Who needs it: code that runs where cudaMalloc/cudaFree are off limits --
// a real-time simulation loop that must not stall (cudaFree synchronises the
// whole device), or a host application whose own allocator has reserved the
// device memory and hands out nothing else.  Such callers can still check how
// divergent a velocity field is (the scale the PCG tolerance is measured
// against) before or after a projection.
//
// The kernel is a variant of the solve's |b|_inf reduction: instead of reading
// the assembled right-hand side from the context's scratch pool, each thread
// forms b for its cells straight from material/u/v/w and the per-block maxima
// go to one file-scope __device__ array instead of allocated scratch.  b is
// the variational matrix's right-hand side with no body force, formed in the
// assembly kernel's operation order, so the result equals bit for bit the
// stats.b_inf of an FP64 solve with options.matrix = XFP_MATRIX_VARIATIONAL
// (xfp_solve_f64 / xfp_project_f64).  It is not the b of a normal-matrix solve
// (which drops solid rows) nor of xfp_project_step_* (which adds force*dt to
// the faces first).  A NaN anywhere in b makes the result NaN, so a blown-up
// field is not reported as finite.
//
// Limits and sharing:
//  * the array holds kMaxBlocks block maxima of kCellsPerBlock cells each, so
//    grids above kMaxCells (268,435,456) cells are rejected; it costs 128 KiB
//    of device memory on every GPU that loads this library's device code, held
//    until the process exits;
//  * every call uses the same array; the completion counter must start each
//    call at zero, so every call clears it on its stream before the kernel,
//    and the last block leaves it at zero.  Two calls whose kernels overlap on
//    the GPU (different streams, or different host threads) race on the array
//    and may return wrong values: serialise them.
//  * every call looks up the array's device address with cudaGetSymbolAddress
//    in the current device's context (a lookup, no allocation), so the address
//    stays right after a cudaDeviceReset re-creates the context.  The first
//    call on a device also loads this file's device code into the context;
//    make that first call before any stream capture begins.
#include <cmath>
#include <cstdio>

#include "xfp.h"
#include "xfp_common.cuh"
#include "xfp_kernels.h"

namespace xfp {
namespace {

constexpr int kThreads = 256;
constexpr int kCellsPerThread = 64;
constexpr long long kCellsPerBlock = (long long)kThreads * kCellsPerThread;  // 16384
constexpr int kMaxBlocks = 16384;
constexpr long long kMaxCells = kCellsPerBlock * kMaxBlocks;  // 2^28

struct RhsInfScratch {
  double block_max[kMaxBlocks];  // one partial per block, written before `done` counts it
  unsigned int done;             // blocks finished in the current call; must start at 0
};

}  // namespace

// The only device memory this entry point uses.  In host code this name is a
// host-side stand-in, not a device address: host code passes the address
// looked up by cudaGetSymbolAddress instead.
static __device__ __align__(256) RhsInfScratch g_rhs_inf_scratch;

namespace {

// a max that keeps a NaN from either operand
__device__ __forceinline__ double nan_max(double a, double b) { return (a > b || a != a) ? a : b; }

__device__ __forceinline__ size_t nu_ix(int ni, int nj, int i, int j, int k) {
  return ((size_t)k * nj + j) * (size_t)(ni + 1) + i;
}
__device__ __forceinline__ size_t nv_ix(int ni, int nj, int i, int j, int k) {
  return ((size_t)k * (nj + 1) + j) * (size_t)ni + i;
}
__device__ __forceinline__ size_t nw_ix(int ni, int nj, int i, int j, int k) {
  return ((size_t)k * nj + j) * (size_t)ni + i;
}

// b of cell (i,j,k), as the assembly forms it (variational_pressuresolver.cpp:
// 294-320): fluid cells sum vsign*u*m over neighbours +i,-i,+j,-j,+k,-k (half
// weight across solid faces); a solid cell collects vsign*u*0.5*m from its
// fluid neighbours in the reference's loop order -x,-y,-z,+z,+y,+x.
__device__ double cell_rhs(const uint8_t* __restrict__ mat, const double* __restrict__ u,
                           const double* __restrict__ v, const double* __restrict__ w,
                           const double* __restrict__ wu, const double* __restrict__ wv,
                           const double* __restrict__ ww, int ni, int nj, int nk, int i, int j, int k) {
  const size_t nn = (size_t)ni * nj;
  const uint8_t m = mat[(size_t)k * nn + (size_t)j * ni + i];
  if (m != MAT_FLUID && m != MAT_SOLID) return 0.0;
  double bb = 0.0;
  const int fluid_order[6] = {0, 1, 2, 3, 4, 5};
  const int solid_order[6] = {1, 3, 5, 4, 2, 0};
#pragma unroll
  for (int t = 0; t < 6; ++t) {
    const int nb = m == MAT_FLUID ? fluid_order[t] : solid_order[t];
    const int di = nb == 0 ? 1 : nb == 1 ? -1 : 0;
    const int dj = nb == 2 ? 1 : nb == 3 ? -1 : 0;
    const int dk = nb == 4 ? 1 : nb == 5 ? -1 : 0;
    const int ii = i + di, jj = j + dj, kk = k + dk;
    if (ii < 0 || jj < 0 || kk < 0 || ii >= ni || jj >= nj || kk >= nk) continue;
    const uint8_t mn = mat[(size_t)kk * nn + (size_t)jj * ni + ii];
    if (m == MAT_SOLID && mn != MAT_FLUID) continue;
    const double vs = (di + dj + dk) > 0 ? -1.0 : 1.0;
    const int fi = i + (di > 0), fj = j + (dj > 0), fk = k + (dk > 0);
    double uf, mf;
    if (di) {
      const size_t f = nu_ix(ni, nj, fi, fj, fk);
      uf = u[f]; mf = wu ? wu[f] : 1.0;
    } else if (dj) {
      const size_t f = nv_ix(ni, nj, fi, fj, fk);
      uf = v[f]; mf = wv ? wv[f] : 1.0;
    } else {
      const size_t f = nw_ix(ni, nj, fi, fj, fk);
      uf = w[f]; mf = ww ? ww[f] : 1.0;
    }
    if (m == MAT_FLUID && mn != MAT_SOLID)
      bb = add_rn(bb, mul_rn(mul_rn(vs, uf), mf));
    else
      bb = add_rn(bb, mul_rn(mul_rn(mul_rn(vs, uf), 0.5), mf));
  }
  return bb;
}

__global__ void __launch_bounds__(kThreads) rhs_inf_kernel(
    const uint8_t* __restrict__ mat, const double* __restrict__ u, const double* __restrict__ v,
    const double* __restrict__ w, const double* __restrict__ wu, const double* __restrict__ wv,
    const double* __restrict__ ww, int ni, int nj, int nk, RhsInfScratch* __restrict__ scratch,
    double* __restrict__ b_inf) {
  const long long ncells = (long long)ni * nj * nk;
  const long long base = (long long)blockIdx.x * kCellsPerBlock;
  double mx = 0.0;
  for (int q = 0; q < kCellsPerThread; ++q) {
    const long long c = base + (long long)q * kThreads + threadIdx.x;
    if (c >= ncells) break;
    const int i = (int)(c % ni);
    const long long jk = c / ni;
    const int j = (int)(jk % nj), k = (int)(jk / nj);
    mx = nan_max(fabs(cell_rhs(mat, u, v, w, wu, wv, ww, ni, nj, nk, i, j, k)), mx);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = nan_max(mx, __shfl_xor_sync(XFP_FULL, mx, o));
  __shared__ double s_warp[kThreads / 32];
  __shared__ bool s_last;
  if ((threadIdx.x & 31) == 0) s_warp[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int q = 0; q < kThreads / 32; ++q) t = nan_max(t, s_warp[q]);
    scratch->block_max[blockIdx.x] = t;
    __threadfence();
    s_last = atomicAdd(&scratch->done, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last) return;
  // last block: every other block's partial is visible (written before its fence)
  __threadfence();
  double t = 0.0;
  for (int q = threadIdx.x; q < (int)gridDim.x; q += kThreads)
    t = nan_max(t, *(volatile const double*)&scratch->block_max[q]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) t = nan_max(t, __shfl_xor_sync(XFP_FULL, t, o));
  if ((threadIdx.x & 31) == 0) s_warp[threadIdx.x >> 5] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = 0.0;
    for (int q = 0; q < kThreads / 32; ++q) r = nan_max(r, s_warp[q]);
    *b_inf = r;
    scratch->done = 0;  // leave the counter ready for the next call
  }
}

int report(char* err, size_t err_len, int rc, const char* msg) {
  if (err && err_len) snprintf(err, err_len, "%s", msg);
  return rc;
}

// Device-side pointers only: a host pointer would fault in the kernel.
bool on_device(const void* p, int dev) {
  if (!p) return true;
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (a.type == cudaMemoryTypeManaged) return true;
  return a.type == cudaMemoryTypeDevice && a.device == dev;
}

}  // namespace
}  // namespace xfp

extern "C" int xfp_rhs_inf_noalloc_f64(int ni, int nj, int nk, const uint8_t* material, const double* u,
                                       const double* v, const double* w, const double* wu,
                                       const double* wv, const double* ww, double* b_inf, void* stream,
                                       char* err, size_t err_len) {
  using namespace xfp;
  if (err && err_len) err[0] = '\0';
  if (ni < 1 || nj < 1 || nk < 1) return report(err, err_len, XFP_ERR_ARGS, "grid sizes must be >= 1");
  const long long ncells = (long long)ni * nj * nk;
  if (ncells > kMaxCells) {
    char msg[160];
    snprintf(msg, sizeof msg,
             "grid of %lld cells exceeds the no-allocation limit of %lld cells "
             "(its fixed scratch holds %d block maxima)",
             ncells, kMaxCells, kMaxBlocks);
    return report(err, err_len, XFP_ERR_ARGS, msg);
  }
  if (!material || !u || !v || !w || !b_inf)
    return report(err, err_len, XFP_ERR_ARGS, "material, u, v, w and b_inf must not be NULL");
  if ((wu == nullptr) != (wv == nullptr) || (wu == nullptr) != (ww == nullptr))
    return report(err, err_len, XFP_ERR_ARGS, "face weights: pass all three or none");
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) {
    cudaGetLastError();
    return report(err, err_len, XFP_ERR_CUDA, "no usable current CUDA device");
  }
  const void* ptrs[] = {material, u, v, w, wu, wv, ww, b_inf};
  for (const void* p : ptrs)
    if (!on_device(p, dev))
      return report(err, err_len, XFP_ERR_ARGS,
                    "every array must be device (or managed) memory on the current device");
  // The array's address in the current context, looked up on every call: a
  // context re-created after cudaDeviceReset maps the array elsewhere.
  void* sym = nullptr;
  cudaError_t se = cudaGetSymbolAddress(&sym, g_rhs_inf_scratch);
  if (se != cudaSuccess || sym == nullptr) {
    cudaGetLastError();
    char msg[160];
    snprintf(msg, sizeof msg, "looking up the fixed scratch failed: %s", cudaGetErrorString(se));
    return report(err, err_len, XFP_ERR_CUDA, msg);
  }
  RhsInfScratch* scratch = static_cast<RhsInfScratch*>(sym);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemsetAsync(&scratch->done, 0, sizeof(unsigned int), st);
  if (e == cudaSuccess) {
    const unsigned blocks = (unsigned)((ncells + kCellsPerBlock - 1) / kCellsPerBlock);
    ++g_kernel_launches;
    rhs_inf_kernel<<<blocks, kThreads, 0, st>>>(material, u, v, w, wu, wv, ww, ni, nj, nk, scratch, b_inf);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    char msg[160];
    snprintf(msg, sizeof msg, "launch failed: %s", cudaGetErrorString(e));
    return report(err, err_len, XFP_ERR_CUDA, msg);
  }
  return XFP_OK;
}
