// xfp_context.h -- the context behind xfp_ctx* and the host helpers shared by
// the single-scene driver (xfp_capi.cu) and the batch driver (xfp_batch.cu).
// Internal to libxfp.
#pragma once

#include <algorithm>
#include <map>
#include <string>
#include <vector>

#include "../../include/xfp.h"
#include "xfp_common.cuh"
#include "xfp_kernels.h"

namespace xfp_host {

constexpr int NBLK_MAX = 148 * 8;   // blocks of the reduction kernels (partials slots)

// A device allocation that only grows.
struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
  cudaError_t ensure(size_t bytes) {
    if (bytes <= cap && p) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    size_t want = std::max<size_t>(bytes, 256);
    cudaError_t e = cudaMalloc(&p, want);
    if (e == cudaSuccess) cap = want;
    return e;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
  template <typename T>
  T* as() const { return reinterpret_cast<T*>(p); }
};

struct BatchState;                      // xfp_batch.cu
void batch_state_free(BatchState* b);

}  // namespace xfp_host

struct xfp_ctx {
  xfp_options opt;
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::string err;
  int nsm = 148;
  using DevBuf = xfp_host::DevBuf;
  // I/O staging (host-pointer mode)
  DevBuf io_mat, io_u, io_v, io_w, io_wu, io_wv, io_ww, io_p, io_gu, io_gv, io_gw;
  // layout
  DevBuf lines, lens, tile_active, tiles, counters, cell_line, group_line;
  // compact arrays
  DevBuf A64[5];                  // diag, ax, ay, az, b (FP64)
  DevBuf A32[5];                  // same in FP32
  DevBuf F64[6], F32[6];          // factor scratch: L and missing per direction
  DevBuf inv64, inv32, L32[3];
  DevBuf x64, r64, x32, r32, s32, z32, s64, z64, dense;
  // control
  DevBuf ctl, scal, scal2, partials, tpartials, sy, sz, trace;
  // particle steps (xfp_particles.cu): staged particles and field, bin keys,
  // indices, boxes, positions, bin starts, box spans, sort/scan scratch
  DevBuf part_io, phi_io, part_key, part_idx, part_box, part_pos, part_sbox, part_spos, part_start, part_span,
      part_tmp;
  // sweep layout (SwTile): tile table, (K,J) -> tile map, cell -> element map
  // and the copies the solves stream (lx, ly, lz, inv, r, y; 8 bytes per
  // element covers every precision)
  DevBuf swt, tile_pos, sw_perm, sw_l[3], sw_inv, sw_r, sw_y;
  // the triangular solves' tile-boundary rows (SweepData::bk, bj), and the
  // largest ni of the layout, which sets the rows per tile
  DevBuf bnd;
  int bnd_ni = 0;
  // host-pointer mode: fluid span per x-line and the two byte counters of
  // the sparse face transfer; bytes moved by the current call; whether its
  // velocities went face-sparse; XFP_HOST_FACES=full turns the sparse
  // transfer off
  DevBuf hio_span, hio_bytes;
  // host-pointer mode: a second stream for the transfers that can run beside
  // the compute stream (the face gather beside the layout build, the dense
  // pressure download beside the apply), and its events; io_pending: the
  // compute stream has still to wait for io_in before it reads the faces
  cudaStream_t io_stream = nullptr;
  cudaEvent_t ev_io_mat = nullptr, ev_io_in = nullptr, ev_io_p = nullptr;
  bool io_pending = false;
  long long h2d_bytes = 0, d2h_bytes = 0;
  int host_faces = 0;
  int host_sparse_ok = 1;
  // xfp_project_step_*: body force fused into assembly and apply, and the
  // extrapolation layers run after the apply (zero outside such a call);
  // xmarker is the extrapolation's layer-marker scratch
  xfp::Force3 force;
  int step_layers = 0;
  DevBuf xmarker;
  long long Msw = 0;
  bool tracing = false;
  // FP32/mixed triangular solves stage their group blocks through shared
  // memory with cp.async (1, the default) or load them into registers (0,
  // XFP_STAGE_SOLVES=0)
  int stage_solves = 1;
  // block cap of the PCG loop's SpMV: 148 x 4 measured best at 256^3 (37.4 us
  // per launch, against 38.7 at 148 x 8 and 54.5 at 148 x 2).  XFP_VEC_BLOCKS
  // overrides, within [148, NBLK_MAX]; the dot's reduction order follows it.
  int vec_blocks = 148 * 4;
  // block cap of the x/r update (two groups in flight per thread): 148 x 2
  // measured best at 256^3 (20.6 us, against 21.5 at 148 x 4 and 26.0 at
  // 148 x 8).  Its |r|_inf is a max, the same in any order.  XFP_XR_BLOCKS
  // overrides, within [148, NBLK_MAX].
  int xr_blocks = 148 * 2;
  // CUDA events around the PCG loop's solve and vector-kernel launches
  // (xfp_stats.ms_sweeps, ms_vec), on every event_every-th iteration; 0 (the
  // default) records none.  An event between two launches serialises them:
  // events on every launch cost 1.3 ms of a 21.8 ms projection at 256^3.
  // XFP_KERNEL_EVENTS=N sets it.
  int event_every = 0;
  int sweep_ord = 0;              // triangular-solve launches of the current PCG loop
  std::vector<int> sweep_ord_of;  // per timed sweep entry: its launch ordinal
  // block cap of the PCG loop's s update: 148 x 8 measured best at 256^3
  // (14.7 us per launch, against 17.0 at 148 x 16, with two groups in flight
  // per thread).  XFP_S_BLOCKS overrides, within [148, 148 x 32].
  int s_blocks = 148 * 8;
  // sizes of the current layout
  int ni = 0, nj = 0, nk = 0, NJt = 0, NKt = 0, nw = 8;
  long long M = 0, rows = 0, nlines_act = 0, ntiles = 0;
  long long nlines_all = 0;       // lines of the layout (nj*nk, or the whole batch's)
  xfp::PcgScalars host_sc{};
  // stats
  double ms_setup = 0, ms_factor = 0, ms_solve = 0, ms_apply = 0;
  int iters = 0, refinements = 0;
  double res = 0, bnorm = 0;
  cudaEvent_t ev[8] = {};
  // device timing of the triangular-solve sweeps (pairs of events, read at the end)
  std::vector<cudaEvent_t> sweep_ev;
  int sweep_ev_used = 0;
  // per timed sweep launch (event pair): 1 when it did work, 0 for the
  // launches a PCG loop issues after convergence (they return at once)
  std::vector<char> sweep_work;
  // the PCG loop's vector kernels, timed the same way: event pairs with the
  // kernel kind (0 SpMV + dot, 1 x/r update, 2 s update) and its PCG iteration
  // (launches after the converged iteration return at once and are dropped)
  std::vector<cudaEvent_t> kern_ev;
  std::vector<int> kern_kind, kern_iter;
  int kern_ev_used = 0;
  long long launches = 0;
  // batched scenes (xfp_project_batch_*): buffers, tables and tuning cache
  xfp_host::BatchState* batch = nullptr;
  // single scenes with options.tile_k == 0: tile height picked per grid shape
  std::map<std::string, int> tuned_nw;
  // xfp_debug_expire_next_sweep: the next sweep launch's boundary waits run out
  bool expire_next_sweep = false;
};

namespace xfp_host {

inline int fail(xfp_ctx* ctx, int code, const std::string& msg) {
  if (ctx) ctx->err = msg;
  return code;
}

#define XFP_CUDA(ctx, call)                                                                    \
  do {                                                                                         \
    cudaError_t _e = (call);                                                                   \
    if (_e != cudaSuccess) {                                                                   \
      return ::xfp_host::fail(ctx, _e == cudaErrorMemoryAllocation ? XFP_ERR_NOMEM : XFP_ERR_CUDA, \
                              std::string(#call) + ": " + cudaGetErrorString(_e));             \
    }                                                                                          \
  } while (0)

// Stage an input array on the device (or use it in place).
template <typename T>
int stage_in(xfp_ctx* ctx, DevBuf& buf, const T* src, size_t n, const T** dev) {
  if (src == nullptr) { *dev = nullptr; return XFP_OK; }
  if (ctx->opt.device_pointers) { *dev = src; return XFP_OK; }
  XFP_CUDA(ctx, buf.ensure(n * sizeof(T)));
  XFP_CUDA(ctx, cudaMemcpyAsync(buf.p, src, n * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
  ctx->h2d_bytes += (long long)(n * sizeof(T));
  *dev = buf.as<T>();
  return XFP_OK;
}

// xfp_capi.cu
size_t ncells(int ni, int nj, int nk);
size_t nu(int ni, int nj, int nk);
size_t nv(int ni, int nj, int nk);
size_t nw_(int ni, int nj, int nk);
long long spin_limit(const xfp_ctx* ctx);
int check_dims(xfp_ctx* ctx, int ni, int nj, int nk, const void* mat);
int ensure_compact(xfp_ctx* ctx, int prec);
int check_sweep_error(xfp_ctx* ctx);


// Sweep-layout copies of the factor (after it is final in the solve type)
// and of r; element slots of lanes without a cell stay zero.
template <typename VT, typename IT, typename CT>
int sweep_copies(xfp_ctx* ctx, const VT* const L[3], const IT* inv, const VT* r, xfp::SweepGrid* gs, int ng,
                 xfp::SweepData<VT, IT, CT>* d) {
  if (ctx->ntiles == 0) return XFP_OK;
  const size_t bytes = (size_t)(ctx->Msw + 8) * 8;
  for (auto& b : ctx->sw_l) XFP_CUDA(ctx, b.ensure(bytes));
  XFP_CUDA(ctx, ctx->sw_inv.ensure(bytes));
  XFP_CUDA(ctx, ctx->sw_r.ensure(bytes));
  XFP_CUDA(ctx, ctx->sw_y.ensure(bytes));
  cudaStream_t st = ctx->stream;
  const int* perm = ctx->sw_perm.as<int>();
  for (int q = 0; q < 3; ++q) {
    XFP_CUDA(ctx, cudaMemsetAsync(ctx->sw_l[q].p, 0, (size_t)ctx->Msw * sizeof(VT), st));
    XFP_CUDA(ctx, xfp::sw_permute<VT>(const_cast<VT*>(L[q]), ctx->sw_l[q].as<VT>(), perm, ctx->M, 0, st));
  }
  XFP_CUDA(ctx, cudaMemsetAsync(ctx->sw_inv.p, 0, (size_t)ctx->Msw * sizeof(IT), st));
  XFP_CUDA(ctx, xfp::sw_permute<IT>(const_cast<IT*>(inv), ctx->sw_inv.as<IT>(), perm, ctx->M, 0, st));
  XFP_CUDA(ctx, cudaMemsetAsync(ctx->sw_r.p, 0, (size_t)ctx->Msw * sizeof(VT), st));
  XFP_CUDA(ctx, xfp::sw_permute<VT>(const_cast<VT*>(r), ctx->sw_r.as<VT>(), perm, ctx->M, 0, st));
  d->lxs = ctx->sw_l[0].as<VT>();
  d->lys = ctx->sw_l[1].as<VT>();
  d->lzs = ctx->sw_l[2].as<VT>();
  d->invs = ctx->sw_inv.as<IT>();
  d->rs = ctx->sw_r.as<VT>();
  d->ys = ctx->sw_y.as<VT>();
  // boundary rows: per active tile, one row per wavefront step it can span,
  // 32 k-edge words and nw j-edge words of P 64-bit words each; zeroed when
  // (re)allocated so no stale word can carry a live generation
  const int P = (int)(sizeof(VT) / 4);
  const long long rows = (long long)ctx->bnd_ni + ctx->nw + 36;
  const size_t kwords = (size_t)ctx->ntiles * rows * 32 * P, jwords = (size_t)ctx->ntiles * rows * ctx->nw * P;
  const size_t bbytes = (kwords + jwords) * sizeof(unsigned long long);
  if (ctx->bnd.cap < bbytes || !ctx->bnd.p) {
    XFP_CUDA(ctx, ctx->bnd.ensure(bbytes));
    XFP_CUDA(ctx, cudaMemsetAsync(ctx->bnd.p, 0, ctx->bnd.cap, st));
  }
  d->bk = ctx->bnd.as<unsigned long long>();
  d->bj = d->bk + kwords;
  for (int q = 0; q < ng; ++q) {
    gs[q].swt = ctx->swt.as<xfp::SwTile>();
    gs[q].tile_pos = ctx->tile_pos.as<int>();
    gs[q].brows = (int)rows;
  }
  return XFP_OK;
}

// Line-layout copy of the sweep-ordered solve result (z, or y after a
// forward solve alone).
template <typename VT>
int sweep_result(xfp_ctx* ctx, VT* out) {
  if (ctx->ntiles == 0) return XFP_OK;
  XFP_CUDA(ctx, xfp::sw_permute<VT>(out, ctx->sw_y.as<VT>(), ctx->sw_perm.as<int>(), ctx->M, 1, ctx->stream));
  return XFP_OK;
}

}  // namespace xfp_host
