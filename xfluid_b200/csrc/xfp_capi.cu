// xfp_capi.cu -- context, device workspace and the C ABI of libxfp (include/xfp.h).
//
// One call runs, on the context's stream:
//   layout   line table + tile list of the material grid          (xfp_layout.cu)
//   assemble the variational system into the compact layout      (xfp_ops.cu)
//   factor   MIC(0) in natural order                              (xfp_sweep.cu)
//   PCG      spmv+dot / x,r update / forward / backward+dot / s update per
//            iteration, convergence read back every check_every iterations
//   output   pressure scattered to the dense grid, velocity update (project)
// Mixed precision wraps the FP32 PCG in FP64 iterative refinement.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <cstdlib>
#include <cstdint>

#include <cuda.h>

#include "../../include/xfp.h"
#include "xfp_common.cuh"
#include "xfp_context.h"
#include "xfp_kernels.h"

using namespace xfp;

namespace xfp_host {

size_t ncells(int ni, int nj, int nk) { return (size_t)ni * nj * nk; }
size_t nu(int ni, int nj, int nk) { return (size_t)(ni + 1) * nj * nk; }
size_t nv(int ni, int nj, int nk) { return (size_t)ni * (nj + 1) * nk; }
size_t nw_(int ni, int nj, int nk) { return (size_t)ni * nj * (nk + 1); }

long long spin_limit(const xfp_ctx* ctx) {
  double ms = ctx->opt.timeout_ms > 0 ? ctx->opt.timeout_ms : 2000.0;
  return (long long)std::max(1e4, ms * 4000.0);  // ~250 ns per backed-off poll
}


int check_dims(xfp_ctx* ctx, int ni, int nj, int nk, const void* mat) {
  if (!ctx) return XFP_ERR_ARGS;
  if (ni < 1 || nj < 1 || nk < 1) return fail(ctx, XFP_ERR_ARGS, "grid sizes must be >= 1");
  if ((long long)ni + nj + nk >= (1LL << 20) || (long long)ni * nj * nk >= (1LL << 31))
    return fail(ctx, XFP_ERR_ARGS, "grid too large");
  if (nj > 65535 * 32) return fail(ctx, XFP_ERR_ARGS, "nj too large");
  if (!mat) return fail(ctx, XFP_ERR_ARGS, "material is NULL");
  return XFP_OK;
}

// ---------------------------------------------------------------- layout
int build_sweep_layout(xfp_ctx* ctx);

int build_layout(xfp_ctx* ctx, const uint8_t* dmat, int ni, int nj, int nk) {
  const int nw = ctx->nw;
  const long long nlines = (long long)nj * nk;
  const int NJt = (nj + 31) / 32, NKt = (nk + nw - 1) / nw;
  XFP_CUDA(ctx, ctx->lines.ensure(nlines * sizeof(Line)));
  XFP_CUDA(ctx, ctx->lens.ensure((nlines + 1) * sizeof(int)));
  XFP_CUDA(ctx, ctx->tile_active.ensure((size_t)NJt * NKt));
  XFP_CUDA(ctx, ctx->tiles.ensure((size_t)NJt * NKt * sizeof(int)));
  XFP_CUDA(ctx, ctx->counters.ensure(4 * sizeof(long long)));
  LayoutDev L{ctx->lines.as<Line>(), ctx->lens.as<int>(), ctx->tile_active.as<unsigned char>(),
              ctx->tiles.as<int>(), ctx->counters.as<long long>()};
  XFP_CUDA(ctx, layout_build(dmat, ni, nj, nk, nw, L, ctx->stream));
  long long cnt[4];
  XFP_CUDA(ctx, cudaMemcpyAsync(cnt, ctx->counters.p, sizeof(cnt), cudaMemcpyDeviceToHost, ctx->stream));
  XFP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  ctx->ni = ni; ctx->nj = nj; ctx->nk = nk;
  ctx->bnd_ni = ni;
  ctx->NJt = NJt; ctx->NKt = NKt;
  ctx->M = cnt[0]; ctx->rows = cnt[1]; ctx->nlines_act = cnt[2]; ctx->ntiles = cnt[3];
  ctx->nlines_all = nlines;
  XFP_CUDA(ctx, ctx->cell_line.ensure((std::max<long long>(ctx->M, 4) + 8) * sizeof(int)));
  XFP_CUDA(ctx, ctx->group_line.ensure((std::max<long long>(ctx->M, 4) / 4 + 8) * sizeof(int)));
  XFP_CUDA(ctx, build_cell_line(ctx->lines.as<Line>(), nlines, ctx->cell_line.as<int>(), ctx->group_line.as<int>(),
                                ctx->stream));
  return build_sweep_layout(ctx);
}

// Tile table of the sweep layout: per-tile spans on the device, block offsets
// scanned here (tile order), table uploaded again.
int build_sweep_layout(xfp_ctx* ctx) {
  const int nt = (int)ctx->ntiles;
  XFP_CUDA(ctx, ctx->swt.ensure(std::max(nt, 1) * sizeof(SwTile)));
  XFP_CUDA(ctx, ctx->tile_pos.ensure((size_t)std::max(ctx->NJt * ctx->NKt, 1) * sizeof(int)));
  ctx->Msw = 0;
  if (nt == 0) return XFP_OK;
  XFP_CUDA(ctx, sw_tiles_build(ctx->lines.as<Line>(), ctx->tiles.as<int>(), nt, ctx->nj, ctx->nk, ctx->nw, ctx->NJt,
                               ctx->swt.as<SwTile>(), ctx->tile_pos.as<int>(), ctx->stream));
  std::vector<SwTile> t(nt);
  XFP_CUDA(ctx, cudaMemcpyAsync(t.data(), ctx->swt.p, nt * sizeof(SwTile), cudaMemcpyDeviceToHost, ctx->stream));
  XFP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  long long off = 0;
  for (auto& e : t) {
    e.off = off;
    off += (long long)ctx->nw * e.ng * 128;
  }
  ctx->Msw = off;
  if (off >= (1LL << 31)) return fail(ctx, XFP_ERR_ARGS, "grid too large for the sweep layout");
  XFP_CUDA(ctx, cudaMemcpyAsync(ctx->swt.p, t.data(), nt * sizeof(SwTile), cudaMemcpyHostToDevice, ctx->stream));
  XFP_CUDA(ctx, ctx->sw_perm.ensure((size_t)(std::max<long long>(ctx->M, 4) + 8) * sizeof(int)));
  XFP_CUDA(ctx, sw_perm_build(ctx->cell_line.as<int>(), ctx->lines.as<Line>(), ctx->nj, ctx->nw, ctx->NJt,
                              ctx->tile_pos.as<int>(), ctx->swt.as<SwTile>(), ctx->M, ctx->sw_perm.as<int>(),
                              ctx->stream));
  XFP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return XFP_OK;
}


int ensure_compact(xfp_ctx* ctx, int prec) {
  const size_t M = (size_t)std::max<long long>(ctx->M, 4) + 8;
  if (prec == XFP_PREC_F64 || prec == XFP_PREC_MIXED) {
    for (auto& b : ctx->A64) XFP_CUDA(ctx, b.ensure(M * 8));
    for (auto& b : ctx->F64) XFP_CUDA(ctx, b.ensure(M * 8));
    XFP_CUDA(ctx, ctx->inv64.ensure(M * 8));
    XFP_CUDA(ctx, ctx->x64.ensure(M * 8));
    XFP_CUDA(ctx, ctx->r64.ensure(M * 8));
  }
  if (prec == XFP_PREC_F64) {
    XFP_CUDA(ctx, ctx->s64.ensure(M * 8));
    XFP_CUDA(ctx, ctx->z64.ensure(M * 8));
    XFP_CUDA(ctx, ctx->x32.ensure(M * 4));  // FP32 output staging
  }
  if (prec == XFP_PREC_F32 || prec == XFP_PREC_MIXED) {
    for (auto& b : ctx->A32) XFP_CUDA(ctx, b.ensure(M * 4));
    XFP_CUDA(ctx, ctx->inv32.ensure(M * 4));
    XFP_CUDA(ctx, ctx->x32.ensure(M * 4));
    XFP_CUDA(ctx, ctx->r32.ensure(M * 4));
    XFP_CUDA(ctx, ctx->s32.ensure(M * 4));
    XFP_CUDA(ctx, ctx->z32.ensure(M * 4));
    for (auto& b : ctx->L32) XFP_CUDA(ctx, b.ensure(M * 4));
  }
  if (prec == XFP_PREC_F32) {
    for (auto& b : ctx->F32) XFP_CUDA(ctx, b.ensure(M * 4));
    XFP_CUDA(ctx, ctx->inv32.ensure(M * 4));
  }
  XFP_CUDA(ctx, ctx->ctl.ensure(sizeof(SweepCtl)));
  XFP_CUDA(ctx, ctx->scal.ensure(sizeof(PcgScalars)));
  XFP_CUDA(ctx, ctx->scal2.ensure(sizeof(PcgScalars)));
  XFP_CUDA(ctx, ctx->partials.ensure(NBLK_MAX * sizeof(double)));
  // z.r partials: one per x-line
  XFP_CUDA(ctx, ctx->tpartials.ensure(std::max<long long>(ctx->nlines_all, 1) * sizeof(double)));
  // stamped tile-boundary words: 4 per cell; zeroed when (re)allocated so no
  // stale word can carry a live generation
  const size_t sbytes = M * 4 * sizeof(unsigned long long);
  for (DevBuf* b : {&ctx->sy, &ctx->sz}) {
    if (b->cap < sbytes || !b->p) {
      XFP_CUDA(ctx, b->ensure(sbytes));
      XFP_CUDA(ctx, cudaMemsetAsync(b->p, 0, b->cap, ctx->stream));
    }
  }
  return XFP_OK;
}

SweepGrid make_grid(xfp_ctx* ctx, PcgScalars* sc, int bwd_mode) {
  SweepGrid g;
  g.ni = ctx->ni; g.nj = ctx->nj; g.nk = ctx->nk;
  g.NJt = ctx->NJt; g.NKt = ctx->NKt;
  g.ntiles = (int)ctx->ntiles;
  g.maxT = ctx->ni + ctx->nj + ctx->nk;
  g.bwd_mode = bwd_mode;
  g.lines = ctx->lines.as<Line>();
  g.tiles = ctx->tiles.as<int>();
  g.ctl = ctx->ctl.as<SweepCtl>();
  g.spin_limit = spin_limit(ctx);
  g.scal = sc;
  g.trace = ctx->tracing ? ctx->trace.as<int>() : nullptr;
  g.stage = ctx->stage_solves;
  return g;
}

template <typename VT, typename IT, typename CT>
int run_sweep(xfp_ctx* ctx, int op, const SweepGrid& g, const SweepData<VT, IT, CT>& d) {
  if (g.ntiles <= 0) return XFP_OK;
  int maxg = sweep_max_grid(op, d, ctx->nw, g.stage);
  if (maxg <= 0) {
    const cudaError_t e = cudaGetLastError();
    return fail(ctx, XFP_ERR_CUDA, std::string("sweep kernel cannot be resident (op ") + std::to_string(op) +
                                       ", tile height " + std::to_string(ctx->nw) + "): " + cudaGetErrorString(e));
  }
  int grid = std::min(maxg, g.ntiles);
  // the forward and backward solve of every event_every-th iteration
  const int ord = op != SWEEP_FACTOR ? ctx->sweep_ord++ : -1;
  const bool timed = ctx->event_every > 0 && ord >= 0 && (ord / 2) % ctx->event_every == 0 &&
                     ctx->sweep_ev_used + 2 <= (int)ctx->sweep_ev.size();
  if (timed) cudaEventRecord(ctx->sweep_ev[ctx->sweep_ev_used], ctx->stream);
  SweepGrid gl = g;
  if (ctx->expire_next_sweep) {
    gl.expect_bias = 1;
    ctx->expire_next_sweep = false;
  }
  XFP_CUDA(ctx, sweep_launch(op, gl, d, ctx->nw, grid, ctx->stream));
  if (timed) {
    cudaEventRecord(ctx->sweep_ev[ctx->sweep_ev_used + 1], ctx->stream);
    ctx->sweep_work[ctx->sweep_ev_used / 2] = 1;
    ctx->sweep_ord_of[ctx->sweep_ev_used / 2] = ord;
    ctx->sweep_ev_used += 2;
  }
  return XFP_OK;
}

// Event pair around one vector-kernel launch of the PCG loop (kind, iteration).
template <typename F>
cudaError_t timed_kernel(xfp_ctx* ctx, int kind, int iter, F&& launch) {
  const bool timed = ctx->event_every > 0 && iter % ctx->event_every == 0 &&
                     ctx->kern_ev_used + 2 <= (int)ctx->kern_ev.size();
  if (timed) cudaEventRecord(ctx->kern_ev[ctx->kern_ev_used], ctx->stream);
  const cudaError_t e = launch();
  if (timed) {
    cudaEventRecord(ctx->kern_ev[ctx->kern_ev_used + 1], ctx->stream);
    ctx->kern_kind[ctx->kern_ev_used / 2] = kind;
    ctx->kern_iter[ctx->kern_ev_used / 2] = iter;
    ctx->kern_ev_used += 2;
  }
  return e;
}

// Sum of the timed durations of the sweep launches that did work (after the
// stream has been synchronised).
double sweep_ms(xfp_ctx* ctx, int* n) {
  double tot = 0;
  int cnt = 0;
  for (int q = 0; q + 1 < ctx->sweep_ev_used; q += 2) {
    if (!ctx->sweep_work[q / 2]) continue;
    float ms = 0;
    if (cudaEventElapsedTime(&ms, ctx->sweep_ev[q], ctx->sweep_ev[q + 1]) == cudaSuccess) {
      tot += ms;
      ++cnt;
    }
  }
  *n = cnt;
  return tot;
}

int check_sweep_error(xfp_ctx* ctx) {
  SweepCtl c;
  XFP_CUDA(ctx, cudaMemcpyAsync(&c, ctx->ctl.p, sizeof(c), cudaMemcpyDeviceToHost, ctx->stream));
  XFP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (c.err && ctx->tracing) {
    std::vector<int> t(ctx->trace.cap / sizeof(int));
    cudaMemcpy(t.data(), ctx->trace.p, ctx->trace.cap, cudaMemcpyDeviceToHost);
    int blk = c.err_thread / ((ctx->nw + 1) * 32);
    fprintf(stderr, "xfp trace: failing block %d, op %d, nw %d (site 0 = not waiting)\n", blk, c.err_op, ctx->nw);
    for (int b = 0; b < 1024; ++b) {
      bool any = false;
      for (int w = 0; w <= ctx->nw; ++w) any |= t[((size_t)b * (ctx->nw + 1) + w) * 4] > 0;
      if (!any && b != blk) continue;
      fprintf(stderr, " block %d:", b);
      for (int w = 0; w <= ctx->nw; ++w) {
        const int* r = &t[((size_t)b * (ctx->nw + 1) + w) * 4];
        fprintf(stderr, " w%d[site %d step %d lane %d pub %d]", w, r[0], r[1], r[3], r[2]);
      }
      fprintf(stderr, "\n");
    }
  }
  if (c.err) {
    char buf[256];
    snprintf(buf, sizeof buf,
             "device wait timed out (site %u, op %d, tile %d, step %d, thread %d, ntiles %lld, seen %016llx, "
             "expect %08x)",
             c.err_where, c.err_op, c.err_tile, c.err_tau, c.err_thread, ctx->ntiles, c.err_word, c.err_expect);
    // clear so the context stays usable
    SweepCtl z{};
    z.gen = c.gen;
    cudaMemcpyAsync(ctx->ctl.p, &z, sizeof(z), cudaMemcpyHostToDevice, ctx->stream);
    cudaStreamSynchronize(ctx->stream);
    return fail(ctx, XFP_ERR_TIMEOUT, buf);
  }
  return XFP_OK;
}

// ---------------------------------------------------------------- factor
// Zero the factor scratch, then the lower sweep.
template <typename VT, typename IT, typename CT>
int factor(xfp_ctx* ctx, const CT* const A[4], CT* const F[6], IT* inv, CT omega, CT ratio) {
  const size_t M = (size_t)ctx->M;
  // the factorisation writes L only where a coupling exists: clear the three L arrays first
  for (int q = 0; q < 3; ++q) XFP_CUDA(ctx, cudaMemsetAsync(F[q], 0, M * sizeof(CT), ctx->stream));
  XFP_CUDA(ctx, cudaMemsetAsync(inv, 0, M * sizeof(IT), ctx->stream));
  SweepData<VT, IT, CT> d;
  d.diag = A[0]; d.ax = A[1]; d.ay = A[2]; d.az = A[3];
  d.flx = F[0]; d.fly = F[1]; d.flz = F[2];
  d.oinv = inv;
  d.sy = ctx->sy.as<unsigned long long>();
  d.sz = ctx->sz.as<unsigned long long>();
  d.omega = omega; d.ratio = ratio;
  SweepGrid g = make_grid(ctx, nullptr, 0);
  return run_sweep<VT, IT, CT>(ctx, SWEEP_FACTOR, g, d);
}

// ---------------------------------------------------------------- PCG
// pcg_solver.h:243-285 on the compact system.  A: coefficient arrays (VT),
// b: rhs (VT), x: solution (VT), L/inv: factor.  DT: dot accumulation type.
template <typename VT, typename IT, typename DT>
int pcg(xfp_ctx* ctx, const VT* const A[4], const VT* b, VT* x, VT* r, VT* s, VT* z,
        const VT* const L[3], const IT* inv, double tol, int maxit, PcgScalars* dsc,
        PcgScalars* hsc) {
  const long long M = ctx->M;
  cudaStream_t st = ctx->stream;
  if (tol < 1e-30) tol = 1e-30;  // set_solver_parameters, pcg_solver.h:237
  XFP_CUDA(ctx, cudaMemsetAsync(x, 0, M * sizeof(VT), st));
  XFP_CUDA(ctx, cudaMemsetAsync(dsc, 0, sizeof(PcgScalars), st));
  XFP_CUDA(ctx, copy_vec<VT>(b, r, M, st));
  XFP_CUDA(ctx, absmax_init<VT>(r, M, dsc, ctx->partials.as<double>(), NBLK_MAX, tol, maxit, st));
  // lines of inactive tiles are never written: their z.r partials stay zero
  XFP_CUDA(ctx, cudaMemsetAsync(ctx->tpartials.p, 0, std::max<long long>(ctx->nlines_all, 1) * sizeof(double), st));
  SweepData<VT, IT, DT> d;
  d.r = r; d.y = z; d.lx = L[0]; d.ly = L[1]; d.lz = L[2]; d.inv = inv;
  d.partials = ctx->tpartials.as<double>();
  d.sy = ctx->sy.as<unsigned long long>();
  d.sz = ctx->sz.as<unsigned long long>();
  SweepGrid gs[2] = {make_grid(ctx, dsc, 0), make_grid(ctx, dsc, 1)};
  int rc;
  if ((rc = sweep_copies<VT, IT, DT>(ctx, L, inv, r, gs, 2, &d)) != XFP_OK) return rc;
  const int first_timed = ctx->sweep_ev_used / 2;
  const int first_kern = ctx->kern_ev_used / 2;
  ctx->sweep_ord = 0;
  const SweepGrid& g0 = gs[0];
  const SweepGrid& g1 = gs[1];
  // with a sweep layout, r is kept in both layouts (update_xr writes both)
  // and z lives in the sweep layout only (update_s reads it through perm)
  const bool swl = ctx->ntiles > 0;
  VT* rsw = swl ? ctx->sw_r.as<VT>() : nullptr;
  const VT* zsw = swl ? ctx->sw_y.as<VT>() : nullptr;
  const int* perm = swl ? ctx->sw_perm.as<int>() : nullptr;
  if ((rc = run_sweep<VT, IT, DT>(ctx, SWEEP_FWD, g0, d)) != XFP_OK) return rc;
  if ((rc = run_sweep<VT, IT, DT>(ctx, SWEEP_BWD, g0, d)) != XFP_OK) return rc;
  if (swl) {
    if ((rc = sweep_result<VT>(ctx, s)) != XFP_OK) return rc;
  } else {
    XFP_CUDA(ctx, copy_vec<VT>(z, s, M, st));
  }
  const int K = ctx->opt.check_every > 0 ? ctx->opt.check_every : 8;
  DT* part = reinterpret_cast<DT*>(ctx->partials.p);
  for (int done_iters = 0;;) {
    for (int q = 0; q < K; ++q) {
      const int it = done_iters + q + 1;   // this launch's PCG iteration (1-based)
      XFP_CUDA(ctx, timed_kernel(ctx, 0, it, [&] {
        return spmv_dot<VT, VT, DT>(A[0], A[1], A[2], A[3], s, z, ctx->lines.as<Line>(), ctx->group_line.as<int>(),
                                    ctx->nj, ctx->nk, M, dsc, part, ctx->vec_blocks, 0, st);
      }));
      XFP_CUDA(ctx, timed_kernel(ctx, 1, it, [&] {
        return update_xr<VT, DT>(x, r, s, z, M, dsc, ctx->partials.as<double>(), ctx->xr_blocks, st, rsw, perm);
      }));
      if ((rc = run_sweep<VT, IT, DT>(ctx, SWEEP_FWD, g1, d)) != XFP_OK) return rc;
      if ((rc = run_sweep<VT, IT, DT>(ctx, SWEEP_BWD, g1, d)) != XFP_OK) return rc;
      XFP_CUDA(ctx, timed_kernel(ctx, 2, it, [&] { return update_s<VT>(s, z, M, dsc, st, zsw, perm, ctx->s_blocks); }));
    }
    done_iters += K;
    XFP_CUDA(ctx, cudaMemcpyAsync(hsc, dsc, sizeof(PcgScalars), cudaMemcpyDeviceToHost, st));
    XFP_CUDA(ctx, cudaStreamSynchronize(st));
    if ((rc = check_sweep_error(ctx)) != XFP_OK) return rc;
    if (hsc->done) break;
    if (done_iters > maxit + 2 * K) return fail(ctx, XFP_ERR_CUDA, "PCG loop did not terminate");
  }
  // the preconditioner's two sweeps, then two per iteration but the last (the
  // converged iteration skips its preconditioner): 2 * iterations did work;
  // the launches after them in the last chunk returned at once
  for (int q = first_timed; q < ctx->sweep_ev_used / 2; ++q)
    if (ctx->sweep_ord_of[q] >= 2 * std::max(hsc->iters, 1)) ctx->sweep_work[q] = 0;
  // vector kernels of this call that ran after convergence: SpMV and the x/r
  // update of iterations past the last, the s update of the last and later
  for (int q = first_kern; q < ctx->kern_ev_used / 2; ++q)
    if (ctx->kern_iter[q] > hsc->iters || (ctx->kern_kind[q] == 2 && ctx->kern_iter[q] >= hsc->iters))
      ctx->kern_kind[q] = -1;
  if (hsc->status == XFP_ERR_BREAKDOWN) return fail(ctx, XFP_ERR_BREAKDOWN, "PCG breakdown: rho is zero or NaN");
  return hsc->status == 0 ? XFP_OK : XFP_NOT_CONVERGED;
}

void ev_record(xfp_ctx* ctx, int i) { cudaEventRecord(ctx->ev[i], ctx->stream); }
float ev_ms(xfp_ctx* ctx, int a, int b) {
  float ms = 0;
  cudaEventElapsedTime(&ms, ctx->ev[a], ctx->ev[b]);
  return ms;
}

// ---------------------------------------------------------------- solve driver
// Assembles, factors and solves.  On return the solution is in x64 (F64,
// MIXED) or x32 (F32) in compact layout.  rhs_from_adjoint: when non-null, the
// assembled b is replaced by G^T g (backward pass) before solving.
//
// Tile height (options.tile_k == 0): the first solve of a grid shape builds
// the layout at each candidate height, assembles and factors in FP32 and
// times two forward+backward sweep pairs; the fastest height is cached in the
// context for that shape and precision.
// The compute stream waits for the face gather of the I/O stream (host-pointer
// mode, face-sparse) before it first reads the velocities.
int inputs_ready(xfp_ctx* ctx) {
  if (!ctx->io_pending) return XFP_OK;
  ctx->io_pending = false;
  XFP_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, ctx->ev_io_in, 0));
  return XFP_OK;
}

template <typename IOT>
int tune_tile_height(xfp_ctx* ctx, int ni, int nj, int nk, const uint8_t* dmat, const IOT* du_, const IOT* dv,
                     const IOT* dw, const IOT* dwu, const IOT* dwv, const IOT* dww) {
  if (ctx->opt.tile_k != 0) {
    ctx->nw = ctx->opt.tile_k;
    return XFP_OK;
  }
  const std::string key = std::to_string(ni) + "x" + std::to_string(nj) + "x" + std::to_string(nk) + ":" +
                          std::to_string(ctx->opt.precision);
  auto it = ctx->tuned_nw.find(key);
  if (it != ctx->tuned_nw.end()) {
    ctx->nw = it->second;
    return XFP_OK;
  }
  cudaStream_t st = ctx->stream;
  float best = 0.f;
  int best_nw = 8;
  if (int rc0 = inputs_ready(ctx)) return rc0;
  cudaEvent_t e0, e1;
  XFP_CUDA(ctx, cudaEventCreate(&e0));
  XFP_CUDA(ctx, cudaEventCreate(&e1));
  int rc = XFP_OK;
  for (int cand : {8, 15, 16}) {
    ctx->nw = cand;
    if ((rc = build_layout(ctx, dmat, ni, nj, nk)) != XFP_OK) break;
    if ((rc = ensure_compact(ctx, XFP_PREC_F32)) != XFP_OK) break;
    if (ctx->ntiles == 0) { best_nw = 8; break; }
    float* A[5];
    for (int q = 0; q < 5; ++q) A[q] = ctx->A32[q].as<float>();
    if (assemble<IOT, float>(dmat, du_, dv, dw, dwu, dwv, dww, ni, nj, nk, ctx->lines.as<Line>(), A[0], A[1], A[2],
                             A[3], A[4], st, ctx->opt.matrix) != cudaSuccess) { rc = fail(ctx, XFP_ERR_CUDA, "assembly failed"); break; }
    float* F[6];
    for (int q = 0; q < 6; ++q) F[q] = ctx->F32[q].as<float>();
    const float* Ac[4] = {A[0], A[1], A[2], A[3]};
    if ((rc = factor<float, float, float>(ctx, Ac, F, ctx->inv32.as<float>(), 0.97f, 0.25f)) != XFP_OK) break;
    SweepData<float, float, float> d;
    d.r = A[4]; d.y = ctx->z32.as<float>(); d.lx = F[0]; d.ly = F[1]; d.lz = F[2]; d.inv = ctx->inv32.as<float>();
    d.partials = ctx->tpartials.as<double>();
    d.sy = ctx->sy.as<unsigned long long>();
    d.sz = ctx->sz.as<unsigned long long>();
    SweepGrid g = make_grid(ctx, nullptr, 0);
    const float* Lc[3] = {F[0], F[1], F[2]};
    if ((rc = sweep_copies<float, float, float>(ctx, Lc, ctx->inv32.as<float>(), A[4], &g, 1, &d)) != XFP_OK) break;
    const int maxg = std::min(sweep_max_grid(SWEEP_FWD, d, cand, g.stage),
                              sweep_max_grid(SWEEP_BWD, d, cand, g.stage));
    if (maxg <= 0) continue;
    const int grid = std::min(maxg, (int)ctx->ntiles);
    cudaError_t e = sweep_launch(SWEEP_FWD, g, d, cand, grid, st);   // warm-up
    if (e == cudaSuccess) e = cudaEventRecord(e0, st);
    for (int q = 0; q < 2 && e == cudaSuccess; ++q) {
      e = sweep_launch(SWEEP_FWD, g, d, cand, grid, st);
      if (e == cudaSuccess) e = sweep_launch(SWEEP_BWD, g, d, cand, grid, st);
    }
    if (e == cudaSuccess) e = cudaEventRecord(e1, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) { rc = fail(ctx, XFP_ERR_CUDA, std::string("tile height timing: ") + cudaGetErrorString(e)); break; }
    if ((rc = check_sweep_error(ctx)) != XFP_OK) break;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (cand == 8 || ms < best) { best = ms; best_nw = cand; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc != XFP_OK) return rc;
  ctx->tuned_nw[key] = best_nw;
  ctx->nw = best_nw;
  return XFP_OK;
}

template <typename IOT>
int solve_core(xfp_ctx* ctx, int ni, int nj, int nk, const uint8_t* dmat, const IOT* du_,
               const IOT* dv, const IOT* dw, const IOT* dwu, const IOT* dwv, const IOT* dww,
               const IOT* adj_gu = nullptr, const IOT* adj_gv = nullptr, const IOT* adj_gw = nullptr) {
  const int prec = ctx->opt.precision;
  cudaStream_t st = ctx->stream;
  int rc;
  ev_record(ctx, 0);
  if ((rc = tune_tile_height<IOT>(ctx, ni, nj, nk, dmat, du_, dv, dw, dwu, dwv, dww)) != XFP_OK) return rc;
  ctx->sweep_ev_used = 0;
  ctx->kern_ev_used = 0;
  if ((rc = build_layout(ctx, dmat, ni, nj, nk)) != XFP_OK) return rc;
  if ((rc = ensure_compact(ctx, prec)) != XFP_OK) return rc;
  if ((rc = inputs_ready(ctx)) != XFP_OK) return rc;
  const Line* lines = ctx->lines.as<Line>();
  const long long M = ctx->M;
  ctx->iters = 0; ctx->refinements = 0; ctx->res = 0; ctx->bnorm = 0;
  PcgScalars* dsc = ctx->scal.as<PcgScalars>();
  PcgScalars& hsc = ctx->host_sc;
  const double tol = ctx->opt.tol, omega = ctx->opt.omega, ratio = ctx->opt.min_diag_ratio;
  const int maxit = ctx->opt.max_iter;

  if (prec == XFP_PREC_F64) {
    double* A[5];
    for (int q = 0; q < 5; ++q) A[q] = ctx->A64[q].as<double>();
    XFP_CUDA(ctx, (assemble<IOT, double>(dmat, du_, dv, dw, dwu, dwv, dww, ni, nj, nk, lines, A[0], A[1], A[2],
                                         A[3], A[4], st, ctx->opt.matrix, ctx->force)));
    if (adj_gu) XFP_CUDA(ctx, (apply_pressure_T<IOT, double>(dmat, dwu, dwv, dww, adj_gu, adj_gv, adj_gw, ni, nj,
                                                             nk, lines, A[4], st)));
    ev_record(ctx, 1);
    double* F[6];
    for (int q = 0; q < 6; ++q) F[q] = ctx->F64[q].as<double>();
    const double* Ac[4] = {A[0], A[1], A[2], A[3]};
    if ((rc = factor<double, double, double>(ctx, Ac, F, ctx->inv64.as<double>(), omega, ratio)) != XFP_OK) return rc;
    if ((rc = check_sweep_error(ctx)) != XFP_OK) return rc;
    ev_record(ctx, 2);
    const double* Lc[3] = {F[0], F[1], F[2]};
    rc = pcg<double, double, double>(ctx, Ac, A[4], ctx->x64.as<double>(), ctx->r64.as<double>(),
                                     ctx->s64.as<double>(), ctx->z64.as<double>(), Lc, ctx->inv64.as<double>(),
                                     tol, maxit, dsc, &hsc);
    ev_record(ctx, 3);
    ctx->iters = hsc.iters; ctx->res = hsc.res; ctx->bnorm = hsc.bnorm;
  } else if (prec == XFP_PREC_F32) {
    float* A[5];
    for (int q = 0; q < 5; ++q) A[q] = ctx->A32[q].as<float>();
    XFP_CUDA(ctx, (assemble<IOT, float>(dmat, du_, dv, dw, dwu, dwv, dww, ni, nj, nk, lines, A[0], A[1], A[2],
                                        A[3], A[4], st, ctx->opt.matrix, ctx->force)));
    if (adj_gu) XFP_CUDA(ctx, (apply_pressure_T<IOT, float>(dmat, dwu, dwv, dww, adj_gu, adj_gv, adj_gw, ni, nj,
                                                            nk, lines, A[4], st)));
    ev_record(ctx, 1);
    float* F[6];
    for (int q = 0; q < 6; ++q) F[q] = ctx->F32[q].as<float>();
    const float* Ac[4] = {A[0], A[1], A[2], A[3]};
    if ((rc = factor<float, float, float>(ctx, Ac, F, ctx->inv32.as<float>(), (float)omega, (float)ratio)) != XFP_OK)
      return rc;
    if ((rc = check_sweep_error(ctx)) != XFP_OK) return rc;
    ev_record(ctx, 2);
    const float* Lc[3] = {F[0], F[1], F[2]};
    rc = pcg<float, float, float>(ctx, Ac, A[4], ctx->x32.as<float>(), ctx->r32.as<float>(), ctx->s32.as<float>(),
                                  ctx->z32.as<float>(), Lc, ctx->inv32.as<float>(), tol, maxit, dsc, &hsc);
    ev_record(ctx, 3);
    ctx->iters = hsc.iters; ctx->res = hsc.res; ctx->bnorm = hsc.bnorm;
  } else {
    // ---- mixed: FP64 system and refinement, FP32 inner PCG ----
    double* A[5];
    for (int q = 0; q < 5; ++q) A[q] = ctx->A64[q].as<double>();
    float* A32[4];
    for (int q = 0; q < 4; ++q) A32[q] = ctx->A32[q].as<float>();
    // the FP32 stencil comes out of the same assembly pass
    XFP_CUDA(ctx, (assemble<IOT, double>(dmat, du_, dv, dw, dwu, dwv, dww, ni, nj, nk, lines, A[0], A[1], A[2],
                                         A[3], A[4], st, ctx->opt.matrix, ctx->force, A32)));
    if (adj_gu) XFP_CUDA(ctx, (apply_pressure_T<IOT, double>(dmat, dwu, dwv, dww, adj_gu, adj_gv, adj_gw, ni, nj,
                                                             nk, lines, A[4], st)));
    ev_record(ctx, 1);
    double* F[6];
    for (int q = 0; q < 6; ++q) F[q] = ctx->F64[q].as<double>();
    const double* Ac[4] = {A[0], A[1], A[2], A[3]};
    if ((rc = factor<float, double, double>(ctx, Ac, F, ctx->inv64.as<double>(), omega, ratio)) != XFP_OK) return rc;
    if ((rc = check_sweep_error(ctx)) != XFP_OK) return rc;
    for (int q = 0; q < 3; ++q) XFP_CUDA(ctx, (convert<double, float>(F[q], ctx->L32[q].as<float>(), M, st)));
    // the pivots are computed in FP64 (above); the FP32 solves stream them rounded to FP32
    XFP_CUDA(ctx, (convert<double, float>(ctx->inv64.as<double>(), ctx->inv32.as<float>(), M, st)));
    ev_record(ctx, 2);
    const float* Lc[3] = {ctx->L32[0].as<float>(), ctx->L32[1].as<float>(), ctx->L32[2].as<float>()};
    const float* A32c[4] = {A32[0], A32[1], A32[2], A32[3]};
    double* x64 = ctx->x64.as<double>();
    double* r64 = ctx->r64.as<double>();
    PcgScalars* osc = ctx->scal2.as<PcgScalars>();
    PcgScalars ho{};
    XFP_CUDA(ctx, cudaMemsetAsync(x64, 0, M * sizeof(double), st));
    XFP_CUDA(ctx, cudaMemsetAsync(osc, 0, sizeof(PcgScalars), st));
    XFP_CUDA(ctx, absmax_init<double>(A[4], M, osc, ctx->partials.as<double>(), NBLK_MAX, tol, 1, st));
    XFP_CUDA(ctx, cudaMemcpyAsync(&ho, osc, sizeof(ho), cudaMemcpyDeviceToHost, st));
    XFP_CUDA(ctx, cudaStreamSynchronize(st));
    const double bnorm = ho.bnorm, target = (tol < 1e-30 ? 1e-30 : tol) * bnorm;
    ctx->bnorm = bnorm;
    double res = bnorm;
    int total = 0, cycles = 0, status = XFP_OK;
    const int max_ref = ctx->opt.max_refine > 0 ? ctx->opt.max_refine : 20;
    const double floor_tol = ctx->opt.inner_tol > 0 ? ctx->opt.inner_tol : 1e-6;
    if (bnorm > 0) {
      status = XFP_NOT_CONVERGED;
      for (cycles = 0; cycles < max_ref && total < maxit; ++cycles) {
        if (cycles > 0) {
          XFP_CUDA(ctx, residual64(A[0], A[1], A[2], A[3], A[4], x64, r64, lines, ni, nj, nk, M, osc,
                                   ctx->partials.as<double>(), NBLK_MAX, st));
          XFP_CUDA(ctx, cudaMemcpyAsync(&ho, osc, sizeof(ho), cudaMemcpyDeviceToHost, st));
          XFP_CUDA(ctx, cudaStreamSynchronize(st));
          res = ho.res;
          if (res <= target) { status = XFP_OK; break; }
          XFP_CUDA(ctx, (convert<double, float>(r64, ctx->r32.as<float>(), M, st)));
        } else {
          XFP_CUDA(ctx, (convert<double, float>(A[4], ctx->r32.as<float>(), M, st)));
        }
        const double inner = std::min(0.5, std::max(floor_tol, 0.5 * target / res));
        // inner rhs lives in s32 scratch's partner: use r32 as b, z32/s32/x32 work
        float* b32 = ctx->A32[4].as<float>();
        XFP_CUDA(ctx, copy_vec<float>(ctx->r32.as<float>(), b32, M, st));
        int irc = pcg<float, float, double>(ctx, A32c, b32, ctx->x32.as<float>(), ctx->r32.as<float>(),
                                            ctx->s32.as<float>(), ctx->z32.as<float>(), Lc,
                                            ctx->inv32.as<float>(), inner, maxit - total, dsc, &hsc);
        if (irc < 0) return irc;
        total += hsc.iters;
        XFP_CUDA(ctx, refine_update(x64, ctx->x32.as<float>(), M, st));
      }
      if (status != XFP_OK) {
        XFP_CUDA(ctx, residual64(A[0], A[1], A[2], A[3], A[4], x64, r64, lines, ni, nj, nk, M, osc,
                                 ctx->partials.as<double>(), NBLK_MAX, st));
        XFP_CUDA(ctx, cudaMemcpyAsync(&ho, osc, sizeof(ho), cudaMemcpyDeviceToHost, st));
        XFP_CUDA(ctx, cudaStreamSynchronize(st));
        res = ho.res;
        if (res <= target) status = XFP_OK;
      }
    }
    ev_record(ctx, 3);
    ctx->iters = total; ctx->refinements = cycles; ctx->res = res;
    rc = status;
  }
  return rc;
}

template <typename IOT>
int solution_dense(xfp_ctx* ctx, IOT* dense) {
  const int prec = ctx->opt.precision;
  const Line* lines = ctx->lines.as<Line>();
  if (prec == XFP_PREC_F32) {
    if (std::is_same<IOT, float>::value) {
      XFP_CUDA(ctx, scatter_dense<float>(ctx->x32.as<float>(), lines, ctx->ni, ctx->nj, ctx->nk, (float*)dense,
                                         ctx->stream));
    } else {
      XFP_CUDA(ctx, ctx->r64.ensure(ctx->M * 8 + 64));
      XFP_CUDA(ctx, (convert<float, double>(ctx->x32.as<float>(), ctx->r64.as<double>(), ctx->M, ctx->stream)));
      XFP_CUDA(ctx, scatter_dense<double>(ctx->r64.as<double>(), lines, ctx->ni, ctx->nj, ctx->nk, (double*)dense,
                                          ctx->stream));
    }
  } else {
    if (std::is_same<IOT, double>::value) {
      XFP_CUDA(ctx, scatter_dense<double>(ctx->x64.as<double>(), lines, ctx->ni, ctx->nj, ctx->nk, (double*)dense,
                                          ctx->stream));
    } else {
      XFP_CUDA(ctx, (convert<double, float>(ctx->x64.as<double>(), ctx->x32.as<float>(), ctx->M, ctx->stream)));
      XFP_CUDA(ctx, scatter_dense<float>(ctx->x32.as<float>(), lines, ctx->ni, ctx->nj, ctx->nk, (float*)dense,
                                         ctx->stream));
    }
  }
  return XFP_OK;
}

// Algorithmic bytes per unknown row and PCG iteration: FP32 vectors, L and
// pivots (the mixed form streams its FP64 pivots as FP32) 112, FP64 224.
double bytes_per_row_iter(int prec) { return prec == XFP_PREC_F64 ? 224.0 : 112.0; }

void fill_stats(xfp_ctx* ctx, xfp_stats* s, int status, double ms_total) {
  if (!s) return;
  memset(s, 0, sizeof(*s));
  s->status = status;
  s->iterations = ctx->iters;
  s->refinements = ctx->refinements;
  s->residual = ctx->res;
  s->b_inf = ctx->bnorm;
  s->rel_residual = ctx->bnorm > 0 ? ctx->res / ctx->bnorm : 0.0;
  s->rows = ctx->rows;
  s->stored = ctx->M;
  s->lines = ctx->nlines_act;
  s->ms_setup = ctx->ms_setup;
  s->ms_factor = ctx->ms_factor;
  s->ms_solve = ctx->ms_solve;
  s->ms_apply = ctx->ms_apply;
  s->ms_total = ms_total;
  const double cells = (double)ctx->ni * ctx->nj * ctx->nk;
  s->bytes = bytes_per_row_iter(ctx->opt.precision) * (double)ctx->rows * ctx->iters + 33.0 * cells +
             24.0 * (double)ctx->rows + 29.0 * cells;
  int n = 0;
  s->ms_sweeps = sweep_ms(ctx, &n);
  s->sweeps = n;
  for (int k = 0; k < 3; ++k) {
    s->ms_vec[k] = 0.0;
    s->vec_launches[k] = 0;
  }
  for (int q = 0; q + 1 < ctx->kern_ev_used; q += 2) {
    const int k = ctx->kern_kind[q / 2];
    float ms = 0;
    if (k < 0 || cudaEventElapsedTime(&ms, ctx->kern_ev[q], ctx->kern_ev[q + 1]) != cudaSuccess) continue;
    s->ms_vec[k] += ms;
    s->vec_launches[k] += 1;
  }
  s->launches = g_kernel_launches - ctx->launches;
  s->tile_k = ctx->nw;
  s->h2d_bytes = ctx->h2d_bytes;
  s->d2h_bytes = ctx->d2h_bytes;
  s->host_faces = ctx->host_faces;
}

// ---------------------------------------------------------------- host I/O
// Whether [p, p + bytes) lies inside one page-locked host allocation that the
// device addresses at the same pointer (unified addressing), so that kernels
// may read and write it in place.  Pageable memory, device memory and ranges
// that leave their allocation answer false; the caller then copies whole
// arrays.  The allocation's extent comes from the driver
// (cuPointerGetAttribute, RANGE_START_ADDR / RANGE_SIZE / MAPPED).
bool host_in_place(const void* p, size_t bytes) {
  if (!p || bytes == 0) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (a.type != cudaMemoryTypeHost || a.devicePointer != p) return false;
  using Fn = CUresult (*)(void*, CUpointer_attribute, CUdeviceptr);
  static const Fn fn = []() -> Fn {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuPointerGetAttribute", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    return reinterpret_cast<Fn>(f);
  }();
  if (!fn) return false;
  unsigned long long start = 0;
  size_t size = 0;
  int mapped = 0;
  const CUdeviceptr d = (CUdeviceptr)(uintptr_t)p;
  if (fn(&start, CU_POINTER_ATTRIBUTE_RANGE_START_ADDR, d) != CUDA_SUCCESS) return false;
  if (fn(&size, CU_POINTER_ATTRIBUTE_RANGE_SIZE, d) != CUDA_SUCCESS) return false;
  if (fn(&mapped, CU_POINTER_ATTRIBUTE_MAPPED, d) != CUDA_SUCCESS || !mapped) return false;
  const uintptr_t b = (uintptr_t)p;
  return b >= start && b - start <= size && bytes <= size - (b - start);
}

// Velocities in: device pointers as they are; page-locked host arrays (all
// three in place, `sparse_ok`) face-sparse -- only the face rows' spans that
// border fluid are read, straight from host memory; otherwise whole-array
// copies.  *sparse tells faces_out which way to go back.
template <typename IOT>
int faces_in(xfp_ctx* ctx, const uint8_t* dmat, int ni, int nj, int nk, const IOT* u, const IOT* v, const IOT* w,
             const IOT** du_, const IOT** dv, const IOT** dw, bool sparse_ok, bool* sparse) {
  *sparse = false;
  if (ctx->io_stream) {
    // a call that stopped early may have left its gather running
    XFP_CUDA(ctx, cudaStreamSynchronize(ctx->io_stream));
    ctx->io_pending = false;
  }
  if (!ctx->opt.device_pointers && sparse_ok && ctx->host_sparse_ok &&
      host_in_place(u, nu(ni, nj, nk) * sizeof(IOT)) && host_in_place(v, nv(ni, nj, nk) * sizeof(IOT)) &&
      host_in_place(w, nw_(ni, nj, nk) * sizeof(IOT))) {
    XFP_CUDA(ctx, ctx->io_u.ensure(nu(ni, nj, nk) * sizeof(IOT)));
    XFP_CUDA(ctx, ctx->io_v.ensure(nv(ni, nj, nk) * sizeof(IOT)));
    XFP_CUDA(ctx, ctx->io_w.ensure(nw_(ni, nj, nk) * sizeof(IOT)));
    XFP_CUDA(ctx, ctx->hio_span.ensure((size_t)std::max<long long>((long long)nj * nk, 1) * sizeof(int2)));
    XFP_CUDA(ctx, ctx->hio_bytes.ensure(2 * sizeof(unsigned long long)));
    // the gather runs on the I/O stream after the material has arrived, beside
    // the layout build on the compute stream; inputs_ready() joins them before
    // the first assembly
    cudaStream_t gs = ctx->io_stream ? ctx->io_stream : ctx->stream;
    if (ctx->io_stream) {
      XFP_CUDA(ctx, cudaEventRecord(ctx->ev_io_mat, ctx->stream));
      XFP_CUDA(ctx, cudaStreamWaitEvent(gs, ctx->ev_io_mat, 0));
    }
    XFP_CUDA(ctx, cudaMemsetAsync(ctx->hio_bytes.p, 0, 2 * sizeof(unsigned long long), gs));
    XFP_CUDA(ctx, fluid_spans(dmat, ni, nj, nk, ctx->hio_span.as<int2>(), gs));
    const IOT* src[3] = {u, v, w};
    IOT* dst[3] = {ctx->io_u.as<IOT>(), ctx->io_v.as<IOT>(), ctx->io_w.as<IOT>()};
    XFP_CUDA(ctx, face_rows_copy<IOT>(ctx->hio_span.as<int2>(), ni, nj, nk, src, dst,
                                      ctx->hio_bytes.as<unsigned long long>(), gs));
    if (ctx->io_stream) {
      XFP_CUDA(ctx, cudaEventRecord(ctx->ev_io_in, gs));
      ctx->io_pending = true;
    }
    *du_ = dst[0];
    *dv = dst[1];
    *dw = dst[2];
    *sparse = true;
    ctx->host_faces = 1;
    return XFP_OK;
  }
  int rc;
  if ((rc = stage_in<IOT>(ctx, ctx->io_u, u, nu(ni, nj, nk), du_))) return rc;
  if ((rc = stage_in<IOT>(ctx, ctx->io_v, v, nv(ni, nj, nk), dv))) return rc;
  if ((rc = stage_in<IOT>(ctx, ctx->io_w, w, nw_(ni, nj, nk), dw))) return rc;
  return XFP_OK;
}

// Velocities out (host-pointer mode): the same face spans written straight
// into the caller's arrays, or whole-array copies.  Faces outside the spans
// are unchanged by the projection, so the caller's copies of them stay right.
template <typename IOT>
int faces_out(xfp_ctx* ctx, int ni, int nj, int nk, const IOT* du_, const IOT* dv, const IOT* dw, IOT* u, IOT* v,
              IOT* w, bool sparse) {
  if (ctx->opt.device_pointers) return XFP_OK;
  if (sparse) {
    const IOT* src[3] = {du_, dv, dw};
    IOT* dst[3] = {u, v, w};
    XFP_CUDA(ctx, face_rows_copy<IOT>(ctx->hio_span.as<int2>(), ni, nj, nk, src, dst,
                                      ctx->hio_bytes.as<unsigned long long>() + 1, ctx->stream));
    return XFP_OK;
  }
  XFP_CUDA(ctx, cudaMemcpyAsync(u, du_, nu(ni, nj, nk) * sizeof(IOT), cudaMemcpyDeviceToHost, ctx->stream));
  XFP_CUDA(ctx, cudaMemcpyAsync(v, dv, nv(ni, nj, nk) * sizeof(IOT), cudaMemcpyDeviceToHost, ctx->stream));
  XFP_CUDA(ctx, cudaMemcpyAsync(w, dw, nw_(ni, nj, nk) * sizeof(IOT), cudaMemcpyDeviceToHost, ctx->stream));
  ctx->d2h_bytes += (long long)((nu(ni, nj, nk) + nv(ni, nj, nk) + nw_(ni, nj, nk)) * sizeof(IOT));
  return XFP_OK;
}

// After the call's last stream synchronisation: the face-sparse byte counts.
int faces_account(xfp_ctx* ctx, bool sparse) {
  if (ctx->io_stream) XFP_CUDA(ctx, cudaStreamSynchronize(ctx->io_stream));
  if (!sparse) return XFP_OK;
  unsigned long long b[2] = {0, 0};
  XFP_CUDA(ctx, cudaMemcpy(b, ctx->hio_bytes.p, sizeof(b), cudaMemcpyDeviceToHost));
  ctx->h2d_bytes += (long long)b[0];
  ctx->d2h_bytes += (long long)b[1];
  return XFP_OK;
}

template <typename IOT>
int project_impl(xfp_ctx* ctx, int ni, int nj, int nk, const uint8_t* mat, IOT* u, IOT* v, IOT* w,
                 const IOT* wu, const IOT* wv, const IOT* ww, IOT* pressure, xfp_stats* stats,
                 bool do_apply) {
  int rc = check_dims(ctx, ni, nj, nk, mat);
  if (rc) return rc;
  if (!u || !v || !w) return fail(ctx, XFP_ERR_ARGS, "velocity arrays must not be NULL");
  if ((wu == nullptr) != (wv == nullptr) || (wu == nullptr) != (ww == nullptr))
    return fail(ctx, XFP_ERR_ARGS, "face weights: pass all three or none");
  if (ctx->opt.matrix == XFP_MATRIX_NORMAL && wu != nullptr)
    return fail(ctx, XFP_ERR_ARGS, "the normal matrix takes no face weights");
  if (!do_apply && !pressure) return fail(ctx, XFP_ERR_ARGS, "pressure output is NULL");
  XFP_CUDA(ctx, cudaSetDevice(ctx->device));
  ctx->launches = g_kernel_launches;
  ctx->h2d_bytes = ctx->d2h_bytes = 0;
  ctx->host_faces = 0;
  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  cudaEventRecord(t0, ctx->stream);
  const uint8_t* dmat;
  const IOT *du_, *dv, *dw, *dwu, *dwv, *dww;
  bool sparse = false;
  if ((rc = stage_in(ctx, ctx->io_mat, mat, ncells(ni, nj, nk), &dmat))) return rc;
  // the extrapolation layers of xfp_project_step_* write faces away from the
  // fluid: those calls move whole arrays
  if ((rc = faces_in<IOT>(ctx, dmat, ni, nj, nk, u, v, w, &du_, &dv, &dw, ctx->step_layers == 0, &sparse)))
    return rc;
  if ((rc = stage_in<IOT>(ctx, ctx->io_wu, wu, nu(ni, nj, nk), &dwu))) return rc;
  if ((rc = stage_in<IOT>(ctx, ctx->io_wv, wv, nv(ni, nj, nk), &dwv))) return rc;
  if ((rc = stage_in<IOT>(ctx, ctx->io_ww, ww, nw_(ni, nj, nk), &dww))) return rc;
  int status = solve_core<IOT>(ctx, ni, nj, nk, dmat, du_, dv, dw, dwu, dwv, dww);
  if (status < 0) {
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    return status;
  }
  IOT* dp;
  if (ctx->opt.device_pointers && pressure) {
    dp = pressure;
  } else {
    XFP_CUDA(ctx, ctx->io_p.ensure(ncells(ni, nj, nk) * sizeof(IOT)));
    dp = ctx->io_p.as<IOT>();
  }
  if ((rc = solution_dense<IOT>(ctx, dp))) return rc;
  // host-pointer mode: the dense pressure is final here; its download runs on
  // the I/O stream beside the apply (which only reads it)
  bool p_async = false;
  if (!ctx->opt.device_pointers && pressure && ctx->io_stream) {
    XFP_CUDA(ctx, cudaEventRecord(ctx->ev_io_p, ctx->stream));
    XFP_CUDA(ctx, cudaStreamWaitEvent(ctx->io_stream, ctx->ev_io_p, 0));
    XFP_CUDA(ctx, cudaMemcpyAsync(pressure, dp, ncells(ni, nj, nk) * sizeof(IOT), cudaMemcpyDeviceToHost,
                                  ctx->io_stream));
    ctx->d2h_bytes += (long long)(ncells(ni, nj, nk) * sizeof(IOT));
    p_async = true;
  }
  if (do_apply) {
    IOT* mu = const_cast<IOT*>(du_);
    IOT* mv = const_cast<IOT*>(dv);
    IOT* mw = const_cast<IOT*>(dw);
    XFP_CUDA(ctx, (apply_pressure<IOT, IOT>(dmat, dwu, dwv, dww, dp, ni, nj, nk, mu, mv, mw, ctx->stream,
                                            ctx->opt.matrix, ctx->force)));
    if (ctx->step_layers > 0) {
      const size_t nm = (size_t)(ni + 1) * (nj + 1) * (nk + 1);
      XFP_CUDA(ctx, ctx->xmarker.ensure(nm * sizeof(short)));
      XFP_CUDA(ctx, extrapolate<IOT>(dmat, ni, nj, nk, mu, mv, mw, ctx->step_layers, ctx->xmarker.as<short>(),
                                     ctx->stream));
    }
  }
  ev_record(ctx, 4);
  if (!ctx->opt.device_pointers) {
    if (pressure && !p_async) {
      XFP_CUDA(ctx, cudaMemcpyAsync(pressure, dp, ncells(ni, nj, nk) * sizeof(IOT), cudaMemcpyDeviceToHost,
                                    ctx->stream));
      ctx->d2h_bytes += (long long)(ncells(ni, nj, nk) * sizeof(IOT));
    }
    if (do_apply && (rc = faces_out<IOT>(ctx, ni, nj, nk, du_, dv, dw, u, v, w, sparse))) return rc;
  }
  if (p_async) {
    // the call's total includes the pressure download
    XFP_CUDA(ctx, cudaEventRecord(ctx->ev_io_mat, ctx->io_stream));
    XFP_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, ctx->ev_io_mat, 0));
  }
  cudaEventRecord(t1, ctx->stream);
  XFP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if ((rc = faces_account(ctx, sparse))) return rc;
  ctx->ms_setup = ev_ms(ctx, 0, 1);
  ctx->ms_factor = ev_ms(ctx, 1, 2);
  ctx->ms_solve = ev_ms(ctx, 2, 3);
  ctx->ms_apply = ev_ms(ctx, 3, 4);
  float tot = 0;
  cudaEventElapsedTime(&tot, t0, t1);
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  fill_stats(ctx, stats, status, tot);
  XFP_CUDA(ctx, cudaGetLastError());
  return status;
}

template <typename IOT>
int apply_impl(xfp_ctx* ctx, int ni, int nj, int nk, const uint8_t* mat, const IOT* wu, const IOT* wv,
               const IOT* ww, const IOT* pressure, IOT* u, IOT* v, IOT* w) {
  int rc = check_dims(ctx, ni, nj, nk, mat);
  if (rc) return rc;
  if (!u || !v || !w || !pressure) return fail(ctx, XFP_ERR_ARGS, "NULL array");
  if (ctx->opt.matrix == XFP_MATRIX_NORMAL && (wu || wv || ww))
    return fail(ctx, XFP_ERR_ARGS, "the normal matrix takes no face weights");
  XFP_CUDA(ctx, cudaSetDevice(ctx->device));
  ctx->h2d_bytes = ctx->d2h_bytes = 0;
  ctx->host_faces = 0;
  const uint8_t* dmat;
  const IOT *du_, *dv, *dw, *dwu, *dwv, *dww, *dp;
  bool sparse = false;
  if ((rc = stage_in(ctx, ctx->io_mat, mat, ncells(ni, nj, nk), &dmat))) return rc;
  if ((rc = faces_in<IOT>(ctx, dmat, ni, nj, nk, u, v, w, &du_, &dv, &dw, true, &sparse))) return rc;
  if ((rc = stage_in<IOT>(ctx, ctx->io_wu, wu, nu(ni, nj, nk), &dwu))) return rc;
  if ((rc = stage_in<IOT>(ctx, ctx->io_wv, wv, nv(ni, nj, nk), &dwv))) return rc;
  if ((rc = stage_in<IOT>(ctx, ctx->io_ww, ww, nw_(ni, nj, nk), &dww))) return rc;
  if ((rc = stage_in<IOT>(ctx, ctx->io_p, pressure, ncells(ni, nj, nk), &dp))) return rc;
  if ((rc = inputs_ready(ctx))) return rc;
  XFP_CUDA(ctx, (apply_pressure<IOT, IOT>(dmat, dwu, dwv, dww, dp, ni, nj, nk, const_cast<IOT*>(du_),
                                          const_cast<IOT*>(dv), const_cast<IOT*>(dw), ctx->stream,
                                          ctx->opt.matrix)));
  if ((rc = faces_out<IOT>(ctx, ni, nj, nk, du_, dv, dw, u, v, w, sparse))) return rc;
  XFP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return faces_account(ctx, sparse);
}

template <typename IOT>
int backward_impl(xfp_ctx* ctx, int ni, int nj, int nk, const uint8_t* mat, const IOT* wu, const IOT* wv,
                  const IOT* ww, const IOT* gu, const IOT* gv, const IOT* gw, IOT* du, IOT* dv, IOT* dw,
                  xfp_stats* stats) {
  int rc = check_dims(ctx, ni, nj, nk, mat);
  if (rc) return rc;
  if (!gu || !gv || !gw || !du || !dv || !dw) return fail(ctx, XFP_ERR_ARGS, "NULL gradient array");
  if (ctx->opt.matrix != XFP_MATRIX_VARIATIONAL)
    return fail(ctx, XFP_ERR_UNSUPPORTED, "the backward projection supports the variational matrix only");
  if ((wu == nullptr) != (wv == nullptr) || (wu == nullptr) != (ww == nullptr))
    return fail(ctx, XFP_ERR_ARGS, "face weights: pass all three or none");
  XFP_CUDA(ctx, cudaSetDevice(ctx->device));
  ctx->launches = g_kernel_launches;
  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  cudaEventRecord(t0, ctx->stream);
  const uint8_t* dmat;
  const IOT *dgu, *dgv, *dgw, *dwu, *dwv, *dww;
  if ((rc = stage_in(ctx, ctx->io_mat, mat, ncells(ni, nj, nk), &dmat))) return rc;
  if ((rc = stage_in<IOT>(ctx, ctx->io_gu, gu, nu(ni, nj, nk), &dgu))) return rc;
  if ((rc = stage_in<IOT>(ctx, ctx->io_gv, gv, nv(ni, nj, nk), &dgv))) return rc;
  if ((rc = stage_in<IOT>(ctx, ctx->io_gw, gw, nw_(ni, nj, nk), &dgw))) return rc;
  if ((rc = stage_in<IOT>(ctx, ctx->io_wu, wu, nu(ni, nj, nk), &dwu))) return rc;
  if ((rc = stage_in<IOT>(ctx, ctx->io_wv, wv, nv(ni, nj, nk), &dwv))) return rc;
  if ((rc = stage_in<IOT>(ctx, ctx->io_ww, ww, nw_(ni, nj, nk), &dww))) return rc;
  // the assembly needs velocities only for b, which the adjoint replaces: use g
  int status = solve_core<IOT>(ctx, ni, nj, nk, dmat, dgu, dgv, dgw, dwu, dwv, dww, dgu, dgv, dgw);
  if (status < 0) return status;
  // lambda to the dense grid, then d = g - D^T lambda
  IOT *ou, *ov, *ow;
  if (ctx->opt.device_pointers) {
    ou = du; ov = dv; ow = dw;
  } else {
    XFP_CUDA(ctx, ctx->io_u.ensure(nu(ni, nj, nk) * sizeof(IOT)));
    XFP_CUDA(ctx, ctx->io_v.ensure(nv(ni, nj, nk) * sizeof(IOT)));
    XFP_CUDA(ctx, ctx->io_w.ensure(nw_(ni, nj, nk) * sizeof(IOT)));
    ou = ctx->io_u.as<IOT>(); ov = ctx->io_v.as<IOT>(); ow = ctx->io_w.as<IOT>();
  }
  const int prec = ctx->opt.precision;
  if (prec == XFP_PREC_F32) {
    XFP_CUDA(ctx, ctx->dense.ensure(ncells(ni, nj, nk) * sizeof(float)));
    XFP_CUDA(ctx, scatter_dense<float>(ctx->x32.as<float>(), ctx->lines.as<Line>(), ni, nj, nk,
                                       ctx->dense.as<float>(), ctx->stream));
    if (std::is_same<IOT, float>::value) {
      XFP_CUDA(ctx, (rhs_T<float, float>(dmat, (const float*)dwu, (const float*)dwv, (const float*)dww,
                                         ctx->dense.as<float>(), ctx->lines.as<Line>(), ni, nj, nk,
                                         (const float*)dgu, (const float*)dgv, (const float*)dgw, (float*)ou,
                                         (float*)ov, (float*)ow, ctx->stream)));
    } else {
      return fail(ctx, XFP_ERR_UNSUPPORTED, "FP32 precision with FP64 I/O is not supported for backward");
    }
  } else {
    XFP_CUDA(ctx, ctx->dense.ensure(ncells(ni, nj, nk) * sizeof(double)));
    XFP_CUDA(ctx, scatter_dense<double>(ctx->x64.as<double>(), ctx->lines.as<Line>(), ni, nj, nk,
                                        ctx->dense.as<double>(), ctx->stream));
    XFP_CUDA(ctx, (rhs_T<IOT, double>(dmat, dwu, dwv, dww, ctx->dense.as<double>(), ctx->lines.as<Line>(), ni, nj,
                                      nk, dgu, dgv, dgw, ou, ov, ow, ctx->stream)));
  }
  ev_record(ctx, 4);
  if (!ctx->opt.device_pointers) {
    XFP_CUDA(ctx, cudaMemcpyAsync(du, ou, nu(ni, nj, nk) * sizeof(IOT), cudaMemcpyDeviceToHost, ctx->stream));
    XFP_CUDA(ctx, cudaMemcpyAsync(dv, ov, nv(ni, nj, nk) * sizeof(IOT), cudaMemcpyDeviceToHost, ctx->stream));
    XFP_CUDA(ctx, cudaMemcpyAsync(dw, ow, nw_(ni, nj, nk) * sizeof(IOT), cudaMemcpyDeviceToHost, ctx->stream));
  }
  cudaEventRecord(t1, ctx->stream);
  XFP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  ctx->ms_setup = ev_ms(ctx, 0, 1);
  ctx->ms_factor = ev_ms(ctx, 1, 2);
  ctx->ms_solve = ev_ms(ctx, 2, 3);
  ctx->ms_apply = ev_ms(ctx, 3, 4);
  float tot = 0;
  cudaEventElapsedTime(&tot, t0, t1);
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  fill_stats(ctx, stats, status, tot);
  return status;
}

// ---------------------------------------------------------------- diagnostics
// Dense FP64 view of a compact array of type T.
template <typename T>
int dump_dense(xfp_ctx* ctx, const T* compact, double* host_out) {
  if (!host_out) return XFP_OK;
  const size_t n = ncells(ctx->ni, ctx->nj, ctx->nk);
  XFP_CUDA(ctx, ctx->dense.ensure(n * sizeof(double)));
  const double* src64;
  if (std::is_same<T, double>::value) {
    src64 = (const double*)compact;
  } else {
    XFP_CUDA(ctx, ctx->io_gw.ensure((ctx->M + 8) * sizeof(double)));
    XFP_CUDA(ctx, (convert<float, double>((const float*)compact, ctx->io_gw.as<double>(), ctx->M, ctx->stream)));
    src64 = ctx->io_gw.as<double>();
  }
  XFP_CUDA(ctx, scatter_dense<double>(src64, ctx->lines.as<Line>(), ctx->ni, ctx->nj, ctx->nk,
                                      ctx->dense.as<double>(), ctx->stream));
  XFP_CUDA(ctx, cudaMemcpyAsync(host_out, ctx->dense.p, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  XFP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return XFP_OK;
}

// VT/IT/CT as in the solve of the context's precision; A: coefficients used by
// the factor (CT) and by the SpMV (VT).  SIT: the inverse-pivot type the
// triangular solves stream (the mixed form factors in FP64 and solves with an
// FP32 copy, as its PCG does); the dumped inv is the factor's own.
template <typename VT, typename IT, typename CT, typename SIT = IT>
int debug_core(xfp_ctx* ctx, const CT* const Af[5], const VT* const Av[4], CT* const F[6], IT* inv,
               const VT* const L[3], const double* dr, double* out[12]) {
  int rc;
  const long long M = ctx->M;
  cudaStream_t st = ctx->stream;
  if ((rc = factor<VT, IT, CT>(ctx, Af, F, inv, (CT)ctx->opt.omega, (CT)ctx->opt.min_diag_ratio))) return rc;
  if (!std::is_same<VT, CT>::value)
    for (int q = 0; q < 3; ++q) XFP_CUDA(ctx, (convert<CT, VT>(F[q], const_cast<VT*>(L[q]), M, st)));
  // r -> compact (VT), sweeps, SpMV
  VT* r = reinterpret_cast<VT*>(ctx->r32.p ? ctx->r32.p : ctx->r64.p);
  VT* z = reinterpret_cast<VT*>(ctx->z32.p ? ctx->z32.p : ctx->z64.p);
  VT* qv = reinterpret_cast<VT*>(ctx->s32.p ? ctx->s32.p : ctx->s64.p);
  if (std::is_same<VT, double>::value) {
    r = (VT*)ctx->r64.p; z = (VT*)ctx->z64.p; qv = (VT*)ctx->s64.p;
  }
  if (dr) {
    XFP_CUDA(ctx, ctx->io_p.ensure(ncells(ctx->ni, ctx->nj, ctx->nk) * sizeof(double)));
    XFP_CUDA(ctx, cudaMemcpyAsync(ctx->io_p.p, dr, ncells(ctx->ni, ctx->nj, ctx->nk) * sizeof(double),
                                  cudaMemcpyHostToDevice, st));
    XFP_CUDA(ctx, ctx->io_gv.ensure((M + 8) * sizeof(double)));
    XFP_CUDA(ctx, gather_compact<double>(ctx->io_p.as<double>(), ctx->lines.as<Line>(), ctx->ni, ctx->nj, ctx->nk,
                                         ctx->io_gv.as<double>(), st));
    if (std::is_same<VT, double>::value)
      XFP_CUDA(ctx, copy_vec<double>(ctx->io_gv.as<double>(), (double*)r, M, st));
    else
      XFP_CUDA(ctx, (convert<double, float>(ctx->io_gv.as<double>(), (float*)r, M, st)));
    const SIT* sinv = reinterpret_cast<const SIT*>(inv);
    if (!std::is_same<SIT, IT>::value) {
      XFP_CUDA(ctx, ctx->inv32.ensure((M + 8) * sizeof(float)));
      XFP_CUDA(ctx, (convert<IT, SIT>(inv, reinterpret_cast<SIT*>(ctx->inv32.p), M, st)));
      sinv = reinterpret_cast<const SIT*>(ctx->inv32.p);
    }
    SweepData<VT, SIT, CT> d;
    d.r = r; d.y = z; d.lx = L[0]; d.ly = L[1]; d.lz = L[2]; d.inv = sinv;
    d.partials = ctx->tpartials.as<double>();
    d.sy = ctx->sy.as<unsigned long long>();
    d.sz = ctx->sz.as<unsigned long long>();
    SweepGrid g = make_grid(ctx, nullptr, 0);
    if ((rc = sweep_copies<VT, SIT, CT>(ctx, L, sinv, r, &g, 1, &d))) return rc;
    if ((rc = run_sweep<VT, SIT, CT>(ctx, SWEEP_FWD, g, d))) return rc;
    // the solve results are in the sweep layout: back to the line layout
    if ((rc = sweep_result<VT>(ctx, z))) return rc;
    XFP_CUDA(ctx, cudaStreamSynchronize(st));
    if ((rc = dump_dense<VT>(ctx, z, out[9]))) return rc;
    if ((rc = run_sweep<VT, SIT, CT>(ctx, SWEEP_BWD, g, d))) return rc;
    if ((rc = sweep_result<VT>(ctx, z))) return rc;
    XFP_CUDA(ctx, (spmv_dot<VT, VT, VT>(Av[0], Av[1], Av[2], Av[3], r, qv, ctx->lines.as<Line>(),
                                        ctx->group_line.as<int>(), ctx->nj, ctx->nk, M, nullptr, (VT*)nullptr,
                                        NBLK_MAX, 1, st)));
  }
  XFP_CUDA(ctx, cudaStreamSynchronize(st));
  if ((rc = check_sweep_error(ctx))) return rc;
  for (int q = 0; q < 5; ++q)
    if ((rc = dump_dense<CT>(ctx, Af[q], out[q]))) return rc;
  if ((rc = dump_dense<IT>(ctx, inv, out[5]))) return rc;
  for (int q = 0; q < 3; ++q)
    if ((rc = dump_dense<CT>(ctx, F[q], out[6 + q]))) return rc;
  if (dr) {
    if ((rc = dump_dense<VT>(ctx, z, out[10]))) return rc;
    if ((rc = dump_dense<VT>(ctx, qv, out[11]))) return rc;
  }
  return XFP_OK;
}

// ---------------------------------------------------------------- steps either side
// The force as FluidSimulator::_applyForces forms it (FluidSimulator.cpp:431-438):
// the summed force times dt, per axis.
Force3 make_force(const double* force, double dt) {
  Force3 f;
  if (!force) return f;
  f.on = 1;
  for (int a = 0; a < 3; ++a) f.d[a] = force[a] * dt;
  return f;
}

template <typename IOT>
int forces_impl(xfp_ctx* ctx, int ni, int nj, int nk, const uint8_t* mat, IOT* u, IOT* v, IOT* w,
                const double* force, double dt) {
  int rc = check_dims(ctx, ni, nj, nk, mat);
  if (rc) return rc;
  if (!u || !v || !w || !force) return fail(ctx, XFP_ERR_ARGS, "NULL array or force");
  XFP_CUDA(ctx, cudaSetDevice(ctx->device));
  const uint8_t* dmat;
  const IOT *du_, *dv, *dw;
  if ((rc = stage_in(ctx, ctx->io_mat, mat, ncells(ni, nj, nk), &dmat))) return rc;
  if ((rc = stage_in<IOT>(ctx, ctx->io_u, u, nu(ni, nj, nk), &du_))) return rc;
  if ((rc = stage_in<IOT>(ctx, ctx->io_v, v, nv(ni, nj, nk), &dv))) return rc;
  if ((rc = stage_in<IOT>(ctx, ctx->io_w, w, nw_(ni, nj, nk), &dw))) return rc;
  XFP_CUDA(ctx, apply_forces<IOT>(dmat, ni, nj, nk, const_cast<IOT*>(du_), const_cast<IOT*>(dv),
                                  const_cast<IOT*>(dw), make_force(force, dt), ctx->stream));
  if (!ctx->opt.device_pointers) {
    XFP_CUDA(ctx, cudaMemcpyAsync(u, du_, nu(ni, nj, nk) * sizeof(IOT), cudaMemcpyDeviceToHost, ctx->stream));
    XFP_CUDA(ctx, cudaMemcpyAsync(v, dv, nv(ni, nj, nk) * sizeof(IOT), cudaMemcpyDeviceToHost, ctx->stream));
    XFP_CUDA(ctx, cudaMemcpyAsync(w, dw, nw_(ni, nj, nk) * sizeof(IOT), cudaMemcpyDeviceToHost, ctx->stream));
  }
  XFP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return XFP_OK;
}

constexpr int kMaxLayers = 30000;   // the layer marker is 16-bit

template <typename IOT>
int extrapolate_impl(xfp_ctx* ctx, int ni, int nj, int nk, const uint8_t* mat, IOT* u, IOT* v, IOT* w,
                     int layers) {
  int rc = check_dims(ctx, ni, nj, nk, mat);
  if (rc) return rc;
  if (!u || !v || !w) return fail(ctx, XFP_ERR_ARGS, "NULL array");
  if (layers < 0 || layers > kMaxLayers) return fail(ctx, XFP_ERR_ARGS, "layers must be in [0, 30000]");
  XFP_CUDA(ctx, cudaSetDevice(ctx->device));
  const uint8_t* dmat;
  const IOT *du_, *dv, *dw;
  if ((rc = stage_in(ctx, ctx->io_mat, mat, ncells(ni, nj, nk), &dmat))) return rc;
  if ((rc = stage_in<IOT>(ctx, ctx->io_u, u, nu(ni, nj, nk), &du_))) return rc;
  if ((rc = stage_in<IOT>(ctx, ctx->io_v, v, nv(ni, nj, nk), &dv))) return rc;
  if ((rc = stage_in<IOT>(ctx, ctx->io_w, w, nw_(ni, nj, nk), &dw))) return rc;
  XFP_CUDA(ctx, ctx->xmarker.ensure((size_t)(ni + 1) * (nj + 1) * (nk + 1) * sizeof(short)));
  XFP_CUDA(ctx, extrapolate<IOT>(dmat, ni, nj, nk, const_cast<IOT*>(du_), const_cast<IOT*>(dv),
                                 const_cast<IOT*>(dw), layers, ctx->xmarker.as<short>(), ctx->stream));
  if (!ctx->opt.device_pointers) {
    XFP_CUDA(ctx, cudaMemcpyAsync(u, du_, nu(ni, nj, nk) * sizeof(IOT), cudaMemcpyDeviceToHost, ctx->stream));
    XFP_CUDA(ctx, cudaMemcpyAsync(v, dv, nv(ni, nj, nk) * sizeof(IOT), cudaMemcpyDeviceToHost, ctx->stream));
    XFP_CUDA(ctx, cudaMemcpyAsync(w, dw, nw_(ni, nj, nk) * sizeof(IOT), cudaMemcpyDeviceToHost, ctx->stream));
  }
  XFP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return XFP_OK;
}

// VariationalPressureSolver::_calculate_divergience on the device.
template <typename IOT>
int divergence_impl(xfp_ctx* ctx, int ni, int nj, int nk, const uint8_t* mat, const IOT* u, const IOT* v,
                    const IOT* w, IOT* div) {
  int rc = check_dims(ctx, ni, nj, nk, mat);
  if (rc) return rc;
  if (!u || !v || !w || !div) return fail(ctx, XFP_ERR_ARGS, "NULL array");
  XFP_CUDA(ctx, cudaSetDevice(ctx->device));
  const uint8_t* dmat;
  const IOT *du_, *dv, *dw;
  if ((rc = stage_in(ctx, ctx->io_mat, mat, ncells(ni, nj, nk), &dmat))) return rc;
  if ((rc = stage_in<IOT>(ctx, ctx->io_u, u, nu(ni, nj, nk), &du_))) return rc;
  if ((rc = stage_in<IOT>(ctx, ctx->io_v, v, nv(ni, nj, nk), &dv))) return rc;
  if ((rc = stage_in<IOT>(ctx, ctx->io_w, w, nw_(ni, nj, nk), &dw))) return rc;
  IOT* dd = div;
  if (!ctx->opt.device_pointers) {
    XFP_CUDA(ctx, ctx->io_p.ensure(ncells(ni, nj, nk) * sizeof(IOT)));
    dd = ctx->io_p.as<IOT>();
  }
  XFP_CUDA(ctx, divergence<IOT>(dmat, ni, nj, nk, du_, dv, dw, dd, ctx->stream));
  if (!ctx->opt.device_pointers)
    XFP_CUDA(ctx, cudaMemcpyAsync(div, dd, ncells(ni, nj, nk) * sizeof(IOT), cudaMemcpyDeviceToHost, ctx->stream));
  XFP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return XFP_OK;
}

// Force fused into assembly and apply, projection, extrapolation on the
// projected velocities, one call.
template <typename IOT>
int step_impl(xfp_ctx* ctx, int ni, int nj, int nk, const uint8_t* mat, IOT* u, IOT* v, IOT* w, const IOT* wu,
              const IOT* wv, const IOT* ww, IOT* pressure, const double* force, double dt, int layers,
              xfp_stats* stats) {
  if (!ctx) return XFP_ERR_ARGS;
  if (layers < 0 || layers > kMaxLayers) return fail(ctx, XFP_ERR_ARGS, "layers must be in [0, 30000]");
  ctx->force = make_force(force, dt);
  ctx->step_layers = layers;
  const int rc = project_impl<IOT>(ctx, ni, nj, nk, mat, u, v, w, wu, wv, ww, pressure, stats, true);
  ctx->force = Force3();
  ctx->step_layers = 0;
  return rc;
}

}  // namespace xfp_host

using namespace xfp_host;

// ============================================================================ C ABI
extern "C" {

const char* xfp_version(void) { return "xfp 0.1 (sm_100a)"; }

void xfp_default_options(xfp_options* o) {
  if (!o) return;
  memset(o, 0, sizeof(*o));
  o->tol = 1e-5;
  o->max_iter = 100;
  o->omega = 0.97;
  o->min_diag_ratio = 0.25;
  o->precision = XFP_PREC_F64;
  o->device_pointers = 0;
  o->device = 0;
  o->check_every = 8;
  o->timeout_ms = 2000.0;
  o->max_refine = 20;
  o->inner_tol = 1e-6;
  o->tile_k = 0;
  o->matrix = XFP_MATRIX_VARIATIONAL;
  o->stream = nullptr;
}

static int validate_options(xfp_ctx* ctx, const xfp_options* o) {
  if (o->precision < XFP_PREC_F64 || o->precision > XFP_PREC_MIXED) return fail(ctx, XFP_ERR_ARGS, "bad precision");
  if (!(o->omega >= 0.0 && o->omega <= 1.0)) return fail(ctx, XFP_ERR_ARGS, "omega must be in [0,1]");
  if (!(o->min_diag_ratio >= 0.0)) return fail(ctx, XFP_ERR_ARGS, "min_diag_ratio must be >= 0");
  if (o->tile_k != 0 && o->tile_k != 8 && o->tile_k != 15 && o->tile_k != 16)
    return fail(ctx, XFP_ERR_ARGS, "tile_k must be 0, 8, 15 or 16");
  if (o->matrix != XFP_MATRIX_VARIATIONAL && o->matrix != XFP_MATRIX_NORMAL)
    return fail(ctx, XFP_ERR_ARGS, "matrix must be XFP_MATRIX_VARIATIONAL or XFP_MATRIX_NORMAL");
  return XFP_OK;
}

int xfp_create(xfp_ctx** out, const xfp_options* opt) {
  if (!out) return XFP_ERR_ARGS;
  *out = nullptr;
  xfp_ctx* ctx = new xfp_ctx();
  xfp_options o;
  xfp_default_options(&o);
  if (opt) o = *opt;
  int rc = validate_options(ctx, &o);
  if (rc) { delete ctx; return rc; }
  ctx->opt = o;
  ctx->device = o.device;
  ctx->nw = o.tile_k ? o.tile_k : 8;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    delete ctx;
    return XFP_ERR_CUDA;
  }
  if (o.device < 0 || o.device >= ndev || cudaSetDevice(o.device) != cudaSuccess) {
    delete ctx;
    return XFP_ERR_ARGS;
  }
  cudaDeviceGetAttribute(&ctx->nsm, cudaDevAttrMultiProcessorCount, o.device);
  if (o.stream) {
    ctx->stream = (cudaStream_t)o.stream;
  } else {
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
      delete ctx;
      return XFP_ERR_CUDA;
    }
    ctx->own_stream = true;
  }
  for (auto& e : ctx->ev) cudaEventCreate(&e);
  if (cudaStreamCreateWithFlags(&ctx->io_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&ctx->ev_io_mat, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&ctx->ev_io_in, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&ctx->ev_io_p, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    ctx->io_stream = nullptr;
  }
  ctx->sweep_ev.resize(2048);
  ctx->sweep_work.assign(1024, 0);
  ctx->sweep_ord_of.assign(1024, 0);
  for (auto& e : ctx->sweep_ev) cudaEventCreate(&e);
  ctx->kern_ev.resize(3072);
  ctx->kern_kind.assign(1536, -1);
  ctx->kern_iter.assign(1536, 0);
  for (auto& e : ctx->kern_ev) cudaEventCreate(&e);
  if (const char* e = getenv("XFP_STAGE_SOLVES")) ctx->stage_solves = atoi(e) != 0;
  if (const char* e = getenv("XFP_VEC_BLOCKS")) ctx->vec_blocks = std::max(148, std::min(xfp_host::NBLK_MAX, atoi(e)));
  if (const char* e = getenv("XFP_KERNEL_EVENTS")) ctx->event_every = std::max(0, atoi(e));
  if (const char* e = getenv("XFP_XR_BLOCKS")) ctx->xr_blocks = std::max(148, std::min(xfp_host::NBLK_MAX, atoi(e)));
  if (const char* e = getenv("XFP_S_BLOCKS")) ctx->s_blocks = std::max(148, std::min(148 * 32, atoi(e)));
  if (const char* e = getenv("XFP_HOST_FACES")) ctx->host_sparse_ok = strcmp(e, "full") != 0;
  if (getenv("XFP_TRACE")) {
    ctx->tracing = true;
    ctx->trace.ensure(1024 * 40 * 4 * sizeof(int));
    cudaMemset(ctx->trace.p, 0xff, ctx->trace.cap);
  }
  if (ctx->ctl.ensure(sizeof(SweepCtl)) != cudaSuccess) { xfp_destroy(ctx); return XFP_ERR_NOMEM; }
  SweepCtl c0{};
  c0.gen = 1;
  cudaMemcpy(ctx->ctl.p, &c0, sizeof(c0), cudaMemcpyHostToDevice);
  *out = ctx;
  return XFP_OK;
}

int xfp_destroy(xfp_ctx* ctx) {
  if (!ctx) return XFP_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  DevBuf* all[] = {&ctx->io_mat, &ctx->io_u, &ctx->io_v, &ctx->io_w, &ctx->io_wu, &ctx->io_wv, &ctx->io_ww,
                   &ctx->io_p, &ctx->io_gu, &ctx->io_gv, &ctx->io_gw, &ctx->lines, &ctx->lens,
                   &ctx->tile_active, &ctx->tiles, &ctx->counters, &ctx->cell_line, &ctx->group_line, &ctx->inv64, &ctx->inv32, &ctx->x64,
                   &ctx->r64, &ctx->x32, &ctx->r32, &ctx->s32, &ctx->z32, &ctx->s64, &ctx->z64, &ctx->dense,
                   &ctx->sy, &ctx->sz, &ctx->bnd, &ctx->ctl, &ctx->scal, &ctx->scal2, &ctx->partials,
                   &ctx->tpartials};
  for (DevBuf* b : all) b->release();
  batch_state_free(ctx->batch);
  ctx->batch = nullptr;
  for (auto& b : ctx->A64) b.release();
  for (auto& b : ctx->A32) b.release();
  for (auto& b : ctx->F64) b.release();
  for (auto& b : ctx->F32) b.release();
  for (auto& b : ctx->L32) b.release();
  for (auto& e : ctx->ev)
    if (e) cudaEventDestroy(e);
  for (auto& e : ctx->sweep_ev)
    if (e) cudaEventDestroy(e);
  for (auto& e : ctx->kern_ev)
    if (e) cudaEventDestroy(e);
  if (ctx->io_stream) {
    cudaStreamSynchronize(ctx->io_stream);
    cudaStreamDestroy(ctx->io_stream);
  }
  for (cudaEvent_t e : {ctx->ev_io_mat, ctx->ev_io_in, ctx->ev_io_p})
    if (e) cudaEventDestroy(e);
  if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return XFP_OK;
}

int xfp_set_options(xfp_ctx* ctx, const xfp_options* opt) {
  if (!ctx || !opt) return XFP_ERR_ARGS;
  int rc = validate_options(ctx, opt);
  if (rc) return rc;
  if (opt->device != ctx->device) return fail(ctx, XFP_ERR_ARGS, "device cannot change on a live context");
  void* keep_stream = ctx->opt.stream;
  ctx->opt = *opt;
  ctx->opt.stream = keep_stream;
  int nw = opt->tile_k ? opt->tile_k : 8;
  ctx->nw = nw;
  return XFP_OK;
}

const char* xfp_last_error(const xfp_ctx* ctx) { return ctx ? ctx->err.c_str() : "no context"; }

int xfp_solve_f64(xfp_ctx* ctx, int ni, int nj, int nk, const uint8_t* material, const double* u,
                  const double* v, const double* w, const double* wu, const double* wv, const double* ww,
                  double* pressure, xfp_stats* stats) {
  return project_impl<double>(ctx, ni, nj, nk, material, const_cast<double*>(u), const_cast<double*>(v),
                              const_cast<double*>(w), wu, wv, ww, pressure, stats, false);
}
int xfp_solve_f32(xfp_ctx* ctx, int ni, int nj, int nk, const uint8_t* material, const float* u,
                  const float* v, const float* w, const float* wu, const float* wv, const float* ww,
                  float* pressure, xfp_stats* stats) {
  return project_impl<float>(ctx, ni, nj, nk, material, const_cast<float*>(u), const_cast<float*>(v),
                             const_cast<float*>(w), wu, wv, ww, pressure, stats, false);
}
int xfp_project_f64(xfp_ctx* ctx, int ni, int nj, int nk, const uint8_t* material, double* u, double* v,
                    double* w, const double* wu, const double* wv, const double* ww, double* pressure,
                    xfp_stats* stats) {
  return project_impl<double>(ctx, ni, nj, nk, material, u, v, w, wu, wv, ww, pressure, stats, true);
}
int xfp_project_f32(xfp_ctx* ctx, int ni, int nj, int nk, const uint8_t* material, float* u, float* v,
                    float* w, const float* wu, const float* wv, const float* ww, float* pressure,
                    xfp_stats* stats) {
  return project_impl<float>(ctx, ni, nj, nk, material, u, v, w, wu, wv, ww, pressure, stats, true);
}
int xfp_apply_pressure_f64(xfp_ctx* ctx, int ni, int nj, int nk, const uint8_t* material, const double* wu,
                           const double* wv, const double* ww, const double* pressure, double* u, double* v,
                           double* w) {
  return apply_impl<double>(ctx, ni, nj, nk, material, wu, wv, ww, pressure, u, v, w);
}
int xfp_apply_pressure_f32(xfp_ctx* ctx, int ni, int nj, int nk, const uint8_t* material, const float* wu,
                           const float* wv, const float* ww, const float* pressure, float* u, float* v,
                           float* w) {
  return apply_impl<float>(ctx, ni, nj, nk, material, wu, wv, ww, pressure, u, v, w);
}
int xfp_project_backward_f64(xfp_ctx* ctx, int ni, int nj, int nk, const uint8_t* material, const double* wu,
                             const double* wv, const double* ww, const double* gu, const double* gv,
                             const double* gw, double* du, double* dv, double* dw, xfp_stats* stats) {
  return backward_impl<double>(ctx, ni, nj, nk, material, wu, wv, ww, gu, gv, gw, du, dv, dw, stats);
}
int xfp_debug_stages(xfp_ctx* ctx, int ni, int nj, int nk, const uint8_t* material, const double* u,
                     const double* v, const double* w, const double* wu, const double* wv, const double* ww,
                     const double* r, double* diag, double* ax, double* ay, double* az, double* b, double* inv,
                     double* lx, double* ly, double* lz, double* y, double* z, double* q) {
  int rc = check_dims(ctx, ni, nj, nk, material);
  if (rc) return rc;
  if (!u || !v || !w) return fail(ctx, XFP_ERR_ARGS, "velocity arrays must not be NULL");
  if (ctx->opt.device_pointers) return fail(ctx, XFP_ERR_UNSUPPORTED, "diagnostics take host pointers");
  XFP_CUDA(ctx, cudaSetDevice(ctx->device));
  const uint8_t* dmat;
  const double *du_, *dv, *dw, *dwu, *dwv, *dww;
  if ((rc = stage_in(ctx, ctx->io_mat, material, ncells(ni, nj, nk), &dmat))) return rc;
  if ((rc = stage_in<double>(ctx, ctx->io_u, u, nu(ni, nj, nk), &du_))) return rc;
  if ((rc = stage_in<double>(ctx, ctx->io_v, v, nv(ni, nj, nk), &dv))) return rc;
  if ((rc = stage_in<double>(ctx, ctx->io_w, w, nw_(ni, nj, nk), &dw))) return rc;
  if ((rc = stage_in<double>(ctx, ctx->io_wu, wu, nu(ni, nj, nk), &dwu))) return rc;
  if ((rc = stage_in<double>(ctx, ctx->io_wv, wv, nv(ni, nj, nk), &dwv))) return rc;
  if ((rc = stage_in<double>(ctx, ctx->io_ww, ww, nw_(ni, nj, nk), &dww))) return rc;
  const int prec = ctx->opt.precision;
  if ((rc = build_layout(ctx, dmat, ni, nj, nk))) return rc;
  if ((rc = ensure_compact(ctx, prec))) return rc;
  if (prec == XFP_PREC_F64) {
    XFP_CUDA(ctx, ctx->s64.ensure((ctx->M + 8) * 8));
    XFP_CUDA(ctx, ctx->z64.ensure((ctx->M + 8) * 8));
  }
  const Line* lines = ctx->lines.as<Line>();
  double* out[12] = {diag, ax, ay, az, b, inv, lx, ly, lz, y, z, q};
  cudaStream_t st = ctx->stream;
  if (prec == XFP_PREC_F64) {
    double* A[5];
    for (int k = 0; k < 5; ++k) A[k] = ctx->A64[k].as<double>();
    XFP_CUDA(ctx, (assemble<double, double>(dmat, du_, dv, dw, dwu, dwv, dww, ni, nj, nk, lines, A[0], A[1], A[2],
                                            A[3], A[4], st, ctx->opt.matrix)));
    double* F[6];
    for (int k = 0; k < 6; ++k) F[k] = ctx->F64[k].as<double>();
    const double* Af[5] = {A[0], A[1], A[2], A[3], A[4]};
    const double* Av[4] = {A[0], A[1], A[2], A[3]};
    const double* L[3] = {F[0], F[1], F[2]};
    return debug_core<double, double, double>(ctx, Af, Av, F, ctx->inv64.as<double>(), L, r, out);
  } else if (prec == XFP_PREC_F32) {
    float* A[5];
    for (int k = 0; k < 5; ++k) A[k] = ctx->A32[k].as<float>();
    XFP_CUDA(ctx, (assemble<double, float>(dmat, du_, dv, dw, dwu, dwv, dww, ni, nj, nk, lines, A[0], A[1], A[2],
                                           A[3], A[4], st, ctx->opt.matrix)));
    float* F[6];
    for (int k = 0; k < 6; ++k) F[k] = ctx->F32[k].as<float>();
    const float* Af[5] = {A[0], A[1], A[2], A[3], A[4]};
    const float* Av[4] = {A[0], A[1], A[2], A[3]};
    const float* L[3] = {F[0], F[1], F[2]};
    return debug_core<float, float, float>(ctx, Af, Av, F, ctx->inv32.as<float>(), L, r, out);
  } else {
    double* A[5];
    for (int k = 0; k < 5; ++k) A[k] = ctx->A64[k].as<double>();
    XFP_CUDA(ctx, (assemble<double, double>(dmat, du_, dv, dw, dwu, dwv, dww, ni, nj, nk, lines, A[0], A[1], A[2],
                                            A[3], A[4], st, ctx->opt.matrix)));
    float* A32[4];
    for (int k = 0; k < 4; ++k) {
      A32[k] = ctx->A32[k].as<float>();
      XFP_CUDA(ctx, (convert<double, float>(A[k], A32[k], ctx->M, st)));
    }
    double* F[6];
    for (int k = 0; k < 6; ++k) F[k] = ctx->F64[k].as<double>();
    const double* Af[5] = {A[0], A[1], A[2], A[3], A[4]};
    const float* Av[4] = {A32[0], A32[1], A32[2], A32[3]};
    const float* L[3] = {ctx->L32[0].as<float>(), ctx->L32[1].as<float>(), ctx->L32[2].as<float>()};
    return debug_core<float, double, double, float>(ctx, Af, Av, F, ctx->inv64.as<double>(), L, r, out);
  }
}

int xfp_project_backward_f32(xfp_ctx* ctx, int ni, int nj, int nk, const uint8_t* material, const float* wu,
                             const float* wv, const float* ww, const float* gu, const float* gv,
                             const float* gw, float* du, float* dv, float* dw, xfp_stats* stats) {
  return backward_impl<float>(ctx, ni, nj, nk, material, wu, wv, ww, gu, gv, gw, du, dv, dw, stats);
}

}  // extern "C"

extern "C" int xfp_debug_expire_next_sweep(xfp_ctx* ctx) {
  if (!ctx) return XFP_ERR_ARGS;
  ctx->expire_next_sweep = true;
  return XFP_OK;
}

int xfp_apply_forces_f64(xfp_ctx* ctx, int ni, int nj, int nk, const uint8_t* material, double* u, double* v,
                         double* w, const double force[3], double dt) {
  return forces_impl<double>(ctx, ni, nj, nk, material, u, v, w, force, dt);
}
int xfp_apply_forces_f32(xfp_ctx* ctx, int ni, int nj, int nk, const uint8_t* material, float* u, float* v,
                         float* w, const double force[3], double dt) {
  return forces_impl<float>(ctx, ni, nj, nk, material, u, v, w, force, dt);
}
int xfp_extrapolate_f64(xfp_ctx* ctx, int ni, int nj, int nk, const uint8_t* material, double* u, double* v,
                        double* w, int layers) {
  return extrapolate_impl<double>(ctx, ni, nj, nk, material, u, v, w, layers);
}
int xfp_extrapolate_f32(xfp_ctx* ctx, int ni, int nj, int nk, const uint8_t* material, float* u, float* v,
                        float* w, int layers) {
  return extrapolate_impl<float>(ctx, ni, nj, nk, material, u, v, w, layers);
}

int xfp_divergence_f64(xfp_ctx* ctx, int ni, int nj, int nk, const uint8_t* material, const double* u, const double* v,
                       const double* w, double* div) {
  if (!ctx) return XFP_ERR_ARGS;
  return divergence_impl<double>(ctx, ni, nj, nk, material, u, v, w, div);
}
int xfp_divergence_f32(xfp_ctx* ctx, int ni, int nj, int nk, const uint8_t* material, const float* u, const float* v,
                       const float* w, float* div) {
  if (!ctx) return XFP_ERR_ARGS;
  return divergence_impl<float>(ctx, ni, nj, nk, material, u, v, w, div);
}
int xfp_project_step_f64(xfp_ctx* ctx, int ni, int nj, int nk, const uint8_t* material, double* u, double* v,
                         double* w, const double* wu, const double* wv, const double* ww, double* pressure,
                         const double force[3], double dt, int layers, xfp_stats* stats) {
  return step_impl<double>(ctx, ni, nj, nk, material, u, v, w, wu, wv, ww, pressure, force, dt, layers, stats);
}
int xfp_project_step_f32(xfp_ctx* ctx, int ni, int nj, int nk, const uint8_t* material, float* u, float* v,
                         float* w, const float* wu, const float* wv, const float* ww, float* pressure,
                         const double force[3], double dt, int layers, xfp_stats* stats) {
  return step_impl<float>(ctx, ni, nj, nk, material, u, v, w, wu, wv, ww, pressure, force, dt, layers, stats);
}
