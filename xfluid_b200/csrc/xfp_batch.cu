// xfp_batch.cu -- xfp_project_batch_{f32,f64}: many independent scenes of
// different sizes projected together.
//
// Every scene gets its own line table, compact slice [base, base+M) of the
// shared compact arrays and its own PCG scalars, so each is solved exactly as
// a single-scene call solves it.  What is shared:
//   * the MIC(0) sweeps: the active tiles of all scenes form one list, merged
//     by wavefront level (J+K), and one persistent launch walks it.  A lone
//     256^3 wavefront leaves most SMs waiting on its dependency chain; the
//     tiles of other scenes fill them.
//   * the vector kernels: one launch per kernel covers all scenes, each scene
//     running the same block decomposition (and so the same reduction order)
//     as its single-scene launch would.
//   * the PCG iteration is captured once as a CUDA graph (check_every
//     iterations: SpMV+dot, x/r update, forward, backward, rho/beta, s update)
//     and replayed until every scene has converged or hit its cap.
//   * the sweep tile height: with options.tile_k == 0 the heights 8, 15 and 16
//     are timed on the first call for a batch shape and the fastest is cached.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <type_traits>
#include <vector>

#include "xfp_context.h"

using namespace xfp;

namespace xfp_host {

struct BatchState {
  DevBuf lines, lens, tile_active, scene_tile_lists, counters;
  DevBuf segs, tiles, tile_scene, scal, scal2, part, tols, maxits;
  DevBuf io, pdense;
  std::vector<BatchSeg> hsegs;
  std::vector<long long> line_base, rows, nlines_act;
  int n = 0, nw = 0, ntiles = 0, blocks_lines = 0, blocks_cells = 0, blocks_groups = 0;
  long long M = 0;
  std::map<std::string, int> tuned;   // batch shape -> sweep tile height
  std::string layout_key;             // shape + tile height of the layout built last
  bool graph_used = false;
};

void batch_state_free(BatchState* b) {
  if (!b) return;
  DevBuf* all[] = {&b->lines, &b->lens, &b->tile_active, &b->scene_tile_lists, &b->counters, &b->segs,
                   &b->tiles, &b->tile_scene, &b->scal, &b->scal2, &b->part,
                   &b->tols, &b->maxits, &b->io, &b->pdense};
  for (DevBuf* d : all) d->release();
  delete b;
}

namespace {

// One scene with its arrays on the device.
template <typename T>
struct DevScene {
  int ni, nj, nk;
  const uint8_t* mat;
  T *u, *v, *w;
  const T *wu, *wv, *ww;
  T* p;
};

std::string shape_key(int n, const xfp_scene* sc, int prec) {
  std::string k = std::to_string(prec) + ":";
  for (int s = 0; s < n; ++s)
    k += std::to_string(sc[s].ni) + "x" + std::to_string(sc[s].nj) + "x" + std::to_string(sc[s].nk) + ",";
  return k;
}

// Line tables, compact slices and the merged tile list for tile height nw.
template <typename T>
int batch_layout(xfp_ctx* ctx, BatchState* B, const std::vector<DevScene<T>>& S, int nw) {
  cudaStream_t st = ctx->stream;
  const int n = (int)S.size();
  std::vector<long long> tile_base(n + 1, 0);
  B->line_base.assign(n + 1, 0);
  for (int s = 0; s < n; ++s) {
    B->line_base[s + 1] = B->line_base[s] + (long long)S[s].nj * S[s].nk;
    const long long NJt = (S[s].nj + 31) / 32, NKt = (S[s].nk + nw - 1) / nw;
    tile_base[s + 1] = tile_base[s] + NJt * NKt;
  }
  const long long nlines = B->line_base[n], ntile_slots = tile_base[n];
  XFP_CUDA(ctx, B->lines.ensure(nlines * sizeof(Line)));
  XFP_CUDA(ctx, B->lens.ensure((nlines + n) * sizeof(int)));
  XFP_CUDA(ctx, B->tile_active.ensure(ntile_slots));
  XFP_CUDA(ctx, B->scene_tile_lists.ensure(ntile_slots * sizeof(int)));
  XFP_CUDA(ctx, B->counters.ensure((size_t)n * 4 * sizeof(long long)));
  Line* lines = B->lines.as<Line>();
  for (int s = 0; s < n; ++s) {
    LayoutDev L{lines + B->line_base[s], B->lens.as<int>() + B->line_base[s] + s,
                B->tile_active.as<unsigned char>() + tile_base[s], B->scene_tile_lists.as<int>() + tile_base[s],
                B->counters.as<long long>() + 4 * s};
    XFP_CUDA(ctx, layout_build(S[s].mat, S[s].ni, S[s].nj, S[s].nk, nw, L, st));
  }
  std::vector<long long> cnt((size_t)n * 4);
  XFP_CUDA(ctx, cudaMemcpyAsync(cnt.data(), B->counters.p, cnt.size() * sizeof(long long), cudaMemcpyDeviceToHost,
                                st));
  XFP_CUDA(ctx, cudaStreamSynchronize(st));
  // compact slices: scene s occupies [base_s, base_s + M_s); line offsets made global
  std::vector<long long> base(n + 1, 0);
  B->rows.assign(n, 0);
  B->nlines_act.assign(n, 0);
  for (int s = 0; s < n; ++s) {
    base[s + 1] = base[s] + cnt[4 * s];
    B->rows[s] = cnt[4 * s + 1];
    B->nlines_act[s] = cnt[4 * s + 2];
  }
  if (base[n] >= (1LL << 31)) return fail(ctx, XFP_ERR_ARGS, "batch too large: more than 2^31 stored cells");
  for (int s = 0; s < n; ++s)
    XFP_CUDA(ctx, offset_lines(lines + B->line_base[s], B->line_base[s + 1] - B->line_base[s], base[s], st));
  // cell -> line index (line numbers local to each scene's table; cells global)
  XFP_CUDA(ctx, ctx->cell_line.ensure((std::max<long long>(base[n], 4) + 8) * sizeof(int)));
  XFP_CUDA(ctx, ctx->group_line.ensure((std::max<long long>(base[n], 4) / 4 + 8) * sizeof(int)));
  for (int s = 0; s < n; ++s)
    XFP_CUDA(ctx, build_cell_line(lines + B->line_base[s], B->line_base[s + 1] - B->line_base[s],
                                  ctx->cell_line.as<int>(), ctx->group_line.as<int>(), st));
  // merge the scenes' tile lists by wavefront level (each list is already in
  // its own topological order, which the merge keeps)
  std::vector<int> all_tiles(ntile_slots > 0 ? ntile_slots : 1);
  if (ntile_slots > 0)
    XFP_CUDA(ctx, cudaMemcpyAsync(all_tiles.data(), B->scene_tile_lists.p, ntile_slots * sizeof(int),
                                  cudaMemcpyDeviceToHost, st));
  XFP_CUDA(ctx, cudaStreamSynchronize(st));
  struct Item {
    int level, scene, idx, packed;
  };
  std::vector<Item> items;
  for (int s = 0; s < n; ++s)
    for (long long q = 0; q < cnt[4 * s + 3]; ++q) {
      const int packed = all_tiles[tile_base[s] + q];
      items.push_back({(packed & 0xffff) + (packed >> 16), s, (int)q, packed});
    }
  std::stable_sort(items.begin(), items.end(), [](const Item& a, const Item& b) {
    return a.level != b.level ? a.level < b.level : a.scene != b.scene ? a.scene < b.scene : a.idx < b.idx;
  });
  const int nt = (int)items.size();
  std::vector<int> tiles(std::max(nt, 1)), tscene(std::max(nt, 1));
  for (int t = 0; t < nt; ++t) {
    tiles[t] = items[t].packed;
    tscene[t] = items[t].scene;
  }
  // per-scene block decomposition of the vector kernels (as a single launch)
  B->hsegs.assign(n, BatchSeg{});
  XFP_CUDA(ctx, B->part.ensure((size_t)n * NBLK_MAX * sizeof(double)));
  int bl = 0, bc = 0, bg = 0;
  for (int s = 0; s < n; ++s) {
    BatchSeg& g = B->hsegs[s];
    const long long nl = (long long)S[s].nj * S[s].nk, Ms = cnt[4 * s];
    g.ni = S[s].ni; g.nj = S[s].nj; g.nk = S[s].nk;
    g.blk_lines = (int)std::max<long long>(1, std::min<long long>((nl + 7) / 8, NBLK_MAX));
    g.blk_lines_start = bl;
    // the cell-based kernels run one thread per 4-cell group (absmax_init and
    // the residual stride over single cells with the same blocks)
    g.blk_cells = (int)std::max<long long>(1, std::min<long long>((Ms / 4 + 255) / 256, NBLK_MAX));
    g.blk_cells_start = bc;
    g.blk_groups = (int)spmv_block_count(Ms, NBLK_MAX);
    g.blk_groups_start = bg;
    g.tile_base = (int)tile_base[s];
    g.base = base[s];
    g.M = Ms;
    g.lines = lines + B->line_base[s];
    g.partials = B->part.as<double>() + (size_t)s * NBLK_MAX;
    g.line_base = B->line_base[s];
    bl += g.blk_lines;
    bc += g.blk_cells;
    bg += g.blk_groups;
  }
  B->blocks_lines = bl;
  B->blocks_cells = bc;
  B->blocks_groups = bg;
  XFP_CUDA(ctx, B->segs.ensure(n * sizeof(BatchSeg)));
  XFP_CUDA(ctx, B->tiles.ensure(tiles.size() * sizeof(int)));
  XFP_CUDA(ctx, B->tile_scene.ensure(tscene.size() * sizeof(int)));
  XFP_CUDA(ctx, cudaMemcpyAsync(B->segs.p, B->hsegs.data(), n * sizeof(BatchSeg), cudaMemcpyHostToDevice, st));
  XFP_CUDA(ctx, cudaMemcpyAsync(B->tiles.p, tiles.data(), tiles.size() * sizeof(int), cudaMemcpyHostToDevice, st));
  XFP_CUDA(ctx, cudaMemcpyAsync(B->tile_scene.p, tscene.data(), tscene.size() * sizeof(int),
                                cudaMemcpyHostToDevice, st));
  // the host vectors above go out of scope: make the copies complete first
  XFP_CUDA(ctx, cudaStreamSynchronize(st));
  B->n = n;
  B->nw = nw;
  B->ntiles = nt;
  B->M = base[n];
  ctx->nw = nw;
  ctx->bnd_ni = 0;
  for (int s = 0; s < n; ++s) ctx->bnd_ni = std::max(ctx->bnd_ni, S[s].ni);
  ctx->M = B->M;
  ctx->ntiles = nt;
  ctx->nlines_all = nlines;
  // Sweep layout over the merged tile list: spans on the device, offsets
  // scanned here, the (scene, K, J) -> tile map filled here, then the cell ->
  // element map scene by scene.
  ctx->Msw = 0;
  if (nt > 0) {
    XFP_CUDA(ctx, ctx->swt.ensure(nt * sizeof(SwTile)));
    XFP_CUDA(ctx, sw_tiles_build_batch(B->tiles.as<int>(), B->tile_scene.as<int>(), B->segs.as<BatchSeg>(), nt, nw,
                                       ctx->swt.as<SwTile>(), st));
    std::vector<SwTile> sw(nt);
    XFP_CUDA(ctx, cudaMemcpyAsync(sw.data(), ctx->swt.p, nt * sizeof(SwTile), cudaMemcpyDeviceToHost, st));
    XFP_CUDA(ctx, cudaStreamSynchronize(st));
    long long off = 0;
    for (auto& e : sw) {
      e.off = off;
      off += (long long)nw * e.ng * 128;
    }
    if (off >= (1LL << 31)) return fail(ctx, XFP_ERR_ARGS, "batch too large for the sweep layout");
    ctx->Msw = off;
    std::vector<int> tpos(std::max<long long>(ntile_slots, 1), -1);
    for (int t = 0; t < nt; ++t) {
      const int sc = tscene[t], J = tiles[t] & 0xffff, K = tiles[t] >> 16;
      tpos[tile_base[sc] + (long long)K * ((S[sc].nj + 31) / 32) + J] = t;
    }
    XFP_CUDA(ctx, ctx->tile_pos.ensure(tpos.size() * sizeof(int)));
    XFP_CUDA(ctx, cudaMemcpyAsync(ctx->swt.p, sw.data(), nt * sizeof(SwTile), cudaMemcpyHostToDevice, st));
    XFP_CUDA(ctx, cudaMemcpyAsync(ctx->tile_pos.p, tpos.data(), tpos.size() * sizeof(int), cudaMemcpyHostToDevice,
                                  st));
    XFP_CUDA(ctx, ctx->sw_perm.ensure((size_t)(std::max<long long>(B->M, 4) + 8) * sizeof(int)));
    for (int sc = 0; sc < n; ++sc)
      XFP_CUDA(ctx, sw_perm_build(ctx->cell_line.as<int>() + base[sc], lines + B->line_base[sc], S[sc].nj, nw,
                                  (S[sc].nj + 31) / 32, ctx->tile_pos.as<int>() + tile_base[sc],
                                  ctx->swt.as<SwTile>(), base[sc + 1] - base[sc], ctx->sw_perm.as<int>() + base[sc],
                                  st, base[sc]));
    XFP_CUDA(ctx, cudaStreamSynchronize(st));
  }
  return XFP_OK;
}

SweepGrid batch_grid(xfp_ctx* ctx, BatchState* B, PcgScalars* sc) {
  SweepGrid g{};
  g.ntiles = B->ntiles;
  g.tiles = B->tiles.as<int>();
  g.ctl = ctx->ctl.as<SweepCtl>();
  g.spin_limit = spin_limit(ctx);
  g.scal = nullptr;
  g.trace = nullptr;
  g.tile_scene = B->tile_scene.as<int>();
  g.segs = B->segs.as<BatchSeg>();
  g.scal_batch = sc;
  g.stage = ctx->stage_solves;
  return g;
}

template <typename VT, typename IT, typename CT>
cudaError_t batch_sweep(xfp_ctx* ctx, BatchState* B, int op, const SweepGrid& g, const SweepData<VT, IT, CT>& d) {
  if (B->ntiles <= 0) return cudaSuccess;
  const int maxg = sweep_max_grid(op, d, B->nw, g.stage);
  if (maxg <= 0) return cudaErrorLaunchOutOfResources;
  return sweep_launch(op, g, d, B->nw, std::min(maxg, B->ntiles), ctx->stream);
}

// Assembly of every scene into the shared compact arrays.
template <typename FT, typename AT>
int batch_assemble(xfp_ctx* ctx, BatchState* B, const std::vector<DevScene<FT>>& S, AT* const A[5]) {
  for (size_t s = 0; s < S.size(); ++s)
    XFP_CUDA(ctx, (assemble<FT, AT>(S[s].mat, S[s].u, S[s].v, S[s].w, S[s].wu, S[s].wv, S[s].ww, S[s].ni, S[s].nj,
                                    S[s].nk, B->hsegs[s].lines, A[0], A[1], A[2], A[3], A[4], ctx->stream)));
  return XFP_OK;
}

// MIC(0) factor of every scene in one sweep launch.
template <typename VT, typename IT, typename CT>
int batch_factor(xfp_ctx* ctx, BatchState* B, const CT* const A[4], CT* const F[6], IT* inv, CT omega, CT ratio) {
  const size_t M = (size_t)std::max<long long>(B->M, 1);
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
  XFP_CUDA(ctx, (batch_sweep<VT, IT, CT>(ctx, B, SWEEP_FACTOR, batch_grid(ctx, B, nullptr), d)));
  return XFP_OK;
}

// PCG (pcg_solver.h:243-285) on every scene at once.  Per-scene tolerance and
// cap come from tol/maxit, or from the device arrays tols/maxits when given.
// On return hsc holds each scene's final scalars.
template <typename VT, typename IT, typename DT>
int batch_pcg(xfp_ctx* ctx, BatchState* B, const VT* const A[4], const VT* b, VT* x, VT* r, VT* s, VT* z,
              const VT* const L[3], const IT* inv, double tol, int maxit, const double* tols, const int* maxits,
              PcgScalars* dsc, std::vector<PcgScalars>& hsc, int maxit_all) {
  cudaStream_t st = ctx->stream;
  const int n = B->n;
  const size_t M = (size_t)std::max<long long>(B->M, 1);
  const BatchSeg* segs = B->segs.as<BatchSeg>();
  int rc0;
  if (tol < 1e-30) tol = 1e-30;
  XFP_CUDA(ctx, cudaMemsetAsync(x, 0, M * sizeof(VT), st));
  XFP_CUDA(ctx, cudaMemsetAsync(dsc, 0, n * sizeof(PcgScalars), st));
  XFP_CUDA(ctx, copy_vec<VT>(b, r, (long long)M, st));
  XFP_CUDA(ctx, batch_absmax_init<VT>(segs, n, B->blocks_cells, r, dsc, tol, maxit, tols, maxits, st));
  SweepData<VT, IT, DT> d;
  d.r = r; d.y = z; d.lx = L[0]; d.ly = L[1]; d.lz = L[2]; d.inv = inv;
  d.partials = ctx->tpartials.as<double>();
  d.sy = ctx->sy.as<unsigned long long>();
  d.sz = ctx->sz.as<unsigned long long>();
  SweepGrid g = batch_grid(ctx, B, dsc);
  // the solves stream the sweep layout (as single scenes do): factor and r
  // copied in, z gathered back through perm
  if ((rc0 = sweep_copies<VT, IT, DT>(ctx, L, inv, r, &g, 1, &d)) != XFP_OK) return rc0;
  const bool swl = B->ntiles > 0;
  VT* rsw = swl ? ctx->sw_r.as<VT>() : nullptr;
  const VT* zsw = swl ? ctx->sw_y.as<VT>() : nullptr;
  const int* perm = swl ? ctx->sw_perm.as<int>() : nullptr;
  const double* lpart = ctx->tpartials.as<double>();
  // lines of inactive tiles are never written: their partials stay zero
  XFP_CUDA(ctx, cudaMemsetAsync(ctx->tpartials.p, 0, std::max<long long>(ctx->nlines_all, 1) * sizeof(double), st));
  XFP_CUDA(ctx, (batch_sweep<VT, IT, DT>(ctx, B, SWEEP_FWD, g, d)));
  XFP_CUDA(ctx, (batch_sweep<VT, IT, DT>(ctx, B, SWEEP_BWD, g, d)));
  XFP_CUDA(ctx, batch_bwd_reduce<DT>(segs, n, lpart, dsc, 0, st));
  if (swl) {
    if ((rc0 = sweep_result<VT>(ctx, s)) != XFP_OK) return rc0;
  } else {
    XFP_CUDA(ctx, copy_vec<VT>(z, s, (long long)M, st));
  }
  auto iteration = [&]() -> cudaError_t {
    cudaError_t e;
    if ((e = batch_spmv_dot<VT, VT, DT>(segs, n, B->blocks_groups, A[0], A[1], A[2], A[3], s, z,
                                        ctx->group_line.as<int>(), dsc, 0, st)))
      return e;
    if ((e = batch_update_xr<VT>(segs, n, B->blocks_cells, x, r, s, z, dsc, st, rsw, perm))) return e;
    if ((e = batch_sweep<VT, IT, DT>(ctx, B, SWEEP_FWD, g, d))) return e;
    if ((e = batch_sweep<VT, IT, DT>(ctx, B, SWEEP_BWD, g, d))) return e;
    if ((e = batch_bwd_reduce<DT>(segs, n, lpart, dsc, 1, st))) return e;
    return batch_update_s<VT>(segs, n, B->blocks_cells, s, z, dsc, st, zsw, perm);
  };
  const int K = ctx->opt.check_every > 0 ? ctx->opt.check_every : 8;
  const int per_iter = B->ntiles > 0 ? 6 : 4;
  // capture K iterations as a graph; if capture is refused, launch directly
  cudaGraphExec_t exec = nullptr;
  {
    cudaGraph_t graph = nullptr;
    const long long before = g_kernel_launches;
    cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      cudaError_t le = cudaSuccess;
      for (int q = 0; q < K && le == cudaSuccess; ++q) le = iteration();
      e = cudaStreamEndCapture(st, &graph);
      if (le != cudaSuccess) e = le;
    }
    if (e == cudaSuccess && graph) e = cudaGraphInstantiate(&exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
      if (exec) cudaGraphExecDestroy(exec);
      exec = nullptr;
      cudaGetLastError();
    }
    g_kernel_launches = before;   // counted per replay below
  }
  B->graph_used = exec != nullptr;
  hsc.assign(n, PcgScalars{});
  int rc = XFP_OK;
  for (int done_iters = 0;;) {
    if (exec) {
      cudaError_t e = cudaGraphLaunch(exec, st);
      if (e != cudaSuccess) { rc = fail(ctx, XFP_ERR_CUDA, std::string("cudaGraphLaunch: ") + cudaGetErrorString(e)); break; }
      g_kernel_launches += (long long)K * per_iter;
    } else {
      for (int q = 0; q < K; ++q) {
        cudaError_t e = iteration();
        if (e != cudaSuccess) { rc = fail(ctx, XFP_ERR_CUDA, std::string("batch iteration: ") + cudaGetErrorString(e)); break; }
      }
      if (rc) break;
    }
    done_iters += K;
    cudaError_t e = cudaMemcpyAsync(hsc.data(), dsc, n * sizeof(PcgScalars), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) { rc = fail(ctx, XFP_ERR_CUDA, std::string("batch scalars: ") + cudaGetErrorString(e)); break; }
    if ((rc = check_sweep_error(ctx)) != XFP_OK) break;
    bool all = true;
    for (int q = 0; q < n; ++q) all &= hsc[q].done != 0;
    if (all) break;
    if (done_iters > maxit_all + 2 * K) { rc = fail(ctx, XFP_ERR_CUDA, "batch PCG loop did not terminate"); break; }
  }
  if (exec) cudaGraphExecDestroy(exec);
  return rc;
}

struct SceneResult {
  int status = XFP_OK, iters = 0, refinements = 0;
  double res = 0, bnorm = 0;
};

// Solve of every scene; the solution ends in x64 (F64, MIXED) or x32 (F32).
template <typename IOT>
int batch_solve(xfp_ctx* ctx, BatchState* B, const std::vector<DevScene<IOT>>& S, std::vector<SceneResult>& out) {
  const int prec = ctx->opt.precision, n = B->n;
  cudaStream_t st = ctx->stream;
  const double tol = ctx->opt.tol, omega = ctx->opt.omega, ratio = ctx->opt.min_diag_ratio;
  const int maxit = ctx->opt.max_iter;
  const long long M = std::max<long long>(B->M, 1);
  XFP_CUDA(ctx, B->scal.ensure(n * sizeof(PcgScalars)));
  XFP_CUDA(ctx, B->scal2.ensure(n * sizeof(PcgScalars)));
  PcgScalars* dsc = B->scal.as<PcgScalars>();
  std::vector<PcgScalars> hsc;
  out.assign(n, SceneResult{});
  int rc;
  if (prec == XFP_PREC_F64 || prec == XFP_PREC_F32) {
    if (prec == XFP_PREC_F64) {
      double* A[5];
      for (int q = 0; q < 5; ++q) A[q] = ctx->A64[q].as<double>();
      if ((rc = batch_assemble<IOT, double>(ctx, B, S, A))) return rc;
      double* F[6];
      for (int q = 0; q < 6; ++q) F[q] = ctx->F64[q].as<double>();
      const double* Ac[4] = {A[0], A[1], A[2], A[3]};
      if ((rc = batch_factor<double, double, double>(ctx, B, Ac, F, ctx->inv64.as<double>(), omega, ratio))) return rc;
      const double* Lc[3] = {F[0], F[1], F[2]};
      rc = batch_pcg<double, double, double>(ctx, B, Ac, A[4], ctx->x64.as<double>(), ctx->r64.as<double>(),
                                             ctx->s64.as<double>(), ctx->z64.as<double>(), Lc,
                                             ctx->inv64.as<double>(), tol, maxit, nullptr, nullptr, dsc, hsc, maxit);
    } else {
      float* A[5];
      for (int q = 0; q < 5; ++q) A[q] = ctx->A32[q].as<float>();
      if ((rc = batch_assemble<IOT, float>(ctx, B, S, A))) return rc;
      float* F[6];
      for (int q = 0; q < 6; ++q) F[q] = ctx->F32[q].as<float>();
      const float* Ac[4] = {A[0], A[1], A[2], A[3]};
      if ((rc = batch_factor<float, float, float>(ctx, B, Ac, F, ctx->inv32.as<float>(), (float)omega,
                                                  (float)ratio)))
        return rc;
      const float* Lc[3] = {F[0], F[1], F[2]};
      rc = batch_pcg<float, float, float>(ctx, B, Ac, A[4], ctx->x32.as<float>(), ctx->r32.as<float>(),
                                          ctx->s32.as<float>(), ctx->z32.as<float>(), Lc, ctx->inv32.as<float>(),
                                          tol, maxit, nullptr, nullptr, dsc, hsc, maxit);
    }
    if (rc < 0) return rc;
    for (int q = 0; q < n; ++q) {
      out[q].iters = hsc[q].iters;
      out[q].res = hsc[q].res;
      out[q].bnorm = hsc[q].bnorm;
      out[q].status = hsc[q].status == XFP_ERR_BREAKDOWN ? XFP_ERR_BREAKDOWN
                      : hsc[q].status == 0               ? XFP_OK
                                                         : XFP_NOT_CONVERGED;
    }
    return XFP_OK;
  }
  // ---- mixed: FP64 system and refinement per scene, FP32 inner PCG ----
  double* A[5];
  for (int q = 0; q < 5; ++q) A[q] = ctx->A64[q].as<double>();
  if ((rc = batch_assemble<IOT, double>(ctx, B, S, A))) return rc;
  float* A32[4];
  for (int q = 0; q < 4; ++q) {
    A32[q] = ctx->A32[q].as<float>();
    XFP_CUDA(ctx, (convert<double, float>(A[q], A32[q], M, st)));
  }
  double* F[6];
  for (int q = 0; q < 6; ++q) F[q] = ctx->F64[q].as<double>();
  const double* Ac[4] = {A[0], A[1], A[2], A[3]};
  if ((rc = batch_factor<float, double, double>(ctx, B, Ac, F, ctx->inv64.as<double>(), omega, ratio))) return rc;
  for (int q = 0; q < 3; ++q) XFP_CUDA(ctx, (convert<double, float>(F[q], ctx->L32[q].as<float>(), M, st)));
  // FP64 pivots, streamed by the FP32 solves rounded to FP32 (as a single scene's mixed solve)
  XFP_CUDA(ctx, (convert<double, float>(ctx->inv64.as<double>(), ctx->inv32.as<float>(), M, st)));
  const float* Lc[3] = {ctx->L32[0].as<float>(), ctx->L32[1].as<float>(), ctx->L32[2].as<float>()};
  const float* A32c[4] = {A32[0], A32[1], A32[2], A32[3]};
  double* x64 = ctx->x64.as<double>();
  double* r64 = ctx->r64.as<double>();
  PcgScalars* osc = B->scal2.as<PcgScalars>();
  const BatchSeg* segs = B->segs.as<BatchSeg>();
  std::vector<PcgScalars> ho(n);
  XFP_CUDA(ctx, cudaMemsetAsync(x64, 0, M * sizeof(double), st));
  XFP_CUDA(ctx, cudaMemsetAsync(osc, 0, n * sizeof(PcgScalars), st));
  XFP_CUDA(ctx, batch_absmax_init<double>(segs, n, B->blocks_cells, A[4], osc, tol, 1, nullptr, nullptr, st));
  XFP_CUDA(ctx, cudaMemcpyAsync(ho.data(), osc, n * sizeof(PcgScalars), cudaMemcpyDeviceToHost, st));
  XFP_CUDA(ctx, cudaStreamSynchronize(st));
  const double t0 = tol < 1e-30 ? 1e-30 : tol;
  std::vector<double> target(n), res(n), tols(n);
  std::vector<int> total(n, 0), cycles(n, 0), maxits(n);
  std::vector<char> fin(n, 0);
  for (int q = 0; q < n; ++q) {
    out[q].bnorm = ho[q].bnorm;
    target[q] = t0 * ho[q].bnorm;
    res[q] = ho[q].bnorm;
    fin[q] = ho[q].bnorm == 0.0;
    out[q].status = fin[q] ? XFP_OK : XFP_NOT_CONVERGED;
  }
  const int max_ref = ctx->opt.max_refine > 0 ? ctx->opt.max_refine : 20;
  const double floor_tol = ctx->opt.inner_tol > 0 ? ctx->opt.inner_tol : 1e-6;
  XFP_CUDA(ctx, B->tols.ensure(n * sizeof(double)));
  XFP_CUDA(ctx, B->maxits.ensure(n * sizeof(int)));
  for (int cyc = 0; cyc < max_ref; ++cyc) {
    if (cyc > 0) {
      XFP_CUDA(ctx, batch_residual64(segs, n, B->blocks_lines, A[0], A[1], A[2], A[3], A[4], x64, r64, osc, st));
      XFP_CUDA(ctx, cudaMemcpyAsync(ho.data(), osc, n * sizeof(PcgScalars), cudaMemcpyDeviceToHost, st));
      XFP_CUDA(ctx, cudaStreamSynchronize(st));
      for (int q = 0; q < n; ++q) {
        if (fin[q]) continue;
        res[q] = ho[q].res;
        if (res[q] <= target[q]) { fin[q] = 1; out[q].status = XFP_OK; }
      }
      XFP_CUDA(ctx, (convert<double, float>(r64, ctx->r32.as<float>(), M, st)));
    } else {
      XFP_CUDA(ctx, (convert<double, float>(A[4], ctx->r32.as<float>(), M, st)));
    }
    bool any = false;
    for (int q = 0; q < n; ++q) {
      const bool run = !fin[q] && total[q] < maxit;
      any |= run;
      tols[q] = run ? std::min(0.5, std::max(floor_tol, 0.5 * target[q] / res[q])) : 0.5;
      maxits[q] = run ? maxit - total[q] : 0;
    }
    if (!any) break;
    XFP_CUDA(ctx, cudaMemcpyAsync(B->tols.p, tols.data(), n * sizeof(double), cudaMemcpyHostToDevice, st));
    XFP_CUDA(ctx, cudaMemcpyAsync(B->maxits.p, maxits.data(), n * sizeof(int), cudaMemcpyHostToDevice, st));
    float* b32 = ctx->A32[4].as<float>();
    XFP_CUDA(ctx, copy_vec<float>(ctx->r32.as<float>(), b32, M, st));
    std::vector<PcgScalars> hin;
    rc = batch_pcg<float, float, double>(ctx, B, A32c, b32, ctx->x32.as<float>(), ctx->r32.as<float>(),
                                         ctx->s32.as<float>(), ctx->z32.as<float>(), Lc, ctx->inv32.as<float>(),
                                          0.5, maxit, B->tols.as<double>(), B->maxits.as<int>(), dsc, hin, maxit);
    if (rc < 0) return rc;
    for (int q = 0; q < n; ++q)
      if (maxits[q] > 0) {
        total[q] += hin[q].iters;
        cycles[q] += 1;
        if (hin[q].status == XFP_ERR_BREAKDOWN) { fin[q] = 1; out[q].status = XFP_ERR_BREAKDOWN; }
      }
    XFP_CUDA(ctx, refine_update(x64, ctx->x32.as<float>(), M, st));
  }
  // scenes that ran out of cycles or iterations: final residual decides
  bool open = false;
  for (int q = 0; q < n; ++q) open |= !fin[q];
  if (open) {
    XFP_CUDA(ctx, batch_residual64(segs, n, B->blocks_lines, A[0], A[1], A[2], A[3], A[4], x64, r64, osc, st));
    XFP_CUDA(ctx, cudaMemcpyAsync(ho.data(), osc, n * sizeof(PcgScalars), cudaMemcpyDeviceToHost, st));
    XFP_CUDA(ctx, cudaStreamSynchronize(st));
    for (int q = 0; q < n; ++q)
      if (!fin[q]) {
        res[q] = ho[q].res;
        if (res[q] <= target[q]) out[q].status = XFP_OK;
      }
  }
  for (int q = 0; q < n; ++q) {
    out[q].iters = total[q];
    out[q].refinements = cycles[q];
    out[q].res = res[q];
  }
  return XFP_OK;
}

// Times one factor and one forward+backward pair over a built layout.
template <typename IOT>
int time_sweeps(xfp_ctx* ctx, BatchState* B, const std::vector<DevScene<IOT>>& S, float* ms) {
  cudaStream_t st = ctx->stream;
  const long long M = std::max<long long>(B->M, 1);
  XFP_CUDA(ctx, B->scal.ensure(B->n * sizeof(PcgScalars)));
  XFP_CUDA(ctx, cudaMemsetAsync(B->scal.p, 0, B->n * sizeof(PcgScalars), st));
  float* A[5];
  for (int q = 0; q < 5; ++q) A[q] = ctx->A32[q].as<float>();
  int rc;
  if ((rc = batch_assemble<IOT, float>(ctx, B, S, A))) return rc;
  float* F[6];
  for (int q = 0; q < 6; ++q) F[q] = ctx->F32[q].as<float>();
  const float* Ac[4] = {A[0], A[1], A[2], A[3]};
  if ((rc = batch_factor<float, float, float>(ctx, B, Ac, F, ctx->inv32.as<float>(), 0.97f, 0.25f))) return rc;
  SweepData<float, float, float> d;
  d.r = A[4]; d.y = ctx->z32.as<float>(); d.lx = F[0]; d.ly = F[1]; d.lz = F[2]; d.inv = ctx->inv32.as<float>();
  d.partials = ctx->tpartials.as<double>();
  d.sy = ctx->sy.as<unsigned long long>();
  d.sz = ctx->sz.as<unsigned long long>();
  SweepGrid g = batch_grid(ctx, B, B->scal.as<PcgScalars>());
  const float* Lf[3] = {F[0], F[1], F[2]};
  if ((rc = sweep_copies<float, float, float>(ctx, Lf, d.inv, d.r, &g, 1, &d))) return rc;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  XFP_CUDA(ctx, (batch_sweep<float, float, float>(ctx, B, SWEEP_FWD, g, d)));   // warm-up
  cudaEventRecord(e0, st);
  for (int q = 0; q < 2; ++q) {
    XFP_CUDA(ctx, (batch_sweep<float, float, float>(ctx, B, SWEEP_FWD, g, d)));
    XFP_CUDA(ctx, (batch_sweep<float, float, float>(ctx, B, SWEEP_BWD, g, d)));
  }
  cudaEventRecord(e1, st);
  XFP_CUDA(ctx, cudaStreamSynchronize(st));
  cudaEventElapsedTime(ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  (void)M;
  return check_sweep_error(ctx);
}

template <typename IOT>
int project_batch(xfp_ctx* ctx, int n, const xfp_scene* scenes, xfp_stats* stats) {
  if (!ctx) return XFP_ERR_ARGS;
  if (n < 1 || !scenes) return fail(ctx, XFP_ERR_ARGS, "batch needs n >= 1 scenes");
  if (ctx->opt.matrix != XFP_MATRIX_VARIATIONAL)
    return fail(ctx, XFP_ERR_UNSUPPORTED, "batched projection supports the variational matrix only");
  for (int s = 0; s < n; ++s) {
    const xfp_scene& c = scenes[s];
    int rc = check_dims(ctx, c.ni, c.nj, c.nk, c.material);
    if (rc) return fail(ctx, rc, "scene " + std::to_string(s) + ": " + ctx->err);
    if (!c.u || !c.v || !c.w) return fail(ctx, XFP_ERR_ARGS, "scene " + std::to_string(s) + ": velocity is NULL");
    if ((c.wu == nullptr) != (c.wv == nullptr) || (c.wu == nullptr) != (c.ww == nullptr))
      return fail(ctx, XFP_ERR_ARGS, "scene " + std::to_string(s) + ": face weights: pass all three or none");
  }
  XFP_CUDA(ctx, cudaSetDevice(ctx->device));
  if (!ctx->batch) ctx->batch = new BatchState();
  BatchState* B = ctx->batch;
  cudaStream_t st = ctx->stream;
  const long long launches0 = g_kernel_launches;
  cudaEvent_t ev[5];
  for (auto& e : ev) cudaEventCreate(&e);
  cudaEventRecord(ev[0], st);

  // ---- inputs on the device (staged into one buffer in host-pointer mode) ----
  std::vector<DevScene<IOT>> S(n);
  const bool host = !ctx->opt.device_pointers;
  size_t io_bytes = 0;
  auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
  for (int s = 0; s < n; ++s) {
    const xfp_scene& c = scenes[s];
    const size_t cells = (size_t)c.ni * c.nj * c.nk;
    const size_t fu = (size_t)(c.ni + 1) * c.nj * c.nk, fv = (size_t)c.ni * (c.nj + 1) * c.nk,
                 fw = (size_t)c.ni * c.nj * (c.nk + 1);
    io_bytes += al(cells) + 2 * al(fu * sizeof(IOT)) + 2 * al(fv * sizeof(IOT)) + 2 * al(fw * sizeof(IOT)) +
                al(cells * sizeof(IOT));
  }
  if (host) XFP_CUDA(ctx, B->io.ensure(io_bytes));
  {
    size_t off = 0;
    auto place = [&](const void* src, size_t bytes) -> void* {
      char* dst = B->io.as<char>() + off;
      off += al(bytes);
      if (src) cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st);
      return dst;
    };
    for (int s = 0; s < n; ++s) {
      const xfp_scene& c = scenes[s];
      DevScene<IOT>& d = S[s];
      d.ni = c.ni; d.nj = c.nj; d.nk = c.nk;
      const size_t cells = (size_t)c.ni * c.nj * c.nk;
      const size_t fu = (size_t)(c.ni + 1) * c.nj * c.nk, fv = (size_t)c.ni * (c.nj + 1) * c.nk,
                   fw = (size_t)c.ni * c.nj * (c.nk + 1);
      if (host) {
        d.mat = (const uint8_t*)place(c.material, cells);
        d.u = (IOT*)place(c.u, fu * sizeof(IOT));
        d.v = (IOT*)place(c.v, fv * sizeof(IOT));
        d.w = (IOT*)place(c.w, fw * sizeof(IOT));
        d.wu = c.wu ? (const IOT*)place(c.wu, fu * sizeof(IOT)) : nullptr;
        d.wv = c.wv ? (const IOT*)place(c.wv, fv * sizeof(IOT)) : nullptr;
        d.ww = c.ww ? (const IOT*)place(c.ww, fw * sizeof(IOT)) : nullptr;
        if (!c.wu) off += al(fu * sizeof(IOT)) + al(fv * sizeof(IOT)) + al(fw * sizeof(IOT));
        d.p = (IOT*)place(nullptr, cells * sizeof(IOT));
      } else {
        d.mat = c.material;
        d.u = (IOT*)c.u; d.v = (IOT*)c.v; d.w = (IOT*)c.w;
        d.wu = (const IOT*)c.wu; d.wv = (const IOT*)c.wv; d.ww = (const IOT*)c.ww;
        d.p = (IOT*)c.pressure;
      }
    }
  }
  // device-pointer mode without a pressure output: a scratch grid per scene
  if (!host) {
    size_t need = 0;
    for (int s = 0; s < n; ++s)
      if (!S[s].p) need += al((size_t)S[s].ni * S[s].nj * S[s].nk * sizeof(IOT));
    if (need) {
      XFP_CUDA(ctx, B->pdense.ensure(need));
      size_t off = 0;
      for (int s = 0; s < n; ++s)
        if (!S[s].p) {
          S[s].p = (IOT*)(B->pdense.as<char>() + off);
          off += al((size_t)S[s].ni * S[s].nj * S[s].nk * sizeof(IOT));
        }
    }
  }

  // ---- layout (tile height tuned per batch shape) ----
  const int prec = ctx->opt.precision;
  const std::string key = shape_key(n, scenes, prec);
  int nw = ctx->opt.tile_k;
  int rc;
  if (nw == 0) {
    auto it = B->tuned.find(key);
    if (it != B->tuned.end()) {
      nw = it->second;
    } else {
      float best = 0;
      int best_nw = 8;
      for (int cand : {8, 15, 16}) {
        if ((rc = batch_layout<IOT>(ctx, B, S, cand))) return rc;
        if ((rc = ensure_compact(ctx, XFP_PREC_F32))) return rc;
        float ms = 0;
        if ((rc = time_sweeps<IOT>(ctx, B, S, &ms))) return rc;
        if (cand == 8 || ms < best) { best = ms; best_nw = cand; }
      }
      B->tuned[key] = best_nw;
      nw = best_nw;
      B->layout_key.clear();
    }
  }
  if ((rc = batch_layout<IOT>(ctx, B, S, nw))) return rc;
  if ((rc = ensure_compact(ctx, prec))) return rc;
  cudaEventRecord(ev[1], st);

  // ---- solve ----
  std::vector<SceneResult> res;
  if ((rc = batch_solve<IOT>(ctx, B, S, res)) < 0) return rc;
  cudaEventRecord(ev[2], st);

  // ---- pressure on the dense grids, velocity update ----
  const long long M = std::max<long long>(B->M, 1);
  const bool sol64 = prec != XFP_PREC_F32;
  const void* xsol = sol64 ? (const void*)ctx->x64.p : (const void*)ctx->x32.p;
  if (sol64 != std::is_same<IOT, double>::value) {
    if (sol64) {
      XFP_CUDA(ctx, (convert<double, float>(ctx->x64.as<double>(), ctx->s32.as<float>(), M, st)));
      xsol = ctx->s32.p;
    } else {
      XFP_CUDA(ctx, ctx->r64.ensure(M * 8 + 64));
      XFP_CUDA(ctx, (convert<float, double>(ctx->x32.as<float>(), ctx->r64.as<double>(), M, st)));
      xsol = ctx->r64.p;
    }
  }
  for (int s = 0; s < n; ++s) {
    const DevScene<IOT>& d = S[s];
    XFP_CUDA(ctx, scatter_dense<IOT>((const IOT*)xsol, B->hsegs[s].lines, d.ni, d.nj, d.nk, d.p, st));
    XFP_CUDA(ctx, (apply_pressure<IOT, IOT>(d.mat, d.wu, d.wv, d.ww, d.p, d.ni, d.nj, d.nk, d.u, d.v, d.w, st)));
  }
  cudaEventRecord(ev[3], st);
  if (host) {
    for (int s = 0; s < n; ++s) {
      const xfp_scene& c = scenes[s];
      const DevScene<IOT>& d = S[s];
      const size_t cells = (size_t)c.ni * c.nj * c.nk;
      const size_t fu = (size_t)(c.ni + 1) * c.nj * c.nk, fv = (size_t)c.ni * (c.nj + 1) * c.nk,
                   fw = (size_t)c.ni * c.nj * (c.nk + 1);
      XFP_CUDA(ctx, cudaMemcpyAsync(c.u, d.u, fu * sizeof(IOT), cudaMemcpyDeviceToHost, st));
      XFP_CUDA(ctx, cudaMemcpyAsync(c.v, d.v, fv * sizeof(IOT), cudaMemcpyDeviceToHost, st));
      XFP_CUDA(ctx, cudaMemcpyAsync(c.w, d.w, fw * sizeof(IOT), cudaMemcpyDeviceToHost, st));
      if (c.pressure)
        XFP_CUDA(ctx, cudaMemcpyAsync(c.pressure, d.p, cells * sizeof(IOT), cudaMemcpyDeviceToHost, st));
    }
  }
  cudaEventRecord(ev[4], st);
  XFP_CUDA(ctx, cudaStreamSynchronize(st));
  float ms[4] = {0, 0, 0, 0};
  for (int q = 0; q < 4; ++q) cudaEventElapsedTime(&ms[q], ev[q], ev[q + 1]);
  for (auto& e : ev) cudaEventDestroy(e);

  int status = XFP_OK;
  for (int s = 0; s < n; ++s) {
    if (res[s].status == XFP_ERR_BREAKDOWN && status == XFP_OK) status = XFP_NOT_CONVERGED;
    if (res[s].status == XFP_NOT_CONVERGED) status = XFP_NOT_CONVERGED;
  }
  if (stats) {
    const long long launches = g_kernel_launches - launches0;
    for (int s = 0; s < n; ++s) {
      xfp_stats& o = stats[s];
      memset(&o, 0, sizeof(o));
      o.status = res[s].status;
      o.iterations = res[s].iters;
      o.refinements = res[s].refinements;
      o.residual = res[s].res;
      o.b_inf = res[s].bnorm;
      o.rel_residual = res[s].bnorm > 0 ? res[s].res / res[s].bnorm : 0.0;
      o.rows = B->rows[s];
      o.stored = B->hsegs[s].M;
      o.lines = B->nlines_act[s];
      // batch-wide timings (the scenes share every launch)
      o.ms_setup = ms[0];
      o.ms_solve = ms[1];
      o.ms_apply = ms[2];
      o.ms_total = ms[0] + ms[1] + ms[2] + ms[3];
      const double bpr = prec == XFP_PREC_F64 ? 224.0 : 112.0;   // FP32 pivots in the mixed solves
      const double cells = (double)scenes[s].ni * scenes[s].nj * scenes[s].nk;
      o.bytes = bpr * (double)o.rows * o.iterations + 33.0 * cells + 24.0 * (double)o.rows + 29.0 * cells;
      o.launches = launches;
      o.tile_k = B->nw;
      o.graph = B->graph_used ? 1 : 0;
    }
  }
  return status;
}

}  // namespace
}  // namespace xfp_host

extern "C" int xfp_project_batch_f32(xfp_ctx* ctx, int n, const xfp_scene* scenes, xfp_stats* stats) {
  return xfp_host::project_batch<float>(ctx, n, scenes, stats);
}
extern "C" int xfp_project_batch_f64(xfp_ctx* ctx, int n, const xfp_scene* scenes, xfp_stats* stats) {
  return xfp_host::project_batch<double>(ctx, n, scenes, stats);
}
