// xfp_kernels.h -- host-side launchers of libxfp's device kernels (internal).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "xfp_common.cuh"

namespace xfp {

enum { SWEEP_FACTOR = 0, SWEEP_FWD = 1, SWEEP_BWD = 2 };

// Kernels launched by this library in this process (every launcher adds its
// launches); a call reports the difference across its own work.
extern long long g_kernel_launches;

// Static description of one sweep launch (tiles, progress words, control).
struct SweepGrid {
  int ni, nj, nk, NJt, NKt, ntiles, maxT;
  int bwd_mode;                 // backward: 0 = initial rho, 1 = beta update
  const Line* lines;            // [nk*nj]
  const int* tiles;             // active tiles, topological order, J | K<<16
  SweepCtl* ctl;
  long long spin_limit;
  PcgScalars* scal;             // forward/backward: skip when done; backward: rho/beta
  int* trace;                   // optional: per (block, warp) {site, step, progress, tile} while waiting
  // Batch of scenes (null for one scene): scene of each tile, per-scene
  // geometry and scalars.  Tiles of a converged scene are skipped, and the
  // backward dot partials are reduced per scene by batch_bwd_reduce.
  const int* tile_scene = nullptr;
  const BatchSeg* segs = nullptr;
  PcgScalars* scal_batch = nullptr;
  // Diagnostic (xfp_debug_expire_next_sweep): the loaders expect boundary
  // words stamped with generation + expect_bias, which no producer writes, so
  // their bounded waits run out.  0 in normal operation.
  unsigned expect_bias = 0;
  // Sweep layout of the solve arrays (one entry per tile of `tiles`), or null:
  // the solves then read the factor and write y in the line layout.
  const SwTile* swt = nullptr;
  // triangular solves of 4-byte types: stage the group blocks through shared
  // memory with cp.async (1) or load them into registers (0)
  int stage = 0;
  // Triangular solves: (scene tile base + K * NJt + J) -> position in
  // `tiles`, or -1 for an inactive tile; and the number of boundary rows per
  // tile (one per wavefront step a tile can span: max ni + tile height + 36).
  const int* tile_pos = nullptr;
  int brows = 0;
};

// Arrays of one sweep.  VT: vector/L type of the solves, IT: invdiag type,
// CT: factor arithmetic (and A input) type.
template <typename VT, typename IT, typename CT>
struct SweepData {
  const VT* r = nullptr;        // forward: rhs r; backward: r for the fused z.r
  VT* y = nullptr;              // forward: out y; backward: in y, out z (in place)
  const VT* lx = nullptr;
  const VT* ly = nullptr;
  const VT* lz = nullptr;
  const IT* inv = nullptr;
  const CT* diag = nullptr;     // factor inputs
  const CT* ax = nullptr;
  const CT* ay = nullptr;
  const CT* az = nullptr;
  CT* flx = nullptr;            // factor outputs: L keyed by the higher cell,
  CT* fly = nullptr;            // lx[c] = L(c,c-1), ly[c] = L(c,c-ni), lz[c] = L(c,c-nn)
  CT* flz = nullptr;
  IT* oinv = nullptr;
  CT omega = CT(0.97), ratio = CT(0.25);
  double* partials = nullptr;   // backward: one z.r partial per x-line (line table order)
  // Tile-boundary values published for neighbouring tiles: per cell up to 4
  // 64-bit words (32-bit payload chunk | launch generation << 32).
  unsigned long long* sy = nullptr;  // to the j-neighbour tile
  unsigned long long* sz = nullptr;  // to the k-neighbour tile
  // Triangular solves: the same words kept by wavefront step instead of by
  // cell, one row per step of the producing tile, so that a step's
  // publication and a loader's poll each touch one contiguous row:
  // bk[((tile * brows + row) * 32 + lane) * P + p] from the tile's k-edge warp,
  // bj[((tile * brows + row) * NW + warp) * P + p] from its j-edge lanes.
  unsigned long long* bk = nullptr;
  unsigned long long* bj = nullptr;
  // Sweep-layout copies (used when SweepGrid::swt is set): the factor, r,
  // and y, which the forward solve writes and the backward solve overwrites
  // with z (the line-layout r and y are then not touched).
  const VT* lxs = nullptr;
  const VT* lys = nullptr;
  const VT* lzs = nullptr;
  const IT* invs = nullptr;
  const VT* rs = nullptr;
  VT* ys = nullptr;
};

// Forward/backward solves (xfp_solve.cu); sweep_launch routes them there.
template <typename VT, typename IT, typename CT>
cudaError_t solve_launch(int op, const SweepGrid& g, const SweepData<VT, IT, CT>& d, int nw, int grid,
                         cudaStream_t st);
template <typename VT, typename IT, typename CT>
int solve_max_grid(int op, int nw, int stage);

#define XFP_SWEEP_DECL(VT, IT, CT)                                                             \
  cudaError_t sweep_launch(int op, const SweepGrid& g, const SweepData<VT, IT, CT>& d, int nw, \
                           int grid, cudaStream_t st);                                         \
  int sweep_max_grid(int op, const SweepData<VT, IT, CT>& d, int nw, int stage = 0);
XFP_SWEEP_DECL(double, double, double)
XFP_SWEEP_DECL(float, float, float)
XFP_SWEEP_DECL(float, double, double)   // mixed form: factorisation only
XFP_SWEEP_DECL(float, float, double)    // mixed form: triangular solves only
#undef XFP_SWEEP_DECL

// ---- sweep layout (xfp_swlayout.cu) ----
// Per-tile step spans of the active tiles (off left 0; the host scans them),
// and the (K*NJt + J) -> tile position map.
cudaError_t sw_tiles_build(const Line* lines, const int* tiles, int ntiles, int nj, int nk, int nw, int NJt,
                           SwTile* swt, int* tile_pos, cudaStream_t st);
// perm[c] = sweep-layout element of stored cell cell_base + c (c < M); the
// line offsets count from cell 0 of the compact arrays.
cudaError_t sw_perm_build(const int* cell_line, const Line* lines, int nj, int nw, int NJt, const int* tile_pos,
                          const SwTile* swt, long long M, int* perm, cudaStream_t st, long long cell_base = 0);
// Batch form of sw_tiles_build: spans of the merged tile list (tile t in scene tile_scene[t]).
cudaError_t sw_tiles_build_batch(const int* tiles, const int* tile_scene, const BatchSeg* segs, int ntiles, int nw,
                                 SwTile* swt, cudaStream_t st);
// dir 0: sw[perm[c]] = line[c]; dir 1: line[c] = sw[perm[c]] for the M stored cells.
template <typename T>
cudaError_t sw_permute(T* line, T* sw, const int* perm, long long M, int dir, cudaStream_t st);

// ---- layout (xfp_layout.cu) ----
// Builds the line table and the active-tile list for a material grid.
// Returns on the host: stored cells M, unknown rows, active lines, active tiles.
struct LayoutDev {
  Line* lines;               // [nk*nj]
  int* line_len_scan;        // scratch [nk*nj + 1]
  unsigned char* tile_active;// [NKt*NJt]
  int* tiles;                // [NKt*NJt]
  long long* counters;       // [4] M, rows, lines, ntiles (device)
};
cudaError_t layout_build(const uint8_t* mat, int ni, int nj, int nk, int tile_k, LayoutDev L,
                         cudaStream_t st);

// ---- assembly / apply / vector kernels (xfp_ops.cu) ----
template <typename FT, typename AT>
cudaError_t assemble(const uint8_t* mat, const FT* u, const FT* v, const FT* w, const FT* wu,
                     const FT* wv, const FT* ww, int ni, int nj, int nk, const Line* lines,
                     AT* diag, AT* ax, AT* ay, AT* az, AT* b, cudaStream_t st,
                     int matrix = XFP_MATRIX_VARIATIONAL, Force3 frc = Force3(),
                     float* const A32[4] = nullptr);   // also write diag..az as FP32 (mixed form)

template <typename T>
cudaError_t scatter_dense(const T* x, const Line* lines, int ni, int nj, int nk, T* dense,
                          cudaStream_t st);
// Host-pointer mode, sparse face transfer (xfp_hostio.cu): fluid span of
// every x-line ({first, last + 1}, or {0, 0}), and the copy of every face
// row's fluid-bordering span of u, v, w from src to dst (either side may be
// page-locked host memory addressed in place); *bytes accumulates the bytes.
cudaError_t fluid_spans(const uint8_t* mat, int ni, int nj, int nk, int2* span, cudaStream_t st);
template <typename T>
cudaError_t face_rows_copy(const int2* span, int ni, int nj, int nk, const T* const src[3], T* const dst[3],
                           unsigned long long* bytes, cudaStream_t st);

template <typename FT, typename PT>
cudaError_t apply_pressure(const uint8_t* mat, const FT* wu, const FT* wv, const FT* ww,
                           const PT* p, int ni, int nj, int nk, FT* u, FT* v, FT* w,
                           cudaStream_t st, int matrix = XFP_MATRIX_VARIATIONAL, Force3 frc = Force3());
// FluidSimulator::_applyForces (FluidSimulator.cpp:429-499) as one pass.
template <typename FT>
cudaError_t apply_forces(const uint8_t* mat, int ni, int nj, int nk, FT* u, FT* v, FT* w, Force3 frc,
                         cudaStream_t st);
// FluidSimulator::_expolateVelocity(layers, axis) for the three axes
// (FluidSimulator.cpp:521-650); marker: scratch of (ni+1)*(nj+1)*(nk+1) shorts.
template <typename FT>
cudaError_t extrapolate(const uint8_t* mat, int ni, int nj, int nk, FT* u, FT* v, FT* w, int layers,
                        short* marker, cudaStream_t st);
template <typename FT>
cudaError_t divergence(const uint8_t* mat, int ni, int nj, int nk, const FT* u, const FT* v, const FT* w, FT* div,
                       cudaStream_t st);
template <typename FT, typename PT>
cudaError_t apply_pressure_T(const uint8_t* mat, const FT* wu, const FT* wv, const FT* ww,
                             const FT* gu, const FT* gv, const FT* gw, int ni, int nj, int nk,
                             const Line* lines, PT* q, cudaStream_t st);
template <typename FT, typename PT>
cudaError_t rhs_T(const uint8_t* mat, const FT* wu, const FT* wv, const FT* ww, const PT* lam,
                  const Line* lines, int ni, int nj, int nk, const FT* gu, const FT* gv,
                  const FT* gw, FT* du, FT* dv, FT* dw, cudaStream_t st);

// PCG vector kernels over the compact arrays (length M).
// z = A s with the fused dot s.z; one thread per aligned 4-cell group
// (group_line maps a group to its line).
template <typename VT, typename AT, typename DT>
cudaError_t spmv_dot(const AT* diag, const AT* ax, const AT* ay, const AT* az, const VT* s, VT* z,
                     const Line* lines, const int* group_line, int nj, int nk, long long M, PcgScalars* sc,
                     DT* partials, int nblk_max, int mode, cudaStream_t st);
// SpMV blocks for M stored cells (the batch gives each scene the same count).
long long spmv_block_count(long long M, int nblk_max);
// cell_line[c] = index of the line storing cell c (for every cell of every
// line); group_line[c / 4] the same per aligned 4-cell group.
cudaError_t build_cell_line(const Line* lines, long long nlines, int* cell_line, int* group_line, cudaStream_t st);
// rsw/perm (optional): the updated r is also stored at rsw[perm[c]].
template <typename VT, typename DT>
cudaError_t update_xr(VT* x, VT* r, const VT* s, const VT* z, long long M, PcgScalars* sc,
                      double* partials, int nblk_max, cudaStream_t st, VT* rsw = nullptr,
                      const int* perm = nullptr);
// zsw/perm (optional): z is read from zsw[perm[c]] instead of z[c].
template <typename VT>
cudaError_t update_s(VT* s, const VT* z, long long M, PcgScalars* sc, cudaStream_t st, const VT* zsw = nullptr,
                     const int* perm = nullptr, int nblk_max = 148 * 16);
template <typename VT>
cudaError_t absmax_init(const VT* b, long long M, PcgScalars* sc, double* partials, int nblk_max,
                        double tol, int maxit, cudaStream_t st);
template <typename A, typename B>
cudaError_t convert(const A* in, B* out, long long n, cudaStream_t st);
template <typename T>
cudaError_t gather_compact(const T* dense, const Line* lines, int ni, int nj, int nk, T* x,
                           cudaStream_t st);
template <typename T>
cudaError_t copy_vec(const T* in, T* out, long long n, cudaStream_t st);

// ---- batch forms: one launch covers every scene of a batch (BatchSeg table,
// nseg scenes, per-scene scalars sc[nseg]); grid = the table's total blocks ----
template <typename VT, typename AT, typename DT>
cudaError_t batch_spmv_dot(const BatchSeg* segs, int nseg, int blocks, const AT* diag, const AT* ax,
                           const AT* ay, const AT* az, const VT* s, VT* z, const int* group_line, PcgScalars* sc,
                           int mode, cudaStream_t st);
// rsw/perm, zsw/perm (optional): as update_xr / update_s, perm indexed by global cell
template <typename VT>
cudaError_t batch_update_xr(const BatchSeg* segs, int nseg, int blocks, VT* x, VT* r, const VT* s,
                            const VT* z, PcgScalars* sc, cudaStream_t st, VT* rsw = nullptr,
                            const int* perm = nullptr);
template <typename VT>
cudaError_t batch_update_s(const BatchSeg* segs, int nseg, int blocks, VT* s, const VT* z, PcgScalars* sc,
                           cudaStream_t st, const VT* zsw = nullptr, const int* perm = nullptr);
// tols/maxits: optional per-scene tolerance and iteration cap (else tol, maxit)
template <typename VT>
cudaError_t batch_absmax_init(const BatchSeg* segs, int nseg, int blocks, const VT* b, PcgScalars* sc,
                              double tol, int maxit, const double* tols, const int* maxits, cudaStream_t st);
cudaError_t batch_residual64(const BatchSeg* segs, int nseg, int blocks, const double* diag, const double* ax,
                             const double* ay, const double* az, const double* b, const double* x, double* r,
                             PcgScalars* sc, cudaStream_t st);
// Per-scene z.r from the backward sweep's per-line partials (line_sum, the
// single-scene order); mode 0: rho, mode 1: beta and rho.
template <typename DT>
cudaError_t batch_bwd_reduce(const BatchSeg* segs, int nseg, const double* line_partials, PcgScalars* sc, int mode,
                             cudaStream_t st);
// ---- semi-Lagrangian MAC self-advection and its adjoint (xfp_advect.cu) ----
template <typename T>
cudaError_t advect(const T* u, const T* v, const T* w, T* ou, T* ov, T* ow, int ni, int nj, int nk, T c,
                   cudaStream_t st);
template <typename T>
cudaError_t advect_adjoint(const T* u, const T* v, const T* w, const T* gu, const T* gv, const T* gw, T* du,
                           T* dv, T* dw, int ni, int nj, int nk, T c, cudaStream_t st);
template <typename T>
cudaError_t box_loss(const T* u, const T* v, const T* w, T* gu, T* gv, T* gw, int ni, int nj, int nk,
                     const double box[6], double* loss, cudaStream_t st);

// Adds base[s] to the offsets of scene s's line table.
cudaError_t offset_lines(Line* lines, long long nlines, long long base, cudaStream_t st);

// Mixed precision: r64 = b64 - A64 x64, |r|_inf and r32 = (float) r64 / scale.
cudaError_t residual64(const double* diag, const double* ax, const double* ay, const double* az,
                       const double* b, const double* x, double* r, const Line* lines, int ni,
                       int nj, int nk, long long M, PcgScalars* sc, double* partials,
                       int nblk_max, cudaStream_t st);
cudaError_t refine_update(double* x64, const float* e32, long long M, cudaStream_t st);

}  // namespace xfp
