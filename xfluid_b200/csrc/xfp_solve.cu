// xfp_solve.cu -- forward and backward triangular solves of the MIC(0)
// preconditioner in xFluid's natural (lexicographic) order, as wavefronts that
// advance in lockstep: one CTA barrier per wavefront step.
//
// Reference semantics (xFluid/xFluid/variationalpressure/pcg_solver.h):
//   forward  solve_lower (column-scatter L y = r)  :192-204
//   backward solve_lower_transpose_in_place        :207-220
// Every update is applied in the reference's column order with separately
// rounded multiplies and subtractions, so the FP64 path is bit-identical to
// the reference (the factorisation is in xfp_sweep.cu).
//
// Work decomposition (the same tiles as the factorisation).  A thread owns
// one x-line (j,k) and walks it in i; a warp holds 32 consecutive j at one k;
// a CTA holds a tile of 32 x NW lines.  Cell (i,j,k) is processed at
// wavefront step tau = i+j+k (mirrored for the backward solve), so at step
// tau a thread needs
//   x-neighbour  its own result of step tau-1          (register)
//   y-neighbour  the neighbouring lane's, step tau-1    (warp shuffle)
//   z-neighbour  the neighbouring warp's, step tau-1    (shared memory)
// and values from the neighbouring tiles, brought in by a loader warp.
//
// Lockstep.  Every compute warp runs every step of the tile's step range
// (cells outside a lane's line are masked to zero) and the step ends at a
// named barrier shared by the compute warps and a gate warp.  After barrier
// tau every z-value of step tau-1 is in shared memory, so the ring between
// warps is a plain double buffer: no stamps, no polling, no back-pressure on
// the per-step path.  A warp-to-warp hand-off costs one barrier, against a
// poll/vote round trip per step for a dataflow pipeline.
//
// Tile boundaries.  Producers publish boundary values in global memory as
// 64-bit words stamped with the launch generation (single-copy atomic, so no
// fence is needed).  The loader warp polls them ahead of the compute warps,
// batch by batch, and forwards every step as soon as its stamps are current
// into a shared ring of plain values; it then raises its progress word.  The
// gate warp lets barrier tau complete only once the loader has forwarded
// step tau, and reports the steps the compute warps have finished, which the
// loader needs before reusing a ring slot.
//
// Tiles are visited in topological order (J+K ascending) and assigned
// round-robin to a fully co-resident grid (cooperative launch), so a CTA only
// waits on tiles that earlier CTAs hold.  The loader's and the gate's waits
// are bounded (spin_limit polls); on expiry the kernel records SweepCtl::err,
// every other wait gives up quickly, all warps still reach the same barriers
// and the host reports XFP_ERR_TIMEOUT.
#include "xfp_sweep_util.cuh"

namespace xfp {
namespace {

constexpr int SRING = 32;   // loader ring depth (steps)
constexpr int SLB = 8;      // loader batch: steps polled together
static_assert(SRING >= SLB + 1, "the loader could wait for a slot the gate cannot free");

// y = t * inv, rounded to the solve type.  The mixed form's solves stream
// its FP64 pivots rounded to FP32 (the pivots themselves are computed in FP64
// by the factorisation), so every solve multiplies in its value type.
template <typename VT, typename IT>
struct Pivot {
  IT v;
  __device__ __forceinline__ explicit Pivot(IT inv) : v(inv) {}
  __device__ __forceinline__ VT mul(VT t) const { return VT(mul_rn((IT)t, v)); }
};

__device__ __forceinline__ void step_barrier(int nthreads) {
  asm volatile("bar.sync 1, %0;" ::"r"(nthreads) : "memory");
}

template <typename VT, int NW>
struct SolveShared {
  VT zr[2][NW][32];   // z hand-off between warps, by step parity
  VT kr[SRING][32];   // k-boundary values from the loader, by step
  VT jr[SRING][NW];   // j-boundary values from the loader, by step
  int tlo[NW], thi[NW];
  int lo, hi, last;
  volatile int lprog;   // last step the loader has forwarded
  volatile int gate;    // last step every compute warp has finished
};

// Group staging (STAGE 1): instead of loading the next group's blocks into
// registers one group ahead, each lane copies its own 16-byte pieces of the
// groups two ahead into a per-warp ring in shared memory with cp.async, waits
// for a group's copies when that group starts, and reads them back from shared
// memory.  On the 256^3 blob scene this took the solve launch from 0.225 to
// 0.189 ms (tile height 16); per-warp bulk copies completed on an mbarrier were
// measured too (0.211 ms).  Used for 4-byte values and pivots (the FP32 and
// mixed solves).
constexpr int STAGE_SLOTS = 3;
template <int OP, typename VT, int NW>
constexpr int stage_bytes() {
  return STAGE_SLOTS * NW * (OP == SWEEP_FWD ? 5 : 6) * 32 * XFP_ALIGN * (int)sizeof(VT);
}
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

template <int OP, typename VT, typename IT, typename CT, int NW, int STAGE>
__global__ void __launch_bounds__((NW + 2) * 32, 1)
    solve_kernel(SweepGrid g, SweepData<VT, IT, CT> d) {
  static_assert(STAGE == 0 || (sizeof(VT) == 4 && sizeof(IT) == 4), "staging holds 4-byte values and pivots");
  static_assert(STAGE == 0 || STAGE == 1, "register loads (0) or cp.async staging (1)");
  extern __shared__ __align__(128) unsigned char stage_smem[];
  constexpr bool REV = (OP == SWEEP_BWD);
  constexpr int P = Words<VT>::P;
  // z.r is accumulated in the dot type: FP32 for the plain FP32 form, FP64 otherwise
  constexpr bool DOT32 = std::is_same<CT, float>::value;
  constexpr int GATE = NW, LOADER = NW + 1;
  constexpr int NT = (NW + 1) * 32;   // threads at the per-step barrier: compute warps + gate
  constexpr int GS = XFP_ALIGN;
  static_assert(GS == 4, "group load/store helpers cover 4-cell groups");
  static_assert(sizeof(VT) * SRING * 32 >= 256 * sizeof(double), "kr doubles as line_sum scratch");
  __shared__ __align__(16) SolveShared<VT, NW> sh;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned gen = ld_volatile_u32(&g.ctl->gen);

  if (g.scal != nullptr && *(volatile int*)&g.scal->done != 0) return;

  for (int pos = blockIdx.x, seq = 0; pos < g.ntiles; pos += gridDim.x, ++seq) {
    const int tpos = REV ? g.ntiles - 1 - pos : pos;
    // the tile's grid: the launch's one scene, or its scene of the batch
    int ni = g.ni, nj = g.nj, nk = g.nk, maxT = g.maxT, NJt = g.NJt, NKt = g.NKt, tbase = 0;
    const Line* lines = g.lines;
    long long line_base = 0;
    if (g.tile_scene != nullptr) {
      const int sid = g.tile_scene[tpos];
      const BatchSeg& S = g.segs[sid];
      // a converged scene's tiles are skipped (its scalars only change between
      // launches, so every CTA of this launch decides the same way)
      if (g.scal_batch != nullptr && *(volatile int*)&g.scal_batch[sid].done != 0) continue;
      ni = S.ni;
      nj = S.nj;
      nk = S.nk;
      maxT = S.ni + S.nj + S.nk;
      NJt = (S.nj + 31) >> 5;
      NKt = (S.nk + NW - 1) / NW;
      tbase = S.tile_base;
      lines = S.lines;
      line_base = S.line_base;
    }
    const int packed = g.tiles[tpos];
    const int J = packed & 0xffff, K = packed >> 16;
    const int j0 = J * 32, k0 = K * NW;
    // First wavefront step a tile (Jt, Kt) can have a stored cell at: its
    // boundary rows are indexed by step - this.  Stored cells include the
    // group padding, i in [-3, ni + 2], so i + j + k runs from 32 Jt + NW Kt - 3
    // to 32 Jt + NW Kt + ni + NW + 32: at most ni + NW + 36 steps.
    auto row_base = [&](int Jt, int Kt) -> int {
      const int lowest = 32 * Jt + NW * Kt - 3;
      return REV ? maxT - (lowest + ni + NW + 35) : lowest;
    };
    const int R = g.brows;

    // ---------------- setup: wavefront ranges, cleared hand-off ring ----------------
    Line L = {0, 0, 0, 0};
    int s = 0;
    if (warp < NW) {
      const int j = j0 + lane, k = k0 + warp;
      if (j < nj && k < nk) L = lines[(size_t)k * nj + j];
      s = j + k;
      int tl = INF_T, th = INT_MIN;
      if (L.len > 0) {
        const int a = L.lo + s, b = L.lo + L.len - 1 + s;
        if (!REV) { tl = a; th = b; } else { tl = maxT - b; th = maxT - a; }
      }
      const int Tlo = __reduce_min_sync(XFP_FULL, tl);
      const int Thi = __reduce_max_sync(XFP_FULL, th);
      if (lane == 0) {
        sh.tlo[warp] = Tlo;
        sh.thi[warp] = Thi;
      }
    }
    for (int q = threadIdx.x; q < 2 * NW * 32; q += blockDim.x) (&sh.zr[0][0][0])[q] = VT(0);
    __syncthreads();
    if (threadIdx.x == 0) {
      int lo = INF_T, hi = INT_MIN;
      for (int w = 0; w < NW; ++w) {
        lo = min(lo, sh.tlo[w]);
        hi = max(hi, sh.thi[w]);
      }
      sh.lo = lo;
      sh.hi = hi;
      sh.lprog = lo - 1;
      sh.gate = lo - 1;
    }
    __syncthreads();
    const int tileLo = sh.lo, tileHi = sh.hi;

    double dot_acc = 0.0;
    float dot_acc_f = 0.0f;

    if (tileLo != INF_T && warp < NW && sh.tlo[warp] == INF_T) {
      // a warp without cells in this tile only keeps the barrier count (its
      // ring slots stay zero)
      for (int tau = tileLo; tau <= tileHi; ++tau) step_barrier(NT);
    } else if (tileLo != INF_T && warp < NW) {
      // ======================= compute warp =======================
      const int zsrc = REV ? warp + 1 : warp - 1;   // producer warp in this tile (or the loader)
      const int zdst = REV ? warp - 1 : warp + 1;   // consumer warp in this tile
      const bool kb = zsrc < 0 || zsrc >= NW;        // fed by the loader (k boundary)
      const bool zdst_in = zdst >= 0 && zdst < NW;
      const bool jb = REV ? (lane == 31) : (lane == 0);    // fed by the loader (j boundary)
      const bool jpub = REV ? (lane == 0) : (lane == 31);  // publish for the j-neighbour tile
      const bool kpub = REV ? (warp == 0) : (warp == NW - 1);

      VT out_x = VT(0), out_y = VT(0);
      // this thread's column of the tile's boundary rows (used by the j-edge
      // lanes and the k-edge warp)
      const int rb_self = row_base(J, K);
      unsigned long long* const bj_me = d.bj + ((size_t)tpos * R * NW + warp) * P;
      unsigned long long* const bk_me = d.bk + ((size_t)tpos * R * 32 + lane) * P;

      // Sweep layout (when the launch has one): this warp's stream of
      // 32-lane blocks, one per group of 4 forward steps.
      const bool swl = g.swt != nullptr;
      SwTile T = {0, 0, 0};
      if (swl) T = g.swt[tpos];
      const long long wbase = T.off + (long long)warp * T.ng * 128 + lane * 4;

      // Grouped access.  A line is stored so that cell (i,j,k) sits at an
      // address = i+j+k (mod GS): at every wavefront step all lanes are at the
      // same position within an aligned group of GS cells, so each lane loads
      // the next GS cells of each array with vector accesses and stores GS
      // results at once.  The group of steps t0..t0+GS-1 is loaded one group
      // ahead into the buffer the previous group has just released.  A group
      // lies entirely inside or outside a line.
      struct Grp {
        VT r[GS], lx[GS], ly[GS], lz[GS], rr[GS];
        IT inv[GS];
      };
      // forward: address phase of step t is t mod GS (increasing cells);
      // backward: (maxT - t) mod GS, cells decreasing
      const int a = REV ? ((maxT + 1) & (GS - 1)) : 0;
      const int base0 = tileLo - ((tileLo - a) & (GS - 1));
      auto group_c4 = [&](int t0) -> int {
        const int ilow = REV ? (maxT - (t0 + GS - 1)) - s : t0 - s;
        const int rel = ilow - L.lo;
        return (unsigned)rel < (unsigned)L.len ? L.off + rel : -1;
      };
      // sweep-layout element of the group of steps t0..t0+GS-1 (clamped into
      // the tile's blocks for the look-ahead past its last group)
      auto sw_at = [&](int t0) -> long long {
        int gi = (REV ? (maxT - t0 - (GS - 1)) : t0) >> 2;
        gi = min(max(gi, T.g0), T.g0 + T.ng - 1);
        return wbase + (long long)(gi - T.g0) * 128;
      };
      // A lane whose group lies outside its line loads nothing: every use of
      // such a group's values is masked by `in`, so the buffer may keep an
      // older group's values (masked lanes fetch no sectors).
      auto load_grp = [&](Grp& G, int c4, long long si) {
        if (c4 < 0) return;
        const int cc = c4;
        if constexpr (OP == SWEEP_FWD) {
          if (swl) ldg(G.r, d.rs + si);
          else ldg(G.r, d.r + cc);
        } else if (swl) {
          ldg(G.r, d.ys + si);
          ldg(G.rr, d.rs + si);
        } else {
          ldg(G.r, d.y + cc);
          ldg(G.rr, d.r + cc);
        }
        if (swl) {
          ldg(G.lx, d.lxs + si);
          ldg(G.ly, d.lys + si);
          ldg(G.lz, d.lzs + si);
          ldg(G.inv, d.invs + si);
        } else {
          ldg(G.lx, d.lx + cc);
          ldg(G.ly, d.ly + cc);
          ldg(G.lz, d.lz + cc);
          ldg(G.inv, d.inv + cc);
        }
      };

      // One wavefront step: everything that needs only this warp's previous
      // step is done before the barrier; after it, the z and boundary inputs
      // of step tau-1 are in shared memory.
      auto step = [&](const int tau, const Grp& G, const int e, const bool in) -> VT {
        const VT vy_sh = REV ? shfl_down_any(out_y) : shfl_up_any(out_y);
        const int slot = tau & (SRING - 1);
        VT res;
        if constexpr (OP == SWEEP_FWD) {
          // solve_lower: columns c-nn, c-ni, c-1 scatter into row c in that
          // order, then result[c] *= invdiag[c]  (pcg_solver.h:198-203)
          const VT px = mul_rn(G.lx[e], out_x);
          const VT py_sh = mul_rn(G.ly[e], vy_sh);
          const Pivot<VT, IT> piv(G.inv[e]);
          step_barrier(NT);
          const VT vz = kb ? sh.kr[slot][lane] : sh.zr[(tau - 1) & 1][zsrc][lane];
          const VT vj = sh.jr[slot][warp];
          const VT py = jb ? mul_rn(G.ly[e], vj) : py_sh;
          VT t = sub_rn(G.r[e], mul_rn(G.lz[e], vz));
          t = sub_rn(t, py);
          t = sub_rn(t, px);
          const VT y = in ? piv.mul(t) : VT(0);
          if (zdst_in) sh.zr[tau & 1][warp][lane] = y;
          out_x = y;
          out_y = y;
          res = y;
          if (in && jpub) {
            uint32_t w[P];
            to_words(y, w);
            unsigned long long* o = bj_me + (size_t)(tau - rb_self) * (NW * P);
#pragma unroll
            for (int p = 0; p < P; ++p) st_gpu64(o + p, stamped(gen, w[p]));
          }
          if (in && kpub) {
            uint32_t w[P];
            to_words(y, w);
            unsigned long long* o = bk_me + (size_t)(tau - rb_self) * (32 * P);
#pragma unroll
            for (int p = 0; p < P; ++p) st_gpu64(o + p, stamped(gen, w[p]));
          }
        } else {
          // solve_lower_transpose_in_place: x[c] -= L(m,c) x[m] for m = c+1,
          // c+ni, c+nn in that order, then x[c] *= invdiag[c]  (:215-218).
          // The products L(m,c) x[m] arrive ready-made from the producers.
          const VT t1 = sub_rn(G.r[e], out_x);
          const VT t2_sh = sub_rn(t1, vy_sh);
          const Pivot<VT, IT> piv(G.inv[e]);
          step_barrier(NT);
          const VT vz = kb ? sh.kr[slot][lane] : sh.zr[(tau - 1) & 1][zsrc][lane];
          const VT vj = sh.jr[slot][warp];
          const VT t2 = jb ? sub_rn(t1, vj) : t2_sh;
          const VT t = sub_rn(t2, vz);
          const VT z = in ? piv.mul(t) : VT(0);
          const VT oz = mul_rn(in ? G.lz[e] : VT(0), z);
          if (zdst_in) sh.zr[tau & 1][warp][lane] = oz;
          const VT rr = in ? G.rr[e] : VT(0);
          if (DOT32) dot_acc_f = in ? __fadd_rn(dot_acc_f, __fmul_rn((float)z, (float)rr)) : dot_acc_f;
          else dot_acc = in ? __dadd_rn(dot_acc, __dmul_rn((double)z, (double)rr)) : dot_acc;
          const VT ox = mul_rn(in ? G.lx[e] : VT(0), z);
          const VT oy = mul_rn(in ? G.ly[e] : VT(0), z);
          out_x = ox;
          out_y = oy;
          res = z;
          if (in && jpub) {
            uint32_t w[P];
            to_words(oy, w);
            unsigned long long* o = bj_me + (size_t)(tau - rb_self) * (NW * P);
#pragma unroll
            for (int p = 0; p < P; ++p) st_gpu64(o + p, stamped(gen, w[p]));
          }
          if (in && kpub) {
            uint32_t w[P];
            to_words(oz, w);
            unsigned long long* o = bk_me + (size_t)(tau - rb_self) * (32 * P);
#pragma unroll
            for (int p = 0; p < P; ++p) st_gpu64(o + p, stamped(gen, w[p]));
          }
        }
        return res;
      };
      auto run_group = [&](int t0, const Grp& G, int c4, long long si) {
        VT yb[GS];
        const bool in = c4 >= 0;
#pragma unroll
        for (int q = 0; q < GS; ++q) {
          const int tau = t0 + q;
          const int e = REV ? GS - 1 - q : q;
          yb[e] = VT(0);
          if (tau >= tileLo && tau <= tileHi) yb[e] = step(tau, G, e, in);
        }
        // with a sweep layout y (forward) and z (backward, in place) go to
        // the sweep-ordered copy, otherwise to the line layout; lanes without
        // a cell in this group store nothing (no solve reads those slots)
        if (in) stg(swl ? d.ys + si : d.y + c4, yb);
      };
      if constexpr (STAGE == 1) {
        // per-warp ring of STAGE_SLOTS group blocks: array a of slot q at
        // [(q * NA + a) * 512 + lane * 16] bytes; copies run two groups ahead
        constexpr int NA = OP == SWEEP_FWD ? 5 : 6;
        constexpr int AB = 32 * GS * (int)sizeof(VT);
        unsigned char* wring = stage_smem + (size_t)warp * STAGE_SLOTS * NA * AB + lane * GS * sizeof(VT);
        auto stage = [&](int slot, int c4, long long si) {
          if (c4 < 0) return;
          unsigned char* b = wring + slot * NA * AB;
          const long long o = swl ? si : (long long)c4;
          if constexpr (OP == SWEEP_FWD) {
            cp_async16(b, (swl ? d.rs : d.r) + o);
          } else {
            cp_async16(b, (swl ? d.ys : d.y) + o);
            cp_async16(b + 5 * AB, (swl ? d.rs : d.r) + o);
          }
          cp_async16(b + 1 * AB, (swl ? d.lxs : d.lx) + o);
          cp_async16(b + 2 * AB, (swl ? d.lys : d.ly) + o);
          cp_async16(b + 3 * AB, (swl ? d.lzs : d.lz) + o);
          cp_async16(b + 4 * AB, (swl ? d.invs : d.inv) + o);
        };
        auto fetch = [&](Grp& G, int slot) {
          const unsigned char* b = wring + slot * NA * AB;
          auto ld4 = [&](VT (&v)[4], const unsigned char* q) {
            const float4 t = *reinterpret_cast<const float4*>(q);
            v[0] = (VT)t.x; v[1] = (VT)t.y; v[2] = (VT)t.z; v[3] = (VT)t.w;
          };
          auto ld4i = [&](IT (&v)[4], const unsigned char* q) {
            const float4 t = *reinterpret_cast<const float4*>(q);
            v[0] = (IT)t.x; v[1] = (IT)t.y; v[2] = (IT)t.z; v[3] = (IT)t.w;
          };
          ld4(G.r, b);
          if constexpr (OP == SWEEP_BWD) ld4(G.rr, b + 5 * AB);
          ld4(G.lx, b + 1 * AB);
          ld4(G.ly, b + 2 * AB);
          ld4(G.lz, b + 3 * AB);
          ld4i(G.inv, b + 4 * AB);
        };
        Grp G{};
        int cA = group_c4(base0), cB = group_c4(base0 + GS), cC;
        long long sA = sw_at(base0), sB = sw_at(base0 + GS), sC;
        stage(0, cA, sA);
        cp_async_commit();
        stage(1, cB, sB);
        cp_async_commit();
        for (int gb = base0; gb <= tileHi; gb += 3 * GS) {
          cC = group_c4(gb + 2 * GS);
          sC = sw_at(gb + 2 * GS);
          stage(2, cC, sC);
          cp_async_commit();
          cp_async_wait<2>();
          if (cA >= 0) fetch(G, 0);
          run_group(gb, G, cA, sA);
          if (gb + GS > tileHi) break;
          cA = group_c4(gb + 3 * GS);
          sA = sw_at(gb + 3 * GS);
          stage(0, cA, sA);
          cp_async_commit();
          cp_async_wait<2>();
          if (cB >= 0) fetch(G, 1);
          run_group(gb + GS, G, cB, sB);
          if (gb + 2 * GS > tileHi) break;
          cB = group_c4(gb + 4 * GS);
          sB = sw_at(gb + 4 * GS);
          stage(1, cB, sB);
          cp_async_commit();
          cp_async_wait<2>();
          if (cC >= 0) fetch(G, 2);
          run_group(gb + 2 * GS, G, cC, sC);
        }
        cp_async_wait<0>();   // the ring is reused by the next tile
      } else
      // Groups are loaded into registers one group ahead (two buffers), or two
      // groups ahead (three buffers) where the register budget allows: the
      // height-8 tile has 10 warps, i.e. about 170 registers per thread (FP32
      // values; FP64 groups are twice the size and stay double-buffered).
      if constexpr (NW <= 8 && sizeof(VT) == 4) {
        Grp GA{}, GB{}, GC{};
        int cA = group_c4(base0), cB = group_c4(base0 + GS);
        long long sA = sw_at(base0), sB = sw_at(base0 + GS);
        load_grp(GA, cA, sA);
        load_grp(GB, cB, sB);
        for (int gb = base0; gb <= tileHi; gb += 3 * GS) {
          const int cC = group_c4(gb + 2 * GS);
          const long long sC = sw_at(gb + 2 * GS);
          load_grp(GC, cC, sC);
          run_group(gb, GA, cA, sA);
          if (gb + GS > tileHi) break;
          cA = group_c4(gb + 3 * GS);
          sA = sw_at(gb + 3 * GS);
          load_grp(GA, cA, sA);
          run_group(gb + GS, GB, cB, sB);
          if (gb + 2 * GS > tileHi) break;
          cB = group_c4(gb + 4 * GS);
          sB = sw_at(gb + 4 * GS);
          load_grp(GB, cB, sB);
          run_group(gb + 2 * GS, GC, cC, sC);
        }
      } else {
      Grp GA{}, GB{};
      int cA = group_c4(base0);
      long long sA = sw_at(base0);
      load_grp(GA, cA, sA);
      for (int gb = base0; gb <= tileHi; gb += 2 * GS) {
        const int cB = group_c4(gb + GS);
        const long long sB = sw_at(gb + GS);
        load_grp(GB, cB, sB);
        run_group(gb, GA, cA, sA);
        if (gb + GS > tileHi) break;
        const int cA2 = group_c4(gb + 2 * GS);
        const long long sA2 = sw_at(gb + 2 * GS);
        load_grp(GA, cA2, sA2);
        run_group(gb + GS, GB, cB, sB);
        cA = cA2;
        sA = sA2;
      }
      }
    } else if (tileLo != INF_T && warp == GATE) {
      // ======================= gate warp =======================
      // Barrier tau completes only once the loader has forwarded step tau;
      // after it, every compute warp has finished step tau-1.
      int seen = tileLo - 1;
      for (int tau = tileLo; tau <= tileHi; ++tau) {
        if (seen < tau) {
          if (lane == 0) {
            seen = sh.lprog;
            if (seen < tau) {
              trace_wait(g, 7, tau);
              Spin sp;
              while ((seen = sh.lprog) < tau) {
                if (!sp.step(g.ctl, g.spin_limit)) {
                  raise_timeout(g.ctl, 7, tpos, tau, OP, (unsigned long long)(unsigned)seen, (unsigned)tau);
                  seen = tileHi;   // proceed: results are void, the host reports the timeout
                  break;
                }
              }
              trace_wait(g, 0, tau);
            }
          }
          seen = __shfl_sync(XFP_FULL, seen, 0);
        }
        step_barrier(NT);
        if (lane == 0) sh.gate = tau - 1;
      }
    } else if (tileLo != INF_T && warp == LOADER) {
      // ======================= loader warp =======================
      // lane r < NW feeds jr column r (line k0+r); every lane l feeds kr
      // column l (line j0+l).  Sources are the neighbouring tiles' stamped
      // boundary values (global), or zero where the source cell has no row.
      const int jc = REV ? j0 + 31 : j0, js = REV ? j0 + 32 : j0 - 1;
      const int kc = REV ? k0 + NW - 1 : k0, ks = REV ? k0 + NW : k0 - 1;
      Line Ljs = {0, 0, 0, 0};
      int sj_c = 0, Sj_lo = INF_T, Sj_hi = INT_MIN;
      {
        const int kr_ = k0 + lane;
        if (lane < NW && kr_ < nk && js >= 0 && js < nj) Ljs = lines[(size_t)kr_ * nj + js];
        sj_c = jc + kr_;
        if (Ljs.len > 0) {
          const int a = Ljs.lo + sj_c, b = Ljs.lo + Ljs.len - 1 + sj_c;
          if (!REV) { Sj_lo = a; Sj_hi = b; } else { Sj_lo = maxT - b; Sj_hi = maxT - a; }
        }
      }
      Line Lks = {0, 0, 0, 0};
      int sk_c = 0, Sk_lo = INF_T, Sk_hi = INT_MIN;
      {
        const int jl = j0 + lane;
        if (jl < nj && ks >= 0 && ks < nk) Lks = lines[(size_t)ks * nj + jl];
        sk_c = jl + kc;
        if (Lks.len > 0) {
          const int a = Lks.lo + sk_c, b = Lks.lo + Lks.len - 1 + sk_c;
          if (!REV) { Sk_lo = a; Sk_hi = b; } else { Sk_lo = maxT - b; Sk_hi = maxT - a; }
        }
      }
      // source tiles of the boundary rows (-1: outside the grid or inactive;
      // then no step needs them, since needj/needk require a source cell)
      const int Jsrc = REV ? J + 1 : J - 1, Ksrc = REV ? K + 1 : K - 1;
      const int tp_j = (Jsrc >= 0 && Jsrc < NJt) ? g.tile_pos[tbase + K * NJt + Jsrc] : -1;
      const int tp_k = (Ksrc >= 0 && Ksrc < NKt) ? g.tile_pos[tbase + Ksrc * NJt + J] : -1;
      const int rb_j = row_base(Jsrc, K), rb_k = row_base(J, Ksrc);
      const unsigned want = gen + g.expect_bias;   // bias != 0 only in the expired-wait diagnostic
      int gate_seen = tileLo - 1;
      bool failed = false;
      for (int base = tileLo; base <= tileHi; base += SLB) {
        // ring space: the slot of step t last held step t-SRING, which the
        // compute warps have used once the gate reports it finished
        const int need = base + SLB - 1 - SRING;
        if (need > gate_seen && !failed) {
          gate_seen = sh.gate;
          if (need > gate_seen) {
            trace_wait(g, 5, base);
            Spin sp;
            while ((gate_seen = sh.gate) < need) {
              if (!sp.step(g.ctl, g.spin_limit)) {
                raise_timeout(g.ctl, 5, tpos, base, OP, (unsigned long long)(unsigned)gate_seen, (unsigned)need);
                failed = true;
                break;
              }
            }
            trace_wait(g, 0, base);
          }
        }
        // Issue the whole batch's loads, then forward every step as soon as
        // its stamps are current: each poll round re-issues the loads of all
        // steps still missing (all in flight together) and forwards the ready
        // prefix.  Step base+q reads the source tile's row of its step
        // base+q-1: one contiguous row per step for the whole warp.
        const long long rj0 = (long long)tp_j * R + (base - 1 - rb_j);
        const long long rk0 = (long long)tp_k * R + (base - 1 - rb_k);
        auto needj = [&](int q) {
          const int tau = base + q;
          return lane < NW && tau <= tileHi && tau >= Sj_lo && tau <= Sj_hi;
        };
        auto needk = [&](int q) {
          const int tau = base + q;
          return tau <= tileHi && tau >= Sk_lo && tau <= Sk_hi;
        };
        auto oj = [&](int q) { return ((size_t)(rj0 + q) * NW + lane) * P; };
        auto ok_ = [&](int q) { return ((size_t)(rk0 + q) * 32 + lane) * P; };
        unsigned long long vj[SLB][P], vk[SLB][P];
#pragma unroll
        for (int q = 0; q < SLB; ++q) {
#pragma unroll
          for (int p = 0; p < P; ++p) {
            vj[q][p] = needj(q) ? ld_gpu64(&d.bj[oj(q) + p]) : 0ull;
            vk[q][p] = needk(q) ? ld_gpu64(&d.bk[ok_(q) + p]) : 0ull;
          }
        }
        const int nsteps = min(SLB, tileHi - base + 1);
        int fwd = 0;         // steps of this batch this lane has forwarded (a prefix)
        int published = 0;   // steps of this batch the progress word covers
        Spin s2;
        for (;;) {
#pragma unroll
          for (int q = 0; q < SLB; ++q) {
            if (q == fwd && q < nsteps) {
              bool rdy = true;
#pragma unroll
              for (int p = 0; p < P; ++p) {
                rdy &= !needj(q) || (uint32_t)(vj[q][p] >> 32) == want;
                rdy &= !needk(q) || (uint32_t)(vk[q][p] >> 32) == want;
              }
              if (rdy || failed) {
                uint32_t wj[P], wk[P];
#pragma unroll
                for (int p = 0; p < P; ++p) {
                  wj[p] = (uint32_t)vj[q][p];
                  wk[p] = (uint32_t)vk[q][p];
                }
                const int slot = (base + q) & (SRING - 1);
                if (lane < NW) sh.jr[slot][lane] = needj(q) ? from_words<VT>(wj) : VT(0);
                sh.kr[slot][lane] = needk(q) ? from_words<VT>(wk) : VT(0);
                fwd = q + 1;
              }
            }
          }
          const int all = __reduce_min_sync(XFP_FULL, fwd);
          if (all > published) {
            __threadfence_block();
            __syncwarp();
            if (lane == 0) sh.lprog = base + all - 1;
            published = all;
          }
          if (all >= nsteps) break;
          if (!failed && !s2.step(g.ctl, g.spin_limit)) {
            raise_timeout(g.ctl, 6, tpos, base + all, OP, 0ull, want);
            failed = true;
          }
          failed = __any_sync(XFP_FULL, failed);
          trace_wait(g, 6, base + all);
#pragma unroll
          for (int q = 0; q < SLB; ++q) {
            if (q >= fwd && !failed) {
#pragma unroll
              for (int p = 0; p < P; ++p) {
                if (needj(q) && (uint32_t)(vj[q][p] >> 32) != want) vj[q][p] = ld_gpu64(&d.bj[oj(q) + p]);
                if (needk(q) && (uint32_t)(vk[q][p] >> 32) != want) vk[q][p] = ld_gpu64(&d.bk[ok_(q) + p]);
              }
            }
          }
        }
        trace_wait(g, 0, base + fwd);
      }
    }

    // ---------------- tile epilogue: dot partial (backward) ----------------
    // One z.r partial per x-line (each lane sums its own line in cell order),
    // so the reduction below is the same for every tile height.
    if (OP == SWEEP_BWD && warp < NW) {
      const int jl = j0 + lane, kl = k0 + warp;
      if (jl < nj && kl < nk)
        d.partials[line_base + (size_t)kl * nj + jl] = DOT32 ? (double)dot_acc_f : dot_acc;
    }
    __syncthreads();
  }

  // ---------------- launch epilogue: last CTA closes the generation ----------------
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    unsigned t = atomicAdd(&g.ctl->finished, 1u);
    sh.last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (OP == SWEEP_BWD && g.scal != nullptr && sh.last) {
    // rho_new = z.r over every line, in line order (line_sum); the loader
    // ring is idle now and serves as its 256-double scratch
    __threadfence();
    const double rho_new = line_sum<DOT32>(d.partials, (long long)g.nj * g.nk, reinterpret_cast<double*>(&sh.kr[0][0]));
    if (threadIdx.x == 0) {
      PcgScalars* sc = g.scal;
      if (g.bwd_mode == 0) {
        sc->rho = rho_new;
        if (rho_new == 0.0 || rho_new != rho_new) { sc->status = -5; sc->done = 1; }
      } else {
        sc->beta = DOT32 ? (double)__fdiv_rn((float)rho_new, (float)sc->rho) : __ddiv_rn(rho_new, sc->rho);
        sc->rho = rho_new;
      }
    }
  }
  if (sh.last && threadIdx.x == 0) {
    __threadfence();
    g.ctl->finished = 0;
    __threadfence();
    atomicExch(&g.ctl->gen, gen + 1);
  }
}

template <int OP, typename VT, typename IT, typename CT, int NW, int STAGE>
cudaError_t prepare(int* max_grid) {
  static int cached = -1;
  static cudaError_t cached_err = cudaSuccess;
  if (cached < 0) {
    int dev = 0, nsm = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const int dyn = STAGE != 0 ? stage_bytes<OP, VT, NW>() : 0;
    cached_err = cudaSuccess;
    if (dyn > 0)
      cached_err = cudaFuncSetAttribute(solve_kernel<OP, VT, IT, CT, NW, STAGE>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
    if (cached_err == cudaSuccess)
      cached_err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, solve_kernel<OP, VT, IT, CT, NW, STAGE>,
                                                                 (NW + 2) * 32, dyn);
    cached = per * nsm;
  }
  *max_grid = cached;
  return cached_err;
}

template <int OP, typename VT, typename IT, typename CT, int NW, int STAGE>
cudaError_t launch_nw(const SweepGrid& g, const SweepData<VT, IT, CT>& d, int grid, cudaStream_t st) {
  int maxg = 0;
  cudaError_t e = prepare<OP, VT, IT, CT, NW, STAGE>(&maxg);
  if (e != cudaSuccess) return e;
  if (grid > maxg) grid = maxg;
  if (grid <= 0) return cudaErrorInvalidConfiguration;
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3((NW + 2) * 32);
  cfg.dynamicSmemBytes = STAGE != 0 ? stage_bytes<OP, VT, NW>() : 0;
  cfg.stream = st;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  ++g_kernel_launches;
  return cudaLaunchKernelEx(&cfg, solve_kernel<OP, VT, IT, CT, NW, STAGE>, g, d);
}

// staged groups for 4-byte values and pivots when the launch asks for them
template <typename VT, typename IT>
constexpr bool can_stage() { return sizeof(VT) == 4 && sizeof(IT) == 4; }

template <int OP, typename VT, typename IT, typename CT, int NW>
cudaError_t launch_stage(const SweepGrid& g, const SweepData<VT, IT, CT>& d, int grid, cudaStream_t st) {
  if constexpr (can_stage<VT, IT>())
    if (g.stage == 1) return launch_nw<OP, VT, IT, CT, NW, 1>(g, d, grid, st);
  return launch_nw<OP, VT, IT, CT, NW, 0>(g, d, grid, st);
}
template <int OP, typename VT, typename IT, typename CT, int NW>
int max_grid_stage(int stage) {
  int maxg = 0;
  if constexpr (can_stage<VT, IT>())
    if (stage == 1) {
      prepare<OP, VT, IT, CT, NW, 1>(&maxg);
      return maxg;
    }
  prepare<OP, VT, IT, CT, NW, 0>(&maxg);
  return maxg;
}

template <int OP, typename VT, typename IT, typename CT>
cudaError_t launch_op(const SweepGrid& g, const SweepData<VT, IT, CT>& d, int nw, int grid, cudaStream_t st) {
  switch (nw) {
    case 8: return launch_stage<OP, VT, IT, CT, 8>(g, d, grid, st);
    case 15: return launch_stage<OP, VT, IT, CT, 15>(g, d, grid, st);
    case 16: return launch_stage<OP, VT, IT, CT, 16>(g, d, grid, st);
    default: return cudaErrorInvalidValue;
  }
}

template <int OP, typename VT, typename IT, typename CT>
int max_grid_op(int nw, int stage) {
  switch (nw) {
    case 8: return max_grid_stage<OP, VT, IT, CT, 8>(stage);
    case 15: return max_grid_stage<OP, VT, IT, CT, 15>(stage);
    case 16: return max_grid_stage<OP, VT, IT, CT, 16>(stage);
    default: return 0;
  }
}

}  // namespace

template <typename VT, typename IT, typename CT>
cudaError_t solve_launch(int op, const SweepGrid& g, const SweepData<VT, IT, CT>& d, int nw, int grid,
                         cudaStream_t st) {
  return op == SWEEP_FWD ? launch_op<SWEEP_FWD, VT, IT, CT>(g, d, nw, grid, st)
                         : launch_op<SWEEP_BWD, VT, IT, CT>(g, d, nw, grid, st);
}
template <typename VT, typename IT, typename CT>
int solve_max_grid(int op, int nw, int stage) {
  return op == SWEEP_FWD ? max_grid_op<SWEEP_FWD, VT, IT, CT>(nw, stage)
                         : max_grid_op<SWEEP_BWD, VT, IT, CT>(nw, stage);
}

#define XFP_SOLVE_INST(VT, IT, CT)                                                                   \
  template cudaError_t solve_launch<VT, IT, CT>(int, const SweepGrid&, const SweepData<VT, IT, CT>&, \
                                                int, int, cudaStream_t);                             \
  template int solve_max_grid<VT, IT, CT>(int, int, int);
XFP_SOLVE_INST(double, double, double)
XFP_SOLVE_INST(float, float, float)
XFP_SOLVE_INST(float, float, double)

}  // namespace xfp
