// xfp_sweep.cu -- MIC(0) factorisation and triangular solves in xFluid's
// natural (lexicographic) order, as persistent dataflow wavefronts.
//
// Reference semantics (xFluid/xFluid/variationalpressure/pcg_solver.h):
//   factor  factor_modified_incomplete_cholesky0  :85-186
//   forward solve_lower (column-scatter L y = r)  :192-204
//   backward solve_lower_transpose_in_place        :207-220
// For the 7-point matrix, cell c=(i,j,k) depends on its lower neighbours
// (i,j,k-1), (i,j-1,k), (i-1,j,k) (forward, factor) or upper ones (backward);
// every update is applied in the reference's column order, with separately
// rounded multiplies and subtractions, so the FP64 path is bit-identical to
// the reference.
//
// Work decomposition.  A thread owns one x-line (j,k) and walks it in i.  A
// warp holds 32 consecutive j at one k; a CTA ("tile") holds NW warps, i.e. a
// 32 x NW block of lines.  Cell (i,j,k) is processed at wavefront step
// tau = i+j+k (forward; mirrored for the backward sweep), so at each step
//   x-neighbour  = the same lane's previous step          (register)
//   y-neighbour  = the neighbouring lane's previous step   (warp shuffle)
//   z-neighbour  = the neighbouring warp's previous step   (shared-memory ring)
// Values of neighbouring tiles come through a loader warp per CTA.
//
// Hand-off without fences.  Every exchanged value travels inside 64-bit words
// that also carry a stamp (the step, or the launch generation): a consumer
// polls the data word itself until the stamp it expects appears.  An aligned
// 64-bit access is single-copy atomic, so no flag/fence pair is needed on the
// per-step path; payloads wider than 32 bits are split into stamped 32-bit
// halves.  Tile boundaries are published the same way in global memory
// (stamped with the launch generation) by the boundary lanes/warps, and the
// loader warp of the consuming tile polls them.  Ring back-pressure uses
// progress counters that consumers publish every few steps, after a warp
// barrier, so every lane has used (in registers) every ring value it read
// before the counter moves; warps issue in order, so those reads are complete.
//
// Tiles are visited in topological order (J+K ascending) and assigned
// round-robin to a fully co-resident grid (cooperative launch), so a CTA only
// waits on tiles earlier CTAs hold.  Every wait is bounded (spin_limit polls);
// on expiry the kernel records SweepCtl::err, all waits drain quickly and the
// host reports XFP_ERR_TIMEOUT.
#include "xfp_sweep_util.cuh"

namespace xfp {

// Consumers publish ring progress every QPUB steps.  Deadlock freedom needs
// RING > QPUB (a producer waits for the consumer to publish the step that
// frees its slot) and LRING >= LB + QPUB - 1 (same for the loader batch).
constexpr int QPUB = 4;  // (RING >= 8 for every payload)

template <int OP, typename VT, typename IT, typename CT>
struct OpTraits {
  // what a producer sends to one consumer direction
  using X = typename std::conditional<OP == SWEEP_FACTOR, Pair<CT>, VT>::type;
  static constexpr int P = Words<X>::P;
  static constexpr int RING = 32 / P;   // intra-CTA ring depth (steps)
  static constexpr int LRING = 64 / P;  // loader ring depth (steps)
  static constexpr int LB = 8 / P;      // loader batch (steps polled together)
  static constexpr int PF = 4;  // cell prefetch depth (steps)
  static_assert(RING > QPUB, "ring must be deeper than the progress interval");
  static_assert(RING * P * 32 * 8 >= 256, "rings must hold the 256-slot line reduction");
  static_assert(LRING >= LB + QPUB - 1, "loader ring too shallow");
};

template <int OP, typename VT, typename IT, typename CT>
__host__ __device__ constexpr size_t smem_bytes(int nw) {
  using T = OpTraits<OP, VT, IT, CT>;
  return 8 * ((size_t)nw * T::RING * T::P * 32 + (size_t)T::LRING * T::P * nw +
              (size_t)T::LRING * T::P * 32) +
         sizeof(int) * (4 * (size_t)nw + 8) + sizeof(double) * (nw + 2);
}

// One CTA per SM is all the bound asks for.  Asking for two made the
// compiler settle at 96 registers and spill inside the step loop, which cost
// more than the second CTA gained; with this bound the FP32/mixed sweeps take
// 104-118 registers without spilling (those at or under 112 still get two
// CTAs per SM from the occupancy query).
template <int OP, typename VT, typename IT, typename CT, int NW>
__global__ void __launch_bounds__((NW + 1) * 32, 1)
    sweep_kernel(SweepGrid g, SweepData<VT, IT, CT> d) {
  using TR = OpTraits<OP, VT, IT, CT>;
  using X = typename TR::X;
  constexpr int P = TR::P, RING = TR::RING, LRING = TR::LRING, LB = TR::LB, PF = TR::PF;
  constexpr bool REV = (OP == SWEEP_BWD);
  constexpr bool DOT32 = std::is_same<VT, float>::value && !std::is_same<IT, double>::value;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned long long* ring = reinterpret_cast<unsigned long long*>(smem_raw);  // [NW][RING][P][32]
  unsigned long long* jring = ring + (size_t)NW * RING * P * 32;              // [LRING][P][NW]
  unsigned long long* kring = jring + (size_t)LRING * P * NW;                 // [LRING][P][32]
  int* s_tlo = reinterpret_cast<int*>(kring + (size_t)LRING * P * 32);        // [NW]
  int* s_thi = s_tlo + NW;                                                    // [NW]
  volatile int* s_prog = s_thi + NW;                                          // [NW] published progress
  int* s_misc = s_thi + 2 * NW;                                               // [NW + 8]
  double* s_red = reinterpret_cast<double*>(s_misc + NW + 8);                 // [NW + 2]

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned gen = ld_volatile_u32(&g.ctl->gen);

  if (OP != SWEEP_FACTOR && g.scal != nullptr && *(volatile int*)&g.scal->done != 0) return;

  // Invalidate the rings: stamps below are unique per (tile sequence, step).
  {
    const size_t nwords = (size_t)(NW * RING * 32 + LRING * NW + LRING * 32) * P;
    for (size_t q = threadIdx.x; q < nwords; q += blockDim.x) ring[q] = ~0ull;
  }
  __syncthreads();

  for (int pos = blockIdx.x, seq = 0; pos < g.ntiles; pos += gridDim.x, ++seq) {
    const int tpos = REV ? g.ntiles - 1 - pos : pos;
    // the tile's grid: the launch's one scene, or its scene of the batch
    int nj = g.nj, nk = g.nk, maxT = g.maxT;
    const Line* lines = g.lines;
    long long line_base = 0;
    if (g.tile_scene != nullptr) {
      const int sid = g.tile_scene[tpos];
      const BatchSeg& S = g.segs[sid];
      // a converged scene's tiles are skipped (its scalars only change between
      // launches, so every CTA of this launch decides the same way)
      if (OP != SWEEP_FACTOR && g.scal_batch != nullptr && *(volatile int*)&g.scal_batch[sid].done != 0) continue;
      nj = S.nj;
      nk = S.nk;
      maxT = S.ni + S.nj + S.nk;
      lines = S.lines;
      line_base = S.line_base;
    }
    const int packed = g.tiles[tpos];
    const int J = packed & 0xffff, K = packed >> 16;
    const int j0 = J * 32, k0 = K * NW;
    const uint32_t tstamp = (uint32_t)(seq & 0x7ff) << 20;   // | step (< 2^20)

    // ---------------- setup: per-warp wavefront ranges ----------------
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
        s_tlo[warp] = Tlo;
        s_thi[warp] = Thi;
        s_prog[warp] = (Tlo == INF_T) ? INF_T : Tlo - 1;
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      int lo = INF_T, hi = INT_MIN;
      for (int w = 0; w < NW; ++w) {
        lo = min(lo, s_tlo[w]);
        hi = max(hi, s_thi[w]);
      }
      s_misc[1] = lo;
      s_misc[2] = hi;
    }
    __syncthreads();
    const int tileLo = s_misc[1], tileHi = s_misc[2];

    double dot_acc = 0.0;
    float dot_acc_f = 0.0f;

    if (warp < NW && s_tlo[warp] != INF_T) {
      // ======================= compute warp =======================
      const int Tlo = s_tlo[warp], Thi = s_thi[warp];
      const int k = k0 + warp;
      const int zsrc = REV ? warp + 1 : warp - 1;   // producer warp in this tile (or the loader)
      const int zdst = REV ? warp - 1 : warp + 1;   // consumer warp in this tile
      const bool zsrc_in = zsrc >= 0 && zsrc < NW;
      const bool zdst_in = zdst >= 0 && zdst < NW;
      const int zsrc_lo = zsrc_in ? s_tlo[zsrc] : 0, zsrc_hi = zsrc_in ? s_thi[zsrc] : -1;
      const int zdst_lo = zdst_in ? s_tlo[zdst] : 0, zdst_hi = zdst_in ? s_thi[zdst] : -1;
      const bool jb = REV ? (lane == 31) : (lane == 0);   // fed by the loader (j boundary)
      const bool kb = !zsrc_in;                            // fed by the loader (k boundary)
      // boundary producers publish stamped values for the neighbouring tiles
      const bool jpub = REV ? (lane == 0) : (lane == 31);
      const bool kpub = REV ? (warp == 0) : (warp == NW - 1);
      unsigned long long* myring = ring + (size_t)warp * RING * P * 32;
      const unsigned long long* zring = zsrc_in ? ring + (size_t)zsrc * RING * P * 32 : nullptr;

      Line Ly = {0, 0, 0, 0}, Lz = {0, 0, 0, 0};
      if (OP == SWEEP_FACTOR) {
        const int j = j0 + lane;
        if (j + 1 < nj && k < nk) Ly = lines[(size_t)k * nj + j + 1];
        if (j < nj && k + 1 < nk) Lz = lines[(size_t)(k + 1) * nj + j];
      }

      // Cell data of the next PF steps is kept in flight in a rotating register
      // buffer.  Loads are unconditional from a clamped index (cell 0 when the
      // step is outside the lane's span) and masked at use, so the step has
      // no divergent branches.
      struct CellData {
        VT r, lx, ly, lz, rr;
        IT inv;
        CT dg, upx, upy, upz;
        int cyup, czup;
      };
      const int di = REV ? -1 : 1;
      auto load_cell = [&](int i) -> CellData {
        CellData cd;
        const bool in = (unsigned)(i - L.lo) < (unsigned)L.len;
        const int c = in ? L.off + (i - L.lo) : 0;
        cd.rr = VT(0);
        cd.r = cd.lx = cd.ly = cd.lz = VT(0);
        cd.inv = IT(0);
        cd.dg = cd.upx = cd.upy = cd.upz = CT(0);
        cd.cyup = cd.czup = -1;
        if constexpr (OP == SWEEP_FWD) {
          cd.r = d.r[c]; cd.lx = d.lx[c]; cd.ly = d.ly[c]; cd.lz = d.lz[c]; cd.inv = d.inv[c];
        } else if constexpr (OP == SWEEP_BWD) {
          cd.r = d.y[c]; cd.lx = d.lx[c]; cd.ly = d.ly[c]; cd.lz = d.lz[c]; cd.inv = d.inv[c];
          cd.rr = d.r[c];
        } else {
          cd.dg = d.diag[c];
          const bool hx = in && (i + 1 - L.lo < L.len);
          const CT ux = d.ax[hx ? c + 1 : 0];
          cd.upx = hx ? ux : CT(0);
          const bool hy = (unsigned)(i - Ly.lo) < (unsigned)Ly.len;
          cd.cyup = hy ? Ly.off + (i - Ly.lo) : -1;
          const CT uy = d.ay[hy ? cd.cyup : 0];
          cd.upy = hy ? uy : CT(0);
          const bool hz = (unsigned)(i - Lz.lo) < (unsigned)Lz.len;
          cd.czup = hz ? Lz.off + (i - Lz.lo) : -1;
          const CT uz = d.az[hz ? cd.czup : 0];
          cd.upz = hz ? uz : CT(0);
        }
        return cd;
      };
      X out_x{}, out_y{};
      int cons_seen = zdst_in ? (int)s_prog[zdst] : INF_T;   // cached consumer progress

      // One wavefront step of this lane's line: wait for the values produced
      // at the previous step, compute the cell and hand its outputs on.  The
      // forward/backward result goes to yout; the caller stores it.
      auto step = [&](const int tau, const CellData& cd, const bool in, const int c, VT& yout) {
        // ---- neighbour values produced at the previous step ----
        // z: previous warp (ring) or the loader (kring); j boundary: loader
        // (jring, one word per warp, read by all lanes as a broadcast).
        const bool zneed = kb || (tau - 1 >= zsrc_lo && tau - 1 <= zsrc_hi);   // warp-uniform
        const uint32_t ez = tstamp | (kb ? tau : tau - 1), ej = tstamp | tau;
        const unsigned long long* zaddr =
            kb ? kring + (size_t)(tau & (LRING - 1)) * P * 32 + lane
               : zring + (size_t)((tau - 1) & (RING - 1)) * P * 32 + lane;
        const unsigned long long* jaddr = jring + (size_t)(tau & (LRING - 1)) * P * NW + warp;
        unsigned long long wz[P], wj[P];
        auto fetch = [&]() {
#pragma unroll
          for (int p = 0; p < P; ++p) {
            wz[p] = zneed ? ld_vol64(zaddr + (size_t)p * 32) : 0ull;
            wj[p] = ld_vol64(jaddr + (size_t)p * NW);
          }
        };
        auto ready = [&]() -> bool {
          bool ok = true;
#pragma unroll
          for (int p = 0; p < P; ++p) {
            ok &= !zneed || (uint32_t)(wz[p] >> 32) == ez;
            ok &= !jb || (uint32_t)(wj[p] >> 32) == ej;
          }
          return ok;
        };
        auto wait_inputs = [&]() {
          fetch();
          if (!__all_sync(XFP_FULL, ready())) {
            trace_wait(g, kb ? 2 : 1, tau);
            Spin sp;
            do {
              if (!sp.step(g.ctl, g.spin_limit)) {
                raise_timeout(g.ctl, kb ? 2 : 1, tpos, tau, OP, wz[0], ez);
                break;
              }
              fetch();
            } while (!__all_sync(XFP_FULL, ready()));
            trace_wait(g, 0, tau);
          }
        };
        auto take_z = [&]() -> X {
          X vz{};
          if (zneed) {
            uint32_t w[P];
#pragma unroll
            for (int p = 0; p < P; ++p) w[p] = (uint32_t)wz[p];
            vz = from_words<X>(w);
          }
          return vz;
        };
        auto take_j = [&]() -> X {
          uint32_t w[P];
#pragma unroll
          for (int p = 0; p < P; ++p) w[p] = (uint32_t)wj[p];
          return from_words<X>(w);
        };
        // ring back-pressure: slot tau%RING last held step tau-RING, which the
        // consumer reads at step tau-RING+1; its progress is published every
        // QPUB steps.  Checked before the inputs arrive, off the critical path.
        auto ring_space = [&]() {
          if (!zdst_in) return;
          const int need = tau - RING + 1;
          if (need > cons_seen && need >= zdst_lo && need <= zdst_hi) {
            trace_wait(g, 4, tau);
            Spin sp;
            while ((cons_seen = s_prog[zdst]) < need) {
              if (!sp.step(g.ctl, g.spin_limit)) {
                raise_timeout(g.ctl, 4, tpos, tau, OP, (unsigned long long)(unsigned)cons_seen, (unsigned)need);
                break;
              }
            }
            trace_wait(g, 0, tau);
          }
        };
        auto ring_put = [&](const X& oz) {
          if (!zdst_in) return;
          uint32_t w[P];
          to_words(oz, w);
          unsigned long long* slot = myring + (size_t)(tau & (RING - 1)) * P * 32 + lane;
#pragma unroll
          for (int p = 0; p < P; ++p) st_vol64(slot + (size_t)p * 32, stamped(tstamp | tau, w[p]));
        };

        X o_x{}, o_y{}, o_z{};
        if constexpr (OP == SWEEP_FWD) {
          // solve_lower: columns c-nn, c-ni, c-1 scatter into row c in that
          // order, then result[c] *= invdiag[c]  (pcg_solver.h:198-203).
          // Everything that does not need the z value is done before waiting
          // for it; after it arrives only the dependent chain and the hand-off
          // to the next warp remain (same roundings, same order).
          const X vy_sh = REV ? shfl_down_any(out_y) : shfl_up_any(out_y);
          const VT px = mul_rn(cd.lx, out_x);
          const VT py_sh = mul_rn(cd.ly, vy_sh);
          ring_space();
          wait_inputs();
          const X vz = take_z();
          VT py = py_sh;
          if (jb) py = mul_rn(cd.ly, take_j());
          VT t = sub_rn(cd.r, mul_rn(cd.lz, vz));
          t = sub_rn(t, py);
          t = sub_rn(t, px);
          const VT y = in ? VT(mul_rn((IT)t, cd.inv)) : VT(0);
          ring_put(y);
          yout = y;
          o_x = y; o_y = y; o_z = y;
        } else if constexpr (OP == SWEEP_BWD) {
          // solve_lower_transpose_in_place: x[c] -= L(m,c) x[m] for m = c+1,
          // c+ni, c+nn in that order, then x[c] *= invdiag[c]  (:215-218).
          // The products L(m,c) x[m] arrive ready-made from the producers;
          // the x and y terms are subtracted before waiting for z.
          const X vy_sh = REV ? shfl_down_any(out_y) : shfl_up_any(out_y);
          const VT t1 = sub_rn(cd.r, out_x);
          const VT t2_sh = sub_rn(t1, vy_sh);
          ring_space();
          wait_inputs();
          const X vz = take_z();
          VT t2 = t2_sh;
          if (jb) t2 = sub_rn(t1, take_j());
          const VT t = sub_rn(t2, vz);
          const VT z = in ? VT(mul_rn((IT)t, cd.inv)) : VT(0);
          o_z = mul_rn(in ? cd.lz : VT(0), z);
          ring_put(o_z);
          yout = z;
          const VT rr = in ? cd.rr : VT(0);
          if (DOT32) dot_acc_f = __fadd_rn(dot_acc_f, __fmul_rn((float)z, (float)rr));
          else dot_acc = __dadd_rn(dot_acc, __dmul_rn((double)z, (double)rr));
          o_x = mul_rn(in ? cd.lx : VT(0), z);
          o_y = mul_rn(in ? cd.ly : VT(0), z);
        } else {
          // factor_modified_incomplete_cholesky0 for column c: updates from
          // columns c-nn, c-ni, c-1 in that order (:137-184), each
          // d -= L*L then d -= omega*L*missing; pivot safeguard (:126-131).
          // the shuffle runs on every lane (full mask); the j-boundary lane
          // then takes its value from the loader instead
          const X vy_sh = REV ? shfl_down_any(out_y) : shfl_up_any(out_y);
          wait_inputs();
          const X vz = take_z();
          X vy = vy_sh;
          if (jb) vy = take_j();
          const bool act = in && cd.dg != CT(0);
          CT dd = cd.dg;
          const X src[3] = {vz, vy, out_x};
#pragma unroll
          for (int t = 0; t < 3; ++t) {
            dd = sub_rn(dd, mul_rn(src[t].a, src[t].a));
            dd = sub_rn(dd, mul_rn(mul_rn(d.omega, src[t].a), src[t].b));
          }
          const CT iv = act ? ((dd < mul_rn(d.ratio, cd.dg)) ? rsqrt_ref(cd.dg) : rsqrt_ref(dd)) : CT(0);
          // column c's entries L(m,c) = A(m,c)*invdiag[c] for m = c+1,
          // c+ni, c+nn, and for each the sum of the other two (dropped fill)
          const CT px = mul_rn(cd.upx, iv), py = mul_rn(cd.upy, iv), pz = mul_rn(cd.upz, iv);
          o_x = {px, add_rn(py, pz)};
          o_y = {py, add_rn(px, pz)};
          o_z = {pz, add_rn(px, py)};
          ring_space();
          ring_put(o_z);
          if (act && cd.upx != CT(0)) d.flx[c + 1] = px;
          if (act && cd.cyup >= 0) d.fly[cd.cyup] = py;
          if (act && cd.czup >= 0) d.flz[cd.czup] = pz;
          if (in) d.oinv[c] = (IT)iv;
        }

        // ---- publish for the other tiles (stamped with the generation) ----
        if (in && jpub) {
          uint32_t w[P];
          to_words(o_y, w);
#pragma unroll
          for (int p = 0; p < P; ++p) st_gpu64(&d.sy[(size_t)c * P + p], stamped(gen, w[p]));
        }
        if (in && kpub) {
          uint32_t w[P];
          to_words(o_z, w);
#pragma unroll
          for (int p = 0; p < P; ++p) st_gpu64(&d.sz[(size_t)c * P + p], stamped(gen, w[p]));
        }
        out_x = o_x;
        out_y = o_y;
        // Progress is published only once every lane has finished the step
        // (a slot is reused as soon as its consumer's progress says it was read).
        if (((tau - Tlo) & (QPUB - 1)) == QPUB - 1) {
          __syncwarp();
          if (lane == 0) {
            s_prog[warp] = tau;
            if (g.trace && !ld_volatile_u32(&g.ctl->err))
              *(volatile int*)&g.trace[((size_t)blockIdx.x * (NW + 1) + warp) * 4 + 2] = tau;
          }
        }
      };

      if constexpr (OP == SWEEP_FACTOR) {
        // pf[q] holds the data of step base+q; it is refilled for step
        // base+q+PF right after use and first read again PF steps later
        // (static indices, no register moves, so the load latency stays hidden).
        const int i0 = REV ? (maxT - Tlo) - s : Tlo - s;
        CellData pf[PF];
#pragma unroll
        for (int q = 0; q < PF; ++q) pf[q] = load_cell(i0 + q * di);
        for (int base = Tlo; base <= Thi; base += PF) {
#pragma unroll
          for (int q = 0; q < PF; ++q) {
            const int tau = base + q;
            if (tau > Thi) break;
            const int i = i0 + (tau - Tlo) * di;
            const CellData cd = pf[q];
            pf[q] = load_cell(i + PF * di);
            const bool in = (unsigned)(i - L.lo) < (unsigned)L.len;
            VT unused;
            step(tau, cd, in, L.off + (i - L.lo), unused);
          }
        }
      } else {
        // Grouped access.  A line is stored so that cell (i,j,k) sits at an
        // address = i+j+k (mod GS): at every wavefront step all lanes of the
        // warp are at the same position within an aligned group of GS cells.
        // Each lane therefore loads the next GS cells of each array with
        // vector accesses and stores GS results at once, instead of touching
        // one 32-byte sector per array per step.  The group covering steps
        // t0..t0+GS-1 is loaded GS steps before use, into the buffer the
        // previous group has just released (two static buffers, no register
        // moves).  A group lies entirely inside or outside the span.
        constexpr int GS = XFP_ALIGN;
        static_assert(GS == 4, "group load/store helpers cover 4-cell groups");
        struct Grp {
          VT r[GS], lx[GS], ly[GS], lz[GS], rr[GS];
          IT inv[GS];
        };
        // forward: address phase of step t is t mod GS (increasing cells);
        // backward: (maxT - t) mod GS, cells decreasing
        const int a = REV ? ((maxT + 1) & (GS - 1)) : 0;
        const int base0 = Tlo - ((Tlo - a) & (GS - 1));
        auto group_c4 = [&](int t0) -> int {
          const int ilow = REV ? (maxT - (t0 + GS - 1)) - s : t0 - s;
          const int rel = ilow - L.lo;
          return (unsigned)rel < (unsigned)L.len ? L.off + rel : -1;
        };
        auto load_grp = [&](Grp& G, int c4) {
          const int cc = c4 >= 0 ? c4 : 0;
          if constexpr (OP == SWEEP_FWD) {
            ldg(G.r, d.r + cc);
          } else {
            ldg(G.r, d.y + cc);
            ldg(G.rr, d.r + cc);
          }
          ldg(G.lx, d.lx + cc);
          ldg(G.ly, d.ly + cc);
          ldg(G.lz, d.lz + cc);
          ldg(G.inv, d.inv + cc);
        };
        auto run_group = [&](int t0, const Grp& G, int c4) {
          VT yb[GS];
#pragma unroll
          for (int q = 0; q < GS; ++q) {
            const int tau = t0 + q;
            const int e = REV ? GS - 1 - q : q;
            yb[e] = VT(0);
            if (tau >= Tlo && tau <= Thi) {
              CellData cd;
              cd.r = G.r[e]; cd.lx = G.lx[e]; cd.ly = G.ly[e]; cd.lz = G.lz[e]; cd.inv = G.inv[e];
              cd.rr = (OP == SWEEP_BWD) ? G.rr[e] : VT(0);
              const bool in = c4 >= 0;
              step(tau, cd, in, (in ? c4 : 0) + e, yb[e]);
            }
          }
          if (c4 >= 0) stg(d.y + c4, yb);
        };
        Grp GA, GB;
        int cA = group_c4(base0);
        load_grp(GA, cA);
        for (int gb = base0; gb <= Thi; gb += 2 * GS) {
          const int cB = group_c4(gb + GS);
          load_grp(GB, cB);
          run_group(gb, GA, cA);
          if (gb + GS > Thi) break;
          const int cA2 = group_c4(gb + 2 * GS);
          load_grp(GA, cA2);
          run_group(gb + GS, GB, cB);
          cA = cA2;
        }
      }
      __syncwarp();
      if (lane == 0) s_prog[warp] = INF_T;
    } else if (warp == NW && tileLo != INF_T) {
      // ======================= loader warp =======================
      // lane r < NW feeds jring row r (line k0+r); every lane l feeds kring
      // column l (line j0+l).  Sources are the neighbouring tiles' stamped
      // boundary values (global), or zero where the source cell has no row.
      const int jc = REV ? j0 + 31 : j0, js = REV ? j0 + 32 : j0 - 1;
      const int kc = REV ? k0 + NW - 1 : k0, ks = REV ? k0 + NW : k0 - 1;
      Line Ljs = {0, 0, 0, 0};
      int sj_c = 0, Sj_lo = INF_T, Sj_hi = INT_MIN;
      {
        const int kr = k0 + lane;
        if (lane < NW && kr < nk && js >= 0 && js < nj) Ljs = lines[(size_t)kr * nj + js];
        sj_c = jc + kr;
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
      int cons_min = tileLo - 1;   // cached min progress over the compute warps
      for (int base = tileLo; base <= tileHi; base += LB) {
        // ring space for the whole batch: slot of step t last held t-LRING,
        // read by its consumers at that same step
        const int need = base + LB - 1 - LRING;
        if (need > cons_min) {
          trace_wait(g, 5, base);
          Spin sp;
          for (;;) {
            int m = INF_T;
            for (int w = 0; w < NW; ++w) m = min(m, (int)s_prog[w]);
            cons_min = m;
            if (cons_min >= need) break;
            if (!sp.step(g.ctl, g.spin_limit)) { raise_timeout(g.ctl, 5, tpos, base, OP, (unsigned long long)(unsigned)cons_min, (unsigned)need); break; }
          }
          trace_wait(g, 0, base);
        }
        // Issue the whole batch's loads, then forward every step to the rings
        // as soon as its stamps are current: each poll round re-issues the
        // loads of all steps still missing (all in flight together) and
        // forwards the ready prefix, so a step reaches the compute warps one
        // round trip after its producer published it, and a round trip can
        // deliver a whole batch.  The source cell of step base+q lies q cells
        // further along the source line (backward: q cells back).
        const int ij0 = REV ? (maxT - base) - sj_c : base - sj_c;
        const int ik0 = REV ? (maxT - base) - sk_c : base - sk_c;
        const int cj0 = Ljs.off + (ij0 - Ljs.lo), ck0 = Lks.off + (ik0 - Lks.lo);
        auto needj = [&](int q) {
          const int tau = base + q;
          return lane < NW && tau <= tileHi && tau >= Sj_lo && tau <= Sj_hi;
        };
        auto needk = [&](int q) {
          const int tau = base + q;
          return tau <= tileHi && tau >= Sk_lo && tau <= Sk_hi;
        };
        auto oj = [&](int q) { return (size_t)(REV ? cj0 - q : cj0 + q) * P; };
        auto ok_ = [&](int q) { return (size_t)(REV ? ck0 - q : ck0 + q) * P; };
        unsigned long long vj[LB][P], vk[LB][P];
#pragma unroll
        for (int q = 0; q < LB; ++q) {
#pragma unroll
          for (int p = 0; p < P; ++p) {
            vj[q][p] = needj(q) ? ld_gpu64(&d.sy[oj(q) + p]) : 0ull;
            vk[q][p] = needk(q) ? ld_gpu64(&d.sz[ok_(q) + p]) : 0ull;
          }
        }
        const int nsteps = min(LB, tileHi - base + 1);
        const unsigned want = gen + g.expect_bias;   // bias != 0 only in the expired-wait diagnostic
        int fwd = 0;   // steps of this batch already forwarded (a prefix)
        Spin s2;
        for (;;) {
#pragma unroll
          for (int q = 0; q < LB; ++q) {
            if (q == fwd && q < nsteps) {
              bool rdy = true;
#pragma unroll
              for (int p = 0; p < P; ++p) {
                rdy &= !needj(q) || (uint32_t)(vj[q][p] >> 32) == want;
                rdy &= !needk(q) || (uint32_t)(vk[q][p] >> 32) == want;
              }
              if (rdy) {
                const uint32_t st = tstamp | (base + q);
                const int slot = (base + q) & (LRING - 1);
#pragma unroll
                for (int p = 0; p < P; ++p) {
                  if (lane < NW)
                    st_vol64(&jring[((size_t)slot * P + p) * NW + lane],
                             stamped(st, needj(q) ? (uint32_t)vj[q][p] : 0u));
                  st_vol64(&kring[((size_t)slot * P + p) * 32 + lane],
                           stamped(st, needk(q) ? (uint32_t)vk[q][p] : 0u));
                }
                fwd = q + 1;
              }
            }
          }
          if (fwd >= nsteps) break;
          if (!s2.step(g.ctl, g.spin_limit)) {
            raise_timeout(g.ctl, 6, tpos, base + fwd, OP, 0ull, want);
            break;
          }
          trace_wait(g, 6, base + fwd);
#pragma unroll
          for (int q = 0; q < LB; ++q) {
            if (q >= fwd) {
#pragma unroll
              for (int p = 0; p < P; ++p) {
                if (needj(q) && (uint32_t)(vj[q][p] >> 32) != want) vj[q][p] = ld_gpu64(&d.sy[oj(q) + p]);
                if (needk(q) && (uint32_t)(vk[q][p] >> 32) != want) vk[q][p] = ld_gpu64(&d.sz[ok_(q) + p]);
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
  __shared__ int s_last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    unsigned t = atomicAdd(&g.ctl->finished, 1u);
    s_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (OP == SWEEP_BWD && g.scal != nullptr && s_last) {
    // rho_new = z.r over every line, in line order (line_sum)
    __threadfence();
    // the rings are idle now (every tile of this CTA is done): 256 doubles of scratch
    const double rho_new = line_sum<DOT32>(d.partials, (long long)g.nj * g.nk, reinterpret_cast<double*>(ring));
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
  if (s_last && threadIdx.x == 0) {
    __threadfence();
    g.ctl->finished = 0;
    __threadfence();
    atomicExch(&g.ctl->gen, gen + 1);
  }
}

// ---------------------------------------------------------------- host side
template <int OP, typename VT, typename IT, typename CT, int NW>
static cudaError_t prepare(int* max_grid) {
  static int cached = -1;
  static cudaError_t cached_err = cudaSuccess;
  if (cached < 0) {
    const size_t sm = smem_bytes<OP, VT, IT, CT>(NW);
    auto kfn = sweep_kernel<OP, VT, IT, CT, NW>;
    cached_err = cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    int dev = 0, nsm = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (cached_err == cudaSuccess)
      cached_err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kfn, (NW + 1) * 32, sm);
    cached = per * nsm;
  }
  *max_grid = cached;
  return cached_err;
}

template <int OP, typename VT, typename IT, typename CT, int NW>
static cudaError_t launch_nw(const SweepGrid& g, const SweepData<VT, IT, CT>& d, int grid, cudaStream_t st) {
  int maxg = 0;
  cudaError_t e = prepare<OP, VT, IT, CT, NW>(&maxg);
  if (e != cudaSuccess) return e;
  if (grid > maxg) grid = maxg;
  if (grid <= 0) return cudaErrorInvalidConfiguration;
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3((NW + 1) * 32);
  cfg.dynamicSmemBytes = smem_bytes<OP, VT, IT, CT>(NW);
  cfg.stream = st;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  ++g_kernel_launches;
  return cudaLaunchKernelEx(&cfg, sweep_kernel<OP, VT, IT, CT, NW>, g, d);
}

template <int OP, typename VT, typename IT, typename CT>
static cudaError_t launch_op(const SweepGrid& g, const SweepData<VT, IT, CT>& d, int nw, int grid,
                             cudaStream_t st) {
  switch (nw) {
    case 8: return launch_nw<OP, VT, IT, CT, 8>(g, d, grid, st);
    case 16: return launch_nw<OP, VT, IT, CT, 16>(g, d, grid, st);
    case 15: return launch_nw<OP, VT, IT, CT, 15>(g, d, grid, st);
    default: return cudaErrorInvalidValue;
  }
}

template <int OP, typename VT, typename IT, typename CT>
static int max_grid_op(int nw) {
  int maxg = 0;
  switch (nw) {
    case 8: prepare<OP, VT, IT, CT, 8>(&maxg); break;
    case 16: prepare<OP, VT, IT, CT, 16>(&maxg); break;
    case 15: prepare<OP, VT, IT, CT, 15>(&maxg); break;
    default: break;
  }
  return maxg;
}

#define XFP_SWEEP_INST(VT, IT, CT)                                                              \
  cudaError_t sweep_launch(int op, const SweepGrid& g, const SweepData<VT, IT, CT>& d, int nw,  \
                           int grid, cudaStream_t st) {                                         \
    switch (op) {                                                                               \
      case SWEEP_FACTOR: return launch_op<SWEEP_FACTOR, VT, IT, CT>(g, d, nw, grid, st);        \
      default: return solve_launch<VT, IT, CT>(op, g, d, nw, grid, st);                         \
    }                                                                                           \
  }                                                                                             \
  int sweep_max_grid(int op, const SweepData<VT, IT, CT>&, int nw) {                            \
    switch (op) {                                                                               \
      case SWEEP_FACTOR: return max_grid_op<SWEEP_FACTOR, VT, IT, CT>(nw);                      \
      default: return solve_max_grid<VT, IT, CT>(op, nw);                                       \
    }                                                                                           \
  }

XFP_SWEEP_INST(double, double, double)
XFP_SWEEP_INST(float, float, float)
XFP_SWEEP_INST(float, double, double)

}  // namespace xfp
