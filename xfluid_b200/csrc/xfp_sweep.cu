// xfp_sweep.cu -- the MIC(0) factorisation in xFluid's natural
// (lexicographic) order, as a persistent dataflow wavefront.  (The triangular
// solves run as lockstep wavefronts in xfp_solve.cu; sweep_launch dispatches
// both.)
//
// Reference semantics (xFluid/xFluid/variationalpressure/pcg_solver.h):
//   factor_modified_incomplete_cholesky0  :85-186
// For the 7-point matrix, cell c=(i,j,k) depends on its lower neighbours
// (i,j,k-1), (i,j-1,k), (i-1,j,k); every update is applied in the reference's
// column order, with separately rounded multiplies and subtractions, so the
// FP64 path is bit-identical to the reference.
//
// Work decomposition.  A thread owns one x-line (j,k) and walks it in i.  A
// warp holds 32 consecutive j at one k; a CTA ("tile") holds NW warps, i.e. a
// 32 x NW block of lines.  Cell (i,j,k) is processed at wavefront step
// tau = i+j+k, so at each step
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
  static_assert(OP == SWEEP_FACTOR, "the triangular solves are in xfp_solve.cu");
  // what a producer sends to one consumer direction: L(m,c) and the sum of the
  // column's other two entries (the dropped fill)
  using X = Pair<CT>;
  static constexpr int P = Words<X>::P;
  static constexpr int RING = 32 / P;   // intra-CTA ring depth (steps)
  static constexpr int LRING = 64 / P;  // loader ring depth (steps)
  static constexpr int LB = 8 / P;      // loader batch (steps polled together)
  static constexpr int PF = 4;  // cell prefetch depth (steps)
  static_assert(RING > QPUB, "ring must be deeper than the progress interval");
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
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned long long* ring = reinterpret_cast<unsigned long long*>(smem_raw);  // [NW][RING][P][32]
  unsigned long long* jring = ring + (size_t)NW * RING * P * 32;              // [LRING][P][NW]
  unsigned long long* kring = jring + (size_t)LRING * P * NW;                 // [LRING][P][32]
  int* s_tlo = reinterpret_cast<int*>(kring + (size_t)LRING * P * 32);        // [NW]
  int* s_thi = s_tlo + NW;                                                    // [NW]
  volatile int* s_prog = s_thi + NW;                                          // [NW] published progress
  int* s_misc = s_thi + 2 * NW;                                               // [NW + 8]

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned gen = ld_volatile_u32(&g.ctl->gen);

  // Invalidate the rings: stamps below are unique per (tile sequence, step).
  {
    const size_t nwords = (size_t)(NW * RING * 32 + LRING * NW + LRING * 32) * P;
    for (size_t q = threadIdx.x; q < nwords; q += blockDim.x) ring[q] = ~0ull;
  }
  __syncthreads();

  for (int pos = blockIdx.x, seq = 0; pos < g.ntiles; pos += gridDim.x, ++seq) {
    const int tpos = pos;
    // the tile's grid: the launch's one scene, or its scene of the batch
    int nj = g.nj, nk = g.nk;
    const Line* lines = g.lines;
    if (g.tile_scene != nullptr) {
      const int sid = g.tile_scene[tpos];
      const BatchSeg& S = g.segs[sid];
      nj = S.nj;
      nk = S.nk;
      lines = S.lines;
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
        tl = a;
        th = b;
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

    if (warp < NW && s_tlo[warp] != INF_T) {
      // ======================= compute warp =======================
      const int Tlo = s_tlo[warp], Thi = s_thi[warp];
      const int k = k0 + warp;
      const int zsrc = warp - 1;   // producer warp in this tile (or the loader)
      const int zdst = warp + 1;   // consumer warp in this tile
      const bool zsrc_in = zsrc >= 0 && zsrc < NW;
      const bool zdst_in = zdst >= 0 && zdst < NW;
      const int zsrc_lo = zsrc_in ? s_tlo[zsrc] : 0, zsrc_hi = zsrc_in ? s_thi[zsrc] : -1;
      const int zdst_lo = zdst_in ? s_tlo[zdst] : 0, zdst_hi = zdst_in ? s_thi[zdst] : -1;
      const bool jb = lane == 0;   // fed by the loader (j boundary)
      const bool kb = !zsrc_in;                            // fed by the loader (k boundary)
      // boundary producers publish stamped values for the neighbouring tiles
      const bool jpub = lane == 31;
      const bool kpub = warp == NW - 1;
      unsigned long long* myring = ring + (size_t)warp * RING * P * 32;
      const unsigned long long* zring = zsrc_in ? ring + (size_t)zsrc * RING * P * 32 : nullptr;

      // the lines above in y and z (their cells take this column's L entries)
      Line Ly = {0, 0, 0, 0}, Lz = {0, 0, 0, 0};
      {
        const int j = j0 + lane;
        if (j + 1 < nj && k < nk) Ly = lines[(size_t)k * nj + j + 1];
        if (j < nj && k + 1 < nk) Lz = lines[(size_t)(k + 1) * nj + j];
      }

      // Cell data of the next PF steps is kept in flight in a rotating register
      // buffer.  Loads are unconditional from a clamped index (cell 0 when the
      // step is outside the lane's span) and masked at use, so the step has
      // no divergent branches.
      struct CellData {
        CT dg, upx, upy, upz;
        int cyup, czup;
      };
      auto load_cell = [&](int i) -> CellData {
        CellData cd;
        const bool in = (unsigned)(i - L.lo) < (unsigned)L.len;
        const int c = in ? L.off + (i - L.lo) : 0;
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
        return cd;
      };
      X out_x{}, out_y{};
      int cons_seen = zdst_in ? (int)s_prog[zdst] : INF_T;   // cached consumer progress

      // One wavefront step of this lane's line: wait for the values produced
      // at the previous step, factor the cell's column and hand its entries on.
      auto step = [&](const int tau, const CellData& cd, const bool in, const int c) {
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
        {
          // factor_modified_incomplete_cholesky0 for column c: updates from
          // columns c-nn, c-ni, c-1 in that order (:137-184), each
          // d -= L*L then d -= omega*L*missing; pivot safeguard (:126-131).
          // the shuffle runs on every lane (full mask); the j-boundary lane
          // then takes its value from the loader instead
          const X vy_sh = shfl_up_any(out_y);
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

      // pf[q] holds the data of step base+q; it is refilled for step
      // base+q+PF right after use and first read again PF steps later
      // (static indices, no register moves, so the load latency stays hidden).
      const int i0 = Tlo - s;
      CellData pf[PF];
#pragma unroll
      for (int q = 0; q < PF; ++q) pf[q] = load_cell(i0 + q);
      for (int base = Tlo; base <= Thi; base += PF) {
#pragma unroll
        for (int q = 0; q < PF; ++q) {
          const int tau = base + q;
          if (tau > Thi) break;
          const int i = i0 + (tau - Tlo);
          const CellData cd = pf[q];
          pf[q] = load_cell(i + PF);
          const bool in = (unsigned)(i - L.lo) < (unsigned)L.len;
          step(tau, cd, in, L.off + (i - L.lo));
        }
      }
      __syncwarp();
      if (lane == 0) s_prog[warp] = INF_T;
    } else if (warp == NW && tileLo != INF_T) {
      // ======================= loader warp =======================
      // lane r < NW feeds jring row r (line k0+r); every lane l feeds kring
      // column l (line j0+l).  Sources are the neighbouring tiles' stamped
      // boundary values (global), or zero where the source cell has no row.
      const int jc = j0, js = j0 - 1;
      const int kc = k0, ks = k0 - 1;
      Line Ljs = {0, 0, 0, 0};
      int sj_c = 0, Sj_lo = INF_T, Sj_hi = INT_MIN;
      {
        const int kr = k0 + lane;
        if (lane < NW && kr < nk && js >= 0 && js < nj) Ljs = lines[(size_t)kr * nj + js];
        sj_c = jc + kr;
        if (Ljs.len > 0) {
          const int a = Ljs.lo + sj_c, b = Ljs.lo + Ljs.len - 1 + sj_c;
          Sj_lo = a;
          Sj_hi = b;
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
          Sk_lo = a;
          Sk_hi = b;
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
        const int ij0 = base - sj_c;
        const int ik0 = base - sk_c;
        const int cj0 = Ljs.off + (ij0 - Ljs.lo), ck0 = Lks.off + (ik0 - Lks.lo);
        auto needj = [&](int q) {
          const int tau = base + q;
          return lane < NW && tau <= tileHi && tau >= Sj_lo && tau <= Sj_hi;
        };
        auto needk = [&](int q) {
          const int tau = base + q;
          return tau <= tileHi && tau >= Sk_lo && tau <= Sk_hi;
        };
        auto oj = [&](int q) { return (size_t)(cj0 + q) * P; };
        auto ok_ = [&](int q) { return (size_t)(ck0 + q) * P; };
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
  int sweep_max_grid(int op, const SweepData<VT, IT, CT>&, int nw, int stage) {                \
    switch (op) {                                                                               \
      case SWEEP_FACTOR: return max_grid_op<SWEEP_FACTOR, VT, IT, CT>(nw);                      \
      default: return solve_max_grid<VT, IT, CT>(op, nw, stage);                                \
    }                                                                                           \
  }

XFP_SWEEP_INST(double, double, double)
XFP_SWEEP_INST(float, float, float)

// The mixed form: the factorisation runs with FP32 L and FP64 pivots
// (float, double, double) and the triangular solves stream FP32 L and the
// pivots rounded to FP32, with FP64 dots (float, float, double).
cudaError_t sweep_launch(int op, const SweepGrid& g, const SweepData<float, double, double>& d, int nw, int grid,
                         cudaStream_t st) {
  return op == SWEEP_FACTOR ? launch_op<SWEEP_FACTOR, float, double, double>(g, d, nw, grid, st)
                            : cudaErrorInvalidValue;
}
int sweep_max_grid(int op, const SweepData<float, double, double>&, int nw, int) {
  return op == SWEEP_FACTOR ? max_grid_op<SWEEP_FACTOR, float, double, double>(nw) : 0;
}
cudaError_t sweep_launch(int op, const SweepGrid& g, const SweepData<float, float, double>& d, int nw, int grid,
                         cudaStream_t st) {
  return op == SWEEP_FACTOR ? cudaErrorInvalidValue : solve_launch<float, float, double>(op, g, d, nw, grid, st);
}
int sweep_max_grid(int op, const SweepData<float, float, double>&, int nw, int stage) {
  return op == SWEEP_FACTOR ? 0 : solve_max_grid<float, float, double>(op, nw, stage);
}

}  // namespace xfp
