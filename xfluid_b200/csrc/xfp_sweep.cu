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
// 32 x NW block of lines.  Cell (i,j,k) is processed at wavefront time
// tau = i+j+k (forward; mirrored for the backward sweep), so at each step
//   x-neighbour  = the same lane's previous step        (register)
//   y-neighbour  = the neighbouring lane's previous step  (warp shuffle)
//   z-neighbour  = the neighbouring warp's previous step  (shared-memory ring,
//                  per-warp progress counters in shared memory)
// Lines of neighbouring tiles arrive through a loader warp per CTA that waits
// on the producing tile's published progress (global memory, release/acquire,
// generation-tagged) and stages the boundary values into shared-memory rings.
// Warps never wait on a global barrier: each waits only on the producers its
// cells actually depend on, so independent regions run concurrently.
//
// Tiles are visited in a topological order (J+K ascending) and assigned
// round-robin to a grid that is fully co-resident (cooperative launch), so a
// CTA only ever waits on tiles that earlier CTAs hold: no deadlock.  Every
// wait is bounded (spin_limit polls); on expiry the kernel records an error in
// SweepCtl::err, all CTAs drain and the host reports XFP_ERR_TIMEOUT.
#include <climits>
#include <type_traits>

#include "xfp_common.cuh"
#include "xfp_kernels.h"

namespace xfp {

constexpr int RING = 16;    // intra-CTA ring depth in wavefront steps
constexpr int LRING = 64;   // loader ring depth
constexpr int PUB = 8;      // publish global progress every PUB steps
constexpr int INF_T = INT_MAX;

template <typename T>
struct Pair {
  T a, b;
};
template <typename T>
__device__ __forceinline__ Pair<T> shfl_up(Pair<T> v, int d) {
  return {__shfl_up_sync(XFP_FULL, v.a, d), __shfl_up_sync(XFP_FULL, v.b, d)};
}
template <typename T>
__device__ __forceinline__ Pair<T> shfl_down(Pair<T> v, int d) {
  return {__shfl_down_sync(XFP_FULL, v.a, d), __shfl_down_sync(XFP_FULL, v.b, d)};
}

template <int OP, typename VT, typename IT, typename CT>
struct OpTraits {
  // ring element: what a producer sends to one consumer direction
  using R = typename std::conditional<OP == SWEEP_FACTOR, Pair<CT>, VT>::type;
};

__device__ __forceinline__ unsigned long long prog_word(unsigned gen, unsigned v) {
  return ((unsigned long long)gen << 32) | v;
}
// Completed-steps value of a progress word for generation gen (0 if stale).
__device__ __forceinline__ unsigned prog_value(unsigned long long w, unsigned gen) {
  return (unsigned)(w >> 32) == gen ? (unsigned)w : 0u;
}

struct Spin {
  long long n = 0;
  __device__ __forceinline__ bool step(const SweepCtl* ctl, long long limit) {
    ++n;
    if (n > 64) __nanosleep(n > 4096 ? 256 : 32);
    if ((n & 63) == 0 && ld_volatile_u32(&ctl->err)) return false;
    return n < limit;
  }
};

__device__ __forceinline__ void raise_timeout(SweepCtl* ctl, unsigned where) {
  atomicOr(&ctl->err, 1u);
  atomicMax(&ctl->err_where, where);
}

template <int OP, typename VT, typename IT, typename CT>
struct Smem {
  using R = typename OpTraits<OP, VT, IT, CT>::R;
  static __host__ __device__ size_t bytes(int nw) {
    size_t b = sizeof(R) * ((size_t)nw * RING * 32 + (size_t)LRING * nw + (size_t)LRING * 32);
    b = (b + 15) & ~size_t(15);
    b += sizeof(int) * (4 * nw + 8) + sizeof(double) * (nw + 2);
    return b;
  }
};

template <int OP, typename VT, typename IT, typename CT, int NW>
__global__ void __launch_bounds__((NW + 1) * 32, 1)
    sweep_kernel(SweepGrid g, SweepData<VT, IT, CT> d) {
  using R = typename OpTraits<OP, VT, IT, CT>::R;
  constexpr bool REV = (OP == SWEEP_BWD);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* ring = reinterpret_cast<R*>(smem_raw);               // [NW][RING][32]
  R* jring = ring + (size_t)NW * RING * 32;               // [LRING][NW]
  R* kring = jring + (size_t)LRING * NW;                  // [LRING][32]
  size_t ofs = sizeof(R) * ((size_t)NW * RING * 32 + (size_t)LRING * NW + (size_t)LRING * 32);
  ofs = (ofs + 15) & ~size_t(15);
  int* s_tlo = reinterpret_cast<int*>(smem_raw + ofs);    // [NW]
  int* s_thi = s_tlo + NW;                                // [NW]
  volatile int* s_prog = s_thi + NW;                      // [NW]
  int* s_misc = s_thi + 2 * NW;                           // [NW + 8]: lprog, tile lo/hi, flags
  volatile int* s_lprog = s_misc;
  double* s_red = reinterpret_cast<double*>(smem_raw + ofs + sizeof(int) * (4 * NW + 8));

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned gen = ld_volatile_u32(&g.ctl->gen);
  const int nj = g.nj, nk = g.nk, maxT = g.maxT;

  bool skip = false;
  if (OP != SWEEP_FACTOR && g.scal != nullptr) skip = *(volatile int*)&g.scal->done != 0;
  if (skip) return;  // converged: nothing runs, generation unchanged

  for (int pos = blockIdx.x; pos < g.ntiles; pos += gridDim.x) {
    if (ld_volatile_u32(&g.ctl->err)) break;
    const int tpos = REV ? g.ntiles - 1 - pos : pos;
    const int packed = g.tiles[tpos];
    const int J = packed & 0xffff, K = packed >> 16;
    const int j0 = J * 32, k0 = K * NW;

    // ---------------- setup: per-warp wavefront ranges ----------------
    Line L = {0, 0, 0, 0};
    int s = 0;
    if (warp < NW) {
      const int j = j0 + lane, k = k0 + warp;
      if (j < nj && k < nk) L = g.lines[(size_t)k * nj + j];
      s = j + k;
      int tl = INF_T, th = INT_MIN;
      if (L.len > 0) {
        int a = L.lo + s, b = L.lo + L.len - 1 + s;
        if (!REV) { tl = a; th = b; } else { tl = maxT - b; th = maxT - a; }
      }
      const int Tlo = __reduce_min_sync(XFP_FULL, tl);
      const int Thi = __reduce_max_sync(XFP_FULL, th);
      if (lane == 0) {
        s_tlo[warp] = Tlo;
        s_thi[warp] = Thi;
        s_prog[warp] = (Tlo == INF_T) ? INF_T : Tlo - 1;
        if (Tlo == INF_T && k < nk) {  // no cells: tell consumers in other tiles
          st_release_u64(&g.prog[(size_t)k * g.NJt + J], prog_word(gen, 0xffffffffu));
        }
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
      *s_lprog = lo == INF_T ? INF_T : lo - 1;
    }
    __syncthreads();
    const int tileLo = s_misc[1], tileHi = s_misc[2];

    double dot_acc = 0.0;
    float dot_acc_f = 0.0f;

    if (warp < NW && s_tlo[warp] != INF_T) {
      // ======================= compute warp =======================
      const int Tlo = s_tlo[warp], Thi = s_thi[warp];
      const int k = k0 + warp;
      const int zsrc = REV ? warp + 1 : warp - 1;   // producer warp in this tile (or loader)
      const int zdst = REV ? warp - 1 : warp + 1;   // consumer warp in this tile
      const bool zsrc_in = zsrc >= 0 && zsrc < NW;
      const bool zdst_in = zdst >= 0 && zdst < NW;
      const int zsrc_lo = zsrc_in ? s_tlo[zsrc] : 0, zsrc_hi = zsrc_in ? s_thi[zsrc] : -1;
      const int zdst_lo = zdst_in ? s_tlo[zdst] : 0, zdst_hi = zdst_in ? s_thi[zdst] : -1;
      const bool jb = REV ? (lane == 31) : (lane == 0);   // lane fed by the loader (j boundary)
      const bool kb = !zsrc_in;                            // warp fed by the loader (k boundary)
      unsigned long long* gprog = &g.prog[(size_t)k * g.NJt + J];
      R* myring = ring + (size_t)warp * RING * 32;
      const R* zring = zsrc_in ? ring + (size_t)zsrc * RING * 32 : nullptr;

      // Upper-neighbour lines for the factor's outgoing values.
      Line Ly = {0, 0, 0, 0}, Lz = {0, 0, 0, 0};
      if (OP == SWEEP_FACTOR) {
        const int j = j0 + lane;
        if (j + 1 < nj && k < nk) Ly = g.lines[(size_t)k * nj + j + 1];
        if (j < nj && k + 1 < nk) Lz = g.lines[(size_t)(k + 1) * nj + j];
      }

      // Values this lane produced at the previous step, per consumer direction.
      R out_x{}, out_y{};
      bool ok = true;
      for (int tau = Tlo; tau <= Thi && ok; ++tau) {
        const int i = REV ? (maxT - tau) - s : tau - s;
        const bool in = (unsigned)(i - L.lo) < (unsigned)L.len;
        const long long c = (long long)L.off + (i - L.lo);

        // ---- cell data (independent of the wavefront) ----
        VT r_c = VT(0), lx_c = VT(0), ly_c = VT(0), lz_c = VT(0);
        IT inv_c = IT(0);
        CT dg = CT(0), upx = CT(0), upy = CT(0), upz = CT(0);
        long long cyup = -1, czup = -1;
        if constexpr (OP == SWEEP_FWD) {
          if (in) { r_c = d.r[c]; lx_c = d.lx[c]; ly_c = d.ly[c]; lz_c = d.lz[c]; inv_c = d.inv[c]; }
        } else if constexpr (OP == SWEEP_BWD) {
          if (in) { r_c = d.y[c]; lx_c = d.lx[c]; ly_c = d.ly[c]; lz_c = d.lz[c]; inv_c = d.inv[c]; }
        } else {
          if (in) {
            dg = d.diag[c];
            if (i + 1 - L.lo < L.len) upx = d.ax[c + 1];
            if ((unsigned)(i - Ly.lo) < (unsigned)Ly.len) {
              cyup = (long long)Ly.off + (i - Ly.lo);
              upy = d.ay[cyup];
            }
            if ((unsigned)(i - Lz.lo) < (unsigned)Lz.len) {
              czup = (long long)Lz.off + (i - Lz.lo);
              upz = d.az[czup];
            }
          }
        }

        // ---- y-neighbour value: neighbouring lane's previous step ----
        R vy = REV ? shfl_down(out_y, 1) : shfl_up(out_y, 1);
        // ---- z-neighbour value ----
        R vz{};
        if (!kb) {
          if (tau - 1 >= zsrc_lo && tau - 1 <= zsrc_hi) {
            Spin spin;
            while (s_prog[zsrc] < tau - 1) {
              if (!spin.step(g.ctl, g.spin_limit)) { raise_timeout(g.ctl, 1); ok = false; break; }
            }
            __threadfence_block();
            vz = zring[(size_t)((tau - 1) & (RING - 1)) * 32 + lane];
          }
        }
        if (jb || kb) {
          if (tau >= tileLo) {
            Spin spin;
            while (*s_lprog < tau) {
              if (!spin.step(g.ctl, g.spin_limit)) { raise_timeout(g.ctl, 2); ok = false; break; }
            }
            __threadfence_block();
            const int slot = tau & (LRING - 1);
            if (jb) vy = jring[(size_t)slot * NW + warp];
            if (kb) vz = kring[(size_t)slot * 32 + lane];
          }
        }
        if (!__all_sync(XFP_FULL, ok)) { ok = false; break; }

        // ---- the cell itself ----
        R o_x{}, o_y{}, o_z{};
        if constexpr (OP == SWEEP_FWD) {
          // solve_lower: columns c-nn, c-ni, c-1 scatter into row c in that
          // order, then result[c] *= invdiag[c]  (pcg_solver.h:198-203)
          VT t = r_c;
          t = sub_rn(t, mul_rn(lz_c, vz));
          t = sub_rn(t, mul_rn(ly_c, vy));
          t = sub_rn(t, mul_rn(lx_c, out_x));
          VT y = in ? VT(mul_rn((IT)t, inv_c)) : VT(0);
          if (in) d.y[c] = y;
          o_x = y; o_y = y; o_z = y;
        } else if constexpr (OP == SWEEP_BWD) {
          // solve_lower_transpose_in_place: x[c] -= L(m,c) x[m] for m = c+1,
          // c+ni, c+nn in that order, then x[c] *= invdiag[c]  (:215-218).
          // Products L(m,c) x[m] arrive ready-made from the producers.
          VT t = r_c;
          t = sub_rn(t, out_x);
          t = sub_rn(t, vy);
          t = sub_rn(t, vz);
          VT z = in ? VT(mul_rn((IT)t, inv_c)) : VT(0);
          if (in) {
            d.y[c] = z;
            const VT rr = d.r[c];
            if (std::is_same<VT, float>::value && !std::is_same<IT, double>::value)
              dot_acc_f = __fadd_rn(dot_acc_f, __fmul_rn((float)z, (float)rr));
            else
              dot_acc = __dadd_rn(dot_acc, __dmul_rn((double)z, (double)rr));
          }
          o_x = mul_rn(lx_c, z);
          o_y = mul_rn(ly_c, z);
          o_z = mul_rn(lz_c, z);
        } else {
          // factor_modified_incomplete_cholesky0 for column c: updates from
          // columns c-nn, c-ni, c-1 in that order (:137-184), each
          // d -= L*L then d -= omega*L*missing; pivot safeguard (:126-131).
          IT inv = IT(0);
          if (in && dg != CT(0)) {
            CT dd = dg;
            const Pair<CT> src[3] = {vz, vy, out_x};
#pragma unroll
            for (int q = 0; q < 3; ++q) {
              dd = sub_rn(dd, mul_rn(src[q].a, src[q].a));
              dd = sub_rn(dd, mul_rn(mul_rn(d.omega, src[q].a), src[q].b));
            }
            CT iv = (dd < mul_rn(d.ratio, dg)) ? rsqrt_ref(dg) : rsqrt_ref(dd);
            inv = (IT)iv;
            // column c's entries L(m,c) = A(m,c)*invdiag[c] for m = c+1,
            // c+ni, c+nn, and for each the sum of the other two (dropped fill)
            const CT px = mul_rn(upx, iv), py = mul_rn(upy, iv), pz = mul_rn(upz, iv);
            o_x = {px, add_rn(py, pz)};
            o_y = {py, add_rn(px, pz)};
            o_z = {pz, add_rn(px, py)};
            if (upx != CT(0)) { d.flx[c + 1] = px; d.fmx[c + 1] = o_x.b; }
            if (cyup >= 0) { d.fly[cyup] = py; d.fmy[cyup] = o_y.b; }
            if (czup >= 0) { d.flz[czup] = pz; d.fmz[czup] = o_z.b; }
          }
          if (in) d.oinv[c] = inv;
        }

        // ---- hand the z-direction value to the consumer warp ----
        if (zdst_in && tau - RING + 1 >= zdst_lo && tau - RING + 1 <= zdst_hi) {
          Spin spin;
          while (s_prog[zdst] < tau - RING + 1) {
            if (!spin.step(g.ctl, g.spin_limit)) { raise_timeout(g.ctl, 3); ok = false; break; }
          }
        }
        myring[(size_t)(tau & (RING - 1)) * 32 + lane] = o_z;
        out_x = o_x;
        out_y = o_y;
        __syncwarp();
        if (lane == 0) {
          __threadfence_block();
          s_prog[warp] = tau;
        }
        if (((tau - Tlo + 1) & (PUB - 1)) == 0 && tau != Thi) {
          __syncwarp();
          if (lane == 0) {
            __threadfence();
            st_release_u64(gprog, prog_word(gen, (unsigned)(tau + 1)));
          }
        }
        if (!__all_sync(XFP_FULL, ok)) { ok = false; break; }
      }
      __syncwarp();
      if (lane == 0) {
        __threadfence();
        if (k < nk) st_release_u64(gprog, prog_word(gen, 0xffffffffu));
        s_prog[warp] = INF_T;
      }
    } else if (warp == NW && tileLo != INF_T) {
      // ======================= loader warp =======================
      // lane r < NW feeds jring row r (line k0+r); every lane l feeds kring
      // column l (line j0+l).
      const int jc = REV ? j0 + 31 : j0, js = REV ? j0 + 32 : j0 - 1;
      const int kc = REV ? k0 + NW - 1 : k0, ks = REV ? k0 + NW : k0 - 1;
      const int Jsrc = REV ? J + 1 : J - 1, Ksrc = REV ? K + 1 : K - 1;
      bool jsrc_tile = Jsrc >= 0 && Jsrc < g.NJt && g.tile_active[(size_t)K * g.NJt + Jsrc];
      bool ksrc_tile = Ksrc >= 0 && Ksrc < g.NKt && g.tile_active[(size_t)Ksrc * g.NJt + J];
      // j source (row r = lane)
      Line Ljs = {0, 0, 0, 0}, Ljc = {0, 0, 0, 0};
      int sj_c = 0, Sj_lo = INF_T, Sj_hi = INT_MIN;
      const unsigned long long* pj = nullptr;
      {
        const int kr = k0 + lane;
        if (lane < NW && kr < nk && js >= 0 && js < nj && jsrc_tile) {
          Ljs = g.lines[(size_t)kr * nj + js];
          if (jc < nj) Ljc = g.lines[(size_t)kr * nj + jc];
          pj = &g.prog[(size_t)kr * g.NJt + Jsrc];
        }
        sj_c = jc + kr;
        if (Ljs.len > 0) {
          int a = Ljs.lo + sj_c, b = Ljs.lo + Ljs.len - 1 + sj_c;
          if (!REV) { Sj_lo = a; Sj_hi = b; } else { Sj_lo = maxT - b; Sj_hi = maxT - a; }
        }
      }
      // k source (column l = lane)
      Line Lks = {0, 0, 0, 0}, Lkc = {0, 0, 0, 0};
      int sk_c = 0, Sk_lo = INF_T, Sk_hi = INT_MIN;
      const unsigned long long* pk = nullptr;
      {
        const int jl = j0 + lane;
        if (jl < nj && ks >= 0 && ks < nk && ksrc_tile) {
          Lks = g.lines[(size_t)ks * nj + jl];
          if (kc < nk) Lkc = g.lines[(size_t)kc * nj + jl];
          pk = &g.prog[(size_t)ks * g.NJt + J];
        }
        sk_c = jl + kc;
        if (Lks.len > 0) {
          int a = Lks.lo + sk_c, b = Lks.lo + Lks.len - 1 + sk_c;
          if (!REV) { Sk_lo = a; Sk_hi = b; } else { Sk_lo = maxT - b; Sk_hi = maxT - a; }
        }
      }
      Spin spin;
      int next = tileLo;
      while (next <= tileHi) {
        // how far the producers allow us to go
        long long lim = (long long)tileHi;
        if (Sj_lo <= Sj_hi) {
          unsigned v = prog_value(ld_acquire_u64(pj), gen);
          long long m = (v >= (unsigned)Sj_hi || v == 0xffffffffu) ? LLONG_MAX : max((long long)v, (long long)Sj_lo - 1);
          lim = min(lim, m);
        }
        if (Sk_lo <= Sk_hi) {
          unsigned v = prog_value(ld_acquire_u64(pk), gen);
          long long m = (v >= (unsigned)Sk_hi || v == 0xffffffffu) ? LLONG_MAX : max((long long)v, (long long)Sk_lo - 1);
          lim = min(lim, m);
        }
        // ring space: every compute warp must have finished tau - LRING
        int minp = INF_T;
        for (int w = 0; w < NW; ++w) minp = min(minp, (int)s_prog[w]);
        if (minp != INF_T) lim = min(lim, (long long)minp + LRING);
        int limit = (int)lim;
        limit = __reduce_min_sync(XFP_FULL, limit);
        if (limit < next) {
          if (!spin.step(g.ctl, g.spin_limit)) { raise_timeout(g.ctl, 4); break; }
          continue;
        }
        spin.n = 0;
        for (int tau = next; tau <= limit; ++tau) {
          const int slot = tau & (LRING - 1);
          if (lane < NW) {
            R v{};
            const int i = REV ? (maxT - tau) - sj_c : tau - sj_c;
            if (tau >= Sj_lo && tau <= Sj_hi) {
              const long long n = (long long)Ljs.off + (i - Ljs.lo);
              if constexpr (OP == SWEEP_FWD) {
                v = ld_relaxed(&d.y[n]);
              } else if constexpr (OP == SWEEP_BWD) {
                v = mul_rn(d.ly[n], ld_relaxed(&d.y[n]));
              } else {
                if ((unsigned)(i - Ljc.lo) < (unsigned)Ljc.len) {
                  const long long cc = (long long)Ljc.off + (i - Ljc.lo);
                  Pair<CT> pr;
                  pr.a = ld_relaxed(&d.fly[cc]);
                  pr.b = ld_relaxed(&d.fmy[cc]);
                  v = pr;
                }
              }
            }
            jring[(size_t)slot * NW + lane] = v;
          }
          {
            R v{};
            const int i = REV ? (maxT - tau) - sk_c : tau - sk_c;
            if (tau >= Sk_lo && tau <= Sk_hi) {
              const long long n = (long long)Lks.off + (i - Lks.lo);
              if constexpr (OP == SWEEP_FWD) {
                v = ld_relaxed(&d.y[n]);
              } else if constexpr (OP == SWEEP_BWD) {
                v = mul_rn(d.lz[n], ld_relaxed(&d.y[n]));
              } else {
                if ((unsigned)(i - Lkc.lo) < (unsigned)Lkc.len) {
                  const long long cc = (long long)Lkc.off + (i - Lkc.lo);
                  Pair<CT> pr;
                  pr.a = ld_relaxed(&d.flz[cc]);
                  pr.b = ld_relaxed(&d.fmz[cc]);
                  v = pr;
                }
              }
            }
            kring[(size_t)slot * 32 + lane] = v;
          }
        }
        __syncwarp();
        if (lane == 0) {
          __threadfence_block();
          *s_lprog = limit;
        }
        next = limit + 1;
      }
    }

    // ---------------- tile epilogue: dot partial (backward) ----------------
    if (OP == SWEEP_BWD) {
      double v = std::is_same<VT, float>::value && !std::is_same<IT, double>::value ? (double)dot_acc_f : dot_acc;
      if (std::is_same<VT, float>::value && !std::is_same<IT, double>::value) {
        float f = dot_acc_f;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) f = __fadd_rn(f, __shfl_xor_sync(XFP_FULL, f, o));
        v = f;
      } else {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = __dadd_rn(v, __shfl_xor_sync(XFP_FULL, v, o));
      }
      if (lane == 0) s_red[warp] = (warp < NW) ? v : 0.0;
    }
    __syncthreads();
    if (OP == SWEEP_BWD && threadIdx.x == 0) {
      if (std::is_same<VT, float>::value && !std::is_same<IT, double>::value) {
        float t = 0.f;
        for (int w = 0; w < NW; ++w) t = __fadd_rn(t, (float)s_red[w]);
        d.partials[tpos] = t;
      } else {
        double t = 0.0;
        for (int w = 0; w < NW; ++w) t = __dadd_rn(t, s_red[w]);
        d.partials[tpos] = t;
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
  if (s_last) {
    __threadfence();
    if (OP == SWEEP_BWD && g.scal != nullptr) {
      // deterministic reduction of the per-tile partials: rho_new = z.r
      double acc = 0.0;
      float accf = 0.f;
      const bool f32 = std::is_same<VT, float>::value && !std::is_same<IT, double>::value;
      if (threadIdx.x == 0) {
        for (int t = 0; t < g.ntiles; ++t) {
          double pv = ld_relaxed(&d.partials[t]);
          if (f32) accf = __fadd_rn(accf, (float)pv); else acc = __dadd_rn(acc, pv);
        }
        const double rho_new = f32 ? (double)accf : acc;
        PcgScalars* sc = g.scal;
        if (g.bwd_mode == 0) {
          sc->rho = rho_new;
          if (rho_new == 0.0 || rho_new != rho_new) { sc->status = -5; sc->done = 1; }
        } else {
          const double beta = f32 ? (double)__fdiv_rn((float)rho_new, (float)sc->rho) : __ddiv_rn(rho_new, sc->rho);
          sc->beta = beta;
          sc->rho = rho_new;
        }
      }
    }
    if (threadIdx.x == 0) {
      g.ctl->finished = 0;
      __threadfence();
      atomicExch(&g.ctl->gen, gen + 1);
    }
  }
}

template <int OP, typename VT, typename IT, typename CT>
static cudaError_t launch_op(const SweepGrid& g, const SweepData<VT, IT, CT>& d, int nw, int grid,
                             cudaStream_t st) {
  size_t sm = Smem<OP, VT, IT, CT>::bytes(nw);
  void* args[] = {(void*)&g, (void*)&d};
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.gridDim = dim3(grid);
  cfg.dynamicSmemBytes = sm;
  cfg.stream = st;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  (void)args;
  switch (nw) {
#define XFP_NW_CASE(N)                                                                       \
  case N: {                                                                                  \
    auto kfn = sweep_kernel<OP, VT, IT, CT, N>;                                              \
    cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);         \
    cfg.blockDim = dim3((N + 1) * 32);                                                       \
    return cudaLaunchKernelEx(&cfg, kfn, g, d);                                              \
  }
    XFP_NW_CASE(8)
    XFP_NW_CASE(16)
#undef XFP_NW_CASE
    default:
      return cudaErrorInvalidValue;
  }
}

template <int OP, typename VT, typename IT, typename CT>
static int max_grid_op(int nw) {
  size_t sm = Smem<OP, VT, IT, CT>::bytes(nw);
  int dev = 0, nsm = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  switch (nw) {
    case 8: {
      auto kfn = sweep_kernel<OP, VT, IT, CT, 8>;
      cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kfn, (8 + 1) * 32, sm);
      break;
    }
    case 16: {
      auto kfn = sweep_kernel<OP, VT, IT, CT, 16>;
      cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kfn, (16 + 1) * 32, sm);
      break;
    }
    default:
      return 0;
  }
  return per * nsm;
}

// ---- explicit entry points (declared in xfp_kernels.h) ----
#define XFP_SWEEP_INST(VT, IT, CT)                                                              \
  cudaError_t sweep_launch(int op, const SweepGrid& g, const SweepData<VT, IT, CT>& d, int nw,  \
                           int grid, cudaStream_t st) {                                         \
    switch (op) {                                                                               \
      case SWEEP_FACTOR: return launch_op<SWEEP_FACTOR, VT, IT, CT>(g, d, nw, grid, st);        \
      case SWEEP_FWD: return launch_op<SWEEP_FWD, VT, IT, CT>(g, d, nw, grid, st);              \
      default: return launch_op<SWEEP_BWD, VT, IT, CT>(g, d, nw, grid, st);                     \
    }                                                                                           \
  }                                                                                             \
  int sweep_max_grid(int op, const SweepData<VT, IT, CT>&, int nw) {                            \
    switch (op) {                                                                               \
      case SWEEP_FACTOR: return max_grid_op<SWEEP_FACTOR, VT, IT, CT>(nw);                      \
      case SWEEP_FWD: return max_grid_op<SWEEP_FWD, VT, IT, CT>(nw);                            \
      default: return max_grid_op<SWEEP_BWD, VT, IT, CT>(nw);                                   \
    }                                                                                           \
  }

XFP_SWEEP_INST(double, double, double)
XFP_SWEEP_INST(float, float, float)
XFP_SWEEP_INST(float, double, double)

}  // namespace xfp
