// Slow tendency + forward-Euler half step for FP32 state, marching along x
// over planes staged in shared memory by the bulk-copy (TMA) engine:
// k_slow_xt.  Same terms per cell as k_slow_xw / k_slow_f32 (WS5 advection
// tendency.py:965-1062, Coriolis :1220-1234, divergence damping, heating
// :1731-1732; in the production form also C2 advection, surface drag,
// sponge, Laplacian / biharmonic diffusion and Newtonian cooling,
// tendency.py:1318-1338, 1488-1514, 1548-1627, 1661-1668; the half step
// integrator.py:346-370), in single precision held to its rounding rather
// than to the reference's operation order: the WS5 derivative is formed as
// its centred sixth-order part less sgn(a) times its dissipative part, two
// fields at a time with the paired FP32 instructions (u with v, theta' with
// w).
//
// A CTA owns R rows (y) by all NZ levels of one x-segment.  Thread t is cell
// (row t / (NZ / KC), level t % (NZ / KC)), and with KC = 2 also that level
// + NZ / 2: the CTA's rows j0..j0+R-1 are consecutive in memory for a fixed
// x, so one x-plane of the CTA with its y-halo (rows j0-3..j0+R+2, periodic)
// is one or two contiguous runs per field.
//
// * The planes arrive by cp.async.bulk, one instruction per run, issued by
//   one thread, completion counted on an mbarrier per ring slot.  w's rows of
//   NZ + 1 floats do not start on 16 bytes: its run is copied as the 16-byte
//   aligned range around it and read from `lead` floats into the slot.  With
//   ny % 4 == 0 a run that wraps in y ends (row ny - 1) and restarts (row 0)
//   on 16 bytes, so its second piece lands, aligned, right after the first;
//   and a run that does not wrap ends at least one row before the array's
//   end, so its aligned range stays inside the array.
// * A ring of 7 plane slots: at step x = i the CTA reads plane i (y- and
//   z-neighbours) and plane i + 3 (the x-window's new column), while planes
//   up to i + 6 are in flight: the copies are issued three steps ahead.
// * Each thread keeps 7-point x-windows of the four fields in registers (and,
//   for the biharmonic, 3-point windows of the inner Laplacians).
//   Steps run in groups of 7 with the group unrolled, so the window's
//   rotation and the ring's slot indices are compile-time: every shared-
//   memory read is a register base plus an immediate (NZ is a template
//   parameter for the same reason).
// * No CTA-wide barrier per step: each slot has a "full" mbarrier (the
//   copies landed) and an "empty" one, on which every warp arrives once it has
//   read the slot's plane for the last time.  Only the thread that issues the
//   next copies into a slot waits for it to be empty, so the warps of a CTA
//   run up to three steps apart.  The issuing passes from warp to warp, step
//   by step, so that no warp carries it all and lags the others.
// * Every wait on an mbarrier is bounded.  A wait that runs out (it cannot
//   by construction: every copy is in bounds) sets stall[0] = 1, waits for
//   the CTA's copies in flight with the same bound, and returns.
#pragma once
#include "kernels.cuh"

namespace ob {

__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long* b, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(b)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* b, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(b)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_test(unsigned long long* b, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_addr(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void mbar_arrive(unsigned long long* b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(b)) : "memory");
}
// Bounded wait for the phase of parity `parity`: false when it did not
// complete within 2^22 tests (each test suspends the thread for up to a
// hardware time limit while the phase is incomplete: about a second or more
// in all).
__device__ __forceinline__ bool mbar_wait(unsigned long long* b, unsigned parity) {
  for (int it = 0; it < (1 << 22); ++it)
    if (mbar_test(b, parity)) return true;
  return false;
}
// orders this thread's earlier shared-memory accesses before its later
// bulk copies (the slot being refilled was read by the generic proxy)
__device__ __forceinline__ void fence_proxy() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes,
                                          unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      ::"r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// 60 d times the WS5 upwind derivative of two fields at once (q[r]: the
// values at offsets r - 3; nsg = -sgn(a) per field, sgn(0) = +1).  The
// stencils of tendency.py:940-959 are C6 - D (a >= 0) and C6 + D (a < 0) with
// C6 = 45 (q1 - q-1) - 9 (q2 - q-2) + (q3 - q-3) and
// D = (q3 + q-3) - 6 (q2 + q-2) + 15 (q1 + q-1) - 20 q0.
__device__ __forceinline__ float2 ws5_pair(const float2 (&q)[7], float2 nsg) {
  const float2 m1 = make_float2(-1.0f, -1.0f);
  const float2 d1 = __ffma2_rn(q[2], m1, q[4]);
  const float2 d2 = __ffma2_rn(q[1], m1, q[5]);
  const float2 d3 = __ffma2_rn(q[0], m1, q[6]);
  const float2 s1 = __fadd2_rn(q[2], q[4]);
  const float2 s2 = __fadd2_rn(q[1], q[5]);
  const float2 s3 = __fadd2_rn(q[0], q[6]);
  float2 c = __ffma2_rn(make_float2(45.0f, 45.0f), d1, d3);
  c = __ffma2_rn(make_float2(-9.0f, -9.0f), d2, c);
  float2 d = __ffma2_rn(make_float2(15.0f, 15.0f), s1, s3);
  d = __ffma2_rn(make_float2(-6.0f, -6.0f), s2, d);
  d = __ffma2_rn(make_float2(-20.0f, -20.0f), q[3], d);
  return __ffma2_rn(nsg, d, c);
}
__device__ __forceinline__ float nsgn(float a) { return a >= 0.0f ? -1.0f : 1.0f; }
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
// Shared-memory plan of k_slow_xt (floats unless stated); KC cells (levels
// k and k + NZ / 2 when KC = 2) per thread; PROD: the production form, whose
// planes also carry the biharmonic's inner Laplacians of u and v.
template <int NZ, int R, int KC = 1, bool PROD = false>
struct SlowXt {
  static constexpr int NT = R * NZ / KC;            // threads
  static constexpr int RH = R + 6;                  // plane rows j0-3 .. j0+R+2
  static constexpr int NW = NZ + 1;                 // w levels
  static constexpr int FS = RH * NZ;                // one u / v / theta' plane
  static constexpr int WS = (RH * NW + 8 + 3) / 4 * 4;  // the w run with its 16-byte margins
  static constexpr int NF = PROD ? 5 : 3;           // full-level fields per plane
  static constexpr int SLOT = NF * FS + WS;
  static constexpr int NSLOT = 7;
  static constexpr size_t smem = (size_t)NSLOT * SLOT * 4 + 2 * NSLOT * 8;  // + mbarriers
  // CTAs per SM: what the shared memory allows (228 KB per SM, 1 KB reserved
  // per CTA), at most 2048 threads, and at least 72 registers a thread (136
  // with two cells per thread, 104 in the production form)
  static constexpr int by_smem = (int)(233472 / (smem + 1024));
  static constexpr int by_regs = 65536 / ((KC == 2 ? 136 : PROD ? 104 : 72) * NT);
  static constexpr int by_thr = 2048 / NT;
  static constexpr int per_sm_min = by_smem < by_regs ? by_smem : by_regs;
  static constexpr int per_sm_cap = per_sm_min < by_thr ? per_sm_min : by_thr;
  static constexpr int per_sm = per_sm_cap < 1 ? 1 : per_sm_cap;
  static_assert(NZ % 4 == 0, "u, v, theta' rows must be whole 16-byte runs");
  // (and ny % 4 == 0, checked by the host, for w's runs)
  static_assert(NT % 32 == 0 && NT <= 1024, "whole warps, one CTA");
  static_assert(KC == 1 || (KC == 2 && NZ % 2 == 0), "one or two cells per thread");
};

// grid = (ny / R, ceil(nx / seg)), block = R * NZ / KC; seg is a multiple of 7.
// OUTMODE 0: out = in + dts * tendency (the half step); 1: out = tendency.
// KC = 2: each thread computes levels k and k + NZ / 2 of its row (twice the
// work between waits, so that a step outlasts more of the copies' latency).
// PROD: the production components as well (k_slow_f32<OUTMODE, true>):
// surface drag, sponge, Laplacian or biharmonic diffusion, Newtonian cooling,
// and centred (C2) or WS5 advection chosen at run time.
// stall: one double (the plan's OB_DIAG_STALL slot).
template <int OUTMODE, int NZ, int R, int KC, bool PROD = false>
__global__ void __launch_bounds__(R * NZ / KC, SlowXt<NZ, R, KC, PROD>::per_sm) k_slow_xt(
    GridK g, SlowK s, int mask, double dts_d, int seg, const float* __restrict__ u,
    const float* __restrict__ v, const float* __restrict__ w, const float* __restrict__ th,
    const float* __restrict__ dmp_u, const float* __restrict__ dmp_v, float* __restrict__ uo,
    float* __restrict__ vo, float* __restrict__ wo, float* __restrict__ tho,
    double* __restrict__ stall) {
  using C = SlowXt<NZ, R, KC, PROD>;
  static_assert(!PROD || KC == 1, "the production form has one cell per thread");
  constexpr int NZC = NZ / KC;  // levels between a thread's cells
  constexpr int NT = C::NT, RH = C::RH, NW = C::NW, FS = C::FS, SLOT = C::SLOT, NF = C::NF;
  extern __shared__ __align__(16) float smx[];
  unsigned long long* bar = reinterpret_cast<unsigned long long*>(smx + C::NSLOT * SLOT);
  const int nx = g.nx, ny = g.ny;
  const int t = threadIdx.x;
  const int row = t / NZC, kb = t - row * NZC;
  const int j0 = blockIdx.x * R, j = j0 + row;
  const int i0 = blockIdx.y * seg;
  const int len = min(seg, nx - i0);
  const int qmax = len + 5;  // last plane (ring index q = x - i0 + 3) the segment reads
  const bool cor = (mask & 2) && s.cor;
  const bool dmp = (mask & 4) && s.damp;
  const bool heat = (mask & 8) && s.heat;
  // production components (k_slow_f32<_, true>)
  const bool ws5 = !PROD || s.adv == 2;
  const bool drg = PROD && (mask & kTendDrag) && s.drag;
  const bool spg = PROD && (mask & kTendSponge) && s.sponge;
  const int dif = (PROD && (mask & kTendDiffusion)) ? s.diff : 0;
  const bool cool = PROD && (mask & kTendCooling) && s.cool;
  const float* lap_u = static_cast<const float*>(s.lap_u);
  const float* lap_v = static_cast<const float*>(s.lap_v);
  const bool lapf = PROD && dif == 2;  // the inner Laplacians ride in the planes
  const float dts = (float)dts_d;
  const float inv60dx = (float)s.inv60dx, inv60dy = (float)s.inv60dy;
  const float inv2dz = (float)s.inv2dz, invdz = (float)s.invdz;
  const float f = cor ? (float)((s.cor == 2) ? s.fy[j] : s.f0) : 0.0f;
  const float u_env = (float)s.u_env, v_env = (float)s.v_env;
  float dth0k[KC], heatz[KC];
#pragma unroll
  for (int c = 0; c < KC; ++c) {
    dth0k[c] = (float)s.dth0[kb + c * NZC];
    heatz[c] = heat ? (float)s.heat_z[kb + c * NZC] : 0.0f;
  }

  // the y-halo'd row block [j0 - 3, j0 + R + 3) mod ny as one or two runs
  // (ny >= R + 6): na rows from global row ga, then nb rows from row 0, which
  // land at plane row na
  int ga = j0 - 3, na = RH, nb = 0;
  if (ga < 0) {
    na = -ga;
    ga += ny;
    nb = RH - na;
  } else if (ga + RH > ny) {
    na = ny - ga;
    nb = RH - na;
  }
  // x-plane of ring plane q (x = i0 - 3 + q, periodic)
  auto plane_x = [&](int q) {
    int px = i0 - 3 + q;
    px += (px < 0) ? nx : 0;
    px -= (px >= nx) ? nx : 0;
    return px;
  };
  // where w's run starts in its slot: its first float's offset mod 4 (the
  // 16-byte aligned copy starts that many floats before it).  The run of
  // plane px starts at float (px ny + ga) NW, and ny % 4 == 0, so the lead is
  // (ga NW) mod 4 for every plane of the CTA.
  const int lead = (ga * NW) & 3;
  unsigned long long* full = bar;
  unsigned long long* empty = bar + C::NSLOT;
  // w's run of plane px: floats [wa, we) and, wrapped, [w2, w2e); piece 1
  // ends at the plane's end (wrapped: aligned there) or at the run's aligned end
  struct WRun {
    size_t wa, we, w2, w2e;
  };
  auto w_run = [&](size_t cb) {
    const size_t w0 = (cb + ga) * NW;
    const size_t w2 = cb * NW;
    return WRun{w0 & ~(size_t)3, nb ? (cb + ny) * NW : (w0 + RH * NW + 3) & ~(size_t)3, w2,
                (w2 + nb * NW + 3) & ~(size_t)3};
  };
  // issue the copies of ring plane q into slot `slot` (free: the caller
  // waited); one thread
  auto issue = [&](int q, int slot) {
    const int px = plane_x(q);
    float* sl = smx + slot * SLOT;
    const size_t cb = (size_t)px * ny;
    const WRun r = w_run(cb);
    const size_t wa = r.wa, we = r.we, w2 = r.w2, w2e = r.w2e;
    const unsigned wbytes = (unsigned)((we - wa) + (nb ? w2e - w2 : 0)) * 4u;
    fence_proxy();
    const int nfc = lapf ? 5 : 3;  // full-level fields copied
    mbar_expect_tx(&full[slot], (unsigned)nfc * FS * 4u + wbytes);
    const float* src[5] = {u, v, th, lap_u, lap_v};
#pragma unroll
    for (int fi = 0; fi < NF; ++fi) {
      if (fi >= nfc) break;
      bulk_load(sl + fi * FS, src[fi] + (cb + ga) * NZ, (unsigned)(na * NZ * 4), &full[slot]);
      if (nb) bulk_load(sl + fi * FS + na * NZ, src[fi] + cb * NZ, (unsigned)(nb * NZ * 4),
                        &full[slot]);
    }
    float* sw = sl + NF * FS;
    bulk_load(sw, w + wa, (unsigned)(we - wa) * 4u, &full[slot]);
    if (nb) bulk_load(sw + (we - wa), w + w2, (unsigned)(w2e - w2) * 4u, &full[slot]);
  };
  const int lane = t & 31, warp = t >> 5;
  constexpr int NWARP = NT / 32;
  // this warp has read plane q for the last time
  auto release = [&](int q) {
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[q % 7]);
  };

  if (t == 0) {
#pragma unroll
    for (int sl = 0; sl < C::NSLOT; ++sl) {
      mbar_init(&full[sl], 1);
      mbar_init(&empty[sl], NWARP);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  int qlast = min(6, qmax);  // the last plane issued
  // planes q = 0..6 (x = i0-3 .. i0+3) into the fresh slots
  if (t == 0)
    for (int q = 0; q <= qlast; ++q) issue(q, q);
  // the windows' first six columns: planes 0..5
  bool ok = true;
#pragma unroll
  for (int q = 0; q < 6; ++q) ok = ok && mbar_wait(&full[q], 0);
  const int pc = (row + 3) * NZ + kb;  // own first cell in a u / v / theta' plane
  const int pw = (row + 3) * NW + kb;  // its level in the w plane (from the lead)
  // x-windows per cell, plane q at index q % 7: (u, v) and (theta', w) pairs
  float2 quv[KC][7], qtw[KC][7];
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    const float* P = smx + q * SLOT;
#pragma unroll
    for (int c = 0; c < KC; ++c) {
      quv[c][q] = f2(P[pc + c * NZC], P[FS + pc + c * NZC]);
      qtw[c][q] = f2(P[2 * FS + pc + c * NZC], P[NF * FS + lead + pw + c * NZC]);
    }
  }
  // the inner Laplacians of u, v at x-1 and x (planes 2 and 3; x+1 comes
  // from the ring each step): the biharmonic's x-neighbours
  float2 lw[3] = {f2(0.0f, 0.0f), f2(0.0f, 0.0f), f2(0.0f, 0.0f)};
  if (lapf) {
    lw[0] = f2(smx[2 * SLOT + 3 * FS + pc], smx[2 * SLOT + 4 * FS + pc]);
    lw[1] = f2(smx[3 * SLOT + 3 * FS + pc], smx[3 * SLOT + 4 * FS + pc]);
  }
  // per-level constants of the production components (one cell per thread)
  const float spa = spg ? (float)s.sp_a[kb] : 0.0f, spah = spg ? (float)s.sp_ah[kb] : 0.0f;
  const float spal = spg ? (float)s.sp_ah[NZ] : 0.0f;  // the lid's
  const float dragk = drg ? (float)(s.drag_cd / s.drag_dz * s.drag_w[kb]) : 0.0f;
  const float dnu = (float)s.diff_nu, rdx2 = (float)(1.0 / s.diff_dx2),
              rdy2 = (float)(1.0 / s.diff_dy2);
  // planes 0..2 are read only here; 7 and 8 refill the slots of 0 and 1
#pragma unroll
  for (int q = 0; q < 3; ++q) release(q);
  for (int q = 7; q < 9; ++q)
    if (q <= qmax) {
      if (t == 0) {
        ok = ok && mbar_wait(&empty[q - 7], 0);
        if (ok) issue(q, q - 7);
      }
      qlast = q;
    }
  // z-neighbours: one-sided differences at the bottom and top levels
  // (tendency.py:1000-1011), as offsets fixed for the thread
  int zm[KC], zp[KC];
  float fz[KC];
#pragma unroll
  for (int c = 0; c < KC; ++c) {
    const int k = kb + c * NZC;
    zm[c] = (k > 0) ? -1 : 0;
    zp[c] = (k < NZ - 1) ? 1 : 0;
    fz[c] = (k == 0 || k == NZ - 1) ? invdz : inv2dz;
  }
  // 32-bit element offsets (the host admits grids of fewer than 2^31 w
  // values)
  const unsigned plane_cells = (unsigned)ny * NZ, plane_w = (unsigned)ny * NW;
  unsigned o = ((unsigned)i0 * ny + j) * NZ + kb;
  unsigned ow = ((unsigned)i0 * ny + j) * NW + kb;
  unsigned col = (unsigned)i0 * ny + j;
  const int pwx = pw + lead;  // this cell's w level in every plane

  int iw = 0;  // the warp that issues this step's copies (lane 0)
  // group gi = s0 / 7 of steps; gp = gi mod 2.  Plane q is the (q / 7)-th
  // fill of slot q % 7, so the wait for plane st + 6 (st = s0 + uu) is on
  // phase parity (gi + (uu >= 1)) mod 2 and the release of plane st + 2 on
  // (gi + (uu >= 5)) mod 2: compile-time offsets, no division per step.
  for (int s0 = 0, gp = 0; ok && s0 < len; s0 += 7, gp ^= 1) {
#pragma unroll
    for (int uu = 0; uu < 7; ++uu) {
      const int st = s0 + uu;  // step: x = i0 + st
      if (ok && st < len) {
        // plane st + 6 (the window's new column) must have landed
        ok = mbar_wait(&full[(uu + 6) % 7], (unsigned)((gp + (uu >= 1 ? 1 : 0)) & 1));
        // refill the slot of plane st + 2 (last read in the previous step)
        // with plane st + 9, once every warp has released it
        if (st + 9 <= qmax) {
          if (warp == iw && lane == 0 && ok) {
            ok = mbar_wait(&empty[(uu + 2) % 7], (unsigned)((gp + (uu >= 5 ? 1 : 0)) & 1));
            if (ok) issue(st + 9, (uu + 2) % 7);
          }
          qlast = st + 9;
        }
        iw = (iw + 1 == NWARP) ? 0 : iw + 1;
        if (!ok) break;

        const float* P = smx + ((uu + 3) % 7) * SLOT;  // plane x
        const float* N = smx + ((uu + 6) % 7) * SLOT;  // plane x + 3
        const float* Pu = P;
        const float* Pv = P + FS;
        const float* Pt = P + 2 * FS;
        const float* Pw = P + NF * FS;
        const float hr = heat ? (float)s.heat_r[col] : 0.0f;
#pragma unroll
        for (int c = 0; c < KC; ++c) {
          const int cp = pc + c * NZC, cw = pwx + c * NZC;
          quv[c][(uu + 6) % 7] = f2(N[cp], N[FS + cp]);
          qtw[c][(uu + 6) % 7] = f2(N[2 * FS + cp], N[NF * FS + pwx + c * NZC]);
          // the windows in x order: x-3 .. x+3
          float2 wuv[7], wtw[7];
#pragma unroll
          for (int r = 0; r < 7; ++r) {
            wuv[r] = quv[c][(uu + r) % 7];
            wtw[r] = qtw[c][(uu + r) % 7];
          }
          const float uc = wuv[3].x, vc = wuv[3].y, wk = wtw[3].y;
          // y-columns of this plane, rows -3..+3
          float2 cuv[7], ctw[7];
#pragma unroll
          for (int r = 0; r < 7; ++r) {
            if (r == 3) continue;  // the centre is the window's
            cuv[r] = f2(Pu[cp + (r - 3) * NZ], Pv[cp + (r - 3) * NZ]);
            ctw[r] = f2(Pt[cp + (r - 3) * NZ], Pw[cw + (r - 3) * NW]);
          }
          cuv[3] = wuv[3];
          ctw[3] = wtw[3];
          const float um = Pu[cp + zm[c]], vm = Pv[cp + zm[c]], tm = Pt[cp + zm[c]];
          const float wp1 = Pw[cw + 1], wm1 = Pw[cw - 1];
          const float wc = 0.5f * (wk + wp1);
          const float uh = 0.5f * (um + uc), vh = 0.5f * (vm + vc);
          const float2 m1 = f2(-1.0f, -1.0f);
          // vertical differences: (u, v) one-sided at the bottom and top
          // levels, (theta' + its base gradient, w on half levels)
          const float2 cuvz = __fmul2_rn(
              __ffma2_rn(f2(um, vm), m1, f2(Pu[cp + zp[c]], Pv[cp + zp[c]])), f2(fz[c], fz[c]));
          const float2 ctwz = __ffma2_rn(__ffma2_rn(f2(tm, wm1), m1, f2(Pt[cp + zp[c]], wp1)),
                                         f2(fz[c], inv2dz), f2(dth0k[c], 0.0f));
          // x and y differences: WS5 (times 60 d) or, in the production form
          // with centred advection, C2 (times 2 d)
          float2 Xuv, Yuv, Xtw, Ytw;
          if (ws5) {
            Xuv = ws5_pair(wuv, f2(nsgn(uc), nsgn(uc)));
            Yuv = ws5_pair(cuv, f2(nsgn(vc), nsgn(vc)));
            Xtw = ws5_pair(wtw, f2(nsgn(uc), nsgn(uh)));
            Ytw = ws5_pair(ctw, f2(nsgn(vc), nsgn(vh)));
          } else {
            Xuv = __ffma2_rn(wuv[2], m1, wuv[4]);
            Yuv = __ffma2_rn(cuv[2], m1, cuv[4]);
            Xtw = __ffma2_rn(wtw[2], m1, wtw[4]);
            Ytw = __ffma2_rn(ctw[2], m1, ctw[4]);
          }
          const float sx = ws5 ? inv60dx : (float)s.inv2dx;
          const float sy = ws5 ? inv60dy : (float)s.inv2dy;
          // tendencies -(u d/dx + v d/dy + w d/dz): (u, v) advected by
          // (uc, vc, wc), (theta', w) by (uc, vc, wc) and (uh, vh, wk)
          const float nux = -uc * sx, nvy = -vc * sy;
          float2 tuv = __fmul2_rn(f2(nux, nux), Xuv);
          tuv = __ffma2_rn(f2(nvy, nvy), Yuv, tuv);
          tuv = __ffma2_rn(f2(-wc, -wc), cuvz, tuv);
          float2 ttw = __fmul2_rn(f2(nux, -uh * sx), Xtw);
          ttw = __ffma2_rn(f2(nvy, -vh * sy), Ytw, ttw);
          ttw = __ffma2_rn(f2(-wc, -wk), ctwz, ttw);
          const unsigned oc = o + c * NZC, owc = ow + c * NZC;
          if (cor) tuv = __ffma2_rn(f2(f, -f), f2(vc - v_env, uc - u_env), tuv);
          if constexpr (PROD) {
            if (drg) {  // the surface wind of the column drives the drag
              const float up0 = Pu[pc - kb] - (float)s.drag_u_env;
              const float vp0 = Pv[pc - kb] - (float)s.drag_v_env;
              const float al = dragk * sqrtf(up0 * up0 + vp0 * vp0);
              tuv = __ffma2_rn(f2(-al, -al),
                               f2(uc - (float)s.drag_u_env, vc - (float)s.drag_v_env), tuv);
            }
            if (spg) {
              tuv = __ffma2_rn(f2(-spa, -spa),
                               f2(uc - (float)s.sp_u_env, vc - (float)s.sp_v_env), tuv);
              ttw.x = ttw.x + (-spa) * wtw[3].x;
            }
            if (dif == 1) {  // 5-point Laplacian of u, v
              const float2 lx = __ffma2_rn(f2(-2.0f, -2.0f), wuv[3], __fadd2_rn(wuv[2], wuv[4]));
              const float2 ly = __ffma2_rn(f2(-2.0f, -2.0f), wuv[3], __fadd2_rn(cuv[2], cuv[4]));
              tuv = __ffma2_rn(f2(dnu, dnu),
                               __ffma2_rn(lx, f2(rdx2, rdx2), __fmul2_rn(ly, f2(rdy2, rdy2))),
                               tuv);
            } else if (dif == 2) {  // 5-point Laplacian of the inner Laplacians
              lw[2] = f2(smx[((uu + 4) % 7) * SLOT + 3 * FS + pc],
                         smx[((uu + 4) % 7) * SLOT + 4 * FS + pc]);
              const float2 yl = f2(P[3 * FS + pc - NZ], P[4 * FS + pc - NZ]);
              const float2 yu = f2(P[3 * FS + pc + NZ], P[4 * FS + pc + NZ]);
              const float2 lx = __ffma2_rn(f2(-2.0f, -2.0f), lw[1], __fadd2_rn(lw[0], lw[2]));
              const float2 ly = __ffma2_rn(f2(-2.0f, -2.0f), lw[1], __fadd2_rn(yl, yu));
              tuv = __ffma2_rn(f2(-dnu, -dnu),
                               __ffma2_rn(lx, f2(rdx2, rdx2), __fmul2_rn(ly, f2(rdy2, rdy2))),
                               tuv);
              lw[0] = lw[1];
              lw[1] = lw[2];
            }
            if (cool) ttw.x = ttw.x + (-(float)s.cool_alpha) * wtw[3].x;
          }
          if (dmp) tuv = __fadd2_rn(tuv, f2(dmp_u[oc], dmp_v[oc]));
          if (heat) ttw.x = ttw.x + hr * heatz[c];
          if (kb + c * NZC == 0) ttw.y = 0.0f;  // w: no advection at the surface
          if (PROD && spg) ttw.y = ttw.y + (-spah) * wk;  // w's sponge, every half level
          if (OUTMODE == 0) {
            tuv = __ffma2_rn(f2(dts, dts), tuv, wuv[3]);
            ttw = __ffma2_rn(f2(dts, dts), ttw, wtw[3]);
          }
          uo[oc] = tuv.x;
          vo[oc] = tuv.y;
          tho[oc] = ttw.x;
          wo[owc] = ttw.y;
          if (kb + c * NZC == NZ - 1) {  // the lid, level nz: the sponge only
            const float tl = (PROD && spg) ? (-spal) * wp1 : 0.0f;
            wo[owc + 1] = OUTMODE == 0 ? wp1 + dts * tl : tl;
          }
        }
        release(st + 3);  // plane x: read for the last time
        o += plane_cells;
        ow += plane_w;
        col += ny;
      }
    }
  }
  if (!ok) {
    // a wait ran out: flag it, and wait with the same bound for the copies
    // into every slot whose latest plane was issued
    *stall = 1.0;
    for (int q = max(0, qlast - 6); q <= qlast; ++q) mbar_wait(&full[q % 7], (q / 7) & 1);
  }
}

}  // namespace ob
