// Register-resident x-pencil kernels for nx = 512 (M = 256), single precision.
//
// The M = 256 point FFT of a column is spread over a 16-lane group (two
// groups per warp): M = 16 x 16, n = n1 + 16 n2, k = 16 k1 + k2.
//   pass 1: lane t = n1 holds z[t + 16 n2] (n2 = 0..15), takes the 16-point
//           DFT over n2 in registers and multiplies by W_256^(t k2);
//   exchange: through a 16 x 17 padded shared-memory block of its own group
//           (only __syncwarp: the group's lanes are one half of a warp);
//   pass 2: lane t = k2 holds the n1 values and takes the 16-point DFT over
//           n1, leaving Z[16 k1 + t] in its registers.
// Against the shared-memory Stockham kernels (pencil.cuh) a column's data
// crosses shared memory once in the FFT instead of three times plus a
// pre/post-processing pass: the real-to-complex pack is fused into pass 1's
// gather, the complex-to-real pre-process likewise, and the R2C split is
// formed from partner lanes with warp shuffles.  Same arithmetic per element
// as k_fx2 / k_ix2 otherwise, in single precision.
// Layouts: state (x, y, z) with z contiguous, w on nz + 1 levels; spectra
// [kx][y][z] with kx in [0, nx/2].  Element indices are 32-bit.
#pragma once
#include "pencil.cuh"

namespace ob {

constexpr int kXrM = 256;  // packed complex FFT length (nx = 512)
constexpr int kXrN = 512;
constexpr int kXrEx = 16 * 17;  // exchange block of one group (complex)

// Row stride (floats) of the level-major tiles: nx plus a pad that puts the
// rows of one warp's z-run on distinct banks.
template <int ZC>
__host__ __device__ constexpr int xr_stride() { return kXrN + 32 / ZC; }

// Pass 1 and pass 2 of a group's 256-point FFT.  tw2[16 k2 + t] = W_256^(t k2)
// (forward sign; conjugated for INV).  On entry a[n2] = z[t + 16 n2]; on exit
// a[k1] = Z[16 k1 + t].  ex: the group's exchange block.  The caller makes
// sure ex is free (a CTA barrier when it aliases other data).
template <class T, bool INV>
__device__ __forceinline__ void xr_pass1(cplx<T> (&a)[16], int t,
                                         const cplx<T>* __restrict__ tw2) {
  dft16<T, INV>(a);
#pragma unroll
  for (int k2 = 1; k2 < 16; ++k2) {
    cplx<T> w = tw2[16 * k2 + t];
    if (INV) w.y = -w.y;
    a[k2] = mul(a[k2], w);
  }
}
template <class T, bool INV>
__device__ __forceinline__ void xr_pass2(cplx<T> (&a)[16], int t, cplx<T>* ex) {
#pragma unroll
  for (int k2 = 0; k2 < 16; ++k2) ex[k2 * 17 + t] = a[k2];
  __syncwarp();
#pragma unroll
  for (int n1 = 0; n1 < 16; ++n1) a[n1] = ex[t * 17 + n1];
  dft16<T, INV>(a);
}

// ---- forward: k_fx3 ----------------------------------------------------------
// Shared memory (bytes): twiddles, then one region that holds in turn the
// level-major state tiles (FP32), the groups' exchange blocks and the spectra
// (arithmetic type T).
template <class T, bool STAGE, int ZC>
__host__ __device__ constexpr size_t fx3_smem() {
  constexpr int B = 3 * ZC, S = xr_stride<ZC>();
  constexpr size_t raw = (size_t)(2 * ZC + (STAGE ? 2 : 1) * (ZC + 1)) * S * 4;
  constexpr size_t ex = (size_t)B * kXrEx * sizeof(cplx<T>);
  constexpr size_t xs = (size_t)(kXrM + 1) * (B + 1) * sizeof(cplx<T>);
  constexpr size_t r1 = raw > ex ? raw : ex;
  return 2 * kXrM * sizeof(cplx<T>) + (r1 > xs ? r1 : xs);
}
template <class T, int ZC>
constexpr int fx3_min_blocks() { return sizeof(T) == 8 ? 2 : (ZC >= 8 ? 2 : 4); }

// Forward x-pencil kernel (k_fx2 semantics, FP32 state, nx = 512):
// rho-weighting, vertical flux divergence (STAGE: of w + sdt b_half, b_half
// the field bh), R2C along x; X0 = i kx' FFTx(rho u) + FFTx(vd),
// X1 = FFTx(rho v).  T = float: the single-precision projection; T = double:
// the FP64 residual transform of the defect correction, with k_fx2's
// operation order in the pack.  3 ZC columns (u, v, d at ZC levels), one
// 16-lane group each.  grid = (ceil(nz/ZC), ny), 48 ZC threads.
// FIELDS (FP32, no stage): the plain half-spectra X0 = FFTx(u), X1 = FFTx(v),
// the Nyquist bin included (what k_fx FX_FIELDS writes; the Helmholtz
// damper's forward x transform); w is not read and the d columns stay zero.
template <class T, bool STAGE, int ZC, bool FIELDS = false>
__global__ void __launch_bounds__(48 * ZC, fx3_min_blocks<T, ZC>()) k_fx3(
    GridK g, const float* __restrict__ u, const float* __restrict__ v,
    const float* __restrict__ w, const float* __restrict__ bh, double sdt,
    const double* __restrict__ rho, const double* __restrict__ rhoh,
    const double* __restrict__ kxd, const cplx<T>* __restrict__ twx,
    cplx<T>* __restrict__ X0, cplx<T>* __restrict__ X1) {
  static_assert(ZC == 2 || ZC == 4 || ZC == 8, "whole warps of 16-lane groups");
  static_assert(sizeof(T) == 4 || !STAGE, "the FP64 form is the residual transform");
  static_assert(!FIELDS || (sizeof(T) == 4 && !STAGE), "the field form is FP32 without a stage");
  constexpr int B = 3 * ZC, NT = 16 * B, M = kXrM, N = kXrN, S = xr_stride<ZC>(), BP = B + 1;
  extern __shared__ __align__(16) unsigned char smem_dyn[];
  cplx<T>* tw2 = reinterpret_cast<cplx<T>*>(smem_dyn);  // [16 k2 + t] = W_256^(t k2)
  cplx<T>* twN = tw2 + M;                               // W_512^k, k < 256
  float* U = reinterpret_cast<float*>(twN + M);         // [ZC][S]
  float* V = U + ZC * S;                                        // [ZC][S]
  float* W = V + ZC * S;                                        // [ZC + 1][S]
  float* BH = W + (ZC + 1) * S;                                 // [ZC + 1][S] (STAGE)
  cplx<T>* ex = reinterpret_cast<cplx<T>*>(U);                  // B x 16 x 17, after the gather
  cplx<T>* XS = reinterpret_cast<cplx<T>*>(U);                  // (M + 1) x BP, after the exchange
  const int ny = g.ny, nz = g.nz;
  const int y = blockIdx.y;
  const int z0 = blockIdx.x * ZC;
  const int tid = threadIdx.x;

  // 1. every tile in flight at once; consecutive threads take consecutive
  //    levels of a row (whole z-runs per warp), rows stored level-major
  for (int e = tid; e < N * ZC; e += NT) {
    const int x = e / ZC, j = e - x * ZC;
    const int z = z0 + j;
    const bool ok = z < nz;
    const int gi = (x * ny + y) * nz + (ok ? z : 0);
    copy_or_zero(&U[j * S + x], u + gi, ok);
    copy_or_zero(&V[j * S + x], v + gi, ok);
  }
  if constexpr (!FIELDS)
    for (int e = tid; e < N * (ZC + 1); e += NT) {
      const int x = e / (ZC + 1), j = e - x * (ZC + 1);
      const int z = z0 + j;  // half levels z0 .. z0+ZC
      const bool ok = z <= nz;
      const int gi = (x * ny + y) * (nz + 1) + (ok ? z : 0);
      copy_or_zero(&W[j * S + x], w + gi, ok);
      if (STAGE) copy_or_zero(&BH[j * S + x], bh + gi, ok);
    }
  cp_commit();
  for (int i = tid; i < M; i += NT) {
    tw2[i] = twx[2 * ((i & 15) * (i >> 4))];  // W_256^m = W_512^(2m)
    twN[i] = twx[i];
  }
  cp_wait<0>();
  __syncthreads();

  // 2. gather with the pack fused: column grp = (field f, level j); lane t
  //    takes z[t + 16 q] = f(2n) + i f(2n+1), n = t + 16 q
  const int grp = tid >> 4, t = tid & 15;
  const int f = grp / ZC, j = grp - f * ZC;
  const int zj = z0 + j;
  const bool ok = zj < nz;
  cplx<T> a[16];
  if (f < 2) {
    const T r = FIELDS ? (T)1 : (ok ? (T)rho[zj] : (T)0);
    const float* R = (f == 0 ? U : V) + j * S + 2 * t;
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      const float2 p = *reinterpret_cast<const float2*>(R + 32 * q);
      a[q] = mk<T>(r * (T)p.x, r * (T)p.y);
    }
  } else if constexpr (sizeof(T) == 8) {
    // the reference's operation order, rounded step by step (as k_fx2)
    const double rl = ok ? rhoh[zj] : 0.0, ru = ok ? rhoh[zj + 1] : 0.0;
    const double dz = g.dz;
    const float* Wl = W + j * S + 2 * t;
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      const float2 wl = *reinterpret_cast<const float2*>(Wl + 32 * q);
      const float2 wu = *reinterpret_cast<const float2*>(Wl + S + 32 * q);
      a[q] = ok ? mk<T>(drn(srn(mrn(ru, (double)wu.x), mrn(rl, (double)wl.x)), dz),
                        drn(srn(mrn(ru, (double)wu.y), mrn(rl, (double)wl.y)), dz))
                : mk<T>((T)0, (T)0);
    }
  } else if constexpr (FIELDS) {
#pragma unroll
    for (int q = 0; q < 16; ++q) a[q] = mk<T>((T)0, (T)0);
  } else {
    const float rl = ok ? (float)rhoh[zj] : 0.0f, ru = ok ? (float)rhoh[zj + 1] : 0.0f;
    const float idz = (float)(1.0 / g.dz);
    const float sd = (float)sdt;
    const float* Wl = W + j * S + 2 * t;
    const float* Bl = BH + j * S + 2 * t;
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      float2 wl = *reinterpret_cast<const float2*>(Wl + 32 * q);
      float2 wu = *reinterpret_cast<const float2*>(Wl + S + 32 * q);
      if (STAGE) {  // provisional stage w (integrator.py:483-490)
        const float2 bl = *reinterpret_cast<const float2*>(Bl + 32 * q);
        const float2 bu = *reinterpret_cast<const float2*>(Bl + S + 32 * q);
        wl.x += sd * bl.x;
        wl.y += sd * bl.y;
        wu.x += sd * bu.x;
        wu.y += sd * bu.y;
      }
      a[q] = ok ? mk<float>((ru * wu.x - rl * wl.x) * idz, (ru * wu.y - rl * wl.y) * idz)
                : mk<float>(0.0f, 0.0f);
    }
  }
  xr_pass1<T, false>(a, t, tw2);
  __syncthreads();  // every gather done: the exchange blocks reuse the tiles' space
  xr_pass2<T, false>(a, t, ex + grp * kXrEx);

  // 3. R2C split, a[s] = Z[k], k = 16 s + t; Z[M - k] is held by the partner
  //    lane (16 - t) mod 16 of the group, at s' = 15 - s (t > 0), or by the
  //    lane itself at (16 - s) mod 16 (t = 0)
  const int plane = (tid & 16) | ((16 - t) & 15);
  __syncthreads();  // every exchange read: the spectra reuse their space
#pragma unroll
  for (int s = 0; s < 16; ++s) {
    const T px = __shfl_sync(0xffffffffu, a[15 - s].x, plane);
    const T py = __shfl_sync(0xffffffffu, a[15 - s].y, plane);
    const cplx<T> zk = a[s];
    const cplx<T> zc = conjg(t == 0 ? a[(16 - s) & 15] : mk<T>(px, py));
    const cplx<T> E = scl(add(zk, zc), (T)0.5);
    const cplx<T> D = sub(zk, zc);
    const cplx<T> O = mk<T>((T)0.5 * D.y, (T)-0.5 * D.x);  // -i/2 * D
    const int k = 16 * s + t;
    const cplx<T> WO = mul(twN[k], O);
    XS[k * BP + grp] = add(E, WO);
    if (k == 0) XS[M * BP + grp] = conjg(sub(E, WO));
  }
  __syncthreads();

  // 4. X0 = i kx' U + D, X1 = V, two adjacent levels per thread
  //    (consecutive threads on consecutive pairs; 16-byte stores of FP32
  //    pairs where the levels start on an even index)
  const bool st2 = sizeof(T) == 4 && (nz & 1) == 0 &&
                   ((reinterpret_cast<size_t>(X0) | reinterpret_cast<size_t>(X1)) & 15) == 0;
  for (int e = tid; e < (M + 1) * (ZC / 2); e += NT) {
    const int k = e / (ZC / 2), jj = 2 * (e - k * (ZC / 2));
    const int z = z0 + jj;
    if (z >= nz) continue;
    const bool two = z + 1 < nz;
    const T kk = (k == M) ? (T)0 : (T)kxd[k];
    const int o = (k * ny + y) * nz + z;
    const cplx<T> x00 = FIELDS ? XS[k * BP + jj]
                               : add(ik(kk, XS[k * BP + jj]), XS[k * BP + 2 * ZC + jj]);
    const cplx<T> x01 = FIELDS ? XS[k * BP + jj + 1]
                               : add(ik(kk, XS[k * BP + jj + 1]), XS[k * BP + 2 * ZC + jj + 1]);
    const cplx<T> x10 = XS[k * BP + ZC + jj], x11 = XS[k * BP + ZC + jj + 1];
    if constexpr (sizeof(T) == 4) {
      if (two && st2) {
        *reinterpret_cast<float4*>(&X0[o]) = make_float4(x00.x, x00.y, x01.x, x01.y);
        *reinterpret_cast<float4*>(&X1[o]) = make_float4(x10.x, x10.y, x11.x, x11.y);
        continue;
      }
    }
    X0[o] = x00;
    X1[o] = x10;
    if (two) {
      X0[o + 1] = x01;
      X1[o + 1] = x11;
    }
  }
}

// ---- inverse: k_ix3 ------------------------------------------------------------
// Columns (groups): [0, ZC] phi at levels z0-1 .. z0+ZC-1 (one halo level),
// [ZC+1, 2ZC] d/dx phi, [2ZC+1, 3ZC] d/dy phi (psi~), 3ZC+1 a zero column
// that makes the group count even (whole warps).
template <int ZC>
struct Ix3Size {
  static constexpr int BG = 3 * ZC + 2;  // groups
  static constexpr int BI = 2 * ZC + 1;  // loaded spectral columns: phi (with halo), psi
  static constexpr int SR = xr_stride<ZC>();
  static constexpr size_t tables = 2 * kXrM * 8 + (((kXrM + 1) * 4 + 15) / 16) * 16;
  static constexpr size_t xi = (size_t)(kXrM + 1) * BI * 8;
  static constexpr size_t ex = (size_t)BG * kXrEx * 8;
  static constexpr size_t zr = (size_t)BG * SR * 4;
  static constexpr size_t regA = xi > ex ? (xi > zr ? xi : zr) : (ex > zr ? ex : zr);
  static constexpr size_t state = (size_t)kXrN * (3 * ZC + 1) * 4;
  static constexpr size_t total = tables + regA + state;
};
template <int ZC>
constexpr int ix3_min_blocks() { return ZC >= 8 ? 2 : 3; }

// Inverse x-pencil kernel with the velocity correction (k_ix2 semantics and
// modes, FP32, nx = 512; in IX_CORRECT and IX_STAGE phi_out may be
// null).  grid = (ceil(nz/ZC), ny), 16 (3 ZC + 2) threads.
// IX_FIELDS: the real C2R outputs of two spectra, u_out = C2R(phs) and
// v_out = C2R(psi) (what k_ix IX_FIELDS writes: the Helmholtz damper's inverse
// x transform); no state is read and nothing else is written.
// Shared memory: twiddles and kx'; region A holding in turn the spectral
// rows, the groups' exchange blocks and the real outputs (level-major rows);
// the state tiles, requested at the start in their own cp.async group so
// that they arrive during the FFT.
template <int MODE, int ZC>
__global__ void __launch_bounds__(16 * (3 * ZC + 2), ix3_min_blocks<ZC>()) k_ix3(
    GridK g, const cplx<float>* __restrict__ phs, const cplx<float>* __restrict__ psi,
    const double* __restrict__ kxd, const cplx<float>* __restrict__ twx, const float* u_in,
    const float* v_in, const float* w_in, const float* __restrict__ bh, double sdt,
    float* u_out, float* v_out, float* w_out, float* phi_out) {
  static_assert(ZC == 2 || ZC == 4 || ZC == 8, "supported z-chunks");
  using SZ = Ix3Size<ZC>;
  constexpr bool STAGE = (MODE == IX_STAGE);
  constexpr int BG = SZ::BG, BI = SZ::BI, SR = SZ::SR, NT = 16 * BG, M = kXrM, N = kXrN;
  extern __shared__ __align__(16) unsigned char smem_dyn[];
  cplx<float>* tw2 = reinterpret_cast<cplx<float>*>(smem_dyn);  // [16 k2 + t] = W_256^(t k2)
  cplx<float>* twN = tw2 + M;                                   // W_512^m, m < 256
  float* kxs = reinterpret_cast<float*>(twN + M);               // kx'[0..M], kx'[M] = 0
  unsigned char* regA = smem_dyn + SZ::tables;
  cplx<float>* XI = reinterpret_cast<cplx<float>*>(regA);       // [M + 1][BI]
  cplx<float>* ex = reinterpret_cast<cplx<float>*>(regA);       // BG x 16 x 17
  float* ZR = reinterpret_cast<float*>(regA);                   // [BG][SR] real outputs
  float* SU = reinterpret_cast<float*>(regA + SZ::regA);        // [x][ZC]
  float* SV = SU + N * ZC;                                      // [x][ZC]
  float* SW = SV + N * ZC;                                      // [x][ZC + 1]
  const int ny = g.ny, nz = g.nz;
  const int y = blockIdx.y;
  const int z0 = blockIdx.x * ZC;
  const int zl = min(z0 + ZC, nz) - 1;  // last level of the chunk
  const int tid = threadIdx.x;

  // 1. spectral rows (first cp.async group), then the state tiles (second);
  //    consecutive threads on consecutive levels of a row
  for (int e = tid; e < (M + 1) * BI; e += NT) {
    const int k = e / BI, b = e - k * BI;
    const int ob = (k * ny + y) * nz;
    if (b <= ZC) {
      const int z = z0 - 1 + b;
      const bool ok = z >= 0 && z < nz;
      copy_or_zero(&XI[e], phs + ob + (ok ? z : 0), ok);
    } else {
      const int z = z0 + b - ZC - 1;
      const bool ok = z < nz;
      copy_or_zero(&XI[e], psi + ob + (ok ? z : 0), ok);
    }
  }
  cp_commit();
  // u, v: 16-byte copies (ZC / 4 per row) where the chunk is whole and the
  // rows start on 16 bytes; 4-byte copies otherwise
  if constexpr (MODE != IX_FIELDS) {
  const bool vec = ZC >= 4 && z0 + ZC <= nz && (nz & 3) == 0 &&
                   ((reinterpret_cast<size_t>(u_in) | reinterpret_cast<size_t>(v_in)) & 15) == 0;
  if (vec) {
    constexpr int Q = ZC >= 4 ? ZC / 4 : 1;
    for (int e = tid; e < N * Q; e += NT) {
      const int x = e / Q, q = e - x * Q;
      const int gi = (x * ny + y) * nz + z0 + 4 * q;
      cp_async(&SU[x * ZC + 4 * q], u_in + gi, 16);
      cp_async(&SV[x * ZC + 4 * q], v_in + gi, 16);
    }
  } else {
    for (int e = tid; e < N * ZC; e += NT) {
      const int x = e / ZC, j = e - x * ZC;
      const int z = z0 + j;
      const bool ok = z < nz;
      const int gi = (x * ny + y) * nz + (ok ? z : 0);
      copy_or_zero(&SU[e], u_in + gi, ok);
      copy_or_zero(&SV[e], v_in + gi, ok);
    }
  }
  for (int e = tid; e < N * (ZC + 1); e += NT) {
    const int x = e / (ZC + 1), j = e - x * (ZC + 1);
    const int z = z0 + j;  // half levels z0 .. z0+ZC
    const bool ok = z <= nz;
    copy_or_zero(&SW[e], w_in + (x * ny + y) * (nz + 1) + (ok ? z : 0), ok);
  }
  }
  cp_commit();
  if (STAGE || MODE == IX_REFINE)
    for (int x = tid; x < N; x += NT) {
      const int c = x * ny + y;
      if (STAGE) prefetch_run(bh + c * (nz + 1) + z0, bh + c * (nz + 1) + zl + 1);
      if (MODE == IX_REFINE) prefetch_run(phi_out + c * nz + z0, phi_out + c * nz + zl);
    }
  for (int i = tid; i < M; i += NT) {
    tw2[i] = twx[2 * ((i & 15) * (i >> 4))];  // W_256^m = W_512^(2m)
    twN[i] = twx[i];
  }
  for (int i = tid; i <= M; i += NT) kxs[i] = (i == M) ? 0.0f : (float)kxd[i];
  cp_wait<1>();  // the spectral rows (the state tiles may still be in flight)
  __syncthreads();

  // 2. gather with the C2R pre-process fused: a[q] = Z[t + 16 q] of column grp
  const int grp = tid >> 4, t = tid & 15;
  int src = 0;
  bool dx = false;
  if (grp <= ZC) {
    src = grp;
  } else if (grp <= 2 * ZC) {
    src = grp - ZC;  // phi~ column of the same level
    dx = true;
  } else {
    src = grp - ZC;  // psi~ (grp = 3 ZC + 1: the zero column)
  }
  const bool zero = grp == 3 * ZC + 1;
  cplx<float> a[16];
#pragma unroll
  for (int q = 0; q < 16; ++q) {
    const int m = t + 16 * q;
    const int mc = M - m;
    cplx<float> xm = zero ? mk<float>(0.0f, 0.0f) : XI[m * BI + src];
    cplx<float> xc = zero ? mk<float>(0.0f, 0.0f) : XI[mc * BI + src];
    if (dx) {
      xm = ik(kxs[m], xm);
      xc = ik(kxs[mc], xc);
    }
    if (m == 0) {
      xm.y = 0.0f;
      xc.y = 0.0f;
    }
    xc = conjg(xc);
    const cplx<float> S = add(xm, xc);
    const cplx<float> D = mul(sub(xm, xc), conjg(twN[m]));
    a[q] = mk<float>(S.x - D.y, S.y + D.x);
  }
  xr_pass1<float, true>(a, t, tw2);
  __syncthreads();  // every gather done: the exchange blocks reuse the rows' space
  xr_pass2<float, true>(a, t, ex + grp * kXrEx);
  // a[k1] = x[2n] + i x[2n+1], n = 16 k1 + t
  __syncthreads();  // every exchange read: the outputs reuse their space
  float* zr = ZR + grp * SR + 2 * t;
#pragma unroll
  for (int k1 = 0; k1 < 16; ++k1)
    *reinterpret_cast<float2*>(zr + 32 * k1) = make_float2(a[k1].x, a[k1].y);
  // the global values the correction reads besides the tiles (STAGE: b_half;
  // IX_REFINE: phi) are loaded here, all at once, so that their latency
  // overlaps the barrier instead of each correction step.  The correction
  // takes two adjacent levels (z, z + 1) of a row per thread.
  constexpr int NPR = N * ZC / 2;             // level pairs of the tile
  constexpr int NP = (NPR + NT - 1) / NT;     // pairs per thread
  float g0[NP], g1[NP], gt[NP];
  if (STAGE || MODE == IX_REFINE) {
#pragma unroll
    for (int i = 0; i < NP; ++i) {
      const int e = tid + i * NT;
      const int x = e / (ZC / 2), j = 2 * (e - x * (ZC / 2));
      const int z = z0 + j;
      g0[i] = g1[i] = gt[i] = 0.0f;
      if (e < NPR && z < nz) {
        const int col = x * ny + y;
        if (STAGE) {
          const float* r = bh + col * (nz + 1);
          g0[i] = r[z];
          if (z + 1 < nz) g1[i] = r[z + 1];
          if (z + 2 >= nz) gt[i] = r[nz];  // the lid (level nz) follows this pair
        } else {
          g0[i] = phi_out[col * nz + z];
          if (z + 1 < nz) g1[i] = phi_out[col * nz + z + 1];
        }
      }
    }
  }
  cp_wait<0>();
  __syncthreads();

  // 3. velocity correction, levels (z, z + 1) of row x per thread;
  //    consecutive threads on consecutive pairs
  const float dzt = (float)g.dz;
  const bool st2 = (nz & 1) == 0 && ((reinterpret_cast<size_t>(u_out) |
                                      reinterpret_cast<size_t>(v_out) |
                                      reinterpret_cast<size_t>(phi_out)) & 7) == 0;
#pragma unroll
  for (int i = 0; i < NP; ++i) {
    const int e = tid + i * NT;
    if (e >= NPR) break;
    const int x = e / (ZC / 2), j = 2 * (e - x * (ZC / 2));
    const int z = z0 + j;
    if (z >= nz) continue;
    const bool two = z + 1 < nz;
    const int col = x * ny + y;
    const int idx = col * nz + z;
    if constexpr (MODE == IX_FIELDS) {
      // phi group j + 1 and psi group 2 ZC + 1 + j hold level z
      const float a0 = ZR[(j + 1) * SR + x], a1 = ZR[(j + 2) * SR + x];
      const float b0 = ZR[(2 * ZC + 1 + j) * SR + x], b1 = ZR[(2 * ZC + 2 + j) * SR + x];
      if (two && st2) {
        *reinterpret_cast<float2*>(&u_out[idx]) = make_float2(a0, a1);
        *reinterpret_cast<float2*>(&v_out[idx]) = make_float2(b0, b1);
      } else {
        u_out[idx] = a0;
        v_out[idx] = b0;
        if (two) {
          u_out[idx + 1] = a1;
          v_out[idx + 1] = b1;
        }
      }
      continue;
    }
    const float phb = ZR[j * SR + x];  // level z - 1
    const float ph0 = ZR[(j + 1) * SR + x];
    const float ph1 = ZR[(j + 2) * SR + x];
    const float gx0 = ZR[(ZC + 1 + j) * SR + x], gx1 = ZR[(ZC + 2 + j) * SR + x];
    const float gy0 = ZR[(2 * ZC + 1 + j) * SR + x], gy1 = ZR[(2 * ZC + 2 + j) * SR + x];
    const float gz0 = (z >= 1) ? drn(srn(ph0, phb), dzt) : 0.0f;
    const float gz1 = drn(srn(ph1, ph0), dzt);
    const float2 su = *reinterpret_cast<const float2*>(&SU[x * ZC + j]);
    const float2 sv = *reinterpret_cast<const float2*>(&SV[x * ZC + j]);
    const int sw = x * (ZC + 1) + j;
    float w0 = SW[sw], w1 = SW[sw + 1];
    if (STAGE) {
      w0 = (float)arn((double)w0, mrn(sdt, (double)g0[i]));
      w1 = (float)arn((double)w1, mrn(sdt, (double)g1[i]));
    }
    const int wi = col * (nz + 1) + z;
    const float p0 = (MODE == IX_REFINE) ? g0[i] + ph0 : ph0;
    const float p1 = (MODE == IX_REFINE) ? g1[i] + ph1 : ph1;
    if (two && st2) {
      *reinterpret_cast<float2*>(&u_out[idx]) = make_float2(su.x - gx0, su.y - gx1);
      *reinterpret_cast<float2*>(&v_out[idx]) = make_float2(sv.x - gy0, sv.y - gy1);
      if (phi_out) *reinterpret_cast<float2*>(&phi_out[idx]) = make_float2(p0, p1);
    } else {
      u_out[idx] = su.x - gx0;
      v_out[idx] = sv.x - gy0;
      if (phi_out) phi_out[idx] = p0;
      if (two) {
        u_out[idx + 1] = su.y - gx1;
        v_out[idx + 1] = sv.y - gy1;
        if (phi_out) phi_out[idx + 1] = p1;
      }
    }
    w_out[wi] = w0 - gz0;
    if (two) w_out[wi + 1] = w1 - gz1;
    // the lid, level nz, after the top level nz - 1 of the column
    const int zt = two ? z + 1 : z;
    if (zt == nz - 1 && (STAGE || w_out != w_in)) {
      float wt = SW[x * (ZC + 1) + (nz - z0)];
      if (STAGE) wt = (float)arn((double)wt, mrn(sdt, (double)gt[i]));
      w_out[col * (nz + 1) + nz] = wt;
    }
  }
}

// ---- y pencils: ny = 512, one warp per column ---------------------------------
// N = 512 = 32 x 16, n = n1 + 32 n2 (n1 < 32, n2 < 16):
//   pass 1: lane n1 takes the 16-point DFT over n2 and multiplies by
//           W_512^(n1 k2) (k2 < 16);
//   exchange: through the column's 16 x 33 padded block (warp-local);
//   pass 2: lane L = k2 + 16 p (p = 0, 1) holds Y[p + 2 m][k2] (m < 16) and
//           takes the 16-point DFT over m: the even (p = 0) and odd (p = 1)
//           halves of the 32-point DFT over n1;
//   radix 2: lanes L and L ^ 16 combine them (shuffles), E + W_32^j O on
//           p = 0 and E - W_32^j O on p = 1.
// Lane L leaves with a[j] = X[16 (j + 16 p) + k2], j < 16.
constexpr int kYrN = 512;
constexpr int kYrEx = 16 * 33;  // exchange block of one column (complex)

// ytw[32 k2 + n1] = W_512^(n1 k2) (forward sign), w32[j] = W_32^j.
// yr_pass1 (DFT over n2 and the twiddles, registers only) and yr_pass2 (the
// exchange through the column's block, the second DFT and the radix-2 step)
// let a caller place a barrier between them when ex aliases other data.
template <class T, bool INV>
__device__ __forceinline__ void yr_pass1(cplx<T> (&a)[16], int lane,
                                         const cplx<T>* __restrict__ ytw) {
  dft16<T, INV>(a);
#pragma unroll
  for (int k2 = 1; k2 < 16; ++k2) {
    cplx<T> w = ytw[32 * k2 + lane];
    if (INV) w.y = -w.y;
    a[k2] = mul(a[k2], w);
  }
}
template <class T, bool INV>
__device__ __forceinline__ void yr_pass2(cplx<T> (&a)[16], int lane,
                                         const cplx<T>* __restrict__ w32, cplx<T>* ex) {
#pragma unroll
  for (int k2 = 0; k2 < 16; ++k2) ex[k2 * 33 + lane] = a[k2];
  __syncwarp();
  const int k2 = lane & 15, p = lane >> 4;
#pragma unroll
  for (int m = 0; m < 16; ++m) a[m] = ex[k2 * 33 + p + 2 * m];
  dft16<T, INV>(a);
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    cplx<T> w = w32[j];
    if (INV) w.y = -w.y;
    const T ox = __shfl_xor_sync(0xffffffffu, a[j].x, 16);
    const T oy = __shfl_xor_sync(0xffffffffu, a[j].y, 16);
    const cplx<T> other = mk<T>(ox, oy);
    // p = 0 holds E, the partner O; p = 1 holds O, the partner E
    a[j] = p == 0 ? add(a[j], mul(w, other)) : sub(other, mul(w, a[j]));
  }
}
template <class T, bool INV>
__device__ __forceinline__ void yr_fft(cplx<T> (&a)[16], int lane,
                                       const cplx<T>* __restrict__ ytw,
                                       const cplx<T>* __restrict__ w32, cplx<T>* ex) {
  yr_pass1<T, INV>(a, lane, ytw);
  yr_pass2<T, INV>(a, lane, w32, ex);
}

template <int ZC>
constexpr int yr_min_blocks() { return ZC >= 8 ? 1 : 3; }

// Shared memory of k_fy3 / k_iy3: twiddles, then one region holding in turn
// the input rows, the columns' exchange blocks and the output rows (complex
// values of type T).
template <int ZC, class T = float>
struct YrSize {
  static constexpr int B = 2 * ZC;   // columns (warps)
  static constexpr int BP = B + 1;   // row stride of the row tiles (odd)
  static constexpr size_t tables = (size_t)(kYrN + 16) * sizeof(cplx<T>);
  static constexpr size_t rows = (size_t)kYrN * BP * sizeof(cplx<T>);
  static constexpr size_t ex = (size_t)B * kYrEx * sizeof(cplx<T>);
  static constexpr size_t total = tables + (rows > ex ? rows : ex);
};

// k_fy2 at ny = 512: d^ = FFTy(X0) + i ky' FFTy(X1) in arithmetic type T,
// stored as TO.  FY_DIV: the projection (T = TO = float); FY_RESID: the
// defect correction's FP64 residual (T = double, TO = float), its Nyquist
// rows (ky = ny/2 or kx = nx/2) zeroed.  Columns: X0 at ZC levels, X1 at ZC
// levels.  grid = (ceil(nz/ZC), nx/2 + 1).
template <int ZC, class T = float, int MODE = FY_DIV, class TO = float>
__global__ void __launch_bounds__(64 * ZC, sizeof(T) == 8 ? 4 : yr_min_blocks<ZC>()) k_fy3(
    GridK g, const cplx<T>* __restrict__ in0, const cplx<T>* __restrict__ in1,
    const double* __restrict__ kyd, const cplx<T>* __restrict__ twy,
    cplx<TO>* __restrict__ out0) {
  using SZ = YrSize<ZC, T>;
  constexpr int B = SZ::B, BP = SZ::BP, NT = 32 * B, N = kYrN;
  extern __shared__ __align__(16) unsigned char smem_dyn[];
  cplx<T>* ytw = reinterpret_cast<cplx<T>*>(smem_dyn);
  cplx<T>* w32 = ytw + N;
  cplx<T>* R = reinterpret_cast<cplx<T>*>(smem_dyn + SZ::tables);  // [N][BP]
  cplx<T>* ex = R;                                                // B x 16 x 33
  const int ny = g.ny, nz = g.nz;
  const int kx = blockIdx.y;
  const int z0 = blockIdx.x * ZC;
  const int tid = threadIdx.x;
  for (int e = tid; e < N * B; e += NT) {
    const int y = e / B, b = e - y * B;
    const int f = b / ZC, j = b - f * ZC;
    const int z = z0 + j;
    const bool ok = z < nz;
    copy_or_zero(&R[y * BP + b], (f == 0 ? in0 : in1) + (kx * ny + y) * nz + (ok ? z : 0), ok);
  }
  cp_commit();
  for (int i = tid; i < N; i += NT) ytw[i] = twy[(i & 31) * (i >> 5)];
  if (tid < 16) w32[tid] = twy[16 * tid];
  cp_wait<0>();
  __syncthreads();
  const int c = tid >> 5, lane = tid & 31;
  cplx<T> a[16];
#pragma unroll
  for (int q = 0; q < 16; ++q) a[q] = R[(lane + 32 * q) * BP + c];
  __syncthreads();  // every gather done: the exchange blocks reuse the rows' space
  yr_fft<T, false>(a, lane, ytw, w32, ex + c * kYrEx);
  __syncthreads();  // every exchange read: the output rows reuse their space
  const int k2 = lane & 15, p = lane >> 4;
#pragma unroll
  for (int j = 0; j < 16; ++j) R[(16 * (j + 16 * p) + k2) * BP + c] = a[j];
  __syncthreads();
  for (int e = tid; e < N * ZC; e += NT) {
    const int ky = e / ZC, j = e - ky * ZC;
    const int z = z0 + j;
    if (z >= nz) continue;
    const T kk = (ky == N / 2) ? (T)0 : (T)kyd[ky];
    cplx<T> d = add(R[ky * BP + j], ik(kk, R[ky * BP + ZC + j]));
    if (MODE == FY_RESID && (ky == N / 2 || kx == g.nx / 2)) d = mk<T>((T)0, (T)0);
    out0[(kx * ny + ky) * nz + z] = mk<TO>((TO)d.x, (TO)d.y);
  }
}

// k_iy2 for FP32 at ny = 512: phi~ = IFFTy(phi^), psi~ = IFFTy(i ky' phi^).
// Columns: phi~ at ZC levels, then psi~ (the gather applies i ky').
template <int ZC>
__global__ void __launch_bounds__(64 * ZC, yr_min_blocks<ZC>()) k_iy3(
    GridK g, const cplx<float>* __restrict__ in0, const double* __restrict__ kyd,
    const cplx<float>* __restrict__ twy, cplx<float>* __restrict__ out0,
    cplx<float>* __restrict__ out1) {
  using SZ = YrSize<ZC>;
  constexpr int B = SZ::B, BP = SZ::BP, NT = 32 * B, N = kYrN;
  extern __shared__ __align__(16) unsigned char smem_dyn[];
  cplx<float>* ytw = reinterpret_cast<cplx<float>*>(smem_dyn);
  cplx<float>* w32 = ytw + N;
  cplx<float>* R = reinterpret_cast<cplx<float>*>(smem_dyn + SZ::tables);  // [N][BP]
  cplx<float>* ex = R;
  const int ny = g.ny, nz = g.nz;
  const int kx = blockIdx.y;
  const int z0 = blockIdx.x * ZC;
  const int tid = threadIdx.x;
  for (int e = tid; e < N * ZC; e += NT) {
    const int y = e / ZC, j = e - y * ZC;
    const int z = z0 + j;
    const bool ok = z < nz;
    copy_or_zero(&R[y * BP + j], in0 + (kx * ny + y) * nz + (ok ? z : 0), ok);
  }
  cp_commit();
  for (int i = tid; i < N; i += NT) ytw[i] = twy[(i & 31) * (i >> 5)];
  if (tid < 16) w32[tid] = twy[16 * tid];
  cp_wait<0>();
  __syncthreads();
  const int c = tid >> 5, lane = tid & 31;
  const int src = c < ZC ? c : c - ZC;
  cplx<float> a[16];
#pragma unroll
  for (int q = 0; q < 16; ++q) {
    const int n = lane + 32 * q;
    a[q] = R[n * BP + src];
    if (c >= ZC) a[q] = ik(n == N / 2 ? 0.0f : (float)kyd[n], a[q]);  // ky' = 0 at Nyquist
  }
  __syncthreads();
  yr_fft<float, true>(a, lane, ytw, w32, ex + c * kYrEx);
  __syncthreads();
  const int k2 = lane & 15, p = lane >> 4;
#pragma unroll
  for (int j = 0; j < 16; ++j) R[(16 * (j + 16 * p) + k2) * BP + c] = a[j];
  __syncthreads();
  for (int e = tid; e < N * ZC; e += NT) {
    const int y = e / ZC, j = e - y * ZC;
    const int z = z0 + j;
    if (z >= nz) continue;
    const int o = (kx * ny + y) * nz + z;
    out0[o] = R[y * BP + j];
    out1[o] = R[y * BP + ZC + j];
  }
}

// The Helmholtz damper's y stage for FP32 at ny = 512 in one pass (what k_fy
// FY_HELM followed by k_iy IY_FIELDS compute): forward y transforms of the U
// and V columns, the divergent-part multipliers
//   out0 = s (Kx^2/K^2 U + (KxKy/K^2)' V),  out1 = s ((KxKy/K^2)' U + Ky^2/K^2 V)
// (the primed cross term zero where exactly one of kx, ky is the Nyquist
// index; s = scale), then inverse y transforms.  The multipliers are formed in
// double as k_fy forms them, once per ky, into a table in shared memory.  In
// place is allowed: each CTA rewrites exactly the columns it read.
// grid = (ceil(nz/ZC), nx/2 + 1), 64 ZC threads.
template <int ZC>
struct HySize {
  static constexpr size_t mult = (size_t)kYrN * 3 * sizeof(float);
  static constexpr size_t total = YrSize<ZC>::total + mult;
};

template <int ZC>
__global__ void __launch_bounds__(64 * ZC, yr_min_blocks<ZC>()) k_hy3(
    GridK g, const cplx<float>* in0, const cplx<float>* in1, const double* __restrict__ kxd,
    const double* __restrict__ kyd, const cplx<float>* __restrict__ twy, double scale,
    cplx<float>* out0, cplx<float>* out1) {
  using SZ = YrSize<ZC>;
  constexpr int B = SZ::B, BP = SZ::BP, NT = 32 * B, N = kYrN;
  extern __shared__ __align__(16) unsigned char smem_dyn[];
  cplx<float>* ytw = reinterpret_cast<cplx<float>*>(smem_dyn);
  cplx<float>* w32 = ytw + N;
  cplx<float>* R = reinterpret_cast<cplx<float>*>(smem_dyn + SZ::tables);  // [N][BP]
  cplx<float>* ex = R;
  float* m3 = reinterpret_cast<float*>(smem_dyn + SZ::total);  // [ky][sxx, syy, sxy]
  const int ny = g.ny, nz = g.nz;
  const int kx = blockIdx.y;
  const int z0 = blockIdx.x * ZC;
  const int tid = threadIdx.x;
  for (int e = tid; e < N * B; e += NT) {
    const int y = e / B, b = e - y * B;
    const int f = b / ZC, j = b - f * ZC;
    const int z = z0 + j;
    const bool ok = z < nz;
    copy_or_zero(&R[y * BP + b], (f == 0 ? in0 : in1) + (kx * ny + y) * nz + (ok ? z : 0), ok);
  }
  cp_commit();
  for (int i = tid; i < N; i += NT) ytw[i] = twy[(i & 31) * (i >> 5)];
  if (tid < 16) w32[tid] = twy[16 * tid];
  for (int ky = tid; ky < N; ky += NT) {
    const double Kx = kxd[kx], Ky = kyd[ky];
    const double K2 = Kx * Kx + Ky * Ky;
    double mxx = 0, myy = 0, mxy = 0;
    if (K2 > 0) {
      mxx = Kx * Kx / K2;
      myy = Ky * Ky / K2;
      const bool nyqx = (kx == g.nx / 2), nyqy = (ky == N / 2);
      mxy = (nyqx != nyqy) ? 0.0 : Kx * Ky / K2;
    }
    m3[3 * ky + 0] = (float)(scale * mxx);
    m3[3 * ky + 1] = (float)(scale * myy);
    m3[3 * ky + 2] = (float)(scale * mxy);
  }
  cp_wait<0>();
  __syncthreads();
  const int c = tid >> 5, lane = tid & 31;
  const int k2 = lane & 15, p = lane >> 4;
  cplx<float> a[16];
#pragma unroll
  for (int q = 0; q < 16; ++q) a[q] = R[(lane + 32 * q) * BP + c];
  __syncthreads();  // every gather done: the exchange blocks reuse the rows' space
  yr_fft<float, false>(a, lane, ytw, w32, ex + c * kYrEx);
  __syncthreads();  // every exchange read: the rows come back in natural order
#pragma unroll
  for (int j = 0; j < 16; ++j) R[(16 * (j + 16 * p) + k2) * BP + c] = a[j];
  __syncthreads();
  for (int e = tid; e < N * ZC; e += NT) {
    const int ky = e / ZC, j = e - ky * ZC;
    const float sxx = m3[3 * ky], syy = m3[3 * ky + 1], sxy = m3[3 * ky + 2];
    const cplx<float> U = R[ky * BP + j], V = R[ky * BP + ZC + j];
    R[ky * BP + j] = mk<float>(sxx * U.x + sxy * V.x, sxx * U.y + sxy * V.y);
    R[ky * BP + ZC + j] = mk<float>(sxy * U.x + syy * V.x, sxy * U.y + syy * V.y);
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < 16; ++q) a[q] = R[(lane + 32 * q) * BP + c];
  __syncthreads();
  yr_fft<float, true>(a, lane, ytw, w32, ex + c * kYrEx);
  __syncthreads();
#pragma unroll
  for (int j = 0; j < 16; ++j) R[(16 * (j + 16 * p) + k2) * BP + c] = a[j];
  __syncthreads();
  for (int e = tid; e < N * B; e += NT) {
    const int y = e / B, b = e - y * B;
    const int f = b / ZC, j = b - f * ZC;
    const int z = z0 + j;
    if (z >= nz) continue;
    (f == 0 ? out0 : out1)[(kx * ny + y) * nz + z] = R[y * BP + b];
  }
}

}  // namespace ob
