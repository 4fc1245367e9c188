// Register-resident pencil kernels for the 1024-point grid lines (nx = 1024
// along x, ny = 1024 along y), single precision, plus the FP64 form of the
// forward x pencil for the defect correction's residual.
//
// x pencils (k_fx4, k_ix4): the packed complex FFT of a grid row has M = 512
// points, one warp per column: M = 32 x 16 with n = n1 + 32 n2, the same
// two-pass warp transform as the 512-point y pencils (yr_pass1 / yr_pass2):
// lane n1 holds z[n1 + 32 n2] (n2 < 16) on entry, and lane L = k2 + 16 p
// leaves with a[j] = Z[16 (j + 16 p) + k2].  The real-to-complex pack is fused
// into the gather, the R2C split is formed from partner lanes with warp
// shuffles (for k2 > 0 the partner of Z[k] holds Z[M - k] at register 15 - j
// in lane (16 - k2) + 16 (1 - p); for k2 = 0 it is lane L ^ 16 at register
// (16 - j) mod 16, or the lane itself at j = 0), and the complex-to-real
// pre-process is fused into the inverse kernel's gather.  Same semantics,
// modes and arithmetic per element as k_fx3 / k_ix3 (nx = 512) and k_fx2 /
// k_ix2 (any nx).
//
// y pencils (k_fy4, k_iy4): a 1024-point column per warp by decimation in
// time: the even and odd samples (16 of each per lane, n = 2 (L + 32 q) and
// n + 1) each take the 512-point warp transform, and X[k] = E[k] + W^k O[k],
// X[k + 512] = E[k] - W^k O[k] (W = W_1024) combine them in registers, since
// lane L holds E and O at the same indices k = 16 (j + 16 p) + k2.
//
// Layouts: state (x, y, z) with z contiguous, w on nz + 1 levels; spectra
// [kx][y][z] with kx in [0, nx/2].  Element indices are 32-bit.
#pragma once
#include "xreg.cuh"

namespace ob {

constexpr int kX4M = 512;   // packed complex FFT length (nx = 1024)
constexpr int kX4N = 1024;
constexpr int kY4N = 1024;  // y pencil length
constexpr int kWEx = 16 * 33;  // exchange block of one warp column (complex)
// twiddle tables: ytw (512), twN / tw1k (512), w32 (16)
constexpr int kX4Tw = 2 * 512 + 16;

// Row stride (floats) of the level-major tiles: nx plus a pad that puts the
// rows of one warp's z-run on distinct banks.
template <int ZC>
__host__ __device__ constexpr int x4_stride() { return kX4N + 32 / ZC; }

// The warp transform's tables from the W_1024^t table tw (1024 entries):
// ytw[32 k2 + n1] = W_512^(n1 k2) = W_1024^(2 n1 k2), w32[j] = W_1024^(32 j),
// twN[k] = W_1024^k (k < 512).
template <class T>
__device__ __forceinline__ void x4_tables(cplx<T>* ytw, cplx<T>* twN, cplx<T>* w32,
                                          const cplx<T>* __restrict__ tw, int tid, int nt) {
  for (int i = tid; i < 512; i += nt) {
    ytw[i] = tw[2 * ((i & 31) * (i >> 5))];
    twN[i] = tw[i];
  }
  if (tid < 16) w32[tid] = tw[32 * tid];
}

// ---- forward x: k_fx4 ------------------------------------------------------------
// Shared memory (bytes): tables, then one region that holds in turn the
// level-major state tiles (FP32), the columns' exchange blocks and the
// spectra (arithmetic type T).  NG: column groups (3: u, v, d; 4: u, v, the
// flux divergence of w and that of b_half, kept apart).
template <class T, bool STAGE, int ZC, int NG = 3>
__host__ __device__ constexpr size_t fx4_smem() {
  constexpr int B = NG * ZC, S = x4_stride<ZC>();
  constexpr size_t raw = (size_t)(2 * ZC + (STAGE ? 2 : 1) * (ZC + 1)) * S * 4;
  constexpr size_t ex = (size_t)B * kWEx * sizeof(cplx<T>);
  constexpr size_t xs = (size_t)(kX4M + 1) * (B + 1) * sizeof(cplx<T>);
  constexpr size_t r1 = raw > ex ? raw : ex;
  return (size_t)kX4Tw * sizeof(cplx<T>) + (r1 > xs ? r1 : xs);
}
template <class T, int ZC>
constexpr int fx4_min_blocks() { return (sizeof(T) == 8 || ZC >= 8) ? 1 : 2; }

// Forward x-pencil kernel (k_fx3 semantics at nx = 1024): rho-weighting,
// vertical flux divergence (STAGE: of w + sdt b_half), R2C along x;
// X0 = i kx' FFTx(rho u) + FFTx(vd), X1 = FFTx(rho v).  T = float: the
// single-precision projection; T = double: the FP64 residual transform of the
// defect correction, with k_fx2's operation order in the pack.  3 ZC columns
// (u, v, d at ZC levels), one warp each.  grid = (ceil(nz/ZC), ny), 96 ZC
// threads.
// NG = 4 (FP32, STAGE): the three fast stages' transforms at once.  The
// stage divergence is linear in sdt, so X0 = i kx' FFTx(rho u) + FFTx(D w),
// X1 = FFTx(rho v) and X2 = FFTx(D b_half), and stage s's X0 is
// X0 + sdt_s X2 (formed by the y pencils); 4 ZC columns, 128 ZC threads.
template <class T, bool STAGE, int ZC, int NG = 3>
__global__ void __launch_bounds__(32 * NG * ZC, fx4_min_blocks<T, ZC>()) k_fx4(
    GridK g, const float* __restrict__ u, const float* __restrict__ v,
    const float* __restrict__ w, const float* __restrict__ bh, double sdt,
    const double* __restrict__ rho, const double* __restrict__ rhoh,
    const double* __restrict__ kxd, const cplx<T>* __restrict__ twx,
    cplx<T>* __restrict__ X0, cplx<T>* __restrict__ X1, cplx<T>* __restrict__ X2) {
  static_assert(ZC == 2 || ZC == 4 || ZC == 8, "supported z-chunks");
  static_assert(sizeof(T) == 4 || !STAGE, "the FP64 form is the residual transform");
  static_assert(NG == 3 || (NG == 4 && STAGE && sizeof(T) == 4), "column groups");
  constexpr int B = NG * ZC, NT = 32 * B, M = kX4M, N = kX4N, S = x4_stride<ZC>(), BP = B + 1;
  extern __shared__ __align__(16) unsigned char smem_dyn[];
  cplx<T>* ytw = reinterpret_cast<cplx<T>*>(smem_dyn);
  cplx<T>* twN = ytw + 512;
  cplx<T>* w32 = twN + 512;
  unsigned char* reg = smem_dyn + kX4Tw * sizeof(cplx<T>);
  float* U = reinterpret_cast<float*>(reg);  // [ZC][S]
  float* V = U + ZC * S;                     // [ZC][S]
  float* W = V + ZC * S;                     // [ZC + 1][S]
  float* BH = W + (ZC + 1) * S;              // [ZC + 1][S] (STAGE)
  cplx<T>* ex = reinterpret_cast<cplx<T>*>(reg);  // B x 16 x 33, after the gather
  cplx<T>* XS = reinterpret_cast<cplx<T>*>(reg);  // (M + 1) x BP, after the exchange
  const int ny = g.ny, nz = g.nz;
  const int y = blockIdx.y;
  const int z0 = blockIdx.x * ZC;
  const int tid = threadIdx.x;

  // 1. every tile in flight at once; consecutive threads take consecutive
  //    levels of a row, rows stored level-major
  for (int e = tid; e < N * ZC; e += NT) {
    const int x = e / ZC, j = e - x * ZC;
    const int z = z0 + j;
    const bool ok = z < nz;
    const int gi = (x * ny + y) * nz + (ok ? z : 0);
    copy_or_zero(&U[j * S + x], u + gi, ok);
    copy_or_zero(&V[j * S + x], v + gi, ok);
  }
  for (int e = tid; e < N * (ZC + 1); e += NT) {
    const int x = e / (ZC + 1), j = e - x * (ZC + 1);
    const int z = z0 + j;  // half levels z0 .. z0+ZC
    const bool ok = z <= nz;
    const int gi = (x * ny + y) * (nz + 1) + (ok ? z : 0);
    copy_or_zero(&W[j * S + x], w + gi, ok);
    if (STAGE) copy_or_zero(&BH[j * S + x], bh + gi, ok);
  }
  cp_commit();
  x4_tables<T>(ytw, twN, w32, twx, tid, NT);
  cp_wait<0>();
  __syncthreads();

  // 2. gather with the pack fused: warp grp = (field f, level j); lane t
  //    takes z[t + 32 q] = f(2n) + i f(2n+1), n = t + 32 q
  const int grp = tid >> 5, t = tid & 31;
  const int f = grp / ZC, j = grp - f * ZC;
  const int zj = z0 + j;
  const bool ok = zj < nz;
  cplx<T> a[16];
  if (f < 2) {
    const T r = ok ? (T)rho[zj] : (T)0;
    const float* R = (f == 0 ? U : V) + j * S + 2 * t;
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      const float2 p = *reinterpret_cast<const float2*>(R + 64 * q);
      a[q] = mk<T>(r * (T)p.x, r * (T)p.y);
    }
  } else if constexpr (sizeof(T) == 8) {
    // the reference's operation order, rounded step by step (as k_fx2)
    const double rl = ok ? rhoh[zj] : 0.0, ru = ok ? rhoh[zj + 1] : 0.0;
    const double dz = g.dz;
    const float* Wl = W + j * S + 2 * t;
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      const float2 wl = *reinterpret_cast<const float2*>(Wl + 64 * q);
      const float2 wu = *reinterpret_cast<const float2*>(Wl + S + 64 * q);
      a[q] = ok ? mk<T>(drn(srn(mrn(ru, (double)wu.x), mrn(rl, (double)wl.x)), dz),
                        drn(srn(mrn(ru, (double)wu.y), mrn(rl, (double)wl.y)), dz))
                : mk<T>((T)0, (T)0);
    }
  } else {
    const float rl = ok ? (float)rhoh[zj] : 0.0f, ru = ok ? (float)rhoh[zj + 1] : 0.0f;
    const float idz = (float)(1.0 / g.dz);
    const float sd = (float)sdt;
    // NG = 4: group 2 differences w, group 3 b_half, each on its own
    const float* Wl = ((NG == 4 && f == 3) ? BH : W) + j * S + 2 * t;
    const float* Bl = BH + j * S + 2 * t;
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      float2 wl = *reinterpret_cast<const float2*>(Wl + 64 * q);
      float2 wu = *reinterpret_cast<const float2*>(Wl + S + 64 * q);
      if (STAGE && NG == 3) {  // provisional stage w (integrator.py:483-490)
        const float2 bl = *reinterpret_cast<const float2*>(Bl + 64 * q);
        const float2 bu = *reinterpret_cast<const float2*>(Bl + S + 64 * q);
        wl.x += sd * bl.x;
        wl.y += sd * bl.y;
        wu.x += sd * bu.x;
        wu.y += sd * bu.y;
      }
      a[q] = ok ? mk<float>((ru * wu.x - rl * wl.x) * idz, (ru * wu.y - rl * wl.y) * idz)
                : mk<float>(0.0f, 0.0f);
    }
  }
  yr_pass1<T, false>(a, t, ytw);
  __syncthreads();  // every gather done: the exchange blocks reuse the tiles' space
  yr_pass2<T, false>(a, t, w32, ex + grp * kWEx);

  // 3. R2C split: a[s] = Z[k], k = 16 (s + 16 p) + k2.  The lanes with
  //    k2 > 0 read their partner values only from lanes with k2 > 0, and the
  //    two lanes with k2 = 0 only from each other, so each lane offers the
  //    register its readers need and one shuffle pair per slot serves all.
  const int k2 = t & 15, p = t >> 4;
  const int partner = k2 ? (16 - k2) + 16 * (1 - p) : (t ^ 16);
  __syncthreads();  // every exchange read: the spectra reuse their space
#pragma unroll
  for (int s = 0; s < 16; ++s) {
    const cplx<T> offer = k2 ? a[15 - s] : a[(16 - s) & 15];
    const T px = __shfl_sync(0xffffffffu, offer.x, partner);
    const T py = __shfl_sync(0xffffffffu, offer.y, partner);
    const cplx<T> zk = a[s];
    const cplx<T> zm = (k2 == 0 && s == 0) ? a[0] : mk<T>(px, py);
    const cplx<T> zc = conjg(zm);
    const cplx<T> E = scl(add(zk, zc), (T)0.5);
    const cplx<T> D = sub(zk, zc);
    const cplx<T> O = mk<T>((T)0.5 * D.y, (T)-0.5 * D.x);  // -i/2 * D
    const int k = 16 * (s + 16 * p) + k2;
    const cplx<T> WO = mul(twN[k], O);
    XS[k * BP + grp] = add(E, WO);
    if (k == 0) XS[M * BP + grp] = conjg(sub(E, WO));
  }
  __syncthreads();

  // 4. X0 = i kx' U + D, X1 = V, two adjacent levels per thread (16-byte
  //    stores of FP32 pairs where the levels start on an even index).  Each
  //    group of 8 ZC threads covers 16 consecutive k at every level pair:
  //    a half-warp reads 16 k of one pair (distinct banks, BP odd), a warp
  //    stores whole 32-byte runs of two pairs per k.
  const bool st2 = sizeof(T) == 4 && (nz & 1) == 0 &&
                   ((reinterpret_cast<size_t>(X0) | reinterpret_cast<size_t>(X1) |
                     reinterpret_cast<size_t>(X2)) & 15) == 0;
  constexpr int G = 16 * (ZC / 2);  // threads of one 16-k group
  for (int e = tid; e < ((M + 1 + 15) / 16) * G; e += NT) {
    const int grp16 = e / G, r = e - grp16 * G;
    const int k = 16 * grp16 + (r & 15), jj = 2 * (r >> 4);
    const int z = z0 + jj;
    if (k > M || z >= nz) continue;
    const bool two = z + 1 < nz;
    const T kk = (k == M) ? (T)0 : (T)kxd[k];
    const int o = (k * ny + y) * nz + z;
    const cplx<T> x00 = add(ik(kk, XS[k * BP + jj]), XS[k * BP + 2 * ZC + jj]);
    const cplx<T> x01 = add(ik(kk, XS[k * BP + jj + 1]), XS[k * BP + 2 * ZC + jj + 1]);
    const cplx<T> x10 = XS[k * BP + ZC + jj], x11 = XS[k * BP + ZC + jj + 1];
    if constexpr (sizeof(T) == 4) {
      if (two && st2) {
        *reinterpret_cast<float4*>(&X0[o]) = make_float4(x00.x, x00.y, x01.x, x01.y);
        *reinterpret_cast<float4*>(&X1[o]) = make_float4(x10.x, x10.y, x11.x, x11.y);
        if constexpr (NG == 4) {
          const cplx<T> x20 = XS[k * BP + 3 * ZC + jj], x21 = XS[k * BP + 3 * ZC + jj + 1];
          *reinterpret_cast<float4*>(&X2[o]) = make_float4(x20.x, x20.y, x21.x, x21.y);
        }
        continue;
      }
    }
    X0[o] = x00;
    X1[o] = x10;
    if constexpr (NG == 4) X2[o] = XS[k * BP + 3 * ZC + jj];
    if (two) {
      X0[o + 1] = x01;
      X1[o + 1] = x11;
      if constexpr (NG == 4) X2[o + 1] = XS[k * BP + 3 * ZC + jj + 1];
    }
  }
}

// ---- inverse x: k_ix4 -------------------------------------------------------------
// Columns (warps): [0, ZC] phi at levels z0-1 .. z0+ZC-1 (one halo level),
// [ZC+1, 2ZC] d/dx phi, [2ZC+1, 3ZC] d/dy phi (psi~).  At ZC = 8 the CTA has
// the SM to itself (registers), so the state tiles the correction reads
// (u, v, w) are staged in shared memory too, requested with the spectra and
// landing during the transforms; at ZC = 2 and 4 (several CTAs per SM) they
// are prefetched into L2 and loaded into registers before the last barrier.
template <int ZC>
struct Ix4Size {
  static constexpr bool SST = (ZC == 8);  // state tiles in shared memory
  static constexpr int BG = 3 * ZC + 1;  // columns (warps)
  static constexpr int BI = 2 * ZC + 1;  // loaded spectral columns: phi (with halo), psi
  static constexpr int SR = x4_stride<ZC>();
  static constexpr size_t tables = kX4Tw * 8 + (((kX4M + 1) * 4 + 15) / 16) * 16;
  static constexpr size_t xi = (size_t)(kX4M + 1) * BI * 8;
  static constexpr size_t ex = (size_t)BG * kWEx * 8;
  static constexpr size_t zr = (size_t)BG * SR * 4;
  static constexpr size_t regA = xi > ex ? (xi > zr ? xi : zr) : (ex > zr ? ex : zr);
  static constexpr size_t state = SST ? (size_t)kX4N * (3 * ZC + 1) * 4 : 0;
  static constexpr size_t total = tables + regA + state;
};
template <int ZC>
constexpr int ix4_min_blocks() { return ZC >= 8 ? 1 : 2; }

// Inverse x-pencil kernel with the velocity correction (k_ix3 semantics at
// nx = 1024; modes IX_CORRECT, IX_STAGE, IX_REFINE; phi_out may be null outside
// IX_REFINE).  grid = (ceil(nz/ZC), ny), 32 (3 ZC + 1) threads.
template <int MODE, int ZC>
__global__ void __launch_bounds__(32 * (3 * ZC + 1), ix4_min_blocks<ZC>()) k_ix4(
    GridK g, const cplx<float>* __restrict__ phs, const cplx<float>* __restrict__ psi,
    const double* __restrict__ kxd, const cplx<float>* __restrict__ twx, const float* u_in,
    const float* v_in, const float* w_in, const float* __restrict__ bh, double sdt,
    float* u_out, float* v_out, float* w_out, float* phi_out) {
  static_assert(ZC == 2 || ZC == 4 || ZC == 8, "supported z-chunks");
  static_assert(MODE == IX_CORRECT || MODE == IX_STAGE || MODE == IX_REFINE, "modes");
  using SZ = Ix4Size<ZC>;
  constexpr bool STAGE = (MODE == IX_STAGE);
  constexpr int BG = SZ::BG, BI = SZ::BI, SR = SZ::SR, NT = 32 * BG, M = kX4M, N = kX4N;
  extern __shared__ __align__(16) unsigned char smem_dyn[];
  cplx<float>* ytw = reinterpret_cast<cplx<float>*>(smem_dyn);
  cplx<float>* twN = ytw + 512;
  cplx<float>* w32 = twN + 512;
  float* kxs = reinterpret_cast<float*>(w32 + 16);  // kx'[0..M], kx'[M] = 0
  unsigned char* regA = smem_dyn + SZ::tables;
  cplx<float>* XI = reinterpret_cast<cplx<float>*>(regA);  // [M + 1][BI]
  cplx<float>* ex = reinterpret_cast<cplx<float>*>(regA);  // BG x 16 x 33
  float* ZR = reinterpret_cast<float*>(regA);              // [BG][SR] real outputs
  constexpr bool SST = SZ::SST;
  float* SU = reinterpret_cast<float*>(regA + SZ::regA);  // [x][ZC] (SST)
  float* SV = SU + N * ZC;                                // [x][ZC]
  float* SW = SV + N * ZC;                                // [x][ZC + 1]
  const int ny = g.ny, nz = g.nz;
  const int y = blockIdx.y;
  const int z0 = blockIdx.x * ZC;
  const int zl = min(z0 + ZC, nz) - 1;  // last level of the chunk
  const int tid = threadIdx.x;

  // 1. spectral rows in one cp.async group; the state rows the correction
  //    reads are prefetched into L2 meanwhile
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
  if constexpr (SST) {
    // u, v: 16-byte copies where the chunk is whole and the rows start on 16
    // bytes, 4-byte copies otherwise; w: 4-byte copies (row stride nz + 1)
    const bool vec = z0 + ZC <= nz && (nz & 3) == 0 &&
                     ((reinterpret_cast<size_t>(u_in) | reinterpret_cast<size_t>(v_in)) & 15) == 0;
    if (vec) {
      for (int e = tid; e < N * (ZC / 4); e += NT) {
        const int x = e / (ZC / 4), q = e - x * (ZC / 4);
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
    cp_commit();
  }
  for (int x = tid; x < N; x += NT) {
    const int c = x * ny + y;
    if (!SST) {
      prefetch_run(u_in + c * nz + z0, u_in + c * nz + zl);
      prefetch_run(v_in + c * nz + z0, v_in + c * nz + zl);
      prefetch_run(w_in + c * (nz + 1) + z0, w_in + c * (nz + 1) + zl + 1);
    }
    if (STAGE) prefetch_run(bh + c * (nz + 1) + z0, bh + c * (nz + 1) + zl + 1);
    if (MODE == IX_REFINE) prefetch_run(phi_out + c * nz + z0, phi_out + c * nz + zl);
  }
  x4_tables<float>(ytw, twN, w32, twx, tid, NT);
  for (int i = tid; i <= M; i += NT) kxs[i] = (i == M) ? 0.0f : (float)kxd[i];
  if constexpr (SST)
    cp_wait<1>();  // the spectra (the state tiles may still be in flight)
  else
    cp_wait<0>();
  __syncthreads();

  // 2. gather with the C2R pre-process fused: a[q] = Z[t + 32 q] of column grp
  const int grp = tid >> 5, t = tid & 31;
  int src;
  bool dx = false;
  if (grp <= ZC) {
    src = grp;
  } else if (grp <= 2 * ZC) {
    src = grp - ZC;  // phi~ column of the same level
    dx = true;
  } else {
    src = grp - ZC;  // psi~
  }
  cplx<float> a[16];
#pragma unroll
  for (int q = 0; q < 16; ++q) {
    const int m = t + 32 * q;
    const int mc = M - m;
    cplx<float> xm = XI[m * BI + src];
    cplx<float> xc = XI[mc * BI + src];
    if (dx) {
      xm = ik(kxs[m], xm);
      xc = ik(kxs[mc], xc);
    }
    if (m == 0) {
      xm.y = 0.0f;
      xc.y = 0.0f;
    }
    xc = conjg(xc);
    const cplx<float> Sm = add(xm, xc);
    const cplx<float> D = mul(sub(xm, xc), conjg(twN[m]));
    a[q] = mk<float>(Sm.x - D.y, Sm.y + D.x);
  }
  yr_pass1<float, true>(a, t, ytw);
  __syncthreads();  // every gather done: the exchange blocks reuse the rows' space
  yr_pass2<float, true>(a, t, w32, ex + grp * kWEx);
  // a[jj] = x[2n] + i x[2n+1], n = 16 (jj + 16 p) + k2
  const int k2 = t & 15, p = t >> 4;
  // The state the correction reads (u, v, w, and b_half or phi) is loaded
  // into registers here, every pair at once, so that the loads overlap the
  // output stores and the barrier.  All loads precede all stores: the outputs
  // may alias the inputs (in-place correction), and each element is read and
  // written by the same thread only.  Two adjacent levels (z, z + 1) of a row
  // per thread; consecutive threads on consecutive pairs.
  constexpr int NPR = N * ZC / 2;          // level pairs of the tile
  constexpr int NP = (NPR + NT - 1) / NT;  // pairs per thread
  const bool st2 = (nz & 1) == 0 && ((reinterpret_cast<size_t>(u_out) |
                                      reinterpret_cast<size_t>(v_out) |
                                      reinterpret_cast<size_t>(phi_out) |
                                      reinterpret_cast<size_t>(u_in) |
                                      reinterpret_cast<size_t>(v_in)) & 7) == 0;
  float su[NP][2], sv[NP][2], sw[NP][2], gg[NP][2], lid[NP];
  auto load_state = [&]() {
  #pragma unroll
    for (int i = 0; i < NP; ++i) {
      const int e = tid + i * NT;
      const int x = e / (ZC / 2), j = 2 * (e - x * (ZC / 2));
      const int z = z0 + j;
      su[i][0] = su[i][1] = sv[i][0] = sv[i][1] = sw[i][0] = sw[i][1] = 0.0f;
      gg[i][0] = gg[i][1] = lid[i] = 0.0f;
      if (e >= NPR || z >= nz) continue;
      const bool two = z + 1 < nz;
      const int col = x * ny + y;
      const int idx = col * nz + z;
      const int wi = col * (nz + 1) + z;
      if constexpr (SST) {
        // the state comes from the shared tiles; the lid too
        if ((two ? z + 1 : z) == nz - 1 && STAGE) lid[i] = bh[col * (nz + 1) + nz];
        if (STAGE) {
          gg[i][0] = bh[wi];
          if (two) gg[i][1] = bh[wi + 1];
        } else if (MODE == IX_REFINE) {
          gg[i][0] = phi_out[idx];
          if (two) gg[i][1] = phi_out[idx + 1];
        }
        continue;
      }
      if (two && st2) {
        const float2 a2 = *reinterpret_cast<const float2*>(&u_in[idx]);
        const float2 b2 = *reinterpret_cast<const float2*>(&v_in[idx]);
        su[i][0] = a2.x;
        su[i][1] = a2.y;
        sv[i][0] = b2.x;
        sv[i][1] = b2.y;
      } else {
        su[i][0] = u_in[idx];
        sv[i][0] = v_in[idx];
        if (two) {
          su[i][1] = u_in[idx + 1];
          sv[i][1] = v_in[idx + 1];
        }
      }
      sw[i][0] = w_in[wi];
      if (two) sw[i][1] = w_in[wi + 1];
      if (STAGE) {
        gg[i][0] = bh[wi];
        if (two) gg[i][1] = bh[wi + 1];
      } else if (MODE == IX_REFINE) {
        gg[i][0] = phi_out[idx];
        if (two) gg[i][1] = phi_out[idx + 1];
      }
      // the lid, level nz, follows the column's top level nz - 1
      if ((two ? z + 1 : z) == nz - 1) {
        lid[i] = w_in[col * (nz + 1) + nz];
        if (STAGE) lid[i] = (float)arn((double)lid[i], mrn(sdt, (double)bh[col * (nz + 1) + nz]));
      }
    }
  };
  // SST: only b_half or phi come from global memory, loaded before the
  // barrier; otherwise the state is loaded after it, once the transform's
  // registers are free (several CTAs per SM cover the latency)
  if constexpr (SST) load_state();
  __syncthreads();  // every exchange read: the outputs reuse their space
  float* zr = ZR + grp * SR + 2 * k2 + 512 * p;
#pragma unroll
  for (int jj = 0; jj < 16; ++jj)
    *reinterpret_cast<float2*>(zr + 32 * jj) = make_float2(a[jj].x, a[jj].y);
  if constexpr (SST) cp_wait<0>();  // this thread's state copies have landed
  __syncthreads();
  if constexpr (!SST) load_state();

  // 3. velocity correction
  const float dzt = (float)g.dz;
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
    const int wi = col * (nz + 1) + z;
    const float phb = ZR[j * SR + x];  // level z - 1
    const float ph0 = ZR[(j + 1) * SR + x];
    const float ph1 = ZR[(j + 2) * SR + x];
    const float gx0 = ZR[(ZC + 1 + j) * SR + x], gx1 = ZR[(ZC + 2 + j) * SR + x];
    const float gy0 = ZR[(2 * ZC + 1 + j) * SR + x], gy1 = ZR[(2 * ZC + 2 + j) * SR + x];
    const float gz0 = (z >= 1) ? drn(srn(ph0, phb), dzt) : 0.0f;
    const float gz1 = drn(srn(ph1, ph0), dzt);
    float w0, w1;
    if constexpr (SST) {
      const float2 u2 = *reinterpret_cast<const float2*>(&SU[x * ZC + j]);
      const float2 v2 = *reinterpret_cast<const float2*>(&SV[x * ZC + j]);
      su[i][0] = u2.x;
      su[i][1] = u2.y;
      sv[i][0] = v2.x;
      sv[i][1] = v2.y;
      w0 = SW[x * (ZC + 1) + j];
      w1 = SW[x * (ZC + 1) + j + 1];
    } else {
      w0 = sw[i][0];
      w1 = sw[i][1];
    }
    if (STAGE) {
      w0 = (float)arn((double)w0, mrn(sdt, (double)gg[i][0]));
      w1 = (float)arn((double)w1, mrn(sdt, (double)gg[i][1]));
    }
    const float p0 = (MODE == IX_REFINE) ? gg[i][0] + ph0 : ph0;
    const float p1 = (MODE == IX_REFINE) ? gg[i][1] + ph1 : ph1;
    if (two && st2) {
      *reinterpret_cast<float2*>(&u_out[idx]) = make_float2(su[i][0] - gx0, su[i][1] - gx1);
      *reinterpret_cast<float2*>(&v_out[idx]) = make_float2(sv[i][0] - gy0, sv[i][1] - gy1);
      if (phi_out) *reinterpret_cast<float2*>(&phi_out[idx]) = make_float2(p0, p1);
    } else {
      u_out[idx] = su[i][0] - gx0;
      v_out[idx] = sv[i][0] - gy0;
      if (phi_out) phi_out[idx] = p0;
      if (two) {
        u_out[idx + 1] = su[i][1] - gx1;
        v_out[idx + 1] = sv[i][1] - gy1;
        if (phi_out) phi_out[idx + 1] = p1;
      }
    }
    w_out[wi] = w0 - gz0;
    if (two) w_out[wi + 1] = w1 - gz1;
    const int zt = two ? z + 1 : z;
    if (zt == nz - 1 && (STAGE || w_out != w_in)) {
      // SST: lid holds b_half at the lid (STAGE) and the level-nz w is in
      // the tile; otherwise lid is the finished lid value
      float wt = lid[i];
      if constexpr (SST) {
        const float wl = SW[x * (ZC + 1) + (nz - z0)];
        wt = STAGE ? (float)arn((double)wl, mrn(sdt, (double)lid[i])) : wl;
      }
      w_out[col * (nz + 1) + nz] = wt;
    }
  }
}

// ---- y pencils: ny = 1024, one warp per column ----------------------------------
// The two 512-point halves (even / odd samples) share one exchange block;
// tables from the W_1024 table twy: ytw, tw1k[k] = W_1024^k (k < 512), w32.
// NI: spectra loaded per level (2; 3 for the shared-stage form of k_fy4)
template <int ZC, int NI = 2>
struct Yr4Size {
  static constexpr int B = 2 * ZC;        // columns (warps)
  static constexpr int BP = NI * ZC + 1;  // row stride of the row tiles (odd)
  static constexpr size_t tables = (size_t)kX4Tw * sizeof(cplx<float>);
  static constexpr size_t rows = (size_t)kY4N * BP * sizeof(cplx<float>);
  static constexpr size_t ex = (size_t)B * kWEx * sizeof(cplx<float>);
  static constexpr size_t total = tables + (rows > ex ? rows : ex);
};
template <int ZC>
constexpr int yr4_min_blocks() { return ZC >= 8 ? 1 : 2; }

// One 1024-point transform of a warp's column.  e[q] = x[2 (L + 32 q)],
// o[q] = x[2 (L + 32 q) + 1] on entry; on exit e[j] = X[k], o[j] = X[k + 512],
// k = 16 (j + 16 p) + k2.  ex: the warp's exchange block (free on entry).
template <bool INV, class T = float>
__device__ __forceinline__ void y4_fft(cplx<T> (&e)[16], cplx<T> (&o)[16], int lane,
                                       const cplx<T>* __restrict__ ytw,
                                       const cplx<T>* __restrict__ w32,
                                       const cplx<T>* __restrict__ tw1k, cplx<T>* ex) {
  yr_pass1<T, INV>(e, lane, ytw);
  yr_pass2<T, INV>(e, lane, w32, ex);
  __syncwarp();  // every lane has read its pass-2 values out of ex
  yr_pass1<T, INV>(o, lane, ytw);
  yr_pass2<T, INV>(o, lane, w32, ex);
  const int k2 = lane & 15, p = lane >> 4;
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    cplx<T> w = tw1k[16 * (j + 16 * p) + k2];
    if (INV) w.y = -w.y;
    const cplx<T> wo = mul(w, o[j]);
    o[j] = sub(e[j], wo);
    e[j] = add(e[j], wo);
  }
}

// k_fy3 (FY_DIV) at ny = 1024: d^ = FFTy(X0) + i ky' FFTy(X1), single
// precision.  Columns: X0 at ZC levels, X1 at ZC levels.
// grid = (ceil(nz/ZC), nx/2 + 1), 64 ZC threads.
// AX: a fast stage from the shared x transforms (k_fx4 with NG = 4): the X0
// column is in0 + sdt in2, formed in the gather (in2 staged as a third
// group of ZC columns).
template <int ZC, bool AX = false>
__global__ void __launch_bounds__(64 * ZC, yr4_min_blocks<ZC>()) k_fy4(
    GridK g, const cplx<float>* __restrict__ in0, const cplx<float>* __restrict__ in1,
    const double* __restrict__ kyd, const cplx<float>* __restrict__ twy,
    cplx<float>* __restrict__ out0, const cplx<float>* __restrict__ in2, float sdt) {
  using SZ = Yr4Size<ZC, AX ? 3 : 2>;
  constexpr int B = SZ::B, BP = SZ::BP, NT = 32 * B, N = kY4N, NL = (AX ? 3 : 2) * ZC;
  extern __shared__ __align__(16) unsigned char smem_dyn[];
  cplx<float>* ytw = reinterpret_cast<cplx<float>*>(smem_dyn);
  cplx<float>* tw1k = ytw + 512;
  cplx<float>* w32 = tw1k + 512;
  cplx<float>* R = reinterpret_cast<cplx<float>*>(smem_dyn + SZ::tables);  // [N][BP]
  cplx<float>* ex = R;                                                    // B x 16 x 33
  const int ny = g.ny, nz = g.nz;
  const int kx = blockIdx.y;
  const int z0 = blockIdx.x * ZC;
  const int tid = threadIdx.x;
  for (int e = tid; e < N * NL; e += NT) {
    const int y = e / NL, b = e - y * NL;
    const int f = b / ZC, j = b - f * ZC;
    const int z = z0 + j;
    const bool ok = z < nz;
    const cplx<float>* src = f == 0 ? in0 : (f == 1 ? in1 : in2);
    copy_or_zero(&R[y * BP + b], src + (kx * ny + y) * nz + (ok ? z : 0), ok);
  }
  cp_commit();
  x4_tables<float>(ytw, tw1k, w32, twy, tid, NT);
  cp_wait<0>();
  __syncthreads();
  const int c = tid >> 5, lane = tid & 31;
  cplx<float> e[16], o[16];
#pragma unroll
  for (int q = 0; q < 16; ++q) {
    const int n = 2 * (lane + 32 * q);
    e[q] = R[n * BP + c];
    o[q] = R[(n + 1) * BP + c];
    if (AX && c < ZC) {  // the stage's X0 = X0 + sdt X2
      const cplx<float> e2 = R[n * BP + 2 * ZC + c], o2 = R[(n + 1) * BP + 2 * ZC + c];
      e[q] = mk<float>(fmaf(sdt, e2.x, e[q].x), fmaf(sdt, e2.y, e[q].y));
      o[q] = mk<float>(fmaf(sdt, o2.x, o[q].x), fmaf(sdt, o2.y, o[q].y));
    }
  }
  __syncthreads();  // every gather done: the exchange blocks reuse the rows' space
  y4_fft<false>(e, o, lane, ytw, w32, tw1k, ex + c * kWEx);
  __syncthreads();  // every exchange read: the output rows reuse their space
  const int k2 = lane & 15, p = lane >> 4;
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const int k = 16 * (j + 16 * p) + k2;
    R[k * BP + c] = e[j];
    R[(k + 512) * BP + c] = o[j];
  }
  __syncthreads();
  for (int e2 = tid; e2 < N * ZC; e2 += NT) {
    const int ky = e2 / ZC, j = e2 - ky * ZC;
    const int z = z0 + j;
    if (z >= nz) continue;
    const float kk = (ky == N / 2) ? 0.0f : (float)kyd[ky];
    out0[(kx * ny + ky) * nz + z] = add(R[ky * BP + j], ik(kk, R[ky * BP + ZC + j]));
  }
}

// k_iy3 at ny = 1024: phi~ = IFFTy(phi^), psi~ = IFFTy(i ky' phi^).
// Columns: phi~ at ZC levels, then psi~ (the gather applies i ky').
template <int ZC>
__global__ void __launch_bounds__(64 * ZC, yr4_min_blocks<ZC>()) k_iy4(
    GridK g, const cplx<float>* __restrict__ in0, const double* __restrict__ kyd,
    const cplx<float>* __restrict__ twy, cplx<float>* __restrict__ out0,
    cplx<float>* __restrict__ out1) {
  using SZ = Yr4Size<ZC>;
  constexpr int B = SZ::B, BP = SZ::BP, NT = 32 * B, N = kY4N;
  extern __shared__ __align__(16) unsigned char smem_dyn[];
  cplx<float>* ytw = reinterpret_cast<cplx<float>*>(smem_dyn);
  cplx<float>* tw1k = ytw + 512;
  cplx<float>* w32 = tw1k + 512;
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
  x4_tables<float>(ytw, tw1k, w32, twy, tid, NT);
  cp_wait<0>();
  __syncthreads();
  const int c = tid >> 5, lane = tid & 31;
  const int src = c < ZC ? c : c - ZC;
  cplx<float> e[16], o[16];
#pragma unroll
  for (int q = 0; q < 16; ++q) {
    const int n = 2 * (lane + 32 * q);
    e[q] = R[n * BP + src];
    o[q] = R[(n + 1) * BP + src];
    if (c >= ZC) {  // ky' = 0 at the Nyquist index
      e[q] = ik(n == N / 2 ? 0.0f : (float)kyd[n], e[q]);
      o[q] = ik((float)kyd[n + 1], o[q]);
    }
  }
  __syncthreads();
  y4_fft<true>(e, o, lane, ytw, w32, tw1k, ex + c * kWEx);
  __syncthreads();
  const int k2 = lane & 15, p = lane >> 4;
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const int k = 16 * (j + 16 * p) + k2;
    R[k * BP + c] = e[j];
    R[(k + 512) * BP + c] = o[j];
  }
  __syncthreads();
  for (int e2 = tid; e2 < N * ZC; e2 += NT) {
    const int y = e2 / ZC, j = e2 - y * ZC;
    const int z = z0 + j;
    if (z >= nz) continue;
    const int o2 = (kx * ny + y) * nz + z;
    out0[o2] = R[y * BP + j];
    out1[o2] = R[y * BP + ZC + j];
  }
}

// The defect correction's FP64 residual y transform at ny = 1024 (k_fy3
// FY_RESID at ny = 512): d^ = FFTy(X0) + i ky' FFTy(X1) in double, zero on
// the Nyquist rows (ky = ny/2 or kx = nx/2), stored as float.  Two levels of
// the two fields, one warp per column: 128 threads, 32 complex doubles per
// lane.  Rows of 2 levels (32-byte runs) against the 16-byte runs of the
// compile-time-chunk Stockham kernel, whose FP64 tiles fit only one level.
struct Yr4dSize {
  static constexpr int ZC = 2, B = 2 * ZC, BP = B + 1;
  static constexpr size_t tables = (size_t)kX4Tw * sizeof(cplx<double>);
  static constexpr size_t rows = (size_t)kY4N * BP * sizeof(cplx<double>);
  static constexpr size_t ex = (size_t)B * kWEx * sizeof(cplx<double>);
  static constexpr size_t total = tables + (rows > ex ? rows : ex);
};

__global__ void __launch_bounds__(128, 2) k_fy4d(GridK g, const cplx<double>* __restrict__ in0,
                                                 const cplx<double>* __restrict__ in1,
                                                 const double* __restrict__ kyd,
                                                 const cplx<double>* __restrict__ twy,
                                                 cplx<float>* __restrict__ out0) {
  using SZ = Yr4dSize;
  constexpr int ZC = SZ::ZC, B = SZ::B, BP = SZ::BP, NT = 32 * B, N = kY4N;
  extern __shared__ __align__(16) unsigned char smem_dyn[];
  cplx<double>* ytw = reinterpret_cast<cplx<double>*>(smem_dyn);
  cplx<double>* tw1k = ytw + 512;
  cplx<double>* w32 = tw1k + 512;
  cplx<double>* R = reinterpret_cast<cplx<double>*>(smem_dyn + SZ::tables);  // [N][BP]
  cplx<double>* ex = R;                                                     // B x 16 x 33
  const int ny = g.ny, nz = g.nz;
  const int tid = threadIdx.x;
  const int nzc = (nz + ZC - 1) / ZC;
  const int nitems = g.nxh * nzc;
  x4_tables<double>(ytw, tw1k, w32, twy, tid, NT);
  for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
  const int kx = item / nzc;
  const int z0 = (item - kx * nzc) * ZC;
  if (item + (int)gridDim.x < nitems) {
    const int nit = item + gridDim.x;
    const int k2_ = nit / nzc, za = (nit - k2_ * nzc) * ZC, zb = min(za + ZC, nz) - 1;
    for (int y = tid; y < N; y += NT) {
      const int ob = (k2_ * ny + y) * nz;
      prefetch_run(in0 + ob + za, in0 + ob + zb);
      prefetch_run(in1 + ob + za, in1 + ob + zb);
    }
  }
  for (int e = tid; e < N * B; e += NT) {
    const int y = e / B, b = e - y * B;
    const int f = b / ZC, j = b - f * ZC;
    const int z = z0 + j;
    const bool ok = z < nz;
    copy_or_zero(&R[y * BP + b], (f == 0 ? in0 : in1) + (kx * ny + y) * nz + (ok ? z : 0), ok);
  }
  cp_commit();
  cp_wait<0>();
  __syncthreads();
  const int c = tid >> 5, lane = tid & 31;
  cplx<double> e[16], o[16];
#pragma unroll
  for (int q = 0; q < 16; ++q) {
    const int n = 2 * (lane + 32 * q);
    e[q] = R[n * BP + c];
    o[q] = R[(n + 1) * BP + c];
  }
  __syncthreads();  // every gather done: the exchange blocks reuse the rows' space
  y4_fft<false, double>(e, o, lane, ytw, w32, tw1k, ex + c * kWEx);
  __syncthreads();  // every exchange read: the output rows reuse their space
  const int k2 = lane & 15, p = lane >> 4;
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const int k = 16 * (j + 16 * p) + k2;
    R[k * BP + c] = e[j];
    R[(k + 512) * BP + c] = o[j];
  }
  __syncthreads();
  for (int e2 = tid; e2 < N * ZC; e2 += NT) {
    const int ky = e2 / ZC, j = e2 - ky * ZC;
    const int z = z0 + j;
    if (z >= nz) continue;
    const double kk = (ky == N / 2) ? 0.0 : kyd[ky];
    cplx<double> d = add(R[ky * BP + j], ik(kk, R[ky * BP + ZC + j]));
    if (ky == N / 2 || kx == g.nx / 2) d = mk<double>(0.0, 0.0);
    out0[(kx * ny + ky) * nz + z] = mk<float>((float)d.x, (float)d.y);
  }
  __syncthreads();  // the next item's copies reuse the rows
  }  // item
}

}  // namespace ob
