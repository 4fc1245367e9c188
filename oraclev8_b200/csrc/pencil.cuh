// x-pencil kernels of the projection with compile-time z-chunks.
//
// Same arithmetic as k_fx (FX_DIV / FX_DIV_STAGE) and k_ix (IX_CORRECT /
// IX_STAGE / IX_REFINE) in kernels.cuh; the data movement is reorganised for
// memory-level parallelism and fewer instructions:
//  * every global input of a CTA is requested at once with cp.async
//    (global -> shared, no register staging), so a CTA's whole tile is in
//    flight in one memory round trip instead of one per batch of loads;
//  * the z-chunk ZC is a template parameter and threads own rows (x or kx)
//    and loop over the ZC levels of the row, so no index needs a division;
//  * k_ix2 loads phi~ once and forms the i kx' phi~ column in its C2R
//    pre-process instead of loading phi~ twice;
//  * the z-chunk sets the bytes a CTA moves per global sector: a row's ZC
//    levels are one contiguous run, so ZC = 8 in FP32 (32-byte runs) needs
//    half the sector operations per byte of ZC = 4.  Shared memory is laid
//    out so that ZC = 8 fits two CTAs per SM: k_ix2 stages its state tiles in
//    the FFT buffer the last pass leaves dead, and the buoyancy rows of the
//    staged kernels are read from L2 (prefetched when the CTA starts).
// Layouts are those of kernels.cuh: state (x, y, z) with z contiguous, w on
// nz + 1 levels; spectra [kx][y][z] with kx in [0, nx/2].  Element indices
// are 32-bit: plan_create bounds nx * ny * (nz + 1) by 2^31.
#pragma once
#include "kernels.cuh"

namespace ob {

// One element global -> shared with cp.async (cp_async / cp_commit / cp_wait:
// common.cuh), or a zero where the source is out of range.
template <class T>
__device__ __forceinline__ void copy_or_zero(T* dst, const T* src, bool ok) {
  if (ok)
    cp_async(dst, src, (int)sizeof(T));
  else
    *dst = (T)0;
}
template <class T>
__device__ __forceinline__ void copy_or_zero(cplx<T>* dst, const cplx<T>* src, bool ok) {
  if (ok)
    cp_async(dst, src, (int)sizeof(cplx<T>));
  else
    *dst = mk<T>((T)0, (T)0);
}

constexpr int kPencilThreads = 256;
// CTAs per SM the launch bounds target: three in FP32; two in FP64, whose
// radix-8 butterflies need more than the 80 registers three CTAs leave.
template <class T>
constexpr int pencil_min_blocks() { return sizeof(T) == 8 ? 2 : 3; }
// x pencils: two CTAs per SM at ZC = 8, where shared memory allows no more
template <class T, int ZC>
constexpr int x2_min_blocks() { return (sizeof(T) == 8 || ZC >= 8) ? 2 : 3; }

// L2 prefetch of the lines holding the run [a, b] (inclusive) of one row
template <class TS>
__device__ __forceinline__ void prefetch_run(const TS* a, const TS* b) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(a));
  if ((reinterpret_cast<size_t>(a) ^ reinterpret_cast<size_t>(b)) >> 7)
    asm volatile("prefetch.global.L2 [%0];" ::"l"(b));
}

// Shared-memory layout of k_fx2 (bytes from the dynamic base), shared by the
// kernel and the host's launch sizing.
struct Fx2Layout {
  size_t tw, bufA, bufB, raw_u, raw_v, raw_w, total;
};
template <class T, class TS, int ZC>
__host__ __device__ inline Fx2Layout fx2_layout(int nx) {
  auto al = [](size_t b) { return (b + 15) & ~size_t(15); };
  const int M = nx / 2;
  const size_t B = 3 * ZC;
  Fx2Layout L;
  L.tw = 0;
  L.bufA = al((size_t)nx * sizeof(cplx<T>));
  const size_t buf = al((size_t)(M + 1) * B * sizeof(cplx<T>));
  L.bufB = L.bufA + buf;
  // raw tiles share the second FFT buffer's space (dead until the first pass)
  L.raw_u = L.bufB;
  L.raw_v = L.raw_u + al((size_t)nx * ZC * sizeof(TS));
  L.raw_w = L.raw_v + al((size_t)nx * ZC * sizeof(TS));
  const size_t raw_end = L.raw_w + al((size_t)nx * (ZC + 1) * sizeof(TS));
  L.total = (L.bufB + buf > raw_end) ? L.bufB + buf : raw_end;
  return L;
}

// x-pencil forward kernel: rho-weighting, vertical flux divergence (STAGE:
// of w + sdt b_half, with b_half = g theta'/theta0 on half levels given as the
// field bh, read from L2), R2C along x; X0 = i kx' FFTx(rho u) + FFTx(vd),
// X1 = FFTx(rho v).  grid = (ceil(nz/ZC), ny).
template <class T, bool STAGE, class TS, int ZC>
__global__ void __launch_bounds__(kPencilThreads, x2_min_blocks<T, ZC>()) k_fx2(
    GridK g, FftPlan px, const TS* __restrict__ u, const TS* __restrict__ v,
    const TS* __restrict__ w, const TS* __restrict__ bh, double sdt,
    const double* __restrict__ rho, const double* __restrict__ rhoh,
    const double* __restrict__ kxd,
    const cplx<T>* __restrict__ twx, cplx<T>* __restrict__ X0, cplx<T>* __restrict__ X1) {
  extern __shared__ __align__(16) unsigned char smem_dyn[];
  const Fx2Layout L = fx2_layout<T, TS, ZC>(g.nx);
  cplx<T>* stw = reinterpret_cast<cplx<T>*>(smem_dyn + L.tw);
  cplx<T>* bufA = reinterpret_cast<cplx<T>*>(smem_dyn + L.bufA);
  cplx<T>* bufB = reinterpret_cast<cplx<T>*>(smem_dyn + L.bufB);
  TS* U = reinterpret_cast<TS*>(smem_dyn + L.raw_u);
  TS* V = reinterpret_cast<TS*>(smem_dyn + L.raw_v);
  TS* W = reinterpret_cast<TS*>(smem_dyn + L.raw_w);
  const int nx = g.nx, ny = g.ny, nz = g.nz, M = g.M;
  constexpr int B = 3 * ZC;
  const int y = blockIdx.y;
  const int z0 = blockIdx.x * ZC;

  // 1. the whole tile in flight at once.  Consecutive threads take
  //    consecutive levels of a row, so a warp's requests cover whole runs of
  //    each row's contiguous z segment (divisions by compile-time widths).
  for (int e = threadIdx.x; e < nx * ZC; e += kPencilThreads) {
    const int x = e / ZC, j = e - x * ZC;
    const int z = z0 + j;
    const bool ok = z < nz;
    const int gi = (x * ny + y) * nz + (ok ? z : 0);
    copy_or_zero(&U[e], u + gi, ok);
    copy_or_zero(&V[e], v + gi, ok);
  }
  for (int e = threadIdx.x; e < nx * (ZC + 1); e += kPencilThreads) {
    const int x = e / (ZC + 1), j = e - x * (ZC + 1);
    const int z = z0 + j;  // half levels z0 .. z0+ZC
    const bool ok = z <= nz;
    const int gi = (x * ny + y) * (nz + 1) + (ok ? z : 0);
    copy_or_zero(&W[e], w + gi, ok);
  }
  cp_commit();
  if (STAGE)
    for (int x = threadIdx.x; x < nx; x += kPencilThreads) {
      const TS* r = bh + (x * ny + y) * (nz + 1);
      prefetch_run(r + z0, r + min(z0 + ZC, nz));
    }
  for (int i = threadIdx.x; i < nx; i += kPencilThreads) stw[i] = twx[i];
  cp_wait<0>();
  __syncthreads();

  // 2. pack rows (2n, 2n+1) into complex inputs z[n] = f[2n] + i f[2n+1];
  //    consecutive threads on consecutive levels (shared-memory rows of B
  //    elements are not read or written with a stride of B across a warp)
  const double dz = g.dz;
  for (int e = threadIdx.x; e < M * ZC; e += kPencilThreads) {
    const int n = e / ZC, j = e - n * ZC;
    {
      const int z = z0 + j;
      const bool ok = z < nz;
      const double r = ok ? rho[z] : 0.0;
      const double rl = ok ? rhoh[z] : 0.0, ru = ok ? rhoh[z + 1] : 0.0;
      T fu[2], fv[2], fd[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int x = 2 * n + h;
        fu[h] = (T)(r * (double)U[x * ZC + j]);
        fv[h] = (T)(r * (double)V[x * ZC + j]);
        double wl = (double)W[x * (ZC + 1) + j];
        double wu = (double)W[x * (ZC + 1) + j + 1];
        if (STAGE && ok) {  // provisional stage w (integrator.py:483-490)
          const TS* r = bh + (x * ny + y) * (nz + 1) + z;
          wl = arn(wl, mrn(sdt, (double)r[0]));
          wu = arn(wu, mrn(sdt, (double)r[1]));
        }
        // the reference's operation order, rounded step by step (no FMA)
        fd[h] = ok ? (T)drn(srn(mrn(ru, wu), mrn(rl, wl)), dz) : (T)0;
      }
      bufA[n * B + j] = mk<T>(fu[0], fu[1]);
      bufA[n * B + ZC + j] = mk<T>(fv[0], fv[1]);
      bufA[n * B + 2 * ZC + j] = mk<T>(fd[0], fd[1]);
    }
  }
  __syncthreads();

  // 3. M-point FFTs of the packed rows, then the real-to-complex split
  cplx<T>* Z = fft_smem<T, false, 8>(bufA, bufB, B, px, stw, 2);
  cplx<T>* X = (Z == bufA) ? bufB : bufA;
  r2c_post<T>(Z, X, M, B, stw);
  __syncthreads();

  // 4. X0 = i kx' U + D, X1 = V (consecutive threads on consecutive levels)
  for (int e = threadIdx.x; e < (M + 1) * ZC; e += kPencilThreads) {
    const int k = e / ZC, j = e - k * ZC;
    const int z = z0 + j;
    if (z >= nz) continue;
    const T kk = (k == M) ? (T)0 : (T)kxd[k];
    const int o = (k * ny + y) * nz + z;
    const cplx<T> Uk = X[k * B + j];
    const cplx<T> Vk = X[k * B + ZC + j];
    const cplx<T> Dk = X[k * B + 2 * ZC + j];
    X0[o] = add(ik(kk, Uk), Dk);
    X1[o] = Vk;
  }
}

// Shared-memory layout of k_ix2: twiddles and the two FFT buffers.  The state
// tiles the correction reads (u, v on ZC levels, w on ZC + 1) go into the
// buffer the last FFT pass leaves dead: nx (3 ZC + 1) elements of TS, which
// the M (3 ZC + 1) complex T of either buffer hold whenever TS is no wider
// than T.
struct Ix2Layout {
  size_t tw, bufX, bufZ, total;
};
template <class T, int ZC>
__host__ __device__ inline Ix2Layout ix2_layout(int nx) {
  auto al = [](size_t b) { return (b + 15) & ~size_t(15); };
  const int M = nx / 2;
  const size_t B = 3 * ZC + 1;
  Ix2Layout L;
  L.tw = 0;
  L.bufX = al((size_t)nx * sizeof(cplx<T>));
  L.bufZ = L.bufX + al((size_t)(M + 1) * B * sizeof(cplx<T>));
  L.total = L.bufZ + al((size_t)M * B * sizeof(cplx<T>));
  return L;
}

// x-pencil inverse kernel with the velocity correction.  Columns of the batch
// (B = 3 ZC + 1): [0, ZC] phi at levels z0-1 .. z0+ZC-1 (one halo level for
// the vertical difference), [ZC+1, 2ZC] d/dx phi, [2ZC+1, 3ZC] d/dy phi.
//   IX_CORRECT: u -= gx, v -= gy, w[k] -= (phi_k - phi_{k-1}) / dz (k >= 1),
//               phi stored (tendency.py:781-788); out may alias in.
//   IX_STAGE:   out = (u_n - gx, v_n - gy, w_n + sdt b_half - gz, phi)
//               (integrator.py:483-500), b_half given as the field bh.
//   IX_REFINE:  as IX_CORRECT but phi_out += phi (a correction potential).
// In IX_CORRECT and IX_STAGE a null phi_out stores no potential (a projection
// whose potential the step overwrites unread).  grid = (ceil(nz/ZC), ny).
template <class T, int MODE, class TS, int ZC>
__global__ void __launch_bounds__(kPencilThreads, x2_min_blocks<T, ZC>()) k_ix2(
    GridK g, FftPlan px, const cplx<T>* __restrict__ phs, const cplx<T>* __restrict__ psi,
    const double* __restrict__ kxd, const cplx<T>* __restrict__ twx, const TS* u_in,
    const TS* v_in, const TS* w_in, const TS* __restrict__ bh, double sdt,
    TS* u_out, TS* v_out, TS* w_out, TS* phi_out) {
  static_assert(sizeof(TS) <= sizeof(T), "the state tiles must fit a dead FFT buffer");
  constexpr bool STAGE = (MODE == IX_STAGE);
  extern __shared__ __align__(16) unsigned char smem_dyn[];
  const Ix2Layout L = ix2_layout<T, ZC>(g.nx);
  cplx<T>* stw = reinterpret_cast<cplx<T>*>(smem_dyn + L.tw);
  cplx<T>* bufX = reinterpret_cast<cplx<T>*>(smem_dyn + L.bufX);
  cplx<T>* bufZ = reinterpret_cast<cplx<T>*>(smem_dyn + L.bufZ);
  const int nx = g.nx, ny = g.ny, nz = g.nz, M = g.M;
  constexpr int B = 3 * ZC + 1;
  const int y = blockIdx.y;
  const int z0 = blockIdx.x * ZC;
  const int zl = min(z0 + ZC, nz) - 1;  // last level of the chunk

  // 1. phi~ (with the halo level) and psi~ rows in flight at once;
  //    consecutive threads on consecutive levels of a row.  The state rows
  //    the correction reads later are prefetched into L2 meanwhile.
  constexpr int BI = 2 * ZC + 1;  // loaded spectral columns per row
  for (int e = threadIdx.x; e < (M + 1) * BI; e += kPencilThreads) {
    const int k = e / BI, b = e - k * BI;
    const int ob = (k * ny + y) * nz;
    if (b <= ZC) {
      const int z = z0 - 1 + b;
      const bool ok = z >= 0 && z < nz;
      copy_or_zero(&bufX[k * B + b], phs + ob + (ok ? z : 0), ok);
    } else {
      const int j = b - ZC - 1;
      const int z = z0 + j;
      const bool ok = z < nz;
      copy_or_zero(&bufX[k * B + 2 * ZC + 1 + j], psi + ob + (ok ? z : 0), ok);
    }
  }
  cp_commit();
  for (int x = threadIdx.x; x < nx; x += kPencilThreads) {
    const int c = x * ny + y;
    prefetch_run(u_in + c * nz + z0, u_in + c * nz + zl);
    prefetch_run(v_in + c * nz + z0, v_in + c * nz + zl);
    prefetch_run(w_in + c * (nz + 1) + z0, w_in + c * (nz + 1) + zl + 1);
    if (STAGE) prefetch_run(bh + c * (nz + 1) + z0, bh + c * (nz + 1) + zl + 1);
    if (MODE == IX_REFINE) prefetch_run(phi_out + c * nz + z0, phi_out + c * nz + zl);
  }
  for (int i = threadIdx.x; i < nx; i += kPencilThreads) stw[i] = twx[i];
  cp_wait<0>();
  __syncthreads();

  // 2. C2R pre-process of every column; the d/dx columns come from the phi~
  //    columns times i kx' (kx' = 0 at the Nyquist index M)
  for (int m = threadIdx.x; m < M; m += kPencilThreads) {
    const cplx<T> twc = conjg(stw[m]);
    const T km = (T)kxd[m];
    const T kc = (m == 0) ? (T)0 : (T)kxd[M - m];  // kx'[M] = 0
#pragma unroll
    for (int c = 0; c < B; ++c) {
      cplx<T> xm, xc;
      if (c >= ZC + 1 && c <= 2 * ZC) {
        const int src = c - ZC;  // phi~ column of the same level
        xm = ik(km, bufX[m * B + src]);
        xc = ik(kc, bufX[(M - m) * B + src]);
      } else {
        xm = bufX[m * B + c];
        xc = bufX[(M - m) * B + c];
      }
      if (m == 0) {
        xm.y = (T)0;
        xc.y = (T)0;
      }
      xc = conjg(xc);
      const cplx<T> S = add(xm, xc);
      const cplx<T> D = mul(sub(xm, xc), twc);
      bufZ[m * B + c] = mk<T>(S.x - D.y, S.y + D.x);
    }
  }
  __syncthreads();

  // 3. inverse M-point FFTs: row x of column c is rz[2 ((x>>1) B + c) + (x&1)]
  cplx<T>* Zr = fft_smem<T, true, 8>(bufZ, bufX, B, px, stw, 2);
  const T* rz = reinterpret_cast<const T*>(Zr);

  // 4. the state tiles into the buffer the last pass read (dead now)
  TS* SU = reinterpret_cast<TS*>(Zr == bufZ ? bufX : bufZ);
  TS* SV = SU + nx * ZC;
  TS* SW = SV + nx * ZC;
  for (int e = threadIdx.x; e < nx * ZC; e += kPencilThreads) {
    const int x = e / ZC, j = e - x * ZC;
    const int z = z0 + j;
    const bool ok = z < nz;
    const int gi = (x * ny + y) * nz + (ok ? z : 0);
    copy_or_zero(&SU[e], u_in + gi, ok);
    copy_or_zero(&SV[e], v_in + gi, ok);
  }
  for (int e = threadIdx.x; e < nx * (ZC + 1); e += kPencilThreads) {
    const int x = e / (ZC + 1), j = e - x * (ZC + 1);
    const int z = z0 + j;  // half levels z0 .. z0+ZC
    const bool ok = z <= nz;
    copy_or_zero(&SW[e], w_in + (x * ny + y) * (nz + 1) + (ok ? z : 0), ok);
  }
  cp_commit();
  cp_wait<0>();
  __syncthreads();

  // 5. velocity correction; consecutive threads on consecutive levels
  const T dzt = (T)g.dz;
  for (int e = threadIdx.x; e < nx * ZC; e += kPencilThreads) {
    const int x = e / ZC, j = e - x * ZC;
    const int z = z0 + j;
    if (z >= nz) continue;
    const int col = x * ny + y;
    const int rb = 2 * ((x >> 1) * B) + (x & 1);
    const int idx = col * nz + z;
    const T phi = rz[rb + 2 * (j + 1)];
    const T phib = rz[rb + 2 * j];
    const T gx = rz[rb + 2 * (ZC + 1 + j)];
    const T gy = rz[rb + 2 * (2 * ZC + 1 + j)];
    const T gz = (z >= 1) ? (T)drn(srn(phi, phib), dzt) : (T)0;
    const int sw = x * (ZC + 1) + j;
    const int wi = col * (nz + 1) + z;
    TS wcz = SW[sw], wt = (TS)0;
    if (STAGE) wcz = (TS)arn((double)wcz, mrn(sdt, (double)bh[wi]));
    if (z == nz - 1) {
      wt = SW[sw + 1];
      if (STAGE) wt = (TS)arn((double)wt, mrn(sdt, (double)bh[wi + 1]));
    }
    u_out[idx] = (TS)((T)SU[e] - gx);
    v_out[idx] = (TS)((T)SV[e] - gy);
    w_out[wi] = (TS)((T)wcz - gz);
    if (z == nz - 1 && (STAGE || w_out != w_in)) w_out[wi + 1] = wt;
    if (MODE == IX_REFINE)
      phi_out[idx] = (TS)((T)phi_out[idx] + phi);
    else if (phi_out)  // null: the caller discards this projection's potential
      phi_out[idx] = (TS)phi;
  }
}

// ---- y pencils ---------------------------------------------------------------
// Same arithmetic as k_fy (FY_DIV / FY_RESID) and k_iy (IY_GRAD), with the
// data movement of the x2 kernels: cp.async tiles, compile-time z-chunk,
// level-fastest thread mapping.  grid = (ceil(nz/ZC), nx/2 + 1).
template <class T, int ZC>
__host__ __device__ inline size_t y2_smem(int ny) {
  auto al = [](size_t b) { return (b + 15) & ~size_t(15); };
  return al((size_t)ny * sizeof(cplx<T>)) + 2 * al((size_t)ny * 2 * ZC * sizeof(cplx<T>));
}

// d^ = FFTy(X1) + i ky' FFTy(X2) (FY_DIV); FY_RESID also zeroes the Nyquist
// rows (kx = nx/2 or ky = ny/2) and may round the result to TO.
template <class T, int MODE, class TO, int ZC>
__global__ void __launch_bounds__(kPencilThreads, pencil_min_blocks<T>()) k_fy2(
    GridK g, FftPlan py, const cplx<T>* __restrict__ in0, const cplx<T>* __restrict__ in1,
    const double* __restrict__ kyd, const cplx<T>* __restrict__ twy,
    cplx<nd_t<TO>>* __restrict__ out0) {
  extern __shared__ __align__(16) unsigned char smem_dyn[];
  constexpr int B = 2 * ZC;
  const int ny = g.ny, nz = g.nz;
  cplx<T>* stw = reinterpret_cast<cplx<T>*>(smem_dyn);
  cplx<T>* bufA = reinterpret_cast<cplx<T>*>(smem_dyn + (((size_t)ny * sizeof(cplx<T>) + 15) & ~size_t(15)));
  cplx<T>* bufB = bufA + (size_t)ny * B;
  const int kx = blockIdx.y;
  const int z0 = blockIdx.x * ZC;
  for (int e = threadIdx.x; e < ny * B; e += kPencilThreads) {
    const int y = e / B, b = e - y * B;
    const int f = b / ZC, j = b - f * ZC;
    const int z = z0 + j;
    const bool ok = z < nz;
    const int o = (kx * ny + y) * nz + (ok ? z : 0);
    copy_or_zero(&bufA[e], (f == 0 ? in0 : in1) + o, ok);
  }
  cp_commit();
  for (int i = threadIdx.x; i < ny; i += kPencilThreads) stw[i] = twy[i];
  cp_wait<0>();
  __syncthreads();
  cplx<T>* R = fft_smem<T, false, 8>(bufA, bufB, B, py, stw, 1);
  for (int e = threadIdx.x; e < ny * ZC; e += kPencilThreads) {
    const int ky = e / ZC, j = e - ky * ZC;
    const int z = z0 + j;
    if (z >= nz) continue;
    const T kk = (ky == ny / 2) ? (T)0 : (T)kyd[ky];
    cplx<T> d = add(R[ky * B + j], ik(kk, R[ky * B + ZC + j]));
    if (MODE == FY_RESID && (ky == ny / 2 || kx == g.nx / 2)) d = mk<T>((T)0, (T)0);
    out0[(kx * ny + ky) * nz + z] = mk<TO>((TO)d.x, (TO)d.y);
  }
}

// phi~ = IFFTy(phi^), psi~ = IFFTy(i ky' phi^) (IY_GRAD with unit scale).
template <class T, int ZC>
__global__ void __launch_bounds__(kPencilThreads, pencil_min_blocks<T>()) k_iy2(
    GridK g, FftPlan py, const cplx<T>* __restrict__ in0, const double* __restrict__ kyd,
    const cplx<T>* __restrict__ twy, cplx<T>* __restrict__ out0, cplx<T>* __restrict__ out1) {
  extern __shared__ __align__(16) unsigned char smem_dyn[];
  constexpr int B = 2 * ZC;
  const int ny = g.ny, nz = g.nz;
  cplx<T>* stw = reinterpret_cast<cplx<T>*>(smem_dyn);
  cplx<T>* bufA = reinterpret_cast<cplx<T>*>(smem_dyn + (((size_t)ny * sizeof(cplx<T>) + 15) & ~size_t(15)));
  cplx<T>* bufB = bufA + (size_t)ny * B;
  const int kx = blockIdx.y;
  const int z0 = blockIdx.x * ZC;
  for (int e = threadIdx.x; e < ny * ZC; e += kPencilThreads) {
    const int ky = e / ZC, j = e - ky * ZC;
    const int z = z0 + j;
    const bool ok = z < nz;
    copy_or_zero(&bufA[ky * B + j], in0 + (kx * ny + ky) * nz + (ok ? z : 0), ok);
  }
  cp_commit();
  for (int i = threadIdx.x; i < ny; i += kPencilThreads) stw[i] = twy[i];
  cp_wait<0>();
  __syncthreads();
  // the d/dy columns: i ky' phi^ (ky' = 0 at the Nyquist row)
  for (int e = threadIdx.x; e < ny * ZC; e += kPencilThreads) {
    const int ky = e / ZC, j = e - ky * ZC;
    const T kk = (ky == ny / 2) ? (T)0 : (T)kyd[ky];
    bufA[ky * B + ZC + j] = ik(kk, bufA[ky * B + j]);
  }
  __syncthreads();
  cplx<T>* R = fft_smem<T, true, 8>(bufA, bufB, B, py, stw, 1);
  for (int e = threadIdx.x; e < ny * ZC; e += kPencilThreads) {
    const int y = e / ZC, j = e - y * ZC;
    const int z = z0 + j;
    if (z >= nz) continue;
    const int o = (kx * ny + y) * nz + z;
    out0[o] = R[y * B + j];
    out1[o] = R[y * B + ZC + j];
  }
}

// Half-level buoyancy field b_half (nz + 1 levels, zero at surface and lid)
// of theta' (equation_set.py:255-263, staggering.py:201-208), with the
// operation order of bhalf(): the fast stages of a step all use the buoyancy
// of the same theta', so it is formed once per step.  One warp per column.
// gth (single-precision plans): g / theta0 per level as float; the field is
// then formed in float, 0.5 (gth[k-1] th[k-1] + gth[k] th[k]), without the
// double divisions.
template <class T>
__global__ void __launch_bounds__(256) k_bhalf(GridK g, const T* __restrict__ th,
                                               const double* __restrict__ theta0,
                                               const float* __restrict__ gth,
                                               T* __restrict__ bh) {
  const int lane = threadIdx.x & 31;
  const long ncol = (long)g.nx * g.ny;
  const int nz = g.nz;
  for (long c = (long)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5); c < ncol;
       c += (long)gridDim.x * (blockDim.x / 32)) {
    const T* thc = th + c * nz;
    if (sizeof(T) == 4 && gth) {
      for (int k = lane; k <= nz; k += 32)
        bh[c * (nz + 1) + k] =
            (k <= 0 || k >= nz)
                ? (T)0
                : (T)(0.5f * (gth[k - 1] * (float)thc[k - 1] + gth[k] * (float)thc[k]));
    } else {
      for (int k = lane; k <= nz; k += 32) bh[c * (nz + 1) + k] = (T)bhalf(thc, k, nz, theta0);
    }
  }
}

}  // namespace ob
