// Device kernels of the LH82 anelastic step.
//
// Projection pipeline (AnelasticProjection.apply_projection,
// oracle_v8/solver/tendency.py:717-790), spectral layout [kx][y|ky][z] with
// kx in [0, nx/2] (real FFT along x), z contiguous:
//   k_fx     x-pencils (fixed y, z-chunk): rho-weighting, vertical flux
//            divergence, R2C along x; emits X1 = i kx' FFTx(rho u) + FFTx(vd)
//            and X2 = FFTx(rho v).
//   k_fy     y-pencils (fixed kx, z-chunk): C2C along y; d^ = FFTy(X1) +
//            i ky' FFTy(X2).
//   k_thomas columns (kx, ky): batched Thomas in z with the zero mode solved on
//            its reduced system; phi^ scaled by 1/(nx ny).
//   k_iy     y-pencils: phi~ = IFFTy(phi^), psi~ = IFFTy(i ky' phi^).
//   k_ix     x-pencils: C2R along x of phi~, i kx' phi~, psi~; applies the
//            velocity correction u -= dphi/dx, v -= dphi/dy,
//            w -= (phi_k - phi_{k-1})/dz and stores phi.
// kx' and ky' are the wavenumbers with the Nyquist entry zeroed: the reference
// takes real(ifft2(i k f^)), which removes exactly that component
// (tendency.py:428-431, 487-491).
#pragma once
#include "fft.cuh"

namespace ob {

// ---------------------------------------------------------------------------
// Buoyancy on half levels: b_half[k] = 0.5 (b[k-1] + b[k]), b = g theta'/theta0,
// zero at surface and lid (equation_set.py:255-263, staggering.py:201-208).
// ---------------------------------------------------------------------------
template <class T>
__device__ __forceinline__ double bhalf(const T* __restrict__ thc, int k, int nz,
                                        const double* __restrict__ theta0) {
  if (k <= 0 || k >= nz) return 0.0;
  const double b0 = drn(mrn(kGravity, (double)thc[k - 1]), theta0[k - 1]);
  const double b1 = drn(mrn(kGravity, (double)thc[k]), theta0[k]);
  return mrn(0.5, arn(b0, b1));
}

// Stage provisional w: w_n + sdt * b_half (integrator.py:483-490).
template <class T>
__device__ __forceinline__ double stage_w(const T* __restrict__ wc, const T* __restrict__ thc,
                                          int k, int nz, double sdt,
                                          const double* __restrict__ theta0) {
  return arn((double)wc[k], mrn(sdt, bhalf(thc, k, nz, theta0)));
}

// Non-deduced alias: template arguments given explicitly (or defaulted) are not
// re-deduced from pointer arguments, so nullptr can be passed for unused ones.
template <class X>
struct nd {
  using type = X;
};
template <class X>
using nd_t = typename nd<X>::type;

// global loads each thread issues before consuming them (memory-level parallelism)
constexpr int kLoadBatch = 4;
// state values per thread k_ix prefetches ahead of its FFT
constexpr int kIxPrefetch = 4;

enum FxMode { FX_DIV = 0, FX_DIV_STAGE = 1, FX_FIELDS = 2 };

// x-pencil forward kernel.  grid = (ny, ceil(nz/zc)).  smem: 2 * (M+1) * B cplx.
// FX_FIELDS transforms `nf` real fields f0..f2 (no weighting) into X0..X2.
template <class T, int MODE, class TS = T>
__global__ void __launch_bounds__(256, 2) k_fx(GridK g, FftPlan px, int zc, int nf,
                                            const nd_t<TS>* __restrict__ f0,
                                            const nd_t<TS>* __restrict__ f1,
                                            const nd_t<TS>* __restrict__ f2,
                                            const nd_t<TS>* __restrict__ th,
                                            double sdt, const double* __restrict__ rho,
                                            const double* __restrict__ rhoh,
                                            const double* __restrict__ theta0,
                                            const double* __restrict__ kxd,
                                            const cplx<T>* __restrict__ twx,
                                            cplx<T>* __restrict__ X0, cplx<T>* __restrict__ X1,
                                            cplx<T>* __restrict__ X2) {
  extern __shared__ __align__(16) unsigned char smem_dyn[];
  // twiddle table staged in shared memory (off the butterflies' critical path)
  cplx<T>* stw = reinterpret_cast<cplx<T>*>(smem_dyn);
  for (int i = threadIdx.x; i < g.nx; i += blockDim.x) stw[i] = twx[i];
  unsigned char* smem_raw = smem_dyn + ((((size_t)g.nx) * sizeof(cplx<T>) + 15) & ~size_t(15));
  const int NF = (MODE == FX_FIELDS) ? nf : 3;
  const int B = NF * zc;
  const int M = g.M;
  cplx<T>* bufA = reinterpret_cast<cplx<T>*>(smem_raw);
  cplx<T>* bufB = bufA + (size_t)(M + 1) * B;
  const int y = blockIdx.y;
  const int z0 = blockIdx.x * zc;
  const int zn = min(zc, g.nz - z0);
  const int nz = g.nz;
  T* rA = reinterpret_cast<T*>(bufA);

  // Load phase: each thread gathers kLoadBatch elements into registers before
  // writing shared memory, so that many global loads are in flight at once.
  const int nel = g.nx * zc;
  for (int e0 = threadIdx.x; e0 < nel; e0 += kLoadBatch * blockDim.x) {
    T va[kLoadBatch][3];
#pragma unroll
    for (int q = 0; q < kLoadBatch; ++q) {
      const int e = e0 + q * blockDim.x;
      va[q][0] = va[q][1] = va[q][2] = (T)0;
      const int x = e / zc;
      const int zl = e - x * zc;
      if (e < nel && zl < zn) {
        const size_t col = (size_t)x * g.ny + y;
        const int z = z0 + zl;
        if (MODE == FX_FIELDS) {
          va[q][0] = (T)f0[col * nz + z];
          if (NF > 1) va[q][1] = (T)f1[col * nz + z];
          if (NF > 2) va[q][2] = (T)f2[col * nz + z];
        } else {
          const double r = rho[z];
          va[q][0] = (T)(r * (double)f0[col * nz + z]);
          va[q][1] = (T)(r * (double)f1[col * nz + z]);
          const TS* wc = f2 + col * (nz + 1);
          double wl, wu;
          if (MODE == FX_DIV_STAGE) {
            const TS* thc = th + col * nz;
            wl = stage_w(wc, thc, z, nz, sdt, theta0);
            wu = stage_w(wc, thc, z + 1, nz, sdt, theta0);
          } else {
            wl = (double)wc[z];
            wu = (double)wc[z + 1];
          }
          va[q][2] = (T)((rhoh[z + 1] * wu - rhoh[z] * wl) / g.dz);
        }
      }
    }
#pragma unroll
    for (int q = 0; q < kLoadBatch; ++q) {
      const int e = e0 + q * blockDim.x;
      if (e >= nel) continue;
      const int x = e / zc;
      const int zl = e - x * zc;
      const int n = x >> 1, odd = x & 1;
#pragma unroll
      for (int f = 0; f < 3; ++f)
        if (f < NF) rA[2 * ((size_t)n * B + f * zc + zl) + odd] = va[q][f];
    }
  }
  __syncthreads();
  cplx<T>* Z = fft_smem<T, false, 4>(bufA, bufB, B, px, stw, 2);
  cplx<T>* X = (Z == bufA) ? bufB : bufA;
  r2c_post<T>(Z, X, M, B, stw);
  __syncthreads();

  const int nout = (M + 1) * zc;
  for (int e = threadIdx.x; e < nout; e += blockDim.x) {
    const int k = e / zc;
    const int zl = e - k * zc;
    if (zl >= zn) continue;
    const size_t o = ((size_t)k * g.ny + y) * nz + z0 + zl;
    if (MODE == FX_FIELDS) {
      for (int f = 0; f < NF; ++f) {
        cplx<T>* dst = f == 0 ? X0 : (f == 1 ? X1 : X2);
        dst[o] = X[(size_t)k * B + f * zc + zl];
      }
    } else {
      const T kk = (k == M) ? (T)0 : (T)kxd[k];
      const cplx<T> U = X[(size_t)k * B + zl];
      const cplx<T> V = X[(size_t)k * B + zc + zl];
      const cplx<T> D = X[(size_t)k * B + 2 * zc + zl];
      X0[o] = add(ik(kk, U), D);
      X1[o] = V;
    }
  }
}

enum FyMode { FY_DIV = 0, FY_FIELDS = 1, FY_HELM = 2, FY_RESID = 3 };

// y-pencil forward kernel.  grid = (nxh, ceil(nz/zc)).  smem: 2 * ny * B cplx.
// FY_DIV: out0 = FFTy(in0) + i ky' FFTy(in1).
// FY_RESID: FY_DIV with the Nyquist rows (kx = nx/2 or ky = ny/2) set to
//   zero: the residual of a defect correction.  The projection cannot make
//   those modes divergence-free (the spectral derivative drops them), so a
//   second projection would only move them; the correction leaves them as
//   the first projection put them.
// FY_FIELDS: out_f = FFTy(in_f) for f < nf.
// FY_HELM: the Helmholtz divergent-part multipliers (tendency.py:1800-1839),
//   out0 = s (Kx^2/K^2 U + (KxKy/K^2)' V), out1 = s ((KxKy/K^2)' U + Ky^2/K^2 V),
//   s = scale; the primed cross term is zero where exactly one of kx, ky is
//   the Nyquist index (there the reference's real() drops it).
// TO: type of the FY_DIV output (narrower than T for the defect correction,
// whose residual divergence is formed in double and handed to a
// single-precision solve); the other modes write T.
template <class T, int MODE, class TO = T>
__global__ void __launch_bounds__(256, 2) k_fy(GridK g, FftPlan py, int zc, int nf,
                                            const cplx<T>* __restrict__ in0,
                                            const cplx<T>* __restrict__ in1,
                                            const double* __restrict__ kxd,
                                            const double* __restrict__ kyd,
                                            const cplx<T>* __restrict__ twy, double scale,
                                            cplx<nd_t<TO>>* __restrict__ out0,
                                            cplx<T>* __restrict__ out1) {
  extern __shared__ __align__(16) unsigned char smem_dyn[];
  // twiddle table staged in shared memory (off the butterflies' critical path)
  cplx<T>* stw = reinterpret_cast<cplx<T>*>(smem_dyn);
  for (int i = threadIdx.x; i < g.ny; i += blockDim.x) stw[i] = twy[i];
  unsigned char* smem_raw = smem_dyn + ((((size_t)g.ny) * sizeof(cplx<T>) + 15) & ~size_t(15));
  const int NF = (MODE == FY_FIELDS) ? nf : 2;
  const int B = NF * zc;
  const int ny = g.ny, nz = g.nz;
  cplx<T>* bufA = reinterpret_cast<cplx<T>*>(smem_raw);
  cplx<T>* bufB = bufA + (size_t)ny * B;
  const int kx = blockIdx.y;
  const int z0 = blockIdx.x * zc;
  const int zn = min(zc, nz - z0);
  const int nel = ny * zc;
  for (int e0 = threadIdx.x; e0 < nel; e0 += kLoadBatch * blockDim.x) {
    cplx<T> va[kLoadBatch][2];
#pragma unroll
    for (int q = 0; q < kLoadBatch; ++q) {
      const int e = e0 + q * blockDim.x;
      const int y = e / zc;
      const int zl = e - y * zc;
      va[q][0] = va[q][1] = mk<T>((T)0, (T)0);
      if (e < nel && zl < zn) {
        const size_t o = ((size_t)kx * ny + y) * nz + z0 + zl;
        va[q][0] = in0[o];
        if (NF > 1) va[q][1] = in1[o];
      }
    }
#pragma unroll
    for (int q = 0; q < kLoadBatch; ++q) {
      const int e = e0 + q * blockDim.x;
      if (e >= nel) continue;
      const int y = e / zc;
      const int zl = e - y * zc;
#pragma unroll
      for (int f = 0; f < 2; ++f)
        if (f < NF) bufA[(size_t)y * B + f * zc + zl] = va[q][f];
    }
  }
  __syncthreads();
  cplx<T>* R = fft_smem<T, false, 4>(bufA, bufB, B, py, stw, 1);
  for (int e = threadIdx.x; e < nel; e += blockDim.x) {
    const int ky = e / zc;
    const int zl = e - ky * zc;
    if (zl >= zn) continue;
    const size_t o = ((size_t)kx * ny + ky) * nz + z0 + zl;
    if (MODE == FY_DIV || MODE == FY_RESID) {
      const T kk = (ky == ny / 2) ? (T)0 : (T)kyd[ky];
      cplx<T> d = add(R[(size_t)ky * B + zl], ik(kk, R[(size_t)ky * B + zc + zl]));
      if (MODE == FY_RESID && (ky == ny / 2 || kx == g.nx / 2)) d = mk<T>((T)0, (T)0);
      out0[o] = mk<TO>((TO)d.x, (TO)d.y);
    } else if constexpr (MODE == FY_FIELDS) {
      for (int f = 0; f < NF; ++f) (f == 0 ? out0 : out1)[o] = R[(size_t)ky * B + f * zc + zl];
    } else {
      const double Kx = kxd[kx], Ky = kyd[ky];
      const double K2 = Kx * Kx + Ky * Ky;
      double mxx = 0, myy = 0, mxy = 0;
      if (K2 > 0) {
        mxx = Kx * Kx / K2;
        myy = Ky * Ky / K2;
        const bool nyqx = (kx == g.nx / 2), nyqy = (ky == ny / 2);
        mxy = (nyqx != nyqy) ? 0.0 : Kx * Ky / K2;
      }
      const cplx<T> U = R[(size_t)ky * B + zl];
      const cplx<T> V = R[(size_t)ky * B + zc + zl];
      const T sxx = (T)(scale * mxx), syy = (T)(scale * myy), sxy = (T)(scale * mxy);
      out0[o] = mk<TO>(sxx * U.x + sxy * V.x, sxx * U.y + sxy * V.y);
      out1[o] = mk<T>(sxy * U.x + syy * V.x, sxy * U.y + syy * V.y);
    }
  }
}

// Thomas tables (double, device), built on the host exactly as
// poisson.py:286-325 builds them.
struct ThomasK {
  const double* a;     // (nz) sub-diagonal, a[0] = 0
  const double* c;     // (nz) super-diagonal, c[nz-1] = 0
  const double* negs;  // (nz) mode-independent part of the diagonal
  const double* rho;   // (nz) rho on full levels (multiplies k^2)
  const double* rhoh;  // (nz+1) rho on half levels (residual operator)
  const double* kx;    // (nx) 2 pi fftfreq
  const double* ky;    // (ny)
  const double* a0;    // (nz-1) zero-mode reduced system
  const double* cp0;
  const double* inv0;
  double dz;
  double scale;        // 1 / (nx ny): inverse-FFT normalisation folded in
};

// Byte offset of a k_thomas CTA's staged columns: after the zero-mode region
// (3 P doubles), rounded up to 16 bytes for the cp.async copies.
__host__ __device__ inline size_t thomas_stage_offset(int P) {
  return ((size_t)3 * P * 8 + 15) & ~size_t(15);
}

// Batched Thomas, one thread per spectral column (kx, ky).  Columns are
// staged through shared memory (coalesced loads of TC consecutive columns);
// the recurrence runs in double with the reference's operation order and no
// FMA contraction (poisson.py:334-383).  diag != nullptr records the
// compatibility residual (poisson.py:233-236) in diag[slot_c] and the
// Parseval form of the discrete-operator residual (poisson.py:263-268) as a
// raw sum of weighted |r^|^2 in diag[slot_d] (normalised on the host).
// dh and ph may alias: a CTA reads only its own columns before writing them.
// The modes are staged and swept in R.  FP64 plans use double throughout (the
// reference's arithmetic).  FP32 plans run two launches over disjoint column
// blocks: the blocks holding a long-wave mode, k^2 Lz^2 < 1, in double, since
// these nearly singular columns amplify rounding by about 1/(k Lz)^2, and
// all other blocks in single precision, with half the shared memory per
// column and so twice the columns in flight per SM.  `blocks` (optional)
// lists the column blocks of the launch (blockIdx.x indexes it); `skip`
// (optional) flags blocks the launch leaves alone.  The zero mode (in the
// first block) is always solved in double, in its own region.
template <class T, int TC, class R = double>
__global__ void __launch_bounds__(TC) k_thomas(GridK g, ThomasK t, const cplx<T>* dh,
                                               cplx<T>* ph, double* diag, int slot_c,
                                               int slot_d, const int* blocks = nullptr,
                                               const unsigned char* skip = nullptr) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const long blk = blocks ? (long)blocks[blockIdx.x] : (long)blockIdx.x;
  if (skip && skip[blk]) return;  // uniform across the block
  const int nz = g.nz;
  const int P = nz + 1;  // padded column stride (bank spread)
  // IL: the sweep type is the data type, so the CTA's columns (one
  // contiguous block) are staged as interleaved (re, im) pairs by cp.async,
  // every copy in flight at once; otherwise converted on the way in.
  constexpr bool IL = sizeof(R) == sizeof(T);
  constexpr int S = IL ? 2 : 1;  // element stride of a staged re / im row
  double* zre = reinterpret_cast<double*>(smem_raw);  // zero mode: P real parts
  double* zim = zre + P;                                // P imag parts
  double* zcp = zim + P;                                // P source copy
  R* sre = reinterpret_cast<R*>(smem_raw + thomas_stage_offset(P));  // TC * P real parts
  R* sim = IL ? sre + 1 : sre + (size_t)TC * P;                      // TC * P imag parts
  R* scp = sre + (size_t)2 * TC * P;                                 // TC * P c' factors
  const long ncols = (long)g.nxh * g.ny;
  const long c0 = blk * TC;
  const int ncl = (int)min((long)TC, ncols - c0);
  const long base = c0 * nz;
  if constexpr (IL) {
    cplx<R>* sc = reinterpret_cast<cplx<R>*>(sre);
    for (int cl = 0; cl < ncl; ++cl)
      for (int k = threadIdx.x; k < nz; k += TC)
        cp_async(&sc[cl * P + k], dh + base + (long)cl * nz + k, (int)sizeof(cplx<T>));
    cp_commit();
    cp_wait<0>();
  } else if constexpr (sizeof(cplx<T>) <= sizeof(R)) {
    // a wider sweep type (FP32 data, FP64 sweep): the pairs are staged by
    // cp.async in the c' area (unused until the sweep, and exactly their
    // size), then widened into the sweep's rows
    cplx<T>* stg = reinterpret_cast<cplx<T>*>(scp);
    for (int cl = 0; cl < ncl; ++cl)
      for (int k = threadIdx.x; k < nz; k += TC)
        cp_async(&stg[cl * P + k], dh + base + (long)cl * nz + k, (int)sizeof(cplx<T>));
    cp_commit();
    cp_wait<0>();
    __syncthreads();
    for (int e = threadIdx.x; e < ncl * nz; e += TC) {
      const int cl = e / nz;
      const int k = e - cl * nz;
      const cplx<T> v = stg[cl * P + k];
      sre[cl * P + k] = (R)v.x;
      sim[cl * P + k] = (R)v.y;
    }
  } else {
    for (int e = threadIdx.x; e < ncl * nz; e += TC) {
      const int cl = e / nz;
      const int k = e - cl * nz;
      const cplx<T> v = dh[base + e];
      sre[cl * P + k] = (R)v.x;
      sim[cl * P + k] = (R)v.y;
    }
  }
  __syncthreads();
  const int cl = threadIdx.x;
  double resid = 0.0;
  if (cl < ncl) {
    const long col = c0 + cl;
    const int kxi = (int)(col / g.ny);
    const int kyi = (int)(col - (long)kxi * g.ny);
    if (col == 0) {
      double* re = zre;
      double* im = zim;
      double* cp = zcp;
      for (int k = 0; k < nz; ++k) {
        re[k] = (double)sre[k * S];
        im[k] = (double)sim[k * S];
      }
      // Zero mode (poisson.py:233-236, 256, 316-325, 367-383): compatibility
      // residual, removal of the column mean, then the reduced (nz-1) system
      // on levels 1..nz-1 with phi(0,0,0) pinned to 0.
      double sr = 0, si = 0;
      for (int k = 0; k < nz; ++k) {
        sr = arn(sr, re[k]);
        si = arn(si, im[k]);
      }
      if (diag) diag[slot_c] = hypot(mrn(sr, t.dz), mrn(si, t.dz));
      const double mr = drn(sr, (double)nz), mi = drn(si, (double)nz);
      for (int k = 0; k < nz; ++k) cp[k] = re[k];  // source, kept for the residual
      const int n0 = nz - 1;
      double pr = mrn(srn(re[1], mr), t.inv0[0]);
      double pi = mrn(srn(im[1], mi), t.inv0[0]);
      re[1] = pr;
      im[1] = pi;
      for (int j = 1; j < n0; ++j) {
        pr = mrn(srn(srn(re[j + 1], mr), mrn(t.a0[j], pr)), t.inv0[j]);
        pi = mrn(srn(srn(im[j + 1], mi), mrn(t.a0[j], pi)), t.inv0[j]);
        re[j + 1] = pr;
        im[j + 1] = pi;
      }
      double xr = pr, xi = pi;
      for (int j = n0 - 2; j >= 0; --j) {
        xr = srn(re[j + 1], mrn(t.cp0[j], xr));
        xi = srn(im[j + 1], mrn(t.cp0[j], xi));
        re[j + 1] = xr;
        im[j + 1] = xi;
      }
      re[0] = 0.0;
      im[0] = 0.0;
      if (diag) {
        // The zero mode of a real field is real.  Residual against the
        // original source, with its z-mean (the domain mean of the physical
        // residual) removed.
        const double dz2 = t.dz * t.dz;
        double rsum = 0, r2 = 0;
        for (int k = 0; k < nz; ++k) {
          const double fu = (k < nz - 1) ? t.rhoh[k + 1] * (re[k + 1] - re[k]) : 0.0;
          const double fl = (k > 0) ? t.rhoh[k] * (re[k] - re[k - 1]) : 0.0;
          const double r = (fu - fl) / dz2 - cp[k];
          rsum += r;
          r2 += r * r;
        }
        resid = r2 - rsum * rsum / nz;
      }
      for (int k = 0; k < nz; ++k) {
        sre[k * S] = (R)re[k];
        sim[k * S] = (R)im[k];
      }
    } else {
      R* re = sre + cl * P * S;
      R* im = sim + cl * P * S;
      R* cp = scp + cl * P;
      const double kx = t.kx[kxi], ky = t.ky[kyi];
      const double ksq = arn(mrn(kx, kx), mrn(ky, ky));
      R b = (R)srn(t.negs[0], mrn(ksq, t.rho[0]));
      R inv = rcprn(b);
      R cpp = mrn((R)t.c[0], inv);
      cp[0] = cpp;
      R pr = mrn(re[0], inv), pi = mrn(im[0], inv);
      re[0] = pr;
      im[0] = pi;
#pragma unroll 4
      for (int k = 1; k < nz; ++k) {
        b = (R)srn(t.negs[k], mrn(ksq, t.rho[k]));
        const R ak = (R)t.a[k];
        const R den = srn(b, mrn(ak, cpp));
        inv = rcprn(den);
        if (k < nz - 1) {
          cpp = mrn((R)t.c[k], inv);
          cp[k] = cpp;
        }
        pr = mrn(srn(re[k * S], mrn(ak, pr)), inv);
        pi = mrn(srn(im[k * S], mrn(ak, pi)), inv);
        re[k * S] = pr;
        im[k * S] = pi;
      }
      R xr = pr, xi = pi;
      for (int k = nz - 2; k >= 0; --k) {
        xr = srn(re[k * S], mrn(cp[k], xr));
        xi = srn(im[k * S], mrn(cp[k], xi));
        re[k * S] = xr;
        im[k * S] = xi;
      }
      if (diag) {
        // r^ = L phi^ - d^, source re-read from global memory
        const double dz2 = t.dz * t.dz;
        double acc = 0;
        for (int k = 0; k < nz; ++k) {
          const double fur = (k < nz - 1) ? t.rhoh[k + 1] * (re[(k + 1) * S] - re[k * S]) : 0.0;
          const double fui = (k < nz - 1) ? t.rhoh[k + 1] * (im[(k + 1) * S] - im[k * S]) : 0.0;
          const double flr = (k > 0) ? t.rhoh[k] * (re[k * S] - re[(k - 1) * S]) : 0.0;
          const double fli = (k > 0) ? t.rhoh[k] * (im[k * S] - im[(k - 1) * S]) : 0.0;
          const cplx<T> src = dh[(size_t)col * nz + k];
          const double rr = (fur - flr) / dz2 - ksq * t.rho[k] * re[k * S] - (double)src.x;
          const double ri = (fui - fli) / dz2 - ksq * t.rho[k] * im[k * S] - (double)src.y;
          acc += rr * rr + ri * ri;
        }
        resid = ((kxi == 0 || 2 * kxi == g.nx) ? 1.0 : 2.0) * acc;
      }
    }
  }
  if (diag) {
    for (int o = 16; o > 0; o >>= 1) resid += __shfl_xor_sync(0xffffffffu, resid, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&diag[slot_d], resid);
  }
  __syncthreads();
  for (int e = threadIdx.x; e < ncl * nz; e += TC) {
    const int c = e / nz;
    const int k = e - c * nz;
    ph[base + e] = mk<T>((T)((double)sre[(c * P + k) * S] * t.scale),
                         (T)((double)sim[(c * P + k) * S] * t.scale));
  }
}

// Single-precision tridiagonal solve over the short-wave column blocks, with
// the level count NZ a compile-time constant: a twisted factorisation (one
// elimination from the top and one from the bottom, two independent chains
// per column, meeting at NZ/2 - 1), each chain on its own thread: threads
// [0, TC) run the top chains of the CTA's TC columns and [TC, 2 TC) the
// bottom ones, with their factors in registers and every loop unrolled, and
// each level's coefficients (negs, rho, a, c, rounded to float on the host)
// one broadcast float4 from shared memory.  The two chains of a column meet
// through shared memory (the 2 x 2 solve at levels NZ/2 - 1, NZ/2), then
// substitute back each on its own half.  Same operations per chain as one
// thread running both, so the same results; twice the warps per SM and half
// the dependent chain per thread.  The diagonal term b = negs - k^2 rho is
// formed in float.  Blocks flagged in `skip` (the long-wave blocks, the zero
// mode's among them) are left to the double launch.  No residual
// diagnostics: the solves that record them run k_thomas.  dh and ph may
// alias (a CTA reads only its own columns before writing them).
// CTAs per SM that the staged columns' shared memory allows (TC = 32), which
// the register bound matches
template <int NZ>
constexpr int thomas_f32_blocks() { return NZ <= 64 ? 12 : 10; }
template <int NZ, int TC>
__global__ void __launch_bounds__(2 * TC, thomas_f32_blocks<NZ>()) k_thomas_f32(
    GridK g, const float4* __restrict__ coef, const double* __restrict__ kxd,
    const double* __restrict__ kyd, float scale, const cplx<float>* dh, cplx<float>* ph,
    const unsigned char* __restrict__ skip) {
  constexpr int P = NZ + 1;  // padded column stride (bank spread)
  constexpr int MT = NZ / 2 - 1;
  constexpr int NT = 2 * TC;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float4* sco = reinterpret_cast<float4*>(smem_raw);          // NZ coefficient quadruples
  cplx<float>* sc = reinterpret_cast<cplx<float>*>(sco + NZ);  // TC * P staged pairs
  __shared__ float meet[2][TC][3];  // (f, d'.re, d'.im) of each chain at its last level
  const long blk = blockIdx.x;
  if (skip[blk]) return;  // uniform across the block
  const long ncols = (long)g.nxh * g.ny;
  const long c0 = blk * TC;
  const int ncl = (int)min((long)TC, ncols - c0);
  const long base = c0 * NZ;
  for (int k = threadIdx.x; k < NZ; k += NT) cp_async(&sco[k], &coef[k], 16);
  for (int e = threadIdx.x; e < ncl * NZ; e += NT) {
    const int cl = e / NZ, k = e - cl * NZ;
    cp_async(&sc[cl * P + k], dh + base + e, 8);
  }
  cp_commit();
  cp_wait<0>();
  __syncthreads();
  const int cl = threadIdx.x % TC;
  const int h = threadIdx.x / TC;  // 0: top chain, 1: bottom chain
  const bool top = h == 0;
  float f[MT + 1];  // top: cp at level t; bottom: ap at level NZ - 1 - t
  float dr = 0.0f, di = 0.0f;
  cplx<float>* s = sc + cl * P;
  if (cl < ncl) {
    const long col = c0 + cl;
    const int kxi = (int)(col / g.ny);
    const int kyi = (int)(col - (long)kxi * g.ny);
    const double kx = kxd[kxi], ky = kyd[kyi];
    const float ksq = (float)arn(mrn(kx, kx), mrn(ky, ky));
    //   top:    cp_k = c_k / (b_k - a_k cp_{k-1}),  dp_k = (d_k - a_k dp_{k-1}) / (...)
    //   bottom: ap_k = a_k / (b_k - c_k ap_{k+1}),  dq_k = (d_k - c_k dq_{k+1}) / (...)
#pragma unroll
    for (int t = 0; t <= MT; ++t) {
      const int k = top ? t : NZ - 1 - t;
      const float4 q = sco[k];  // (negs, rho, a, c)
      const float el = top ? q.z : q.w, fa = top ? q.w : q.z;
      const float bk = srn(q.x, mrn(ksq, q.y));
      const float iv = rcprn(t == 0 ? bk : srn(bk, mrn(el, f[t > 0 ? t - 1 : 0])));
      f[t] = mrn(fa, iv);
      const cplx<float> d = s[k];
      dr = mrn(t == 0 ? d.x : srn(d.x, mrn(el, dr)), iv);
      di = mrn(t == 0 ? d.y : srn(d.y, mrn(el, di)), iv);
      s[k] = mk<float>(dr, di);
      // loads may run ahead within a group of four levels, not further: the
      // unrolled sweep would otherwise hoist every level's loads into
      // registers that the factors need
      if ((t & 3) == 3) asm volatile("" ::: "memory");
    }
    meet[h][cl][0] = f[MT];
    meet[h][cl][1] = dr;
    meet[h][cl][2] = di;
  }
  __syncthreads();
  if (cl < ncl) {
    // meeting point: x_MT = dp_MT - cp_MT x_{MT+1},  x_{MT+1} = dq_{MT+1} - ap_{MT+1} x_MT
    const float cpm = meet[0][cl][0], tr = meet[0][cl][1], ti = meet[0][cl][2];
    const float apm = meet[1][cl][0], br = meet[1][cl][1], bi = meet[1][cl][2];
    const float den = rcprn(srn(1.0f, mrn(cpm, apm)));
    float xr = mrn(srn(tr, mrn(cpm, br)), den);
    float xi = mrn(srn(ti, mrn(cpm, bi)), den);
    if (!top) {
      xr = srn(br, mrn(apm, xr));
      xi = srn(bi, mrn(apm, xi));
    }
    s[top ? MT : MT + 1] = mk<float>(xr, xi);
#pragma unroll
    for (int t = 1; t <= MT; ++t) {
      const int k = top ? MT - t : MT + 1 + t;
      const cplx<float> d = s[k];
      const float fk = f[MT - t];
      xr = srn(d.x, mrn(fk, xr));
      xi = srn(d.y, mrn(fk, xi));
      s[k] = mk<float>(xr, xi);
      if ((t & 3) == 0) asm volatile("" ::: "memory");
    }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < ncl * NZ; e += NT) {
    const int c = e / NZ, k = e - c * NZ;
    const cplx<float> v = sc[c * P + k];
    ph[base + e] = mk<float>(v.x * scale, v.y * scale);
  }
}

enum IyMode { IY_GRAD = 0, IY_FIELDS = 1 };

// y-pencil inverse kernel.  grid = (nxh, ceil(nz/zc)).  smem 2 * ny * B cplx.
// IY_GRAD: out0 = IFFTy(in0), out1 = IFFTy(i ky' in0).
// IY_FIELDS: out_f = IFFTy(scale * in_f), f < nf.
template <class T, int MODE>
__global__ void __launch_bounds__(256, 2) k_iy(GridK g, FftPlan py, int zc, int nf,
                                            const cplx<T>* __restrict__ in0,
                                            const cplx<T>* __restrict__ in1,
                                            const double* __restrict__ kyd,
                                            const cplx<T>* __restrict__ twy, double scale,
                                            cplx<T>* __restrict__ out0,
                                            cplx<T>* __restrict__ out1) {
  extern __shared__ __align__(16) unsigned char smem_dyn[];
  // twiddle table staged in shared memory (off the butterflies' critical path)
  cplx<T>* stw = reinterpret_cast<cplx<T>*>(smem_dyn);
  for (int i = threadIdx.x; i < g.ny; i += blockDim.x) stw[i] = twy[i];
  unsigned char* smem_raw = smem_dyn + ((((size_t)g.ny) * sizeof(cplx<T>) + 15) & ~size_t(15));
  const int NF = (MODE == IY_FIELDS) ? nf : 2;
  const int B = NF * zc;
  const int ny = g.ny, nz = g.nz;
  cplx<T>* bufA = reinterpret_cast<cplx<T>*>(smem_raw);
  cplx<T>* bufB = bufA + (size_t)ny * B;
  const int kx = blockIdx.y;
  const int z0 = blockIdx.x * zc;
  const int zn = min(zc, nz - z0);
  const int nel = ny * zc;
  const T s = (T)scale;
  for (int e0 = threadIdx.x; e0 < nel; e0 += kLoadBatch * blockDim.x) {
    cplx<T> va[kLoadBatch][2];
#pragma unroll
    for (int q = 0; q < kLoadBatch; ++q) {
      const int e = e0 + q * blockDim.x;
      const int ky = e / zc;
      const int zl = e - ky * zc;
      va[q][0] = va[q][1] = mk<T>((T)0, (T)0);
      if (e < nel && zl < zn) {
        const size_t o = ((size_t)kx * ny + ky) * nz + z0 + zl;
        va[q][0] = scl(in0[o], s);
        if (MODE == IY_FIELDS && NF > 1) va[q][1] = scl(in1[o], s);
      }
    }
#pragma unroll
    for (int q = 0; q < kLoadBatch; ++q) {
      const int e = e0 + q * blockDim.x;
      if (e >= nel) continue;
      const int ky = e / zc;
      const int zl = e - ky * zc;
      if (MODE == IY_GRAD) {
        const T kk = (ky == ny / 2) ? (T)0 : (T)kyd[ky];
        bufA[(size_t)ky * B + zl] = va[q][0];
        bufA[(size_t)ky * B + zc + zl] = ik(kk, va[q][0]);
      } else {
#pragma unroll
        for (int f = 0; f < 2; ++f)
          if (f < NF) bufA[(size_t)ky * B + f * zc + zl] = va[q][f];
      }
    }
  }
  __syncthreads();
  cplx<T>* R = fft_smem<T, true>(bufA, bufB, B, py, stw, 1);
  for (int e = threadIdx.x; e < nel; e += blockDim.x) {
    const int y = e / zc;
    const int zl = e - y * zc;
    if (zl >= zn) continue;
    const size_t o = ((size_t)kx * ny + y) * nz + z0 + zl;
    out0[o] = R[(size_t)y * B + zl];
    if (NF > 1) out1[o] = R[(size_t)y * B + zc + zl];
  }
}

enum IxMode { IX_CORRECT = 0, IX_STAGE = 1, IX_GRAD = 2, IX_FIELDS = 3, IX_REFINE = 4 };

// x-pencil inverse kernel.  grid = (ny, ceil(nz/zc)).  smem: (M+1)*B + M*B cplx,
// B = 3 zc + 1 (correction/grad: phi with one halo level below, d/dx, d/dy)
// or nf * zc (IX_FIELDS).
//   IX_CORRECT: in place, u -= gx, v -= gy, w[k] -= (phi_k - phi_{k-1})/dz
//               (1 <= k <= nz-1), phi stored (tendency.py:781-788).
//   IX_STAGE:   u_out = u_n - gx, v_out = v_n - gy, w_out = w_n + sdt b_half
//               - gz, phi_out = phi (the RK3 stage provisional state,
//               integrator.py:483-500).
//   IX_GRAD:    gx, gy (full levels), gz (nz+1 half levels, zero ends)
//               (tendency.py:487-500).
//   IX_FIELDS:  real outputs of nf spectra.
// In IX_CORRECT and IX_STAGE a null phi_out stores no potential.
template <class T, int MODE, class TS = T>
__global__ void __launch_bounds__(256, 2) k_ix(GridK g, FftPlan px, int zc, int nf,
                                            const cplx<T>* __restrict__ phs,
                                            const cplx<T>* __restrict__ psi,
                                            const cplx<T>* __restrict__ s2,
                                            const double* __restrict__ kxd,
                                            const cplx<T>* __restrict__ twx,
                                            const nd_t<TS>* u_in, const nd_t<TS>* v_in,
                                            const nd_t<TS>* w_in,
                                            const nd_t<TS>* __restrict__ th, double sdt,
                                            const double* __restrict__ theta0, nd_t<TS>* u_out,
                                            nd_t<TS>* v_out, nd_t<TS>* w_out,
                                            nd_t<TS>* phi_out) {
  extern __shared__ __align__(16) unsigned char smem_dyn[];
  // twiddle table staged in shared memory (off the butterflies' critical path)
  cplx<T>* stw = reinterpret_cast<cplx<T>*>(smem_dyn);
  for (int i = threadIdx.x; i < g.nx; i += blockDim.x) stw[i] = twx[i];
  unsigned char* smem_raw = smem_dyn + ((((size_t)g.nx) * sizeof(cplx<T>) + 15) & ~size_t(15));
  const bool fields = (MODE == IX_FIELDS);
  const int B = fields ? nf * zc : 3 * zc + 1;
  const int M = g.M;
  const int nz = g.nz;
  cplx<T>* bufX = reinterpret_cast<cplx<T>*>(smem_raw);  // (M+1) * B
  cplx<T>* bufZ = bufX + (size_t)(M + 1) * B;             // M * B
  const int y = blockIdx.y;
  const int z0 = blockIdx.x * zc;
  const int zn = min(zc, nz - z0);

  // load spectra X[k][b], kLoadBatch elements per thread in flight
  const int nel = (M + 1) * B;
  for (int e0 = threadIdx.x; e0 < nel; e0 += kLoadBatch * blockDim.x) {
    cplx<T> va[kLoadBatch];
#pragma unroll
    for (int q = 0; q < kLoadBatch; ++q) {
      const int e = e0 + q * blockDim.x;
      const int k = e / B;
      const int bb = e - k * B;
      cplx<T> v = mk<T>((T)0, (T)0);
      if (e < nel) {
        const size_t rowo = ((size_t)k * g.ny + y) * nz;
        if (fields) {
          const int f = bb / zc, zl = bb - f * zc;
          if (zl < zn) v = (f == 0 ? phs : (f == 1 ? psi : s2))[rowo + z0 + zl];
        } else if (bb <= zc) {
          // phi at level z0 - 1 + bb (bb = 0 is the halo below the chunk)
          const int z = z0 - 1 + bb;
          if (z >= 0 && bb <= zn) v = phs[rowo + z];
        } else if (bb <= 2 * zc) {
          const int zl = bb - zc - 1;
          if (zl < zn) {
            const T kk = (k == M) ? (T)0 : (T)kxd[k];
            v = ik(kk, phs[rowo + z0 + zl]);
          }
        } else {
          const int zl = bb - 2 * zc - 1;
          if (zl < zn) v = psi[rowo + z0 + zl];
        }
      }
      va[q] = v;
    }
#pragma unroll
    for (int q = 0; q < kLoadBatch; ++q) {
      const int e = e0 + q * blockDim.x;
      if (e < nel) bufX[e] = va[q];
    }
  }
  // Prefetch the state values this thread will correct, so their load
  // latency overlaps the shared-memory FFT below (CORRECT / STAGE modes).
  const int nout = g.nx * zc;
  const bool pre = (MODE == IX_CORRECT || MODE == IX_STAGE || MODE == IX_REFINE) &&
                   nout <= kIxPrefetch * (int)blockDim.x;
  TS pu[kIxPrefetch], pv[kIxPrefetch], pw[kIxPrefetch], pt[kIxPrefetch];
  if (pre) {
#pragma unroll
    for (int q = 0; q < kIxPrefetch; ++q) {
      const int e = threadIdx.x + q * blockDim.x;
      pu[q] = pv[q] = pw[q] = pt[q] = (TS)0;
      const int x = e / zc;
      const int zl = e - x * zc;
      if (e < nout && zl < zn) {
        const int z = z0 + zl;
        const size_t col = (size_t)x * g.ny + y;
        const size_t idx = col * nz + z;
        const size_t wi = col * (nz + 1) + z;
        pu[q] = u_in[idx];
        pv[q] = v_in[idx];
        if (MODE != IX_STAGE) {
          pw[q] = w_in[wi];
          if (z == nz - 1) pt[q] = w_in[wi + 1];
        } else {
          const TS* wc = w_in + col * (nz + 1);
          const TS* thc = th + col * nz;
          pw[q] = (TS)stage_w(wc, thc, z, nz, sdt, theta0);
          if (z == nz - 1) pt[q] = (TS)stage_w(wc, thc, nz, nz, sdt, theta0);
        }
      }
    }
  }
  __syncthreads();
  c2r_pre<T>(bufX, bufZ, M, B, stw);
  __syncthreads();
  cplx<T>* Zr = fft_smem<T, true>(bufZ, bufX, B, px, stw, 2);
  const T* rz = reinterpret_cast<const T*>(Zr);
  // real value of batch bb at x: rz[2 * ((x >> 1) * B + bb) + (x & 1)]

#pragma unroll 1
  for (int e = threadIdx.x, q = 0; e < nout; e += blockDim.x, ++q) {
    const int x = e / zc;
    const int zl = e - x * zc;
    if (zl >= zn) continue;
    const int z = z0 + zl;
    const size_t rb = 2 * ((size_t)(x >> 1) * B) + (x & 1);
    const size_t col = (size_t)x * g.ny + y;
    const size_t idx = col * nz + z;
    if (fields) {
      for (int f = 0; f < nf; ++f) {
        TS* dst = f == 0 ? u_out : (f == 1 ? v_out : w_out);
        dst[idx] = (TS)rz[rb + 2 * (f * zc + zl)];
      }
      continue;
    }
    const T phi = rz[rb + 2 * (zl + 1)];
    const T phib = rz[rb + 2 * zl];
    const T gx = rz[rb + 2 * (zc + 1 + zl)];
    const T gy = rz[rb + 2 * (2 * zc + 1 + zl)];
    const T gz = (z >= 1) ? (T)((phi - phib) / (T)g.dz) : (T)0;
    const size_t wi = col * (nz + 1) + z;
    if (MODE == IX_GRAD) {
      u_out[idx] = (TS)gx;
      v_out[idx] = (TS)gy;
      w_out[wi] = (TS)gz;
      if (z == nz - 1) w_out[wi + 1] = (TS)0;
      continue;
    }
    TS uc, vc, wc, wt;
    if (pre) {
      // q < kIxPrefetch whenever pre holds; select the register without
      // dynamic indexing of the arrays
      uc = pu[0]; vc = pv[0]; wc = pw[0]; wt = pt[0];
#pragma unroll
      for (int r = 1; r < kIxPrefetch; ++r)
        if (q == r) { uc = pu[r]; vc = pv[r]; wc = pw[r]; wt = pt[r]; }
    } else {
      uc = u_in[idx];
      vc = v_in[idx];
      if (MODE != IX_STAGE) {
        wc = w_in[wi];
        wt = (z == nz - 1) ? w_in[wi + 1] : (TS)0;
      } else {
        const TS* wcol = w_in + col * (nz + 1);
        const TS* thc = th + col * nz;
        wc = (TS)stage_w(wcol, thc, z, nz, sdt, theta0);
        wt = (z == nz - 1) ? (TS)stage_w(wcol, thc, nz, nz, sdt, theta0) : (TS)0;
      }
    }
    // the spectral type T may be wider than the state type TS (defect
    // correction of a single-precision state): subtract in T, store in TS
    u_out[idx] = (TS)((T)uc - gx);
    v_out[idx] = (TS)((T)vc - gy);
    w_out[wi] = (TS)((T)wc - gz);
    if (z == nz - 1 && (MODE == IX_STAGE || w_out != w_in)) w_out[wi + 1] = wt;
    if (MODE == IX_REFINE)
      phi_out[idx] = (TS)((T)phi_out[idx] + phi);
    else if (phi_out)  // null: the caller discards this projection's potential
      phi_out[idx] = (TS)phi;
  }
}

// ---------------------------------------------------------------------------
// Fused slow tendency + forward-Euler half step (integrator.py:346-370).
// Components, summed in OperatorConfig slot order (operator_config.py:147-160):
// advection (tendency.py:965-1062), Coriolis (tendency.py:1220-1234),
// divergence damping (precomputed spectral tendency, added here) and
// diabatic heating (tendency.py:1731-1732).
// ---------------------------------------------------------------------------
struct SlowK {
  int adv;            // OB_ADV_*
  int cor;            // 0 none, 1 f-plane, 2 beta-plane
  int heat;
  int damp;
  double f0, u_env, v_env;
  const double* fy;     // (ny)
  const double* dth0;   // (nz) d theta0 / dz (tendency.py:1013-1016)
  const double* heat_r; // (nx*ny)
  const double* heat_z; // (nz)
  double inv2dx, inv2dy, inv60dx, inv60dy, inv2dz, invdz;
  // production components, in slot order after Coriolis (operator_config.py:147-160)
  int drag, sponge, diff, cool;
  double drag_cd, drag_dz, drag_u_env, drag_v_env;
  const double* drag_w;  // (nz) max(0, 1 - z / H_bl)
  double sp_u_env, sp_v_env;
  const double* sp_a;    // (nz) full levels
  const double* sp_ah;   // (nz+1) half levels
  double diff_nu, diff_dx2, diff_dy2;
  const void* lap_u;     // biharmonic: lap(u), lap(v) of this slow half (element type T)
  const void* lap_v;
  double cool_alpha;
};

// mask bits of the production components (OB_TEND_*)
constexpr int kTendDrag = 16, kTendSponge = 32, kTendDiffusion = 64, kTendCooling = 128;

// Periodic 5-point horizontal Laplacian of q at o, in the reference's order
// ((q[i+1] - 2 q) + q[i-1]) / dx2 + ((q[j+1] - 2 q) + q[j-1]) / dy2
// (tendency.py:1551-1558, 1608-1613).  off[2], off[3]: offsets of i-1, i+1.
template <class T, class A>
__device__ __forceinline__ A lap5(const T* __restrict__ q, int o, const int* offx,
                                  const int* offy, A dx2, A dy2) {
  const A c = (A)q[o];
  return ((A)q[o + offx[3]] - (A)2 * c + (A)q[o + offx[2]]) / dx2 +
         ((A)q[o + offy[3]] - (A)2 * c + (A)q[o + offy[2]]) / dy2;
}

// The same Laplacian with the spacings' reciprocals, for single-precision
// state: two multiplies where lap5 takes two IEEE divisions (the FP32 path is
// held to its rounding, not to the reference's operation order).
__device__ __forceinline__ float lap5r(const float* __restrict__ q, int o, const int* offx,
                                       const int* offy, float rdx2, float rdy2) {
  const float c = q[o];
  return (q[o + offx[3]] - 2.0f * c + q[o + offx[2]]) * rdx2 +
         (q[o + offy[3]] - 2.0f * c + q[o + offy[2]]) * rdy2;
}

// WS5 upwind derivative along one horizontal axis.  cols[r] are the linear
// column indices of the neighbours i-3, i-2, i-1, i+1, i+2, i+3 (periodic);
// the value at neighbour r, level k is q[cols[r] * nzk + k].  Only the six
// points of the stencil a selects are loaded (tendency.py:940-959).
template <class T>
__device__ __forceinline__ double ddx_ws5(const T* __restrict__ q, int o, const int* off,
                                          double a, double inv60d) {
  // off[0..5] = offsets of i-3, i-2, i-1, i+1, i+2, i+3 relative to o
  const double qm3 = q[o + off[0]], qm2 = q[o + off[1]], qm1 = q[o + off[2]];
  const double q0 = q[o], qp1 = q[o + off[3]], qp2 = q[o + off[4]], qp3 = q[o + off[5]];
  if (a >= 0.0)
    return (-2.0 * qm3 + 15.0 * qm2 - 60.0 * qm1 + 20.0 * q0 + 30.0 * qp1 - 3.0 * qp2) * inv60d;
  return (2.0 * qp3 - 15.0 * qp2 + 60.0 * qp1 - 20.0 * q0 - 30.0 * qm1 + 3.0 * qm2) * inv60d;
}

template <class T>
__device__ __forceinline__ double ddx_c2(const T* __restrict__ q, int o, const int* off,
                                         double inv2d) {
  return ((double)q[o + off[3]] - (double)q[o + off[2]]) * inv2d;
}

// One thread per (i, j, k), k in [0, nz] (k = nz only updates w).
// grid = (ceil(ny / blockDim.y), nx); blockDim.x strides k.
// OUTMODE 0: out = in + dts * tendency (state update); 1: out = tendency.
// PROD: with the production components (surface drag, sponge, horizontal
// diffusion, Newtonian cooling); without them the kernel compiles as before.
template <class T, int OUTMODE, bool PROD = false>
__global__ void __launch_bounds__(256) k_slow(GridK g, SlowK s, int mask, double dts,
                                              const T* __restrict__ u, const T* __restrict__ v,
                                              const T* __restrict__ w,
                                              const T* __restrict__ th,
                                              const T* __restrict__ dmp_u,
                                              const T* __restrict__ dmp_v, T* __restrict__ uo,
                                              T* __restrict__ vo, T* __restrict__ wo,
                                              T* __restrict__ tho) {
  const int i = blockIdx.y;
  const int j = blockIdx.x * blockDim.y + threadIdx.y;
  if (j >= g.ny) return;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int nzw = nz + 1;
  const bool adv = (mask & 1) && s.adv;
  const bool cor = (mask & 2) && s.cor;
  const bool dmp = (mask & 4) && s.damp;
  const bool heat = (mask & 8) && s.heat;
  const bool drg = PROD && (mask & kTendDrag) && s.drag;
  const bool spg = PROD && (mask & kTendSponge) && s.sponge;
  const int dif = (PROD && (mask & kTendDiffusion)) ? s.diff : 0;
  const bool col_ = PROD && (mask & kTendCooling) && s.cool;
  // periodic neighbour columns
  int ix[6], jy[6];
  const int dd[6] = {-3, -2, -1, 1, 2, 3};
#pragma unroll
  for (int r = 0; r < 6; ++r) {
    int a = i + dd[r];
    a += (a < 0) ? nx : 0;
    a -= (a >= nx) ? nx : 0;
    ix[r] = a;
    int b = j + dd[r];
    b += (b < 0) ? ny : 0;
    b -= (b >= ny) ? ny : 0;
    jy[r] = b;
  }
  // 32-bit element offsets: plan_create bounds nx * ny * (nz + 1) by 2^31
  const int col = i * ny + j;
  int offx[6], offy[6], offxw[6], offyw[6];
#pragma unroll
  for (int r = 0; r < 6; ++r) {
    offx[r] = (ix[r] - i) * ny * nz;
    offy[r] = (jy[r] - j) * nz;
    offxw[r] = (ix[r] - i) * ny * nzw;
    offyw[r] = (jy[r] - j) * nzw;
  }
  const bool ws5 = (s.adv == 2);
  for (int k = threadIdx.x; k <= nz; k += blockDim.x) {
    const int o = col * nz + k;
    const int ow = col * nzw + k;
    if (k < nz) {
      const double uc = u[o], vc = v[o], thc = th[o];
      double tu = 0.0, tv = 0.0, tt = 0.0;
      if (adv) {
        const double wc = 0.5 * ((double)w[ow] + (double)w[ow + 1]);
        double czu, czv, czt;
        if (k == 0) {
          czu = ((double)u[o + 1] - uc) * s.invdz;
          czv = ((double)v[o + 1] - vc) * s.invdz;
          czt = ((double)th[o + 1] - thc) * s.invdz;
        } else if (k == nz - 1) {
          czu = (uc - (double)u[o - 1]) * s.invdz;
          czv = (vc - (double)v[o - 1]) * s.invdz;
          czt = (thc - (double)th[o - 1]) * s.invdz;
        } else {
          czu = ((double)u[o + 1] - (double)u[o - 1]) * s.inv2dz;
          czv = ((double)v[o + 1] - (double)v[o - 1]) * s.inv2dz;
          czt = ((double)th[o + 1] - (double)th[o - 1]) * s.inv2dz;
        }
        double xu, yu, xv, yv, xt, yt;
        if (ws5) {
          xt = ddx_ws5(th, o, offx, uc, s.inv60dx);
          yt = ddx_ws5(th, o, offy, vc, s.inv60dy);
          xu = ddx_ws5(u, o, offx, uc, s.inv60dx);
          yu = ddx_ws5(u, o, offy, vc, s.inv60dy);
          xv = ddx_ws5(v, o, offx, uc, s.inv60dx);
          yv = ddx_ws5(v, o, offy, vc, s.inv60dy);
        } else {
          xt = ddx_c2(th, o, offx, s.inv2dx);
          yt = ddx_c2(th, o, offy, s.inv2dy);
          xu = ddx_c2(u, o, offx, s.inv2dx);
          yu = ddx_c2(u, o, offy, s.inv2dy);
          xv = ddx_c2(v, o, offx, s.inv2dx);
          yv = ddx_c2(v, o, offy, s.inv2dy);
        }
        tt = -(uc * xt + vc * yt + wc * (czt + s.dth0[k]));
        tu = -(uc * xu + vc * yu + wc * czu);
        tv = -(uc * xv + vc * yv + wc * czv);
      }
      if (cor) {
        const double f = (s.cor == 2) ? s.fy[j] : s.f0;
        tu = tu + f * (vc - s.v_env);
        tv = tv + (-f) * (uc - s.u_env);
      }
      if (drg) {  // SurfaceDragComponent (tendency.py:1318-1338)
        const double up0 = (double)u[col * nz] - s.drag_u_env;
        const double vp0 = (double)v[col * nz] - s.drag_v_env;
        const double al = s.drag_cd * sqrt(up0 * up0 + vp0 * vp0) / s.drag_dz * s.drag_w[k];
        tu = tu + (-al) * (uc - s.drag_u_env);
        tv = tv + (-al) * (vc - s.drag_v_env);
      }
      if (spg) {  // SpongeDampingComponent (tendency.py:1489-1508)
        const double a = s.sp_a[k];
        tu = tu + (-a) * (uc - s.sp_u_env);
        tv = tv + (-a) * (vc - s.sp_v_env);
        tt = tt + (-a) * thc;
      }
      if (dif == 1) {  // HorizontalDiffusionComponent (tendency.py:1548-1562)
        tu = tu + s.diff_nu * lap5<T, double>(u, o, offx, offy, s.diff_dx2, s.diff_dy2);
        tv = tv + s.diff_nu * lap5<T, double>(v, o, offx, offy, s.diff_dx2, s.diff_dy2);
      } else if (dif == 2) {  // HyperDiffusionComponent (tendency.py:1615-1621)
        const T* lu = static_cast<const T*>(s.lap_u);
        const T* lv = static_cast<const T*>(s.lap_v);
        tu = tu + (-s.diff_nu) * lap5<T, double>(lu, o, offx, offy, s.diff_dx2, s.diff_dy2);
        tv = tv + (-s.diff_nu) * lap5<T, double>(lv, o, offx, offy, s.diff_dx2, s.diff_dy2);
      }
      if (col_) tt = tt + (-s.cool_alpha) * thc;  // NewtonianCooling (tendency.py:1661-1662)
      if (dmp) {
        tu = tu + (double)dmp_u[o];
        tv = tv + (double)dmp_v[o];
      }
      if (heat) tt = tt + s.heat_r[col] * s.heat_z[k];
      if (OUTMODE == 0) {
        uo[o] = (T)(uc + dts * tu);
        vo[o] = (T)(vc + dts * tv);
        tho[o] = (T)(thc + dts * tt);
      } else {
        uo[o] = (T)tu;
        vo[o] = (T)tv;
        tho[o] = (T)tt;
      }
    }
    // w on half level k
    {
      const double wk = w[ow];
      double tw = 0.0;
      if (adv && k > 0 && k < nz) {
        const double uh = 0.5 * ((double)u[o - 1] + (double)u[o]);
        const double vh = 0.5 * ((double)v[o - 1] + (double)v[o]);
        const double czw = ((double)w[ow + 1] - (double)w[ow - 1]) * s.inv2dz;
        double xw, yw;
        if (ws5) {
          xw = ddx_ws5(w, ow, offxw, uh, s.inv60dx);
          yw = ddx_ws5(w, ow, offyw, vh, s.inv60dy);
        } else {
          xw = ddx_c2(w, ow, offxw, s.inv2dx);
          yw = ddx_c2(w, ow, offyw, s.inv2dy);
        }
        tw = -(uh * xw + vh * yw + wk * czw);
      }
      if (spg) tw = tw + (-s.sp_ah[k]) * wk;  // sponge on half levels (tendency.py:1506)
      if (OUTMODE == 0)
        wo[ow] = (T)(wk + dts * tw);
      else
        wo[ow] = (T)tw;
    }
  }
}

// WS5 upwind derivative in single precision: only the six points the upwind
// side selects are loaded.  With s = +1 (a >= 0) or -1,
//   d = s (-2 q[-3s] + 15 q[-2s] - 60 q[-s] + 20 q[0] + 30 q[s] - 3 q[2s]) / (60 d),
// the two branches of ddx_ws5 with the second one's terms negated.
__device__ __forceinline__ float ddx_ws5f(const float* __restrict__ q, int o, const int* off,
                                          float a, float inv60d) {
  // off[0..5] = offsets of i-3, i-2, i-1, i+1, i+2, i+3 relative to o
  const bool up = a >= 0.0f;
  const int m3 = up ? off[0] : off[5], m2 = up ? off[1] : off[4], m1 = up ? off[2] : off[3];
  const int p1 = up ? off[3] : off[2], p2 = up ? off[4] : off[1];
  const float d = -2.0f * q[o + m3] + 15.0f * q[o + m2] - 60.0f * q[o + m1] + 20.0f * q[o] +
                  30.0f * q[o + p1] - 3.0f * q[o + p2];
  return (up ? d : -d) * inv60d;
}

// The fused slow tendency of k_slow for single-precision state, computed in
// single precision: the FP32 state's own rounding (2^-24 of each field) is
// the accuracy floor of this path, and FP32 arithmetic needs no conversion
// of the loaded values and half the registers of the double form.  Same
// terms, summation order and boundary treatment as k_slow.
template <int OUTMODE, bool PROD = false>
__global__ void __launch_bounds__(256, PROD ? 5 : 4) k_slow_f32(GridK g, SlowK s, int mask, double dts_d,
                                                     const float* __restrict__ u,
                                                     const float* __restrict__ v,
                                                     const float* __restrict__ w,
                                                     const float* __restrict__ th,
                                                     const float* __restrict__ dmp_u,
                                                     const float* __restrict__ dmp_v,
                                                     float* __restrict__ uo, float* __restrict__ vo,
                                                     float* __restrict__ wo,
                                                     float* __restrict__ tho) {
  const int i = blockIdx.y;
  const int j = blockIdx.x * blockDim.y + threadIdx.y;
  if (j >= g.ny) return;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int nzw = nz + 1;
  const bool adv = (mask & 1) && s.adv;
  const bool cor = (mask & 2) && s.cor;
  const bool dmp = (mask & 4) && s.damp;
  const bool heat = (mask & 8) && s.heat;
  const float dts = (float)dts_d;
  const float inv60dx = (float)s.inv60dx, inv60dy = (float)s.inv60dy;
  const float inv2dx = (float)s.inv2dx, inv2dy = (float)s.inv2dy;
  const float inv2dz = (float)s.inv2dz, invdz = (float)s.invdz;
  const float f = cor ? (float)((s.cor == 2) ? s.fy[j] : s.f0) : 0.0f;
  const float u_env = (float)s.u_env, v_env = (float)s.v_env;
  const bool drg = PROD && (mask & kTendDrag) && s.drag;
  const bool spg = PROD && (mask & kTendSponge) && s.sponge;
  const int dif = (PROD && (mask & kTendDiffusion)) ? s.diff : 0;
  const bool col_ = PROD && (mask & kTendCooling) && s.cool;
  const float dnu = (float)s.diff_nu, rdx2 = (float)(1.0 / s.diff_dx2),
              rdy2 = (float)(1.0 / s.diff_dy2);
  int offx[6], offy[6], offxw[6], offyw[6];
  const int dd[6] = {-3, -2, -1, 1, 2, 3};
#pragma unroll
  for (int r = 0; r < 6; ++r) {
    int a = i + dd[r];
    a += (a < 0) ? nx : 0;
    a -= (a >= nx) ? nx : 0;
    int b = j + dd[r];
    b += (b < 0) ? ny : 0;
    b -= (b >= ny) ? ny : 0;
    offx[r] = (a - i) * ny * nz;
    offy[r] = (b - j) * nz;
    offxw[r] = (a - i) * ny * nzw;
    offyw[r] = (b - j) * nzw;
  }
  const int col = i * ny + j;
  const float hr = heat ? (float)s.heat_r[col] : 0.0f;
  const bool ws5 = (s.adv == 2);
  for (int k = threadIdx.x; k <= nz; k += blockDim.x) {
    const int o = col * nz + k;
    const int ow = col * nzw + k;
    if (k < nz) {
      const float uc = u[o], vc = v[o], thc = th[o];
      float tu = 0.0f, tv = 0.0f, tt = 0.0f;
      if (adv) {
        const float wc = 0.5f * (w[ow] + w[ow + 1]);
        float czu, czv, czt;
        if (k == 0) {
          czu = (u[o + 1] - uc) * invdz;
          czv = (v[o + 1] - vc) * invdz;
          czt = (th[o + 1] - thc) * invdz;
        } else if (k == nz - 1) {
          czu = (uc - u[o - 1]) * invdz;
          czv = (vc - v[o - 1]) * invdz;
          czt = (thc - th[o - 1]) * invdz;
        } else {
          czu = (u[o + 1] - u[o - 1]) * inv2dz;
          czv = (v[o + 1] - v[o - 1]) * inv2dz;
          czt = (th[o + 1] - th[o - 1]) * inv2dz;
        }
        float xu, yu, xv, yv, xt, yt;
        if (ws5) {
          xt = ddx_ws5f(th, o, offx, uc, inv60dx);
          yt = ddx_ws5f(th, o, offy, vc, inv60dy);
          xu = ddx_ws5f(u, o, offx, uc, inv60dx);
          yu = ddx_ws5f(u, o, offy, vc, inv60dy);
          xv = ddx_ws5f(v, o, offx, uc, inv60dx);
          yv = ddx_ws5f(v, o, offy, vc, inv60dy);
        } else {
          xt = (th[o + offx[3]] - th[o + offx[2]]) * inv2dx;
          yt = (th[o + offy[3]] - th[o + offy[2]]) * inv2dy;
          xu = (u[o + offx[3]] - u[o + offx[2]]) * inv2dx;
          yu = (u[o + offy[3]] - u[o + offy[2]]) * inv2dy;
          xv = (v[o + offx[3]] - v[o + offx[2]]) * inv2dx;
          yv = (v[o + offy[3]] - v[o + offy[2]]) * inv2dy;
        }
        tt = -(uc * xt + vc * yt + wc * (czt + (float)s.dth0[k]));
        tu = -(uc * xu + vc * yu + wc * czu);
        tv = -(uc * xv + vc * yv + wc * czv);
      }
      if (cor) {
        tu = tu + f * (vc - v_env);
        tv = tv + (-f) * (uc - u_env);
      }
      if (drg) {
        const float du_env = (float)s.drag_u_env, dv_env = (float)s.drag_v_env;
        const float up0 = u[col * nz] - du_env, vp0 = v[col * nz] - dv_env;
        const float al = (float)s.drag_cd * sqrtf(up0 * up0 + vp0 * vp0) / (float)s.drag_dz *
                         (float)s.drag_w[k];
        tu = tu + (-al) * (uc - du_env);
        tv = tv + (-al) * (vc - dv_env);
      }
      if (spg) {
        const float a = (float)s.sp_a[k];
        tu = tu + (-a) * (uc - (float)s.sp_u_env);
        tv = tv + (-a) * (vc - (float)s.sp_v_env);
        tt = tt + (-a) * thc;
      }
      if (dif == 1) {
        tu = tu + dnu * lap5r(u, o, offx, offy, rdx2, rdy2);
        tv = tv + dnu * lap5r(v, o, offx, offy, rdx2, rdy2);
      } else if (dif == 2) {
        const float* lu = static_cast<const float*>(s.lap_u);
        const float* lv = static_cast<const float*>(s.lap_v);
        tu = tu + (-dnu) * lap5r(lu, o, offx, offy, rdx2, rdy2);
        tv = tv + (-dnu) * lap5r(lv, o, offx, offy, rdx2, rdy2);
      }
      if (col_) tt = tt + (-(float)s.cool_alpha) * thc;
      if (dmp) {
        tu = tu + dmp_u[o];
        tv = tv + dmp_v[o];
      }
      if (heat) tt = tt + hr * (float)s.heat_z[k];
      if (OUTMODE == 0) {
        uo[o] = uc + dts * tu;
        vo[o] = vc + dts * tv;
        tho[o] = thc + dts * tt;
      } else {
        uo[o] = tu;
        vo[o] = tv;
        tho[o] = tt;
      }
    }
    // w on half level k
    {
      const float wk = w[ow];
      float tw = 0.0f;
      if (adv && k > 0 && k < nz) {
        const float uh = 0.5f * (u[o - 1] + u[o]);
        const float vh = 0.5f * (v[o - 1] + v[o]);
        const float czw = (w[ow + 1] - w[ow - 1]) * inv2dz;
        float xw, yw;
        if (ws5) {
          xw = ddx_ws5f(w, ow, offxw, uh, inv60dx);
          yw = ddx_ws5f(w, ow, offyw, vh, inv60dy);
        } else {
          xw = (w[ow + offxw[3]] - w[ow + offxw[2]]) * inv2dx;
          yw = (w[ow + offyw[3]] - w[ow + offyw[2]]) * inv2dy;
        }
        tw = -(uh * xw + vh * yw + wk * czw);
      }
      if (spg) tw = tw + (-(float)s.sp_ah[k]) * wk;
      if (OUTMODE == 0)
        wo[ow] = wk + dts * tw;
      else
        wo[ow] = tw;
    }
  }
}

// k_slow_f32 marching along x.  A CTA covers TJ = 8 rows j, a z-chunk of 32
// levels at a time, and KXW consecutive x cells.  Each thread keeps, for its
// (j, k), a 7-point window of u, v, theta', w along x in registers (the x
// stencils' points; one new column loaded per step), and the CTA shares, per
// x step, a plane of the four fields over its rows plus three halo rows on
// either side and one halo level above and below (the y and z neighbours),
// double-buffered so that one barrier per step suffices.  Global loads per
// cell: about 7, against about 48 gathered loads of k_slow_f32, whose x
// neighbours come from the columns other CTAs own (seven L2 reads of every
// value).  Same arithmetic, terms and order as k_slow_f32.
// Requires ny % 8 == 0 and nx % KXW == 0.  grid = (ny / 8, nx / KXW),
// block = (32, 8).
constexpr int KXW = 16;
constexpr int kXwRows = 8 + 6;   // plane rows: j0-3 .. j0+10
constexpr int kXwCols = 32 + 2;  // plane columns: k0-1 .. k0+32

__device__ __forceinline__ float ws5_win(const float (&q)[7], float a, float inv60d) {
  // q[r] = value at offset r - 3
  const bool up = a >= 0.0f;
  const float m3 = up ? q[0] : q[6], m2 = up ? q[1] : q[5], m1 = up ? q[2] : q[4];
  const float p1 = up ? q[4] : q[2], p2 = up ? q[5] : q[1];
  const float d = -2.0f * m3 + 15.0f * m2 - 60.0f * m1 + 20.0f * q[3] + 30.0f * p1 - 3.0f * p2;
  return (up ? d : -d) * inv60d;
}
// the same over plane column c: rows r0-3 .. r0+3, row stride kXwCols
__device__ __forceinline__ float ws5_col(const float* P, int r0, int c, float a, float inv60d) {
  const bool up = a >= 0.0f;
  const int s = up ? kXwCols : -kXwCols;
  const float* q = P + r0 * kXwCols + c;
  const float d = -2.0f * q[-3 * s] + 15.0f * q[-2 * s] - 60.0f * q[-s] + 20.0f * q[0] +
                  30.0f * q[s] - 3.0f * q[2 * s];
  return (up ? d : -d) * inv60d;
}

template <int OUTMODE>
__global__ void __launch_bounds__(256, 3) k_slow_xw(GridK g, SlowK s, int mask, double dts_d,
                                                    const float* __restrict__ u,
                                                    const float* __restrict__ v,
                                                    const float* __restrict__ w,
                                                    const float* __restrict__ th,
                                                    const float* __restrict__ dmp_u,
                                                    const float* __restrict__ dmp_v,
                                                    float* __restrict__ uo, float* __restrict__ vo,
                                                    float* __restrict__ wo,
                                                    float* __restrict__ tho) {
  __shared__ float plane[2][4][kXwRows * kXwCols];
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int nzw = nz + 1;
  const int lane = threadIdx.x, row = threadIdx.y;
  const int tid = row * 32 + lane;
  const int j0 = blockIdx.x * 8, j = j0 + row;
  const int i0 = blockIdx.y * KXW;
  const int r0 = row + 3;  // own plane row
  const bool adv = (mask & 1) && s.adv;
  const bool cor = (mask & 2) && s.cor;
  const bool dmp = (mask & 4) && s.damp;
  const bool heat = (mask & 8) && s.heat;
  const bool ws5 = (s.adv == 2);
  const float dts = (float)dts_d;
  const float inv60dx = (float)s.inv60dx, inv60dy = (float)s.inv60dy;
  const float inv2dx = (float)s.inv2dx, inv2dy = (float)s.inv2dy;
  const float inv2dz = (float)s.inv2dz, invdz = (float)s.invdz;
  const float f = cor ? (float)((s.cor == 2) ? s.fy[j] : s.f0) : 0.0f;
  const float u_env = (float)s.u_env, v_env = (float)s.v_env;
  // halo row this thread loads (rows 0-2: j0-3..j0-1, rows 5-7: j0+8..j0+10)
  const int hrow = row < 3 ? row : (row >= 5 ? row + 6 : -1);
  int jh = j0 - 3 + (hrow < 0 ? 0 : hrow);
  jh += (jh < 0) ? ny : 0;
  jh -= (jh >= ny) ? ny : 0;
  // k-halo value this thread loads: field kf, plane row kr, end ke
  const int kf = tid / 28, krem = tid - kf * 28, kr = krem >> 1, ke = krem & 1;
  int jk = j0 - 3 + kr;
  jk += (jk < 0) ? ny : 0;
  jk -= (jk >= ny) ? ny : 0;
  // field f: 0 u, 1 v, 2 theta', 3 w (nz + 1 levels)
  auto fptr = [&](int f_) { return f_ == 0 ? u : (f_ == 1 ? v : th); };

  for (int k0 = 0; k0 < nz; k0 += 32) {
    const int k = k0 + lane;
    const bool kin = k < nz;
    // per-level constants of this thread's level, once per chunk
    const float dth0k = (adv && kin) ? (float)s.dth0[k] : 0.0f;
    const float heatz = (heat && kin) ? (float)s.heat_z[k] : 0.0f;
    auto at = [&](int ii, int jj, int f_) -> float {  // cell (ii, jj, k) of field f_
      return f_ < 3 ? fptr(f_)[(ii * ny + jj) * nz + k] : w[(ii * ny + jj) * nzw + k];
    };
    // the global values of step x = ii: the window's new column (x + 3), the
    // halo row's four fields and the level-halo value at x (software
    // pipelined: loaded one step ahead of their use)
    float nu, nv, nt, nw, hv[4], kv;
    auto load_step = [&](int ii) {
      int in = ii + 3;
      in -= (in >= nx) ? nx : 0;
      nu = kin ? at(in, j, 0) : 0.0f;
      nv = kin ? at(in, j, 1) : 0.0f;
      nt = kin ? at(in, j, 2) : 0.0f;
      nw = kin ? at(in, j, 3) : 0.0f;
      if (hrow >= 0) {
#pragma unroll
        for (int f_ = 0; f_ < 4; ++f_) {
          float val = 0.0f;
          if (kin) val = at(ii, jh, f_);
          else if (f_ == 3 && k == nz) val = w[(ii * ny + jh) * nzw + nz];
          hv[f_] = val;
        }
      }
      kv = 0.0f;
      if (tid < 4 * 28) {
        const int kk = ke ? k0 + 32 : k0 - 1;
        const int lim = kf < 3 ? nz : nzw;
        if (kk >= 0 && kk < lim)
          kv = kf < 3 ? fptr(kf)[(ii * ny + jk) * nz + kk] : w[(ii * ny + jk) * nzw + kk];
      }
    };
    // prefill the windows with x = i0-3 .. i0+2
    float qu[7], qv[7], qt[7], qw[7];
#pragma unroll
    for (int r = 1; r < 7; ++r) {
      int ii = i0 - 4 + r;
      ii += (ii < 0) ? nx : 0;
      qu[r] = kin ? at(ii, j, 0) : 0.0f;
      qv[r] = kin ? at(ii, j, 1) : 0.0f;
      qt[r] = kin ? at(ii, j, 2) : 0.0f;
      qw[r] = kin ? at(ii, j, 3) : 0.0f;
    }
    load_step(i0);
    for (int step = 0; step < KXW; ++step) {
      const int i = i0 + step;
#pragma unroll
      for (int r = 0; r < 6; ++r) {
        qu[r] = qu[r + 1];
        qv[r] = qv[r + 1];
        qt[r] = qt[r + 1];
        qw[r] = qw[r + 1];
      }
      qu[6] = nu;
      qv[6] = nv;
      qt[6] = nt;
      qw[6] = nw;
      // this step's plane: own row from the window centres, halo rows and
      // levels from the values loaded one step ahead (the lid w at level nz
      // included)
      float* P = &plane[step & 1][0][0];
      const int c = lane + 1;
      P[0 * kXwRows * kXwCols + r0 * kXwCols + c] = qu[3];
      P[1 * kXwRows * kXwCols + r0 * kXwCols + c] = qv[3];
      P[2 * kXwRows * kXwCols + r0 * kXwCols + c] = qt[3];
      P[3 * kXwRows * kXwCols + r0 * kXwCols + c] =
          kin ? qw[3] : (k == nz ? w[(i * ny + j) * nzw + nz] : 0.0f);
      if (hrow >= 0) {
#pragma unroll
        for (int f_ = 0; f_ < 4; ++f_) P[f_ * kXwRows * kXwCols + hrow * kXwCols + c] = hv[f_];
      }
      if (tid < 4 * 28) P[kf * kXwRows * kXwCols + kr * kXwCols + (ke ? kXwCols - 1 : 0)] = kv;
      if (step + 1 < KXW) load_step(i + 1);
      __syncthreads();
      if (kin) {
        const float* Pu = P;
        const float* Pv = P + kXwRows * kXwCols;
        const float* Pt = P + 2 * kXwRows * kXwCols;
        const float* Pw = P + 3 * kXwRows * kXwCols;
        const int pc = r0 * kXwCols + c;
        const int col = i * ny + j;
        const int o = col * nz + k;
        const int ow = col * nzw + k;
        const float uc = qu[3], vc = qv[3], thc = qt[3];
        float tu = 0.0f, tv = 0.0f, tt = 0.0f;
        if (adv) {
          const float wc = 0.5f * (Pw[pc] + Pw[pc + 1]);
          float czu, czv, czt;
          if (k == 0) {
            czu = (Pu[pc + 1] - uc) * invdz;
            czv = (Pv[pc + 1] - vc) * invdz;
            czt = (Pt[pc + 1] - thc) * invdz;
          } else if (k == nz - 1) {
            czu = (uc - Pu[pc - 1]) * invdz;
            czv = (vc - Pv[pc - 1]) * invdz;
            czt = (thc - Pt[pc - 1]) * invdz;
          } else {
            czu = (Pu[pc + 1] - Pu[pc - 1]) * inv2dz;
            czv = (Pv[pc + 1] - Pv[pc - 1]) * inv2dz;
            czt = (Pt[pc + 1] - Pt[pc - 1]) * inv2dz;
          }
          float xu, yu, xv, yv, xt, yt;
          if (ws5) {
            xt = ws5_win(qt, uc, inv60dx);
            yt = ws5_col(Pt, r0, c, vc, inv60dy);
            xu = ws5_win(qu, uc, inv60dx);
            yu = ws5_col(Pu, r0, c, vc, inv60dy);
            xv = ws5_win(qv, uc, inv60dx);
            yv = ws5_col(Pv, r0, c, vc, inv60dy);
          } else {
            xt = (qt[4] - qt[2]) * inv2dx;
            yt = (Pt[pc + kXwCols] - Pt[pc - kXwCols]) * inv2dy;
            xu = (qu[4] - qu[2]) * inv2dx;
            yu = (Pu[pc + kXwCols] - Pu[pc - kXwCols]) * inv2dy;
            xv = (qv[4] - qv[2]) * inv2dx;
            yv = (Pv[pc + kXwCols] - Pv[pc - kXwCols]) * inv2dy;
          }
          tt = -(uc * xt + vc * yt + wc * (czt + dth0k));
          tu = -(uc * xu + vc * yu + wc * czu);
          tv = -(uc * xv + vc * yv + wc * czv);
        }
        if (cor) {
          tu = tu + f * (vc - v_env);
          tv = tv + (-f) * (uc - u_env);
        }
        if (dmp) {
          tu = tu + dmp_u[o];
          tv = tv + dmp_v[o];
        }
        if (heat) tt = tt + (float)s.heat_r[col] * heatz;
        if (OUTMODE == 0) {
          uo[o] = uc + dts * tu;
          vo[o] = vc + dts * tv;
          tho[o] = thc + dts * tt;
        } else {
          uo[o] = tu;
          vo[o] = tv;
          tho[o] = tt;
        }
        // w on half level k
        const float wk = qw[3];
        float tw = 0.0f;
        if (adv && k > 0) {
          const float uh = 0.5f * (Pu[pc - 1] + uc);
          const float vh = 0.5f * (Pv[pc - 1] + vc);
          const float czw = (Pw[pc + 1] - Pw[pc - 1]) * inv2dz;
          float xw, yw;
          if (ws5) {
            xw = ws5_win(qw, uh, inv60dx);
            yw = ws5_col(Pw, r0, c, vh, inv60dy);
          } else {
            xw = (qw[4] - qw[2]) * inv2dx;
            yw = (Pw[pc + kXwCols] - Pw[pc - kXwCols]) * inv2dy;
          }
          tw = -(uh * xw + vh * yw + wk * czw);
        }
        wo[ow] = OUTMODE == 0 ? wk + dts * tw : tw;
        if (k == nz - 1) {  // the lid, level nz: no tendency
          const float wl = Pw[pc + 1];
          wo[ow + 1] = OUTMODE == 0 ? wl : 0.0f;
        }
      }
    }
    __syncthreads();  // the next chunk's first step rewrites plane 0
  }
}

// lap(u), lap(v) of one slow half for the biharmonic diffusion: the
// reference applies its 5-point Laplacian twice and rounds the inner one to a
// field (tendency.py:1608-1621), so it is formed as one.  One thread per cell;
// grid = (ceil(ny nz / 256), nx), so that an x plane is one grid row and the
// only division is r / nz (32-bit: nx ny (nz + 1) < 2^31, plan_create).
template <class T>
__global__ void __launch_bounds__(256) k_lap2(GridK g, const T* __restrict__ u,
                                              const T* __restrict__ v, double dx2, double dy2,
                                              T* __restrict__ lu, T* __restrict__ lv) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int pl = ny * nz;
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= pl) return;
  const int i = blockIdx.y;
  const int j = r / nz;
  {
    const int ip = i + 1 == nx ? 0 : i + 1, im = i == 0 ? nx - 1 : i - 1;
    const int jp = j + 1 == ny ? 0 : j + 1, jm = j == 0 ? ny - 1 : j - 1;
    const int o = i * pl + r;
    const int offx[6] = {0, 0, (im - i) * pl, (ip - i) * pl, 0, 0};
    const int offy[6] = {0, 0, (jm - j) * nz, (jp - j) * nz, 0, 0};
    if (sizeof(T) == 8) {
      lu[o] = (T)lap5<T, double>(u, o, offx, offy, dx2, dy2);
      lv[o] = (T)lap5<T, double>(v, o, offx, offy, dx2, dy2);
    } else {
      const float rdx2 = (float)(1.0 / dx2), rdy2 = (float)(1.0 / dy2);
      lu[o] = (T)lap5r((const float*)u, o, offx, offy, rdx2, rdy2);
      lv[o] = (T)lap5r((const float*)v, o, offx, offy, rdx2, rdy2);
    }
  }
}

// IntensityCapComponent.compute_tendency (tendency.py:1396-1403), elementwise.
template <class T>
__global__ void __launch_bounds__(256) k_intensity_cap(const T* __restrict__ u,
                                                       const T* __restrict__ v, long n,
                                                       double v_cap, double tau, double u_env,
                                                       double v_env, T* __restrict__ du,
                                                       T* __restrict__ dv) {
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n;
       e += (long)gridDim.x * blockDim.x) {
    if constexpr (sizeof(T) == 8) {
      const double up = (double)u[e] - u_env, vp = (double)v[e] - v_env;
      const double spd = sqrt(up * up + vp * vp);
      const double excess = fmax(0.0, spd - v_cap);
      const double alpha = excess / (tau * fmax(spd, 1e-6));
      du[e] = (T)(-alpha * up);
      dv[e] = (T)(-alpha * vp);
    } else {
      // single-precision fields: single-precision arithmetic (the tendency
      // is held to the FP32 rounding of the state)
      const float up = (float)u[e] - (float)u_env, vp = (float)v[e] - (float)v_env;
      const float spd = sqrtf(up * up + vp * vp);
      const float excess = fmaxf(0.0f, spd - (float)v_cap);
      const float alpha = excess / ((float)tau * fmaxf(spd, 1e-6f));
      du[e] = (T)(-alpha * up);
      dv[e] = (T)(-alpha * vp);
    }
  }
}

// dw_dt of the buoyancy component (nz+1 levels).
template <class T>
__global__ void k_buoyancy(GridK g, const T* __restrict__ th, const double* __restrict__ theta0,
                           T* __restrict__ dw) {
  const size_t ncol = (size_t)g.nx * g.ny;
  const int nzw = g.nz + 1;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < ncol * nzw;
       e += (size_t)gridDim.x * blockDim.x) {
    const size_t col = e / nzw;
    const int k = (int)(e - col * nzw);
    dw[e] = (T)bhalf(th + col * g.nz, k, g.nz, theta0);
  }
}

// Vertical part of apply_operator plus rho * horizontal Laplacian term
// (poisson.py:171-200): out = rho * lap + vert(phi).
template <class T>
__global__ void k_apply_vert(GridK g, const T* __restrict__ phi, const T* __restrict__ lap,
                             const double* __restrict__ rho, const double* __restrict__ rhoh,
                             T* __restrict__ out) {
  const size_t n = (size_t)g.nx * g.ny * g.nz;
  const double dz2 = g.dz * g.dz;
  const int nz = g.nz;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
       e += (size_t)gridDim.x * blockDim.x) {
    const int k = (int)(e % nz);
    const double p = phi[e];
    double vert;
    const double fu = (k < nz - 1) ? rhoh[k + 1] * ((double)phi[e + 1] - p) : 0.0;
    const double fl = (k > 0) ? rhoh[k] * (p - (double)phi[e - 1]) : 0.0;
    if (k == 0)
      vert = fu / dz2;
    else if (k == nz - 1)
      vert = -fl / dz2;
    else
      vert = (fu - fl) / dz2;
    out[e] = (T)(rho[k] * (double)lap[e] + vert);
  }
}

// k^2-weighted copy for the horizontal Laplacian: out = -k^2 * in.
template <class T>
__global__ void k_neg_ksq(GridK g, const cplx<T>* __restrict__ in, const double* __restrict__ kxd,
                          const double* __restrict__ kyd, cplx<T>* __restrict__ out) {
  const size_t n = (size_t)g.nxh * g.ny * g.nz;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
       e += (size_t)gridDim.x * blockDim.x) {
    const size_t col = e / g.nz;
    const int kx = (int)(col / g.ny), ky = (int)(col - (size_t)kx * g.ny);
    const double k2 = kxd[kx] * kxd[kx] + kyd[ky] * kyd[ky];
    out[e] = scl(in[e], (T)(-k2));
  }
}

// ---------------------------------------------------------------------------
// Step diagnostics (integrator.py:287-295): max|u|, max|v|, max|w|, max|th|,
// sum(phi), min/max phi[:, :, 0].  Two-stage deterministic reduction.
// ---------------------------------------------------------------------------
struct DiagPart {
  double mu, mv, mw, mt, sp, pmin, pmax, pad;
};

// Maximum and minimum that propagate NaN as NumPy's max / min do (fmax and
// fmin would drop it): once either operand is NaN the result stays NaN.
__device__ __forceinline__ double nan_max(double m, double x) { return (x > m || x != x) ? x : m; }
__device__ __forceinline__ double nan_min(double m, double x) { return (x < m || x != x) ? x : m; }
__device__ __forceinline__ float nan_maxf(float m, float x) { return (x > m || x != x) ? x : m; }

template <class T>
__global__ void __launch_bounds__(256) k_diag_partial(GridK g, const T* __restrict__ u,
                                                      const T* __restrict__ v,
                                                      const T* __restrict__ w,
                                                      const T* __restrict__ th,
                                                      const T* __restrict__ phi, DiagPart* part) {
  const size_t n = (size_t)g.nx * g.ny * g.nz;
  const size_t nw = (size_t)g.nx * g.ny * (g.nz + 1);
  double mu = 0, mv = 0, mw = 0, mt = 0, sp = 0, pmin = INFINITY, pmax = -INFINITY;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  const size_t first = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  bool done = false;
  if constexpr (sizeof(T) == 4) {
    // single precision: float4 loads where sizes and pointers allow; the
    // maxima of |.| are exact in float, the phi sum stays in double
    const size_t al = reinterpret_cast<size_t>(u) | reinterpret_cast<size_t>(v) |
                      reinterpret_cast<size_t>(w) | reinterpret_cast<size_t>(th) |
                      reinterpret_cast<size_t>(phi);
    if ((n & 3) == 0 && (nw & 3) == 0 && (al & 15) == 0) {
      float fu = 0.0f, fv = 0.0f, fw = 0.0f, ft = 0.0f;
      const float4* u4 = reinterpret_cast<const float4*>(u);
      const float4* v4 = reinterpret_cast<const float4*>(v);
      const float4* t4 = reinterpret_cast<const float4*>(th);
      const float4* p4 = reinterpret_cast<const float4*>(phi);
      const float4* w4 = reinterpret_cast<const float4*>(w);
      auto amax = [](float m, float4 a) {
        return nan_maxf(nan_maxf(nan_maxf(m, fabsf(a.x)), nan_maxf(fabsf(a.y), fabsf(a.z))),
                        fabsf(a.w));
      };
      for (size_t e = first; e < n / 4; e += stride) {
        const float4 a = u4[e], b = v4[e], c = t4[e], d = p4[e];
        fu = amax(fu, a);
        fv = amax(fv, b);
        ft = amax(ft, c);
        sp += (double)d.x;
        sp += (double)d.y;
        sp += (double)d.z;
        sp += (double)d.w;
      }
      for (size_t e = first; e < nw / 4; e += stride) fw = amax(fw, w4[e]);
      mu = fu;
      mv = fv;
      mw = fw;
      mt = ft;
      done = true;
    }
  }
  if (!done) {
    for (size_t e = first; e < n; e += stride) {
      mu = nan_max(mu, fabs((double)u[e]));
      mv = nan_max(mv, fabs((double)v[e]));
      mt = nan_max(mt, fabs((double)th[e]));
      sp += (double)phi[e];
    }
    for (size_t e = first; e < nw; e += stride) mw = nan_max(mw, fabs((double)w[e]));
  }
  // surface level k = 0 of every column
  const size_t ncol = (size_t)g.nx * g.ny;
  for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < ncol; c += stride) {
    const double p = phi[c * g.nz];
    pmin = nan_min(pmin, p);
    pmax = nan_max(pmax, p);
  }
  __shared__ double red[8][8];
  double vals[7] = {mu, mv, mw, mt, sp, pmin, pmax};
#pragma unroll
  for (int q = 0; q < 7; ++q) {
    double x = vals[q];
    for (int o = 16; o > 0; o >>= 1) {
      const double y = __shfl_xor_sync(0xffffffffu, x, o);
      x = (q == 4) ? x + y : (q == 5 ? nan_min(x, y) : nan_max(x, y));
    }
    vals[q] = x;
  }
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0)
    for (int q = 0; q < 7; ++q) red[wid][q] = vals[q];
  __syncthreads();
  if (threadIdx.x == 0) {
    const int nw_ = blockDim.x >> 5;
    double r[7];
    for (int q = 0; q < 7; ++q) r[q] = red[0][q];
    for (int ww = 1; ww < nw_; ++ww)
      for (int q = 0; q < 7; ++q)
        r[q] = (q == 4) ? r[q] + red[ww][q]
                        : (q == 5 ? nan_min(r[q], red[ww][q]) : nan_max(r[q], red[ww][q]));
    DiagPart p;
    p.mu = r[0];
    p.mv = r[1];
    p.mw = r[2];
    p.mt = r[3];
    p.sp = r[4];
    p.pmin = r[5];
    p.pmax = r[6];
    p.pad = 0;
    part[blockIdx.x] = p;
  }
}

// One warp combines the per-CTA partials (fixed order: lane-strided, then a
// butterfly), so the result does not depend on timing.  It also raises the
// plan's sticky blow-up flag diag[14] (OB_DIAG_BLOWUP): 1 for a non-finite
// value in any field, 2 for max|u| above umax_limit (> 0), the blow-up test
// of the reference's harness (measure_lh82_phase3.py:129-130).
__global__ void k_diag_final(const DiagPart* part, int np, double ncell, double umax_limit,
                             double* diag) {
  if (blockIdx.x != 0 || threadIdx.x >= 32) return;
  double mu = 0, mv = 0, mw = 0, mt = 0, sp = 0, pmin = INFINITY, pmax = -INFINITY;
  for (int b = threadIdx.x; b < np; b += 32) {
    const DiagPart q = part[b];
    mu = nan_max(mu, q.mu);
    mv = nan_max(mv, q.mv);
    mw = nan_max(mw, q.mw);
    mt = nan_max(mt, q.mt);
    sp += q.sp;
    pmin = nan_min(pmin, q.pmin);
    pmax = nan_max(pmax, q.pmax);
  }
  for (int o = 16; o > 0; o >>= 1) {
    mu = nan_max(mu, __shfl_xor_sync(0xffffffffu, mu, o));
    mv = nan_max(mv, __shfl_xor_sync(0xffffffffu, mv, o));
    mw = nan_max(mw, __shfl_xor_sync(0xffffffffu, mw, o));
    mt = nan_max(mt, __shfl_xor_sync(0xffffffffu, mt, o));
    sp += __shfl_xor_sync(0xffffffffu, sp, o);
    pmin = nan_min(pmin, __shfl_xor_sync(0xffffffffu, pmin, o));
    pmax = nan_max(pmax, __shfl_xor_sync(0xffffffffu, pmax, o));
  }
  if (threadIdx.x != 0) return;
  const double mean = sp / ncell;
  diag[0] = mu;
  diag[1] = mv;
  diag[2] = mw;
  diag[3] = mt;
  diag[4] = pmin - mean;
  diag[5] = pmax - mean;
  const bool finite = isfinite(mu) && isfinite(mv) && isfinite(mw) && isfinite(mt) &&
                      isfinite(sp) && isfinite(pmin) && isfinite(pmax);
  double flag = diag[14];
  if (!finite) flag = fmax(flag, 1.0);
  else if (umax_limit > 0.0 && mu > umax_limit) flag = fmax(flag, 2.0);
  diag[14] = flag;
}

}  // namespace ob
