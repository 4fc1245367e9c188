// Persistent, software-pipelined pencil kernels of the projection.
//
// Each CTA walks a strided list of work items (pencil, z-chunk), z-chunk
// fastest so that concurrently processed items cover adjacent bytes of every
// row.  While the FFT of item i runs out of shared memory, the raw inputs of
// item i+1 stream into a second shared-memory stage buffer with cp.async
// (Ampere-style asynchronous copies, no register staging), so DRAM keeps
// working through the compute phase:
//
//   issue(i0 -> raw[0]); commit
//   for each item i:  issue(i+1 -> raw[(n+1)&1]); commit; wait_group 1;
//                     __syncthreads; process(i, raw[n&1]); __syncthreads
//
// Semantics are those of k_fx / k_fy / k_iy / k_ix in kernels.cuh (same
// spectral layout and arithmetic); only the data movement differs.
#pragma once
#include "kernels.cuh"

namespace ob {

// cp_async / cp_commit / cp_wait: common.cuh
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

// buoyancy on half level k from a shared-memory theta' column whose entry j
// holds level (zlo + j); zero at surface and lid (equation_set.py:255-263)
template <class T>
__device__ __forceinline__ double bhalf_s(const T* thc, int zlo, int k, int nz,
                                          const double* __restrict__ theta0) {
  if (k <= 0 || k >= nz) return 0.0;
  const double b0 = drn(mrn(kGravity, (double)thc[k - 1 - zlo]), theta0[k - 1]);
  const double b1 = drn(mrn(kGravity, (double)thc[k - zlo]), theta0[k]);
  return mrn(0.5, arn(b0, b1));
}

// Pipeline driver.  Issue(item, stage) enqueues the copies of one item;
// Process(item, stage) consumes it.  Both are called by all threads.
template <class Issue, class Process>
__device__ __forceinline__ void pipeline(int ntot, unsigned char* raw0, unsigned char* raw1,
                                         Issue&& issue, Process&& process) {
  int t = blockIdx.x;
  if (t < ntot) issue(t, raw0);
  cp_commit();
  for (int n = 0; t < ntot; ++n, t += gridDim.x) {
    const int tn = t + gridDim.x;
    unsigned char* cur = (n & 1) ? raw1 : raw0;
    unsigned char* nxt = (n & 1) ? raw0 : raw1;
    if (tn < ntot) issue(tn, nxt);
    cp_commit();
    cp_wait<1>();
    __syncthreads();
    process(t, cur);
    __syncthreads();
  }
  cp_wait<0>();
}

// ---------------------------------------------------------------------------
// x-pencil forward: rho u, rho v, vertical flux divergence -> R2C along x.
// Raw stage per item: u [nx][zc], v [nx][zc], w [nx][zc+1] (levels z0..z0+zc),
// theta' [nx][zc+2] (levels z0-1..z0+zc, stage mode).
// ---------------------------------------------------------------------------
template <class T>
__host__ __device__ inline size_t fxp_raw_elems(int nx, int zc, bool stage) {
  return (size_t)nx * (2 * zc + (zc + 1) + (stage ? zc + 2 : 0));
}

template <class T, bool STAGE>
__global__ void __launch_bounds__(256, 2) k_fxp(GridK g, FftPlan px, int zc,
                                                const T* __restrict__ u, const T* __restrict__ v,
                                                const T* __restrict__ w, const T* __restrict__ th,
                                                double sdt, const double* __restrict__ rho,
                                                const double* __restrict__ rhoh,
                                                const double* __restrict__ theta0,
                                                const double* __restrict__ kxd,
                                                const cplx<T>* __restrict__ twx,
                                                cplx<T>* __restrict__ X0, cplx<T>* __restrict__ X1) {
  extern __shared__ __align__(16) unsigned char smem_dyn[];
  // twiddle table staged in shared memory (off the butterflies' critical path)
  cplx<T>* stw = reinterpret_cast<cplx<T>*>(smem_dyn);
  for (int i = threadIdx.x; i < g.nx; i += blockDim.x) stw[i] = twx[i];
  unsigned char* smem_raw = smem_dyn + ((((size_t)g.nx) * sizeof(cplx<T>) + 15) & ~size_t(15));
  const int nx = g.nx, ny = g.ny, nz = g.nz, M = g.M;
  const int B = 3 * zc;
  const int Bs = B | 1;  // odd row stride: spreads shared-memory banks
  const int nzc = (nz + zc - 1) / zc;
  const size_t rawb = ((fxp_raw_elems<T>(nx, zc, STAGE) * sizeof(T)) + 15) & ~size_t(15);
  unsigned char* raw0 = smem_raw;
  unsigned char* raw1 = smem_raw + rawb;
  cplx<T>* bufA = reinterpret_cast<cplx<T>*>(smem_raw + 2 * rawb);
  cplx<T>* bufB = bufA + (size_t)(M + 1) * Bs;
  const int zw = zc + 1, zt = zc + 2;
  const FastDiv fzc(zc), fzw(zw), fzt(zt), fnzc(nzc);

  auto issue = [&](int t, unsigned char* raw) {
    const int y = fnzc.div(t);
    const int z0 = (t - y * nzc) * zc;
    const int zn = min(zc, nz - z0);
    T* ru = reinterpret_cast<T*>(raw);
    T* rv = ru + (size_t)nx * zc;
    T* rw = rv + (size_t)nx * zc;
    T* rt = rw + (size_t)nx * zw;
    for (int e = threadIdx.x; e < nx * zc; e += blockDim.x) {
      const int x = fzc.div(e), l = e - x * zc;
      const size_t o = ((size_t)x * ny + y) * nz + z0 + (l < zn ? l : 0);
      copy_or_zero(ru + e, u + o, l < zn);
      copy_or_zero(rv + e, v + o, l < zn);
    }
    for (int e = threadIdx.x; e < nx * zw; e += blockDim.x) {
      const int x = fzw.div(e), l = e - x * zw;
      copy_or_zero(rw + e, w + ((size_t)x * ny + y) * (nz + 1) + z0 + (l <= zn ? l : 0),
                   l <= zn);
    }
    if (STAGE) {
      for (int e = threadIdx.x; e < nx * zt; e += blockDim.x) {
        const int x = fzt.div(e), l = e - x * zt;
        const int z = z0 - 1 + l;
        const bool ok = z >= 0 && z < nz && l <= zn + 1;
        copy_or_zero(rt + e, th + ((size_t)x * ny + y) * nz + (ok ? z : 0), ok);
      }
    }
  };

  auto process = [&](int t, unsigned char* raw) {
    const int y = fnzc.div(t);
    const int z0 = (t - y * nzc) * zc;
    const int zn = min(zc, nz - z0);
    const T* ru = reinterpret_cast<const T*>(raw);
    const T* rv = ru + (size_t)nx * zc;
    const T* rw = rv + (size_t)nx * zc;
    const T* rt = rw + (size_t)nx * zw;
    T* rA = reinterpret_cast<T*>(bufA);
    for (int e = threadIdx.x; e < nx * zc; e += blockDim.x) {
      const int x = fzc.div(e), l = e - x * zc;
      T a = (T)0, b = (T)0, c = (T)0;
      if (l < zn) {
        const int z = z0 + l;
        const double r = rho[z];
        a = (T)(r * (double)ru[e]);
        b = (T)(r * (double)rv[e]);
        double wl = (double)rw[x * zw + l], wu = (double)rw[x * zw + l + 1];
        if (STAGE) {
          const T* tc = rt + x * zt;  // entry j = level z0 - 1 + j
          wl = arn(wl, mrn(sdt, bhalf_s(tc, z0 - 1, z, nz, theta0)));
          wu = arn(wu, mrn(sdt, bhalf_s(tc, z0 - 1, z + 1, nz, theta0)));
        }
        c = (T)((rhoh[z + 1] * wu - rhoh[z] * wl) / g.dz);
      }
      const int n = x >> 1, odd = x & 1;
      rA[2 * ((size_t)n * Bs + l) + odd] = a;
      rA[2 * ((size_t)n * Bs + zc + l) + odd] = b;
      rA[2 * ((size_t)n * Bs + 2 * zc + l) + odd] = c;
    }
    __syncthreads();
    cplx<T>* Z = fft_smem<T, false, 4>(bufA, bufB, B, Bs, px, stw, 2);
    cplx<T>* X = (Z == bufA) ? bufB : bufA;
    r2c_post<T>(Z, X, M, B, stw, Bs);
    __syncthreads();
    for (int e = threadIdx.x; e < (M + 1) * zc; e += blockDim.x) {
      const int k = fzc.div(e), l = e - k * zc;
      if (l >= zn) continue;
      const size_t o = ((size_t)k * ny + y) * nz + z0 + l;
      const T kk = (k == M) ? (T)0 : (T)kxd[k];
      X0[o] = add(ik(kk, X[(size_t)k * Bs + l]), X[(size_t)k * Bs + 2 * zc + l]);
      X1[o] = X[(size_t)k * Bs + zc + l];
    }
  };
  pipeline(ny * nzc, raw0, raw1, issue, process);
}

// ---------------------------------------------------------------------------
// y-pencil forward (DIV): d^ = FFTy(X1) + i ky' FFTy(X2).  The raw stage is
// already the FFT input layout [y][2 zc] (field-major within a row).
// ---------------------------------------------------------------------------
template <class T>
__global__ void __launch_bounds__(256, 2) k_fyp(GridK g, FftPlan py, int zc,
                                                const cplx<T>* __restrict__ in0,
                                                const cplx<T>* __restrict__ in1,
                                                const double* __restrict__ kyd,
                                                const cplx<T>* __restrict__ twy,
                                                cplx<T>* __restrict__ out0) {
  extern __shared__ __align__(16) unsigned char smem_dyn[];
  // twiddle table staged in shared memory (off the butterflies' critical path)
  cplx<T>* stw = reinterpret_cast<cplx<T>*>(smem_dyn);
  for (int i = threadIdx.x; i < g.ny; i += blockDim.x) stw[i] = twy[i];
  unsigned char* smem_raw = smem_dyn + ((((size_t)g.ny) * sizeof(cplx<T>) + 15) & ~size_t(15));
  const int ny = g.ny, nz = g.nz;
  const int B = 2 * zc;
  const int Bs = B | 1;
  const int nzc = (nz + zc - 1) / zc;
  const size_t rawb = (size_t)ny * Bs * sizeof(cplx<T>);
  unsigned char* raw0 = smem_raw;
  unsigned char* raw1 = smem_raw + rawb;
  cplx<T>* work = reinterpret_cast<cplx<T>*>(smem_raw + 2 * rawb);
  const FastDiv fzc(zc), fB(B), fnzc(nzc);

  auto issue = [&](int t, unsigned char* raw) {
    const int kx = fnzc.div(t);
    const int z0 = (t - kx * nzc) * zc;
    const int zn = min(zc, nz - z0);
    cplx<T>* r = reinterpret_cast<cplx<T>*>(raw);
    for (int e = threadIdx.x; e < ny * B; e += blockDim.x) {
      const int y = fB.div(e), bb = e - y * B;
      const int f = bb >= zc, l = bb - f * zc;
      const size_t o = ((size_t)kx * ny + y) * nz + z0 + l;
      copy_or_zero(r + (size_t)y * Bs + bb, (f ? in1 : in0) + (l < zn ? o : 0), l < zn);
    }
  };
  auto process = [&](int t, unsigned char* raw) {
    const int kx = fnzc.div(t);
    const int z0 = (t - kx * nzc) * zc;
    const int zn = min(zc, nz - z0);
    cplx<T>* R = fft_smem<T, false, 4>(reinterpret_cast<cplx<T>*>(raw), work, B, Bs, py, stw, 1);
    for (int e = threadIdx.x; e < ny * zc; e += blockDim.x) {
      const int ky = fzc.div(e), l = e - ky * zc;
      if (l >= zn) continue;
      const T kk = (ky == ny / 2) ? (T)0 : (T)kyd[ky];
      out0[((size_t)kx * ny + ky) * nz + z0 + l] =
          add(R[(size_t)ky * Bs + l], ik(kk, R[(size_t)ky * Bs + zc + l]));
    }
  };
  pipeline(g.nxh * nzc, raw0, raw1, issue, process);
}

// ---------------------------------------------------------------------------
// y-pencil inverse (GRAD): phi~ = IFFTy(phi^), psi~ = IFFTy(i ky' phi^).
// ---------------------------------------------------------------------------
template <class T>
__global__ void __launch_bounds__(256, 2) k_iyp(GridK g, FftPlan py, int zc,
                                                const cplx<T>* __restrict__ in0,
                                                const double* __restrict__ kyd,
                                                const cplx<T>* __restrict__ twy, double scale,
                                                cplx<T>* __restrict__ out0,
                                                cplx<T>* __restrict__ out1) {
  extern __shared__ __align__(16) unsigned char smem_dyn[];
  // twiddle table staged in shared memory (off the butterflies' critical path)
  cplx<T>* stw = reinterpret_cast<cplx<T>*>(smem_dyn);
  for (int i = threadIdx.x; i < g.ny; i += blockDim.x) stw[i] = twy[i];
  unsigned char* smem_raw = smem_dyn + ((((size_t)g.ny) * sizeof(cplx<T>) + 15) & ~size_t(15));
  const int ny = g.ny, nz = g.nz;
  const int B = 2 * zc;
  const int Bs = B | 1;
  const int nzc = (nz + zc - 1) / zc;
  const size_t rawb = (size_t)ny * zc * sizeof(cplx<T>);
  unsigned char* raw0 = smem_raw;
  unsigned char* raw1 = smem_raw + rawb;
  cplx<T>* bufA = reinterpret_cast<cplx<T>*>(smem_raw + 2 * rawb);
  cplx<T>* bufB = bufA + (size_t)ny * Bs;
  const T s = (T)scale;
  const FastDiv fzc(zc), fnzc(nzc);

  auto issue = [&](int t, unsigned char* raw) {
    const int kx = fnzc.div(t);
    const int z0 = (t - kx * nzc) * zc;
    const int zn = min(zc, nz - z0);
    cplx<T>* r = reinterpret_cast<cplx<T>*>(raw);
    for (int e = threadIdx.x; e < ny * zc; e += blockDim.x) {
      const int y = fzc.div(e), l = e - y * zc;
      const size_t o = ((size_t)kx * ny + y) * nz + z0 + l;
      copy_or_zero(r + e, in0 + (l < zn ? o : 0), l < zn);
    }
  };
  auto process = [&](int t, unsigned char* raw) {
    const int kx = fnzc.div(t);
    const int z0 = (t - kx * nzc) * zc;
    const int zn = min(zc, nz - z0);
    const cplx<T>* r = reinterpret_cast<const cplx<T>*>(raw);
    for (int e = threadIdx.x; e < ny * zc; e += blockDim.x) {
      const int ky = fzc.div(e), l = e - ky * zc;
      const cplx<T> val = scl(r[e], s);
      const T kk = (ky == ny / 2) ? (T)0 : (T)kyd[ky];
      bufA[(size_t)ky * Bs + l] = val;
      bufA[(size_t)ky * Bs + zc + l] = ik(kk, val);
    }
    __syncthreads();
    cplx<T>* R = fft_smem<T, true>(bufA, bufB, B, Bs, py, stw, 1);
    for (int e = threadIdx.x; e < ny * zc; e += blockDim.x) {
      const int y = fzc.div(e), l = e - y * zc;
      if (l >= zn) continue;
      const size_t o = ((size_t)kx * ny + y) * nz + z0 + l;
      out0[o] = R[(size_t)y * Bs + l];
      out1[o] = R[(size_t)y * Bs + zc + l];
    }
  };
  pipeline(g.nxh * nzc, raw0, raw1, issue, process);
}

// ---------------------------------------------------------------------------
// x-pencil inverse + velocity correction (CORRECT: in place; STAGE: anchor
// state in, provisional + projected stage state out).
// Raw stage: phi~ [M+1][zc+1] (levels z0-1..z0+zc-1), psi~ [M+1][zc],
// u [nx][zc], v [nx][zc], w [nx][zc+1] (levels z0..z0+zc), theta' [nx][zc+1]
// (levels z0-1..z0+zc-1, stage mode).
// ---------------------------------------------------------------------------
template <class T>
__host__ __device__ inline size_t ixp_raw_bytes(int nx, int zc, bool stage) {
  const int M = nx / 2;
  size_t b = (size_t)(M + 1) * (2 * zc + 1) * 2 * sizeof(T);
  b += (size_t)nx * (2 * zc + (zc + 1) + (stage ? zc + 1 : 0)) * sizeof(T);
  return (b + 15) & ~size_t(15);
}

template <class T, bool STAGE>
__global__ void __launch_bounds__(256, 2) k_ixp(GridK g, FftPlan px, int zc,
                                                const cplx<T>* __restrict__ phs,
                                                const cplx<T>* __restrict__ psi,
                                                const double* __restrict__ kxd,
                                                const cplx<T>* __restrict__ twx, const T* u_in,
                                                const T* v_in, const T* w_in,
                                                const T* __restrict__ th, double sdt,
                                                const double* __restrict__ theta0, T* u_out,
                                                T* v_out, T* w_out, T* phi_out) {
  extern __shared__ __align__(16) unsigned char smem_dyn[];
  // twiddle table staged in shared memory (off the butterflies' critical path)
  cplx<T>* stw = reinterpret_cast<cplx<T>*>(smem_dyn);
  for (int i = threadIdx.x; i < g.nx; i += blockDim.x) stw[i] = twx[i];
  unsigned char* smem_raw = smem_dyn + ((((size_t)g.nx) * sizeof(cplx<T>) + 15) & ~size_t(15));
  const int nx = g.nx, ny = g.ny, nz = g.nz, M = g.M;
  const int B = 3 * zc + 1;
  const int Bs = B | 1;
  const int nzc = (nz + zc - 1) / zc;
  const size_t rawb = ixp_raw_bytes<T>(nx, zc, STAGE);
  unsigned char* raw0 = smem_raw;
  unsigned char* raw1 = smem_raw + rawb;
  cplx<T>* bufX = reinterpret_cast<cplx<T>*>(smem_raw + 2 * rawb);  // (M+1) * Bs
  cplx<T>* bufZ = bufX + (size_t)(M + 1) * Bs;                        // M * Bs
  const int zp = zc + 1;  // phi~ levels per row
  const int zw = zc + 1;
  const FastDiv fzc(zc), fzp(zp), fB(B), fnzc(nzc);

  auto issue = [&](int t, unsigned char* raw) {
    const int y = fnzc.div(t);
    const int z0 = (t - y * nzc) * zc;
    const int zn = min(zc, nz - z0);
    cplx<T>* rp = reinterpret_cast<cplx<T>*>(raw);
    cplx<T>* rs = rp + (size_t)(M + 1) * zp;
    T* ru = reinterpret_cast<T*>(rs + (size_t)(M + 1) * zc);
    T* rv = ru + (size_t)nx * zc;
    T* rw = rv + (size_t)nx * zc;
    T* rt = rw + (size_t)nx * zw;
    for (int e = threadIdx.x; e < (M + 1) * zp; e += blockDim.x) {
      const int k = fzp.div(e), l = e - k * zp;
      const int z = z0 - 1 + l;
      const bool ok = z >= 0 && l <= zn;
      copy_or_zero(rp + e, phs + ((size_t)k * ny + y) * nz + (ok ? z : 0), ok);
    }
    for (int e = threadIdx.x; e < (M + 1) * zc; e += blockDim.x) {
      const int k = fzc.div(e), l = e - k * zc;
      copy_or_zero(rs + e, psi + ((size_t)k * ny + y) * nz + z0 + (l < zn ? l : 0), l < zn);
    }
    for (int e = threadIdx.x; e < nx * zc; e += blockDim.x) {
      const int x = fzc.div(e), l = e - x * zc;
      const size_t o = ((size_t)x * ny + y) * nz + z0 + (l < zn ? l : 0);
      copy_or_zero(ru + e, u_in + o, l < zn);
      copy_or_zero(rv + e, v_in + o, l < zn);
    }
    for (int e = threadIdx.x; e < nx * zw; e += blockDim.x) {
      const int x = fzp.div(e), l = e - x * zw;
      copy_or_zero(rw + e, w_in + ((size_t)x * ny + y) * (nz + 1) + z0 + (l <= zn ? l : 0),
                   l <= zn);
    }
    if (STAGE) {
      for (int e = threadIdx.x; e < nx * zp; e += blockDim.x) {
        const int x = fzp.div(e), l = e - x * zp;
        const int z = z0 - 1 + l;
        const bool ok = z >= 0 && l <= zn;
        copy_or_zero(rt + e, th + ((size_t)x * ny + y) * nz + (ok ? z : 0), ok);
      }
    }
  };

  auto process = [&](int t, unsigned char* raw) {
    const int y = fnzc.div(t);
    const int z0 = (t - y * nzc) * zc;
    const int zn = min(zc, nz - z0);
    const cplx<T>* rp = reinterpret_cast<const cplx<T>*>(raw);
    const cplx<T>* rs = rp + (size_t)(M + 1) * zp;
    const T* ru = reinterpret_cast<const T*>(rs + (size_t)(M + 1) * zc);
    const T* rv = ru + (size_t)nx * zc;
    const T* rw = rv + (size_t)nx * zc;
    const T* rt = rw + (size_t)nx * zw;
    // C2R pre-process straight from the raw rows: batch bb < zc+1 is phi~ at
    // level z0-1+bb, the next zc are i kx' phi~, the last zc are psi~
    auto X = [&](int k, int bb) -> cplx<T> {
      if (bb <= zc) return rp[k * zp + bb];
      if (bb <= 2 * zc) {
        const T kk = (k == M) ? (T)0 : (T)kxd[k];
        return ik(kk, rp[k * zp + (bb - zc)]);
      }
      return rs[k * zc + (bb - 2 * zc - 1)];
    };
    for (int e = threadIdx.x; e < M * B; e += blockDim.x) {
      const int m = fB.div(e), bb = e - m * B;
      cplx<T> xm = X(m, bb);
      cplx<T> xc = X(M - m, bb);
      if (m == 0) {
        xm.y = (T)0;
        xc.y = (T)0;
      }
      xc = conjg(xc);
      const cplx<T> S = add(xm, xc);
      const cplx<T> D = mul(sub(xm, xc), conjg(stw[m]));
      bufZ[(size_t)m * Bs + bb] = mk<T>(S.x - D.y, S.y + D.x);
    }
    __syncthreads();
    cplx<T>* Zr = fft_smem<T, true>(bufZ, bufX, B, Bs, px, stw, 2);
    const T* rz = reinterpret_cast<const T*>(Zr);
    for (int e = threadIdx.x; e < nx * zc; e += blockDim.x) {
      const int x = fzc.div(e), l = e - x * zc;
      if (l >= zn) continue;
      const int z = z0 + l;
      const size_t rb = 2 * ((size_t)(x >> 1) * Bs) + (x & 1);
      const T phi = rz[rb + 2 * (l + 1)];
      const T phib = rz[rb + 2 * l];
      const T gx = rz[rb + 2 * (zc + 1 + l)];
      const T gy = rz[rb + 2 * (2 * zc + 1 + l)];
      const T gz = (z >= 1) ? (T)((phi - phib) / (T)g.dz) : (T)0;
      const size_t col = (size_t)x * ny + y;
      const size_t idx = col * nz + z;
      const size_t wi = col * (nz + 1) + z;
      T wc = rw[x * zw + l];
      T wt = rw[x * zw + l + 1];
      if (STAGE) {
        const T* tc = rt + x * zp;  // entry j = level z0 - 1 + j
        wc = (T)arn((double)wc, mrn(sdt, bhalf_s(tc, z0 - 1, z, nz, theta0)));
      }
      u_out[idx] = ru[e] - gx;
      v_out[idx] = rv[e] - gy;
      w_out[wi] = wc - gz;
      if (z == nz - 1 && (STAGE || w_out != w_in)) w_out[wi + 1] = wt;
      phi_out[idx] = phi;
    }
  };
  pipeline(ny * nzc, raw0, raw1, issue, process);
}

}  // namespace ob
