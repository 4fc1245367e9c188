// Vortex diagnostics read-outs (oracle_v8/diagnostics.py:40-220) and the
// sub-cell centre refinement (oracle_v8/run_translation_test.py:115-161).
//
// The per-cell values are formed in the reference's operation order, with
// products rounded before they are summed (__dmul_rn / __dadd_rn keep the
// compiler from contracting them into FMAs that NumPy does not do):
//  * level-band column means: NumPy's mean over a boolean-indexed band is a
//    sequential sum from the first selected level (k_vd_band_mean);
//  * the positive vorticity column mean of the refinement is a mean over a
//    contiguous axis, which NumPy forms by its pairwise summation
//    (pairwise_sum: 8 accumulators, blocks of at most 128) (k_vd_zpos);
//  * argmax follows numpy.argmax: the larger value wins, the first index wins
//    ties, and the first NaN wins over every number.
// Domain sums (kinetic energy, enstrophy, rings, the centroid) are
// deterministic fixed-order trees; they differ from NumPy's pairwise order by
// rounding only.
#pragma once
#include "common.cuh"

namespace ob {

constexpr int kVdThreads = 256;
constexpr int kVdMaxPairwise = 128;  // levels of one pairwise block

struct VdMax {
  double v;
  long long i;
};

// numpy.argmax's order: does (v2, i2) beat (v, i)?
__device__ __forceinline__ bool vd_beats(double v2, long long i2, double v, long long i) {
  const bool n2 = isnan(v2), n1 = isnan(v);
  if (n1 || n2) return n1 && n2 ? i2 < i : n2;
  return v2 > v || (v2 == v && i2 < i);
}

__device__ __forceinline__ void vd_warp_max(VdMax& a) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double v2 = __shfl_xor_sync(0xffffffffu, a.v, o);
    const long long i2 = __shfl_xor_sync(0xffffffffu, a.i, o);
    if (vd_beats(v2, i2, a.v, a.i)) {
      a.v = v2;
      a.i = i2;
    }
  }
}

// Block argmax; the result is valid in thread 0.
__device__ VdMax vd_block_max(VdMax a) {
  __shared__ double sv[kVdThreads / 32];
  __shared__ long long si[kVdThreads / 32];
  vd_warp_max(a);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    sv[warp] = a.v;
    si[warp] = a.i;
  }
  __syncthreads();
  if (threadIdx.x == 0)
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w)
      if (vd_beats(sv[w], si[w], a.v, a.i)) {
        a.v = sv[w];
        a.i = si[w];
      }
  __syncthreads();
  return a;
}

// Block sum in a fixed order; the result is valid in thread 0.
__device__ double vd_block_sum(double s) {
  __shared__ double red[kVdThreads / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s = __dadd_rn(s, __shfl_xor_sync(0xffffffffu, s, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    s = red[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) s = __dadd_rn(s, red[w]);
  }
  __syncthreads();
  return s;
}

// |(u - u_env, v - v_env)| as NumPy forms it: each square rounded, then added.
template <class T>
__device__ __forceinline__ double vd_speed(const T* __restrict__ u, const T* __restrict__ v,
                                           long long o, double ue, double ve) {
  const double up = (double)u[o] - ue, vp = (double)v[o] - ve;
  return sqrt(__dadd_rn(__dmul_rn(up, up), __dmul_rn(vp, vp)));
}

// Cell-centre distance from (cx, cy): x = (ix + 0.5) dx, no periodic wrap
// (diagnostics.py:40-50).
__device__ __forceinline__ double vd_radius(int ix, int iy, double dx, double dy, double cx,
                                            double cy) {
  const double a = __dmul_rn((double)ix + 0.5, dx) - cx;
  const double b = __dmul_rn((double)iy + 0.5, dy) - cy;
  return sqrt(__dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b)));
}

// Per-CTA argmax partial of the perturbation speed over the listed levels
// (ascending) of every column; the flat index is (col * nz + k).
template <class T>
__global__ void __launch_bounds__(kVdThreads) k_vd_speed_max(
    const T* __restrict__ u, const T* __restrict__ v, long long ncol, int nz,
    const int* __restrict__ lev, int nlev, double ue, double ve, VdMax* __restrict__ part) {
  VdMax a{-INFINITY, 0x7fffffffffffffffLL};
  const long long n = ncol * nlev;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const long long col = e / nlev;
    const int k = lev[e - col * nlev];
    const long long o = col * nz + k;
    const double s = vd_speed(u, v, o, ue, ve);
    if (vd_beats(s, o, a.v, a.i)) {
      a.v = s;
      a.i = o;
    }
  }
  a = vd_block_max(a);
  if (threadIdx.x == 0) part[blockIdx.x] = a;
}

// Final argmax over the partials, in one CTA.
__global__ void __launch_bounds__(kVdThreads) k_vd_max_final(const VdMax* __restrict__ part,
                                                             int npart, VdMax* __restrict__ out) {
  VdMax a{-INFINITY, 0x7fffffffffffffffLL};
  for (int b = threadIdx.x; b < npart; b += blockDim.x)
    if (vd_beats(part[b].v, part[b].i, a.v, a.i)) a = part[b];
  a = vd_block_max(a);
  if (threadIdx.x == 0) *out = a;
}

// Column means of u and v over the listed levels: a sequential sum from the
// first listed level, divided by the count (NumPy's mean of u[:, :, band]).
template <class T>
__global__ void __launch_bounds__(kVdThreads) k_vd_band_mean(
    const T* __restrict__ u, const T* __restrict__ v, long long ncol, int nz,
    const int* __restrict__ lev, int nlev, double* __restrict__ um, double* __restrict__ vm) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncol;
       c += (long long)gridDim.x * blockDim.x) {
    const T* uc = u + c * nz;
    const T* vc = v + c * nz;
    double su = (double)uc[lev[0]], sv = (double)vc[lev[0]];
    for (int l = 1; l < nlev; ++l) {
      su = __dadd_rn(su, (double)uc[lev[l]]);
      sv = __dadd_rn(sv, (double)vc[lev[l]]);
    }
    um[c] = su / (double)nlev;
    vm[c] = sv / (double)nlev;
  }
}

// zeta = (v[i+1] - v[i-1]) / (2 dx) - (u[j+1] - u[j-1]) / (2 dy), periodic
// (diagnostics.py:175-178), with the window's argmax partials
// (r < window ? zeta : -inf) and the partial sums of zeta^2.
__global__ void __launch_bounds__(kVdThreads) k_vd_zeta(
    const double* __restrict__ um, const double* __restrict__ vm, int nx, int ny, double dx,
    double dy, double cx, double cy, double window, double* __restrict__ zeta,
    VdMax* __restrict__ part, double* __restrict__ sq) {
  VdMax a{-INFINITY, 0x7fffffffffffffffLL};
  double s2 = 0.0;
  const long long ncol = (long long)nx * ny;
  const double tdx = 2.0 * dx, tdy = 2.0 * dy;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncol;
       c += (long long)gridDim.x * blockDim.x) {
    const int ix = (int)(c / ny), iy = (int)(c - (long long)ix * ny);
    const int ip = ix + 1 == nx ? 0 : ix + 1, im = ix == 0 ? nx - 1 : ix - 1;
    const int jp = iy + 1 == ny ? 0 : iy + 1, jm = iy == 0 ? ny - 1 : iy - 1;
    const double dvdx = (vm[(long long)ip * ny + iy] - vm[(long long)im * ny + iy]) / tdx;
    const double dudy = (um[(long long)ix * ny + jp] - um[(long long)ix * ny + jm]) / tdy;
    const double z = dvdx - dudy;
    zeta[c] = z;
    s2 = __dadd_rn(s2, __dmul_rn(z, z));
    const double w = vd_radius(ix, iy, dx, dy, cx, cy) < window ? z : -INFINITY;
    if (vd_beats(w, c, a.v, a.i)) {
      a.v = w;
      a.i = c;
    }
  }
  a = vd_block_max(a);
  s2 = vd_block_sum(s2);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = a;
    sq[blockIdx.x] = s2;
  }
}

// Partial sums of (u - u_env)^2 + (v - v_env)^2 over every cell.
template <class T>
__global__ void __launch_bounds__(kVdThreads) k_vd_ke(const T* __restrict__ u,
                                                      const T* __restrict__ v, long long n,
                                                      double ue, double ve,
                                                      double* __restrict__ part) {
  double s = 0.0;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const double up = (double)u[e] - ue, vp = (double)v[e] - ve;
    s = __dadd_rn(s, __dadd_rn(__dmul_rn(up, up), __dmul_rn(vp, vp)));
  }
  s = vd_block_sum(s);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// Sum of the partials in one CTA (fixed order).
__global__ void __launch_bounds__(kVdThreads) k_vd_sum_final(const double* __restrict__ part,
                                                             int npart, double* __restrict__ out) {
  double s = 0.0;
  for (int b = threadIdx.x; b < npart; b += blockDim.x) s = __dadd_rn(s, part[b]);
  s = vd_block_sum(s);
  if (threadIdx.x == 0) *out = s;
}

// Ring sums of the deep-layer winds for the ventilation flow
// (diagnostics.py:150-166), one CTA over the disk's bounding box
// [i0, i1) x [j0, j1).  out[3 b + 0..2] = (cells, sum u, sum v) of ring b
// (edges[b] <= r < edges[b + 1]); ring nb is the disk r < r_vent.
__global__ void __launch_bounds__(kVdThreads) k_vd_rings(
    const double* __restrict__ um, const double* __restrict__ vm, int ny, int i0, int i1,
    int j0, int j1, double dx, double dy, double cx, double cy,
    const double* __restrict__ edges, int nb, double r_vent, double* __restrict__ out) {
  const int bw = j1 - j0;
  const long long nbox = (long long)(i1 - i0) * bw;
  for (int b = 0; b <= nb; ++b) {
    const double lo = b < nb ? edges[b] : -INFINITY;
    const double hi = b < nb ? edges[b + 1] : r_vent;
    double cnt = 0.0, su = 0.0, sv = 0.0;
    for (long long e = threadIdx.x; e < nbox; e += blockDim.x) {
      const int ix = i0 + (int)(e / bw), iy = j0 + (int)(e % bw);
      const double r = vd_radius(ix, iy, dx, dy, cx, cy);
      if (r >= lo && r < hi) {
        const long long c = (long long)ix * ny + iy;
        cnt += 1.0;
        su = __dadd_rn(su, um[c]);
        sv = __dadd_rn(sv, vm[c]);
      }
    }
    cnt = vd_block_sum(cnt);
    su = vd_block_sum(su);
    sv = vd_block_sum(sv);
    if (threadIdx.x == 0) {
      out[3 * b + 0] = cnt;
      out[3 * b + 1] = su;
      out[3 * b + 2] = sv;
    }
  }
}

// Element-at-a-time form of NumPy's pairwise_sum for n <= 128: below 8
// elements a sequential sum from 0; otherwise 8 strided accumulators over the
// multiple-of-8 prefix, combined as ((r0+r1)+(r2+r3))+((r4+r5)+(r6+r7)), then
// the remainder added in order.
template <class F>
__device__ __forceinline__ double vd_pairwise(F f, int n) {
  if (n < 8) {
    double r = 0.0;
    for (int i = 0; i < n; ++i) r = __dadd_rn(r, f(i));
    return r;
  }
  double r[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) r[j] = f(j);
  const int m = n - (n % 8);
  for (int i = 8; i < m; i += 8) {
#pragma unroll
    for (int j = 0; j < 8; ++j) r[j] = __dadd_rn(r[j], f(i + j));
  }
  double s = __dadd_rn(__dadd_rn(__dadd_rn(r[0], r[1]), __dadd_rn(r[2], r[3])),
                       __dadd_rn(__dadd_rn(r[4], r[5]), __dadd_rn(r[6], r[7])));
  for (int i = m; i < n; ++i) s = __dadd_rn(s, f(i));
  return s;
}

// Positive low-level vorticity column mean of the refinement
// (run_translation_test.py:134-139): levels [0, nz/2), spacing dx on both
// axes, max(dv/dx - du/dy, 0), NumPy's pairwise mean over the levels.
template <class T>
__global__ void __launch_bounds__(kVdThreads) k_vd_zpos(const T* __restrict__ u,
                                                        const T* __restrict__ v, int nx, int ny,
                                                        int nz, double dx,
                                                        double* __restrict__ zp) {
  const long long ncol = (long long)nx * ny;
  const int nzh = nz / 2;
  const double tdx = 2.0 * dx;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncol;
       c += (long long)gridDim.x * blockDim.x) {
    const int ix = (int)(c / ny), iy = (int)(c - (long long)ix * ny);
    const int ip = ix + 1 == nx ? 0 : ix + 1, im = ix == 0 ? nx - 1 : ix - 1;
    const int jp = iy + 1 == ny ? 0 : iy + 1, jm = iy == 0 ? ny - 1 : iy - 1;
    const T* vp = v + ((long long)ip * ny + iy) * nz;
    const T* vmn = v + ((long long)im * ny + iy) * nz;
    const T* up = u + ((long long)ix * ny + jp) * nz;
    const T* umn = u + ((long long)ix * ny + jm) * nz;
    auto f = [&](int k) {
      const double dvdx = ((double)vp[k] - (double)vmn[k]) / tdx;
      const double dudy = ((double)up[k] - (double)umn[k]) / tdx;
      return fmax(dvdx - dudy, 0.0);
    };
    zp[c] = vd_pairwise(f, nzh) / (double)nzh;
  }
}

// The [1, 2, 1] / 4 smoothing along x, then along y (periodic), in NumPy's
// order: (z[i-1] + 2 z[i]) + z[i+1], times 0.25.
__device__ __forceinline__ double vd_s121(double a, double b, double c) {
  return __dmul_rn(__dadd_rn(__dadd_rn(a, __dmul_rn(2.0, b)), c), 0.25);
}

__global__ void __launch_bounds__(kVdThreads) k_vd_smooth(const double* __restrict__ zp, int nx,
                                                          int ny, double* __restrict__ zs) {
  const long long ncol = (long long)nx * ny;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncol;
       c += (long long)gridDim.x * blockDim.x) {
    const int ix = (int)(c / ny), iy = (int)(c - (long long)ix * ny);
    const int ip = ix + 1 == nx ? 0 : ix + 1, im = ix == 0 ? nx - 1 : ix - 1;
    const int jp = iy + 1 == ny ? 0 : iy + 1, jm = iy == 0 ? ny - 1 : iy - 1;
    auto zx = [&](int j) {
      return vd_s121(zp[(long long)im * ny + j], zp[(long long)ix * ny + j],
                     zp[(long long)ip * ny + j]);
    };
    zs[c] = vd_s121(zx(jm), zx(iy), zx(jp));
  }
}

// One centroid iteration of the refinement over the patch [i0, i1) x [j0, j1)
// of the smoothed field: out = (sum w, sum i w, sum j w) with w = zs^2.
__global__ void __launch_bounds__(kVdThreads) k_vd_centroid(const double* __restrict__ zs,
                                                            int ny, int i0, int i1, int j0,
                                                            int j1, double* __restrict__ out) {
  const int bw = j1 - j0;
  const long long nbox = (long long)(i1 - i0) * bw;
  double t = 0.0, sx = 0.0, sy = 0.0;
  for (long long e = threadIdx.x; e < nbox; e += blockDim.x) {
    const int ix = i0 + (int)(e / bw), iy = j0 + (int)(e % bw);
    const double z = zs[(long long)ix * ny + iy];
    const double w = __dmul_rn(z, z);
    t = __dadd_rn(t, w);
    sx = __dadd_rn(sx, __dmul_rn((double)ix, w));
    sy = __dadd_rn(sy, __dmul_rn((double)iy, w));
  }
  t = vd_block_sum(t);
  sx = vd_block_sum(sx);
  sy = vd_block_sum(sy);
  if (threadIdx.x == 0) {
    out[0] = t;
    out[1] = sx;
    out[2] = sy;
  }
}

}  // namespace ob
