// Storm-centre reductions of the theta' surface-pressure tracker
// (storm_tracker.py:64-98 proxy and window, :191-203 masked argmin, :115-188
// vorticity field).  The column integrals and the argmin / max reductions run
// on the device (warp shuffles, one deterministic two-stage reduction); the
// scalar decision logic (parabolic refine, continuity gate, fall-backs) stays
// on the host, as in the reference.
#pragma once
#include "common.cuh"

namespace ob {

constexpr int kTrackThreads = 256;  // 8 warps per CTA

// Per-CTA partial of the masked argmin: the smallest interior value with its
// first C-order index (ix * ny + iy), and the largest value of the whole
// field, for the raw anomaly and for the windowed one.
struct TrackPart {
  double rmin, rmax, wmin, wmax;
  long long ridx, widx;
};

// Device result; the same layout as OracleTrackFix in the C header.
struct TrackFixD {
  double mean;
  double raw_min, raw_max;
  long long raw_idx;
  double raw_nb[5];
  double win_min, win_max;
  long long win_idx;
  double win_nb[5];
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// (value, index) minimum with the first index winning ties: numpy's argmin.
__device__ __forceinline__ void cand_min(double& v, long long& i, double v2, long long i2) {
  if (v2 < v || (v2 == v && i2 < i)) {
    v = v2;
    i = i2;
  }
}

__device__ __forceinline__ void warp_cand_min(double& v, long long& i) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double v2 = __shfl_xor_sync(0xffffffffu, v, o);
    const long long i2 = __shfl_xor_sync(0xffffffffu, i, o);
    cand_min(v, i, v2, i2);
  }
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// p_sfc(x, y) = -trapz(rho0 * (g theta' / theta0), z): one warp per column,
// lanes along z (coalesced in the z-contiguous layout).  Each trapezoid is
// (z[k+1] - z[k]) * (f[k+1] + f[k]) / 2, the operation order of numpy.trapz.
// part[blockIdx.x] = sum of this CTA's p values (for the domain mean).
template <class T>
__global__ void __launch_bounds__(kTrackThreads) k_track_psfc(
    int ncol, int nz, const T* __restrict__ th, const double* __restrict__ z,
    const double* __restrict__ rho0, const double* __restrict__ theta0,
    double* __restrict__ p, double* __restrict__ part) {
  __shared__ double red[kTrackThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nwarps = gridDim.x * (kTrackThreads / 32);
  double acc = 0.0;
  for (int c = blockIdx.x * (kTrackThreads / 32) + warp; c < ncol; c += nwarps) {
    const T* col = th + (size_t)c * nz;
    double s = 0.0;
    for (int k = lane; k < nz - 1; k += 32) {
      const double f0 = rho0[k] * ((kGravity * (double)col[k]) / theta0[k]);
      const double f1 = rho0[k + 1] * ((kGravity * (double)col[k + 1]) / theta0[k + 1]);
      s += ((z[k + 1] - z[k]) * (f1 + f0)) / 2.0;
    }
    s = -warp_sum(s);
    if (lane == 0) {
      p[c] = s;
      acc += s;
    }
  }
  if (lane == 0) red[warp] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kTrackThreads / 32; ++w) t += red[w];
    part[blockIdx.x] = t;
  }
}

struct TrackWin {
  int on;              // a previous fix exists (storm_tracker.py:91-98)
  double lx, ly;       // last position in cells (last_pos / dx)
  double r0;           // window radius in cells
};

// Windowed anomaly a * exp(-r^2 / (2 r0^2)), r measured in cells from the
// last fix (storm_tracker.py:91-98 operation order).
__device__ __forceinline__ double track_window(double a, int ix, int iy, const TrackWin& w) {
  const double dxc = (double)ix - w.lx, dyc = (double)iy - w.ly;
  const double r2 = dxc * dxc + dyc * dyc;
  return a * exp(-r2 / (2.0 * (w.r0 * w.r0)));
}

// Block-wide mean of p from the psfc partials; every CTA sums them in the same
// fixed order, so all CTAs see the same mean.
__device__ double track_mean(const double* __restrict__ part, int npart, long long ncol) {
  __shared__ double red[kTrackThreads / 32];
  __shared__ double mean_s;
  double s = 0.0;
  for (int i = threadIdx.x; i < npart; i += blockDim.x) s += part[i];
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kTrackThreads / 32; ++w) t += red[w];
    mean_s = t / (double)ncol;
  }
  __syncthreads();
  return mean_s;
}

// Masked argmin partials (storm_tracker.py:191-203): interior minimum with
// its first index and whole-field maximum, for the anomaly p - mean and, when
// a previous fix exists, for its windowed form.
__global__ void __launch_bounds__(kTrackThreads) k_track_min(
    int nx, int ny, int margin, TrackWin win, const double* __restrict__ p,
    const double* __restrict__ part, int npart, TrackPart* __restrict__ out) {
  __shared__ TrackPart red[kTrackThreads / 32];
  const double mean = track_mean(part, npart, (long long)nx * ny);
  const long long n = (long long)nx * ny;
  double rmin = INFINITY, rmax = -INFINITY, wmin = INFINITY, wmax = -INFINITY;
  long long ridx = -1, widx = -1;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int ix = (int)(i / ny), iy = (int)(i - (long long)ix * ny);
    const double a = p[i] - mean;
    const bool inner = ix >= margin && ix < nx - margin && iy >= margin && iy < ny - margin;
    rmax = fmax(rmax, a);
    if (inner) cand_min(rmin, ridx, a, i);
    if (win.on) {
      const double b = track_window(a, ix, iy, win);
      wmax = fmax(wmax, b);
      if (inner) cand_min(wmin, widx, b, i);
    }
  }
  warp_cand_min(rmin, ridx);
  warp_cand_min(wmin, widx);
  rmax = warp_max(rmax);
  wmax = warp_max(wmax);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = TrackPart{rmin, rmax, wmin, wmax, ridx, widx};
  __syncthreads();
  if (threadIdx.x == 0) {
    TrackPart t = red[0];
    for (int w = 1; w < kTrackThreads / 32; ++w) {
      cand_min(t.rmin, t.ridx, red[w].rmin, red[w].ridx);
      cand_min(t.wmin, t.widx, red[w].wmin, red[w].widx);
      t.rmax = fmax(t.rmax, red[w].rmax);
      t.wmax = fmax(t.wmax, red[w].wmax);
    }
    out[blockIdx.x] = t;
  }
}

// Final reduction (one CTA) and the 5-point neighbourhood of each chosen
// cell for the host's parabolic sub-cell refine (storm_tracker.py:206-227).
// When the interior minimum does not lie below the field maximum (a constant
// field, or no interior), numpy's argmin of the masked copy is index 0.
__global__ void __launch_bounds__(kTrackThreads) k_track_final(
    int nx, int ny, TrackWin win, const double* __restrict__ p, const double* __restrict__ part,
    int npart, const TrackPart* __restrict__ parts, int nparts, TrackFixD* __restrict__ fix) {
  const double mean = track_mean(part, npart, (long long)nx * ny);
  if (threadIdx.x != 0) return;
  TrackPart t = parts[0];
  for (int b = 1; b < nparts; ++b) {
    cand_min(t.rmin, t.ridx, parts[b].rmin, parts[b].ridx);
    cand_min(t.wmin, t.widx, parts[b].wmin, parts[b].widx);
    t.rmax = fmax(t.rmax, parts[b].rmax);
    t.wmax = fmax(t.wmax, parts[b].wmax);
  }
  fix->mean = mean;
  fix->raw_min = t.rmin;
  fix->raw_max = t.rmax;
  fix->win_min = t.wmin;
  fix->win_max = t.wmax;
  const long long ri = (t.ridx >= 0 && t.rmin < t.rmax) ? t.ridx : 0;
  const long long wi = (t.widx >= 0 && t.wmin < t.wmax) ? t.widx : 0;
  fix->raw_idx = ri;
  fix->win_idx = win.on ? wi : ri;
  for (int s = 0; s < 2; ++s) {
    const long long c = s == 0 ? ri : (win.on ? wi : ri);
    const int ix = (int)(c / ny), iy = (int)(c - (long long)ix * ny);
    const int nbx[5] = {ix, ix - 1, ix + 1, ix, ix};
    const int nby[5] = {iy, iy, iy, iy - 1, iy + 1};
    double* nb = s == 0 ? fix->raw_nb : fix->win_nb;
    for (int q = 0; q < 5; ++q) {
      const int x = nbx[q], y = nby[q];
      double v = 0.0;
      if (x >= 0 && x < nx && y >= 0 && y < ny) {
        v = p[(size_t)x * ny + y] - mean;
        if (s == 1 && win.on) v = track_window(v, x, y, win);
      }
      nb[q] = v;
    }
  }
}

// Column-mean positive relative vorticity over the lower half of the levels
// (storm_tracker.py:130-139): zeta = dv/dx - du/dy by periodic centred
// differences with spacing dx on both axes; zcol = mean_k max(zeta, 0).
// One warp per column, lanes along z.
template <class T>
__global__ void __launch_bounds__(kTrackThreads) k_track_zcol(
    int nx, int ny, int nz, const T* __restrict__ u, const T* __restrict__ v, double dx,
    double* __restrict__ zcol) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nwarps = gridDim.x * (kTrackThreads / 32);
  const int nzh = nz / 2;
  const int ncol = nx * ny;
  for (int c = blockIdx.x * (kTrackThreads / 32) + warp; c < ncol; c += nwarps) {
    const int ix = c / ny, iy = c - ix * ny;
    const size_t xp = ((size_t)((ix + 1) % nx) * ny + iy) * nz;
    const size_t xm = ((size_t)((ix + nx - 1) % nx) * ny + iy) * nz;
    const size_t yp = ((size_t)ix * ny + (iy + 1) % ny) * nz;
    const size_t ym = ((size_t)ix * ny + (iy + ny - 1) % ny) * nz;
    double s = 0.0;
    for (int k = lane; k < nzh; k += 32) {
      const double dvdx = ((double)v[xp + k] - (double)v[xm + k]) / (2.0 * dx);
      const double dudy = ((double)u[yp + k] - (double)u[ym + k]) / (2.0 * dx);
      s += fmax(dvdx - dudy, 0.0);
    }
    s = warp_sum(s);
    if (lane == 0) zcol[c] = s / (double)nzh;
  }
}

}  // namespace ob
