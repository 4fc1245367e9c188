// Holland-vortex state fill (vortex_init.py:330-370): the per-cell expansion
// of the host's column and radial tables into (u, v, w, theta', phi).
#pragma once
#include "common.cuh"

namespace ob {

// One warp per (x, y) column, lanes along z.  col[4 * c + {0,1,2,3}] =
// (r, V_t(r), sin(phi), cos(phi)) of column c; S (nz) is the wind's vertical
// structure; tab (nr x nz, C order) the theta' radial profiles on the radial
// grid rr (nr, increasing).  theta' is numpy.interp(r, rr, tab[:, k]): the
// bracketing index by binary search, then slope * (r - rr[j]) + tab[j, k]
// with slope = (tab[j+1, k] - tab[j, k]) / (rr[j+1] - rr[j]), values beyond
// the grid clamped to the end values; u = (-V_t S) sin + u_env,
// v = (V_t S) cos + v_env (each product rounded before the sum); w = phi = 0.
template <class T>
__global__ void __launch_bounds__(256) k_vortex_fill(
    int ncol, int nz, int nr, const double* __restrict__ col, const double* __restrict__ S,
    const double* __restrict__ rr, const double* __restrict__ tab, double u_env, double v_env,
    T* __restrict__ u, T* __restrict__ v, T* __restrict__ w, T* __restrict__ th,
    T* __restrict__ phi) {
  const int lane = threadIdx.x & 31;
  const int nwarps = gridDim.x * (blockDim.x / 32);
  for (int c = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5); c < ncol; c += nwarps) {
    const double r = col[4 * (size_t)c], vt = col[4 * (size_t)c + 1];
    const double sn = col[4 * (size_t)c + 2], cs = col[4 * (size_t)c + 3];
    // bracket: rr[j] <= r < rr[j + 1]; mode 0 interior, 1 left end, 2 right end
    int mode = 0, j = 0;
    if (r < rr[0]) {
      mode = 1;
    } else if (r >= rr[nr - 1]) {
      mode = 2;
    } else {
      int lo = 0, hi = nr - 1;  // rr[lo] <= r < rr[hi]
      while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (rr[mid] <= r) lo = mid; else hi = mid;
      }
      j = lo;
    }
    const double dr = mode == 0 ? __dsub_rn(r, rr[j]) : 0.0;
    const double drr = mode == 0 ? __dsub_rn(rr[j + 1], rr[j]) : 1.0;
    const size_t o = (size_t)c * nz;
    for (int k = lane; k < nz; k += 32) {
      double t;
      if (mode == 1) {
        t = tab[k];
      } else if (mode == 2) {
        t = tab[(size_t)(nr - 1) * nz + k];
      } else {
        const double a = tab[(size_t)j * nz + k], b = tab[(size_t)(j + 1) * nz + k];
        const double slope = __ddiv_rn(__dsub_rn(b, a), drr);
        t = __dadd_rn(__dmul_rn(slope, dr), a);
      }
      const double vk = __dmul_rn(vt, S[k]);
      th[o + k] = (T)t;
      u[o + k] = (T)__dadd_rn(__dmul_rn(-vk, sn), u_env);
      v[o + k] = (T)__dadd_rn(__dmul_rn(vk, cs), v_env);
      phi[o + k] = (T)0;
    }
    for (int k = lane; k <= nz; k += 32) w[(size_t)c * (nz + 1) + k] = (T)0;
  }
}

}  // namespace ob
