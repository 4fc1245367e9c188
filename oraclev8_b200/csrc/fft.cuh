// Shared-memory mixed-radix (2, 3, 4, 5, 16) Stockham FFT, executed by a whole CTA
// on a batch of B transforms stored [n][b] (batch index innermost, matching
// the z-contiguous global layout so loads and stores stay coalesced).
//
// Pass s with radix R combines R sub-transforms of length Ns into length Ns*R:
//   v[r] = in[j + r*M/R] * W_{Ns*R}^{r*(j mod Ns)},  V = DFT_R(v),
//   out[(j - j mod Ns)*R + j mod Ns + q*Ns] = V[q].
// Twiddles come from one table W_N^t (t < N) with W_M^s = W_N^{s*N/M}.
#pragma once
#include "common.cuh"

namespace ob {

// Small DFTs in registers.  Each size is its own function and dft_small
// selects one with `if constexpr`, so no template instantiates a call cycle
// (force-inlined functions must never recurse).
template <class T, bool INV>
__device__ __forceinline__ void dft2(cplx<T>* v) {
  const cplx<T> a = v[0], b = v[1];
  v[0] = add(a, b);
  v[1] = sub(a, b);
}

template <class T, bool INV>
__device__ __forceinline__ void dft4(cplx<T>* v) {
  const cplx<T> t0 = add(v[0], v[2]), t1 = sub(v[0], v[2]);
  const cplx<T> t2 = add(v[1], v[3]), t3 = rot<T, INV>(sub(v[1], v[3]));
  v[0] = add(t0, t2);
  v[2] = sub(t0, t2);
  v[1] = add(t1, t3);
  v[3] = sub(t1, t3);
}

template <class T, bool INV>
__device__ __forceinline__ void dft3(cplx<T>* v) {
  const T h = (T)0.86602540378443864676;  // sin(2*pi/3)
  const cplx<T> s = add(v[1], v[2]);
  const cplx<T> d = sub(v[1], v[2]);
  const cplx<T> m = mk<T>(v[0].x - (T)0.5 * s.x, v[0].y - (T)0.5 * s.y);
  const cplx<T> r = rot<T, INV>(scl(d, h));
  v[0] = add(v[0], s);
  v[1] = add(m, r);
  v[2] = sub(m, r);
}

template <class T, bool INV>
__device__ __forceinline__ void dft5(cplx<T>* v) {
  const T c1 = (T)0.30901699437494742410, c2 = (T)-0.80901699437494742410;
  const T s1 = (T)0.95105651629515357212, s2 = (T)0.58778525229247312917;
  const cplx<T> a1 = add(v[1], v[4]), b1 = sub(v[1], v[4]);
  const cplx<T> a2 = add(v[2], v[3]), b2 = sub(v[2], v[3]);
  const cplx<T> p1 = mk<T>(v[0].x + c1 * a1.x + c2 * a2.x, v[0].y + c1 * a1.y + c2 * a2.y);
  const cplx<T> p2 = mk<T>(v[0].x + c2 * a1.x + c1 * a2.x, v[0].y + c2 * a1.y + c1 * a2.y);
  const cplx<T> q1 = rot<T, INV>(mk<T>(s1 * b1.x + s2 * b2.x, s1 * b1.y + s2 * b2.y));
  const cplx<T> q2 = rot<T, INV>(mk<T>(s2 * b1.x - s1 * b2.x, s2 * b1.y - s1 * b2.y));
  v[0] = add(v[0], add(a1, a2));
  v[1] = add(p1, q1);
  v[4] = sub(p1, q1);
  v[2] = add(p2, q2);
  v[3] = sub(p2, q2);
}

// a * W, W = exp(-+ i theta) with (c, s) = (cos theta, sin theta):
// forward multiplies by (c - i s), inverse by (c + i s)
template <class T, bool INV>
__device__ __forceinline__ cplx<T> twc(cplx<T> a, T c, T s) {
  return INV ? mk<T>(a.x * c - a.y * s, a.x * s + a.y * c)
             : mk<T>(a.x * c + a.y * s, a.y * c - a.x * s);
}

// 8-point DFT: two 4-point DFTs of the even and odd samples combined with
// W_8^k (radix-2 decimation in time)
template <class T, bool INV>
__device__ __forceinline__ void dft8(cplx<T>* v) {
  const T h = (T)0.70710678118654752440;  // cos(pi/4) = sin(pi/4)
  cplx<T> e[4] = {v[0], v[2], v[4], v[6]};
  cplx<T> o[4] = {v[1], v[3], v[5], v[7]};
  dft4<T, INV>(e);
  dft4<T, INV>(o);
  o[1] = twc<T, INV>(o[1], h, h);
  o[2] = rot<T, INV>(o[2]);
  o[3] = twc<T, INV>(o[3], -h, h);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    v[k] = add(e[k], o[k]);
    v[k + 4] = sub(e[k], o[k]);
  }
}

// 16-point DFT: two 8-point DFTs combined with W_16^k
template <class T, bool INV>
__device__ __forceinline__ void dft16(cplx<T>* v) {
  const T c1 = (T)0.92387953251128675613, s1 = (T)0.38268343236508977173;  // pi/8
  const T h = (T)0.70710678118654752440;
  cplx<T> e[8], o[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    e[k] = v[2 * k];
    o[k] = v[2 * k + 1];
  }
  dft8<T, INV>(e);
  dft8<T, INV>(o);
  o[1] = twc<T, INV>(o[1], c1, s1);
  o[2] = twc<T, INV>(o[2], h, h);
  o[3] = twc<T, INV>(o[3], s1, c1);
  o[4] = rot<T, INV>(o[4]);
  o[5] = twc<T, INV>(o[5], -s1, c1);
  o[6] = twc<T, INV>(o[6], -h, h);
  o[7] = twc<T, INV>(o[7], -c1, s1);
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    v[k] = add(e[k], o[k]);
    v[k + 8] = sub(e[k], o[k]);
  }
}

template <class T, int R, bool INV>
__device__ __forceinline__ void dft_small(cplx<T>* v) {
  if constexpr (R == 2) dft2<T, INV>(v);
  else if constexpr (R == 3) dft3<T, INV>(v);
  else if constexpr (R == 4) dft4<T, INV>(v);
  else if constexpr (R == 5) dft5<T, INV>(v);
  else if constexpr (R == 8) dft8<T, INV>(v);
  else if constexpr (R == 16) dft16<T, INV>(v);
}

template <class T, int R, bool INV>
__device__ __forceinline__ void stockham_pass(const cplx<T>* __restrict__ in,
                                              cplx<T>* __restrict__ out, int M, int B, int Bs,
                                              const FastDiv& fB, int Ns, const FastDiv& fNs,
                                              const cplx<T>* __restrict__ tw, int twstep) {
  const int MR = M / R;
  const int total = MR * B;
#pragma unroll (R >= 8 ? 1 : 2)
  for (int it = threadIdx.x; it < total; it += blockDim.x) {
    const int j = fB.div(it);
    const int bb = it - j * B;
    const int k = j - fNs.div(j) * Ns;
    cplx<T> v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = in[(j + r * MR) * Bs + bb];
    if (Ns > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) {
        cplx<T> w = tw[r * k * twstep];
        if (INV) w.y = -w.y;
        v[r] = mul(v[r], w);
      }
    }
    dft_small<T, R, INV>(v);
    const int base = (j - k) * R + k;
#pragma unroll
    for (int q = 0; q < R; ++q) out[(base + q * Ns) * Bs + bb] = v[q];
  }
}

// Runs all passes on B transforms stored with row stride Bs >= B; returns
// the buffer holding the result (a or b).  Caller must __syncthreads()
// before (input ready); this returns after a barrier.
// MAXR: largest radix compiled into the caller.  Kernels whose plans stop at
// radix 4 instantiate fft_smem<.., 4> so the 16-point butterfly (and its
// register pressure) is not part of them; MAXR = 8 compiles radices 2-5 and 8
// (plans from a radix-8-first factorisation) and not 16.
template <class T, bool INV, int MAXR = 16>
__device__ cplx<T>* fft_smem(cplx<T>* a, cplx<T>* b, int B, int Bs, const FftPlan& p,
                             const cplx<T>* __restrict__ tw, int tws) {
  const FastDiv fB((unsigned)B);
  int Ns = 1;
  for (int s = 0; s < p.np; ++s) {
    const int R = p.r[s];
    const int step = (p.M / (Ns * R)) * tws;
    switch (R) {
      case 2: stockham_pass<T, 2, INV>(a, b, p.M, B, Bs, fB, Ns, p.ns[s], tw, step); break;
      case 3: stockham_pass<T, 3, INV>(a, b, p.M, B, Bs, fB, Ns, p.ns[s], tw, step); break;
      case 4: stockham_pass<T, 4, INV>(a, b, p.M, B, Bs, fB, Ns, p.ns[s], tw, step); break;
      case 8:
        if constexpr (MAXR == 8) stockham_pass<T, 8, INV>(a, b, p.M, B, Bs, fB, Ns, p.ns[s], tw, step);
        break;
      case 16:
        if constexpr (MAXR >= 16) stockham_pass<T, 16, INV>(a, b, p.M, B, Bs, fB, Ns, p.ns[s], tw, step);
        break;
      default: stockham_pass<T, 5, INV>(a, b, p.M, B, Bs, fB, Ns, p.ns[s], tw, step); break;
    }
    __syncthreads();
    cplx<T>* t = a;
    a = b;
    b = t;
    Ns *= R;
  }
  return a;
}

template <class T, bool INV, int MAXR = 16>
__device__ cplx<T>* fft_smem(cplx<T>* a, cplx<T>* b, int B, const FftPlan& p,
                             const cplx<T>* __restrict__ tw, int tws) {
  return fft_smem<T, INV, MAXR>(a, b, B, B, p, tw, tws);
}

// R2C post-process.  Z holds the M-point FFT of z[n] = x[2n] + i x[2n+1];
// writes X[k], k = 0..M (M+1 bins) of the N = 2M real transform into X
// (layout [k][b]).  twN[t] = exp(-2 pi i t / N).
template <class T>
__device__ void r2c_post(const cplx<T>* __restrict__ Z, cplx<T>* __restrict__ X, int M, int B,
                         const cplx<T>* __restrict__ twN, int Bs = 0) {
  if (Bs == 0) Bs = B;
  const FastDiv fB((unsigned)B);
  const int half = M / 2;
  const int total = (half + 1) * B;
  for (int e = threadIdx.x; e < total; e += blockDim.x) {
    const int k = fB.div(e);
    const int bb = e - k * B;
    const cplx<T> zk = Z[(k == M ? 0 : k) * Bs + bb];
    const cplx<T> zc = conjg(Z[(k == 0 ? 0 : M - k) * Bs + bb]);
    const cplx<T> E = scl(add(zk, zc), (T)0.5);
    const cplx<T> D = sub(zk, zc);
    const cplx<T> O = mk<T>((T)0.5 * D.y, (T)-0.5 * D.x);  // -i/2 * D
    const cplx<T> WO = mul(twN[k], O);
    X[k * Bs + bb] = add(E, WO);
    X[(M - k) * Bs + bb] = conjg(sub(E, WO));
  }
}

// C2R pre-process: from X[k], k = 0..M (imag of X[0], X[M] ignored), build
// Z[m] (m < M) whose inverse M-point FFT is x[2n] + i x[2n+1] (unnormalised).
template <class T>
__device__ void c2r_pre(const cplx<T>* __restrict__ X, cplx<T>* __restrict__ Z, int M, int B,
                        const cplx<T>* __restrict__ twN) {
  const FastDiv fB((unsigned)B);
  const int total = M * B;
  for (int e = threadIdx.x; e < total; e += blockDim.x) {
    const int m = fB.div(e);
    const int bb = e - m * B;
    cplx<T> xm = X[m * B + bb];
    cplx<T> xc = X[(M - m) * B + bb];
    if (m == 0) {
      xm.y = (T)0;
      xc.y = (T)0;
    }
    xc = conjg(xc);
    const cplx<T> S = add(xm, xc);
    const cplx<T> D = mul(sub(xm, xc), conjg(twN[m]));
    Z[m * B + bb] = mk<T>(S.x - D.y, S.y + D.x);  // S + i D
  }
}

}  // namespace ob
