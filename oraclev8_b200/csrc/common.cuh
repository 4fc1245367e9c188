// Shared device helpers for the LH82 step kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ob {

// Interleaved complex value; 8-byte (float) or 16-byte (double) aligned so a
// warp moves it with one vector load per lane.
template <class T>
struct __align__(2 * sizeof(T)) cplx {
  T x, y;
};

template <class T>
__device__ __forceinline__ cplx<T> mk(T a, T b) {
  cplx<T> c;
  c.x = a;
  c.y = b;
  return c;
}
template <class T>
__device__ __forceinline__ cplx<T> add(cplx<T> a, cplx<T> b) { return mk<T>(a.x + b.x, a.y + b.y); }
template <class T>
__device__ __forceinline__ cplx<T> sub(cplx<T> a, cplx<T> b) { return mk<T>(a.x - b.x, a.y - b.y); }
template <class T>
__device__ __forceinline__ cplx<T> mul(cplx<T> a, cplx<T> b) {
  return mk<T>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <class T>
__device__ __forceinline__ cplx<T> conjg(cplx<T> a) { return mk<T>(a.x, -a.y); }
template <class T>
__device__ __forceinline__ cplx<T> scl(cplx<T> a, T s) { return mk<T>(a.x * s, a.y * s); }
// multiply by -i (forward) or +i (inverse)
template <class T, bool INV>
__device__ __forceinline__ cplx<T> rot(cplx<T> a) {
  return INV ? mk<T>(-a.y, a.x) : mk<T>(a.y, -a.x);
}
// i * k * a  (k real): the spectral derivative multiplier
template <class T>
__device__ __forceinline__ cplx<T> ik(T k, cplx<T> a) { return mk<T>(-k * a.y, k * a.x); }

// Round-to-nearest arithmetic without FMA contraction, for the sequences
// whose rounding must follow the reference's NumPy operation order.
__device__ __forceinline__ double mrn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double arn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double srn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double drn(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float mrn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float arn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float srn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float drn(float a, float b) { return __fdiv_rn(a, b); }
// correctly rounded 1 / a: the value drn(1, a) gives, without the general
// division's operand scaling
__device__ __forceinline__ double rcprn(double a) { return __drcp_rn(a); }
__device__ __forceinline__ float rcprn(float a) { return __frcp_rn(a); }

// ---- cp.async (global -> shared, asynchronous, no register staging) --------
__device__ __forceinline__ void cp_async(void* smem, const void* gmem, int bytes) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  if (bytes == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
  else if (bytes == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem));
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// Grid description passed by value to every kernel.
struct GridK {
  int nx, ny, nz;
  int M;        // nx / 2 (length of the packed complex FFT along x)
  int nxh;      // nx / 2 + 1 (R2C modes along x)
  double dx, dy, dz;
};

// Division by a runtime-invariant divisor d >= 1 as a multiply-high, add and
// shift (Granlund & Montgomery, 1994): q = (umulhi(m, n) + n) >> l with
// l = ceil(log2 d), m = floor(2^32 (2^l - d) / d) + 1.  Exact for n < 2^31.
struct FastDiv {
  unsigned d, m, l;
  __host__ __device__ FastDiv() : d(1), m(1), l(0) {}
  __host__ __device__ explicit FastDiv(unsigned dd) : d(dd), m(1), l(0) {
    while ((1u << l) < d) ++l;
    m = (unsigned)((((unsigned long long)1 << 32) * ((1ull << l) - d)) / d + 1ull);
  }
  __device__ __forceinline__ int div(int n) const {
    return (int)((__umulhi(m, (unsigned)n) + (unsigned)n) >> l);
  }
};

// Mixed-radix factor list of a complex FFT length, with the invariant
// divisors of each Stockham pass (Ns = product of the earlier radices).
struct FftPlan {
  int M;
  int np;
  int r[16];
  FastDiv ns[16];
};

constexpr double kGravity = 9.81;  // oracle_v8/constants.py:25

}  // namespace ob
