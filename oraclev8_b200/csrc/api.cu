// C ABI of the B200 LH82 step library.  See include/oracle_b200.h.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <cstring>
#include <array>
#include <functional>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/oracle_b200.h"
#include "kernels.cuh"
#include "pencil.cuh"
#include "xreg.cuh"
#include "xreg4.cuh"
#include "slowx.cuh"
#include "tracker.cuh"
#include "vdiag.cuh"
#include "init.cuh"

using namespace ob;

namespace {

thread_local std::string g_err;

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

#define OB_CUDA(call)                                                                    \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return fail(OB_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_),   \
                  __FILE__, __LINE__);                                                   \
  } while (0)

#define OB_LAUNCHED()                                                                    \
  do {                                                                                   \
    cudaError_t e_ = cudaGetLastError();                                                 \
    if (e_ != cudaSuccess)                                                               \
      return fail(OB_ERR_CUDA, "kernel launch failed: %s (%s:%d)", cudaGetErrorString(e_), \
                  __FILE__, __LINE__);                                                   \
  } while (0)

#define RC(x)            \
  do {                   \
    int rc_ = (x);       \
    if (rc_) return rc_; \
  } while (0)

constexpr int kThomasCols = 32;
constexpr int kFftThreads = 256;
constexpr size_t kSmemBudget = 112 * 1024;  // two CTAs per SM
constexpr size_t kSmemMax = 227 * 1024;

bool factorize(int M, FftPlan& p, bool radix16 = true) {
  p.M = M;
  p.np = 0;
  int m = M;
  auto push = [&](int r) {
    if (p.np >= 16) return false;
    p.r[p.np++] = r;
    return true;
  };
  // large radices first: each pass is one trip through shared memory.  A
  // stand-alone radix-8 pass is not used (see the kernel notes on the
  // misaligned-address fault); 8 is factored as 4 x 2.
  for (int r : {16, 4})
    while (m > 1 && m % r == 0 && (radix16 || r != 16)) {
      if (!push(r)) return false;
      m /= r;
    }
  const int rs[3] = {2, 3, 5};
  for (int r : rs)
    while (m % r == 0 && m > 1) {
      if (!push(r)) return false;
      m /= r;
    }
  int ns = 1;
  for (int s = 0; s < p.np; ++s) {
    p.ns[s] = FastDiv((unsigned)ns);
    ns *= p.r[s];
  }
  return m == 1;
}

// Radix-8-first factorisation for the kernels compiled with fft_smem<.., 8>.
bool factorize8(int M, FftPlan& p) {
  p.M = M;
  p.np = 0;
  int m = M;
  for (int r : {8, 4, 2, 3, 5})
    while (m > 1 && m % r == 0) {
      if (p.np >= 16) return false;
      p.r[p.np++] = r;
      m /= r;
    }
  int ns = 1;
  for (int s = 0; s < p.np; ++s) {
    p.ns[s] = FastDiv((unsigned)ns);
    ns *= p.r[s];
  }
  return m == 1;
}

// 2 pi fftfreq(n, d=L/n), with NumPy's operation order (numpy/fft/_helper.py),
// into k[0..n).
void fill_wavenumbers(double* k, int n, double L) {
  const double d = L / n;
  const double val = 1.0 / ((double)n * d);
  const int N = (n - 1) / 2 + 1;
  for (int i = 0; i < n; ++i) {
    const long si = (i < N) ? i : (long)i - n;
    k[i] = (2.0 * M_PI) * ((double)si * val);
  }
}
std::vector<double> wavenumbers(int n, double L) {
  std::vector<double> k(n);
  fill_wavenumbers(k.data(), n, L);
  return k;
}

// W_N^t = exp(-2 pi i t / N), t < N, evaluated in long double, into tw[0..N).
template <class T>
void fill_twiddles(cplx<T>* tw, int N) {
  for (int t = 0; t < N; ++t) {
    const long double a = -2.0L * 3.14159265358979323846264338327950288L * (long double)t /
                          (long double)N;
    tw[t].x = (T)cosl(a);
    tw[t].y = (T)sinl(a);
  }
}
template <class T>
std::vector<cplx<T>> twiddles(int N) {
  std::vector<cplx<T>> tw(N);
  fill_twiddles<T>(tw.data(), N);
  return tw;
}

// Host tables of the anelastic Poisson solver, written into caller-provided
// arrays, shared by oracle_b200_plan_create and the allocation-free solve so
// that the two cannot drift apart:
//   rh[nz + 1]   rho on half levels: interior means, boundary copies
//                (tendency.py:748-754);
//   a, c, negs[nz]  the vertical operator's sub / super diagonals and the
//                negated sum of the flux weights, Neumann edge rows
//                (poisson.py:286-315);
//   a0, cp0, inv0[nz - 1]  forward-elimination factors of the zero mode's
//                reduced system with phi(0, 0, 0) pinned (poisson.py:316-325).
struct SolverTables {
  double *rh, *a, *c, *negs, *a0, *cp0, *inv0;
};
void fill_solver_tables(int nz, double dz, const double* rf, const SolverTables& t) {
  double* rh = t.rh;
  for (int k = 1; k < nz; ++k) rh[k] = 0.5 * (rf[k - 1] + rf[k]);
  rh[0] = rf[0];
  rh[nz] = rf[nz - 1];
  const double dz2 = dz * dz;
  auto rl = [&](int k) { return rh[k] / dz2; };
  auto ru = [&](int k) { return rh[k + 1] / dz2; };
  for (int k = 0; k < nz; ++k) {
    t.a[k] = rl(k);
    t.c[k] = ru(k);
    t.negs[k] = -(rl(k) + ru(k));
  }
  t.a[0] = 0.0;
  t.c[nz - 1] = 0.0;
  t.negs[0] = -ru(0);
  t.negs[nz - 1] = -rl(nz - 1);
  // the reduced system's rows j = 0 .. n0 - 1 are levels 1 .. nz - 1
  const int n0 = nz - 1;
  auto a0 = [&](int j) { return j == 0 ? 0.0 : (j == n0 - 1 ? rl(nz - 1) : rl(j + 1)); };
  auto b0 = [&](int j) { return j == n0 - 1 ? -rl(nz - 1) : -(rl(j + 1) + ru(j + 1)); };
  auto c0 = [&](int j) { return j == n0 - 1 ? 0.0 : ru(j + 1); };
  for (int j = 0; j < n0; ++j) t.a0[j] = a0(j);
  t.inv0[0] = 1.0 / b0(0);
  t.cp0[0] = c0(0) * t.inv0[0];
  for (int j = 1; j < n0; ++j) {
    const double den = b0(j) - t.a0[j] * t.cp0[j - 1];
    t.inv0[j] = 1.0 / den;
    t.cp0[j] = (j < n0 - 1) ? c0(j) * t.inv0[j] : 0.0;
  }
}

}  // namespace

struct OraclePlan {
  int prec = 0;
  GridK g{};
  int buoyancy = 0, projection = 0, advection = 0, coriolis = 0, damping = 0, heating = 0;
  double f0 = 0, u_env = 0, v_env = 0, epsilon = 0;
  // production slow components (OracleComponentDesc)
  int drag = 0, sponge = 0, diffusion = 0, cooling = 0;
  double drag_cd = 0, drag_dz = 1, drag_u_env = 0, drag_v_env = 0;
  double sponge_u_env = 0, sponge_v_env = 0;
  double diff_nu = 0, diff_dx2 = 1, diff_dy2 = 1, cool_alpha = 0;
  double blowup_u = 0;  // max|u| limit of the blow-up flag (0: non-finite values only)
  double *drag_w = nullptr, *sp_a = nullptr, *sp_ah = nullptr;
  void *Lu = nullptr, *Lv = nullptr;  // biharmonic: the inner Laplacians
  int diag_every = 60;
  long solve_count = 0;
  FftPlan px{}, py{};    // radix-16-first plans (inverse kernels)
  FftPlan pxf{}, pyf{};  // radix-4-first plans (forward kernels: lower register pressure)
  int zc_fx = 1, zc_fy = 1, zc_iy = 1, zc_ix = 1;
  // x-pencil kernels with compile-time z-chunks (pencil.cuh); 0 = not used
  FftPlan px8{}, py8{};
  bool px8_ok = false, py8_ok = false;  // nx/2 and ny factor into 8, 4, 2, 3, 5
  int zc2_fx = 0, zc2_fxs = 0, zc2_ix = 0, zc2_fy = 0, zc2_iy = 0;
  // register-resident x pencils of FP32 plans at nx = 512 (z-chunk, 0 = off): the
  // projection's forward and inverse kernels, and the FP64 residual transform
  int zc3_fx = 0, zc3_fxs = 0, zc3_ix = 0, zc3_fxd = 0;
  int zc3_fy = 0;  // register-resident FP32 y pencils (ny = 512): z-chunk, 0 = off
  int zc3_fyd = 0;  // the FP64 residual y transform at ny = 512 (register form): 0 or 2
  int thomas_fast = 1;  // FP32 short-wave sweep with a compile-time level count
  // register-resident pencils of the 1024-point lines (xreg4.cuh), FP32 plans:
  // forward x (stage / correction), inverse x, the FP64 residual x transform,
  // and the y pencils (ny = 1024); z-chunk, 0 = off
  int zc4_fxs = 0, zc4_fx = 0, zc4_ix = 0, zc4_fxd = 0, zc4_fy = 0, zc4_iy = 0, zc4_fyd = 0;
  // the three fast stages from one forward x transform of the anchor state
  // (k_fx4 with four column groups into S4..S6, then k_fy4 forming each
  // stage's divergence spectrum): its z-chunk, 0 = off; needs zc4_fy
  int zc4_fxsh = 0;
  // FP32 slow tendency: 0 the gather form, 1 marching along x (k_slow_xw),
  // 4 / 8 marching along x over bulk-copied planes of 4 / 8 rows (k_slow_xt)
  int slow_xw = 1;
  // FP64 defect correction of single-precision plans: a double-precision
  // shadow descriptor (own twiddles and spectral buffers, shared tables)
  OraclePlan* dbl = nullptr;
  int refine_passes = 0, refine_every = 1;
  long step_count = 0;
  int capturing = 0;  // recording a step graph: no solver-residual logging
  size_t esz = 8;  // element size of T
  // device constants
  double *kx = nullptr, *ky = nullptr, *rho = nullptr, *rhoh = nullptr, *theta0 = nullptr;
  double *dth0 = nullptr, *fy = nullptr, *heat_r = nullptr, *heat_z = nullptr;
  double *ta = nullptr, *tc = nullptr, *tnegs = nullptr, *ta0 = nullptr, *tcp0 = nullptr,
         *tinv0 = nullptr;
  void *twx = nullptr, *twy = nullptr;
  // scratch
  void *S1 = nullptr, *S2 = nullptr, *S3 = nullptr;           // spectral
  // the shared stage transforms (allocated where zc4_fxsh can be on):
  // S4 = i kx' FFTx(rho u) + FFTx(D w), S5 = FFTx(rho v), S6 = FFTx(D b_half)
  void *S4 = nullptr, *S5 = nullptr, *S6 = nullptr;
  void *Au = nullptr, *Av = nullptr, *Aw = nullptr, *Ath = nullptr, *Aphi = nullptr;
  void *Su = nullptr, *Sv = nullptr, *Sw = nullptr, *Sphi = nullptr;
  void *Du = nullptr, *Dv = nullptr;                         // damper / temp
  void* Bh = nullptr;  // half-level buoyancy of the step's anchor theta' (nz + 1 levels)
  double* diag = nullptr;
  DiagPart* parts = nullptr;
  int nparts = 0;
  std::vector<void*> allocs;
  size_t scratch_bytes = 0;
  cudaMemPool_t pool = nullptr;   // device memory pool (plan_pool)
  cudaStream_t astream = nullptr; // private stream ordering set-up work
  // split FP32 Thomas solve: the column blocks holding a long-wave mode
  // (k^2 Lz^2 < 1), as a list and as per-block flags, and the side stream
  // and fork/join events that run their double launch beside the rest
  int* lw_blocks = nullptr;
  unsigned char* lw_flag = nullptr;
  int n_lw = 0;
  float* tcoef = nullptr;  // FP32 plans: (negs, rho, a, c) per level, as float4
  float* gth = nullptr;    // FP32 plans: g / theta0 per level
  cudaStream_t aux = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // launch accounting and optional per-kernel-class event timing
  long launches = 0;
  int profiling = 0;
  struct Mark {
    int cls;
    cudaEvent_t a, b;
  };
  std::vector<Mark> marks;
  // timing events, created when profiling is switched on and reused: a
  // profiled launch records two of them and creates none
  std::vector<cudaEvent_t> ev_pool;
  size_t ev_next = 0;
};

namespace {

// Plan memory comes from one stream-ordered pool per device that keeps the
// blocks it is given back (release threshold = max).  A loop that retires
// and creates plans (a serving loop) then reuses the same device memory: no
// page mapping per plan, and no device-wide synchronisation on release, which
// cudaFree implies.
std::mutex g_pool_mu;
constexpr int kMaxDevices = 64;
cudaMemPool_t g_pools[kMaxDevices] = {};

int plan_pool(cudaMemPool_t* out) {
  int dev = 0;
  OB_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return fail(OB_ERR_UNSUPPORTED, "device index %d", dev);
  std::lock_guard<std::mutex> lk(g_pool_mu);
  if (!g_pools[dev]) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    OB_CUDA(cudaMemPoolCreate(&pool, &props));
    unsigned long long keep = ~0ull;
    OB_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    g_pools[dev] = pool;
  }
  *out = g_pools[dev];
  return OB_OK;
}

// Allocations are ordered on the plan's private set-up stream; plan_create
// synchronises that stream before returning, after which the memory may be
// used on any stream.
template <class P>
int dalloc(OraclePlan* p, P** out, size_t bytes) {
  void* q = nullptr;
  cudaError_t e = cudaMallocFromPoolAsync(&q, bytes, p->pool, p->astream);
  if (e == cudaErrorMemoryAllocation) {
    // give blocks the pool holds for reuse back to the device, then retry
    cudaGetLastError();
    OB_CUDA(cudaStreamSynchronize(p->astream));
    OB_CUDA(cudaMemPoolTrimTo(p->pool, 0));
    e = cudaMallocFromPoolAsync(&q, bytes, p->pool, p->astream);
  }
  if (e != cudaSuccess)
    return fail(OB_ERR_CUDA, "plan allocation of %zu bytes failed: %s", bytes,
                cudaGetErrorString(e));
  p->allocs.push_back(q);
  p->scratch_bytes += bytes;
  *out = reinterpret_cast<P*>(q);
  return OB_OK;
}

int upload(OraclePlan* p, double** out, const double* host, size_t n) {
  int rc = dalloc(p, out, n * sizeof(double));
  if (rc) return rc;
  OB_CUDA(cudaMemcpyAsync(*out, host, n * sizeof(double), cudaMemcpyHostToDevice, p->astream));
  return OB_OK;
}

// Release a plan's memory in the order of `st` (the pool reuses it once the
// work queued on `st` before this point is done) and free the descriptor.
void release_plan(OraclePlan* p, cudaStream_t st) {
  delete p->dbl;  // owns no allocations: its buffers are in p->allocs
  for (cudaEvent_t e : p->ev_pool) cudaEventDestroy(e);
  for (void* q : p->allocs) cudaFreeAsync(q, st);
  if (p->astream) cudaStreamDestroy(p->astream);
  if (p->aux) cudaStreamDestroy(p->aux);
  if (p->ev_fork) cudaEventDestroy(p->ev_fork);
  if (p->ev_join) cudaEventDestroy(p->ev_join);
  delete p;
}

int pick_zc(int nz, size_t per_zc, size_t fixed) {
  int best = 1;
  for (int zc : {16, 8, 4, 2, 1}) {
    if (zc > nz && zc > 1) continue;
    if (fixed + per_zc * (size_t)zc <= kSmemBudget) {
      best = zc;
      break;
    }
  }
  return best;
}

// bytes of a twiddle table of n complex entries staged at the start of the
// FFT kernels' dynamic shared memory
size_t tw_bytes(const OraclePlan* p, int n) { return ((size_t)n * 2 * p->esz + 15) & ~size_t(15); }
size_t smem_fx(const OraclePlan* p, int nf) {
  return tw_bytes(p, p->g.nx) + 2ull * (p->g.M + 1) * nf * p->zc_fx * 2 * p->esz;
}
size_t smem_fy(const OraclePlan* p, int nf, int zc) {
  return tw_bytes(p, p->g.ny) + 2ull * p->g.ny * nf * zc * 2 * p->esz;
}
size_t smem_ix(const OraclePlan* p, int B) {
  return tw_bytes(p, p->g.nx) + (size_t)(2 * p->g.M + 1) * B * 2 * p->esz;
}
// staging in the sweep type plus the zero mode's double region (k_thomas)
size_t smem_thomas(const OraclePlan* p, size_t rsz = 8) {
  return thomas_stage_offset(p->g.nz + 1) + 3ull * kThomasCols * (p->g.nz + 1) * rsz;
}

template <class K>
int x2_attr(K kernel) {
  OB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemMax));
  OB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  return OB_OK;
}

template <class T, class TS, int ZC>
int x2_attrs_zc() {
  int rc;
  if constexpr (sizeof(TS) == sizeof(T)) {
    if ((rc = x2_attr(k_fy2<T, FY_DIV, T, ZC>)) || (rc = x2_attr(k_iy2<T, ZC>))) return rc;
  }
  if ((rc = x2_attr(k_fx2<T, false, TS, ZC>)) || (rc = x2_attr(k_fx2<T, true, TS, ZC>)) ||
      (rc = x2_attr(k_ix2<T, IX_CORRECT, TS, ZC>)) || (rc = x2_attr(k_ix2<T, IX_STAGE, TS, ZC>)))
    return rc;
  if constexpr (sizeof(TS) == 4)
    if ((rc = x2_attr(k_ix2<T, IX_REFINE, TS, ZC>))) return rc;
  return OB_OK;
}

template <class T, bool STAGE, int ZC>
int xr_attr_fx3() {
  OB_CUDA(cudaFuncSetAttribute(k_fx3<T, STAGE, ZC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)fx3_smem<T, STAGE, ZC>()));
  return OB_OK;
}

template <int MODE, int ZC>
int xr_attr_ix3() {
  OB_CUDA(cudaFuncSetAttribute(k_ix3<MODE, ZC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)Ix3Size<ZC>::total));
  return OB_OK;
}
template <int ZC>
int xr_attrs_ix3() {
  int rc;
  if ((rc = xr_attr_ix3<IX_CORRECT, ZC>()) || (rc = xr_attr_ix3<IX_STAGE, ZC>()) ||
      (rc = xr_attr_ix3<IX_REFINE, ZC>()) || (rc = xr_attr_ix3<IX_FIELDS, ZC>()))
    return rc;
  OB_CUDA(cudaFuncSetAttribute(k_fx3<float, false, ZC, true>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)fx3_smem<float, false, ZC>()));
  return OB_OK;
}

template <int ZC>
int yr_attrs() {
  OB_CUDA(cudaFuncSetAttribute(k_fy3<ZC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)YrSize<ZC>::total));
  OB_CUDA(cudaFuncSetAttribute(k_iy3<ZC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)YrSize<ZC>::total));
  OB_CUDA(cudaFuncSetAttribute(k_hy3<ZC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)HySize<ZC>::total));
  return OB_OK;
}

template <class T, bool STAGE, int ZC>
int xr4_attr_fx() {
  OB_CUDA(cudaFuncSetAttribute(k_fx4<T, STAGE, ZC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)fx4_smem<T, STAGE, ZC>()));
  return OB_OK;
}
template <int ZC>
int xr4_attrs_zc() {
  int rc;
  if ((rc = xr4_attr_fx<float, false, ZC>()) || (rc = xr4_attr_fx<float, true, ZC>()))
    return rc;
  OB_CUDA(cudaFuncSetAttribute(k_fx4<float, true, ZC, 4>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)fx4_smem<float, true, ZC, 4>()));
  OB_CUDA(cudaFuncSetAttribute(k_fy4<ZC, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)Yr4Size<ZC, 3>::total));
  if constexpr (ZC <= 4)
    if ((rc = xr4_attr_fx<double, false, ZC>())) return rc;
  for (auto k : {k_ix4<IX_CORRECT, ZC>, k_ix4<IX_STAGE, ZC>, k_ix4<IX_REFINE, ZC>})
    OB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)Ix4Size<ZC>::total));
  OB_CUDA(cudaFuncSetAttribute(k_fy4<ZC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)Yr4Size<ZC>::total));
  if constexpr (ZC == 2)
    OB_CUDA(cudaFuncSetAttribute(k_fy4d, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)Yr4dSize::total));
  OB_CUDA(cudaFuncSetAttribute(k_iy4<ZC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)Yr4Size<ZC>::total));
  return OB_OK;
}

template <class T>
int set_x2_attrs() {
  int rc;
  if constexpr (sizeof(T) == 4)
    if ((rc = xr4_attrs_zc<2>()) || (rc = xr4_attrs_zc<4>()) || (rc = xr4_attrs_zc<8>()))
      return rc;
  if constexpr (sizeof(T) == 4) {
    if ((rc = yr_attrs<2>()) || (rc = yr_attrs<4>()) || (rc = yr_attrs<8>())) return rc;
  } else {  // the defect correction's FP64 residual y transform
    OB_CUDA(cudaFuncSetAttribute(k_fy3<2, double, FY_RESID, float>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)YrSize<2, double>::total));
  }
  if constexpr (sizeof(T) == 4) {
    if ((rc = xr_attrs_ix3<2>()) || (rc = xr_attrs_ix3<4>()) || (rc = xr_attrs_ix3<8>()))
      return rc;
    if ((rc = xr_attr_fx3<float, false, 2>()) || (rc = xr_attr_fx3<float, true, 2>()) ||
        (rc = xr_attr_fx3<float, false, 4>()) || (rc = xr_attr_fx3<float, true, 4>()) ||
        (rc = xr_attr_fx3<float, false, 8>()) || (rc = xr_attr_fx3<float, true, 8>()) ||
        (rc = xr_attr_fx3<double, false, 2>()) || (rc = xr_attr_fx3<double, false, 4>()))
      return rc;
  }
  if ((rc = x2_attrs_zc<T, T, 1>()) || (rc = x2_attrs_zc<T, T, 2>()) ||
      (rc = x2_attrs_zc<T, T, 4>()) || (rc = x2_attrs_zc<T, T, 8>()))
    return rc;
  if constexpr (sizeof(T) == 8) {  // residual transforms of the FP32 defect correction
    for (auto k : {k_fx2<double, false, float, 1>, k_fx2<double, false, float, 2>,
                   k_fx2<double, false, float, 4>, k_fx2<double, false, float, 8>})
      if ((rc = x2_attr(k))) return rc;
    for (auto k : {k_fy2<double, FY_RESID, float, 1>, k_fy2<double, FY_RESID, float, 2>,
                   k_fy2<double, FY_RESID, float, 4>, k_fy2<double, FY_RESID, float, 8>})
      if ((rc = x2_attr(k))) return rc;
  }
  return OB_OK;
}

int slow_xt_attrs(int nz);

template <class T>
int set_smem_attrs() {
  const int mx = (int)kSmemMax;
  if constexpr (sizeof(T) == 4)
    for (int nz : {32, 48, 64, 80})
      if (int rc = slow_xt_attrs(nz)) return rc;
  OB_CUDA(cudaFuncSetAttribute(k_fx<T, FX_DIV>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
  OB_CUDA(cudaFuncSetAttribute(k_fx<T, FX_DIV_STAGE>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
  OB_CUDA(cudaFuncSetAttribute(k_fx<T, FX_FIELDS>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
  OB_CUDA(cudaFuncSetAttribute(k_fy<T, FY_DIV>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
  OB_CUDA(cudaFuncSetAttribute(k_fy<T, FY_FIELDS>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
  OB_CUDA(cudaFuncSetAttribute(k_fy<T, FY_HELM>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
  OB_CUDA(cudaFuncSetAttribute(k_iy<T, IY_GRAD>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
  OB_CUDA(cudaFuncSetAttribute(k_iy<T, IY_FIELDS>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
  OB_CUDA(cudaFuncSetAttribute(k_ix<T, IX_CORRECT>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
  OB_CUDA(cudaFuncSetAttribute(k_ix<T, IX_STAGE>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
  OB_CUDA(cudaFuncSetAttribute(k_ix<T, IX_GRAD>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
  OB_CUDA(cudaFuncSetAttribute(k_ix<T, IX_FIELDS>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
  OB_CUDA(cudaFuncSetAttribute(k_thomas<T, kThomasCols>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
  OB_CUDA(cudaFuncSetAttribute(k_fx<double, FX_DIV, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
  OB_CUDA(cudaFuncSetAttribute(k_fy<double, FY_RESID, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
  OB_CUDA(cudaFuncSetAttribute(k_ix<float, IX_REFINE>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
  return set_x2_attrs<T>();
}

// Kernel attributes are per function and device: set them once per device.
template <class T>
int set_smem_attrs_once() {
  static std::mutex mu;
  static bool done[kMaxDevices] = {};
  int dev = 0;
  OB_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  const bool known = dev >= 0 && dev < kMaxDevices;
  if (known && done[dev]) return OB_OK;
  if (int rc = set_smem_attrs<T>()) return rc;
  if (known) done[dev] = true;
  return OB_OK;
}

ThomasK thomas_args(const OraclePlan* p) {
  ThomasK t;
  t.a = p->ta;
  t.c = p->tc;
  t.negs = p->tnegs;
  t.rho = p->rho;
  t.rhoh = p->rhoh;
  t.kx = p->kx;
  t.ky = p->ky;
  t.a0 = p->ta0;
  t.cp0 = p->tcp0;
  t.inv0 = p->tinv0;
  t.dz = p->g.dz;
  t.scale = 1.0 / ((double)p->g.nx * (double)p->g.ny);
  return t;
}

// Brackets one kernel launch: counts it and, when profiling is on, records a
// pair of events on the launch stream so per-class device time can be summed.
// Next event of the plan's timing pool (grown only when a profiled run
// outlasts the events created up front).
cudaEvent_t pool_event(OraclePlan* p) {
  if (p->ev_next == p->ev_pool.size()) {
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    p->ev_pool.push_back(e);
  }
  return p->ev_pool[p->ev_next++];
}

struct Launch {
  OraclePlan* p;
  cudaStream_t st;
  int cls;
  cudaEvent_t a = nullptr, b = nullptr;
  Launch(OraclePlan* p_, int cls_, cudaStream_t st_) : p(p_), st(st_), cls(cls_) {
    p->launches++;
    if (p->profiling) {
      a = pool_event(p);
      b = pool_event(p);
      cudaEventRecord(a, st);
    }
  }
  ~Launch() {
    if (a && b) {
      cudaEventRecord(b, st);
      p->marks.push_back({cls, a, b});
    }
  }
};

dim3 grid_x(const OraclePlan* p, int zc) { return dim3((p->g.nz + zc - 1) / zc, p->g.ny); }
dim3 grid_y(const OraclePlan* p, int zc) { return dim3((p->g.nz + zc - 1) / zc, p->g.nxh); }

// ---- x2 pencil kernels (pencil.cuh) ----------------------------------------
// Shared memory per CTA the x-pencil z-chunk choice aims at.  k_ix2's time
// follows the bytes it moves per global sector (a row's ZC levels are one
// run): at nx = 512, FP32, 5.9 / 2.3 / 1.66 ms per step at ZC = 2 / 4 / 8,
// the last at two CTAs per SM, so it gets two CTAs' worth.  The FP32 forward
// kernel measured faster at ZC = 4 with three or more CTAs per SM (1.41 ms
// per step) than at ZC = 8 with two (1.48 ms).
template <class T>
size_t x2_smem_budget(int kind) {
  return (sizeof(T) == 4 && kind < 2) ? 74 * 1024 : 112 * 1024;
}
// y pencils (complex rows of ZC levels, at least 16-byte runs): three CTAs
// per SM in FP32, two in FP64
template <class T>
size_t y2_smem_budget() {
  return sizeof(T) == 4 ? 74 * 1024 : 112 * 1024;
}

// Dynamic shared memory of a k_fx2 (kinds 0 and 1: plain and staged) or k_ix2
// (kind 2) launch with z-chunk zc.
template <class T, class TS>
size_t x2_smem(int kind, int zc, int nx) {
  switch (zc) {
#define OB_X2_CASE(Z)                                                                  \
  case Z:                                                                              \
    return kind < 2 ? fx2_layout<T, TS, Z>(nx).total : ix2_layout<T, Z>(nx).total;
    OB_X2_CASE(1)
    OB_X2_CASE(2)
    OB_X2_CASE(4)
    OB_X2_CASE(8)
#undef OB_X2_CASE
  }
  return ~size_t(0);
}

// Largest z-chunk in {8, 4, 2, 1} (no larger than nz) whose tile fits the
// per-CTA budget of the kernels' target occupancy, else the largest that fits
// one CTA; 0 when none fits.  The chunk is then raised, where one CTA still
// holds it, until a row's run of state is 16 bytes (4 FP32 / 2 FP64 levels):
// the x pencils' time follows the sector operations per byte more than the
// CTAs per SM.  At 1024^2 x 80 the FP64 step took 98.3 ms per step with
// 1-level inverse chunks at two CTAs per SM and 79.5 ms with 2-level chunks at
// one; the FP32-refined step 60.9 ms with 2-level chunks and 46.2 ms with 4.
template <class T, class TS>
int pick_x2_zc(int kind, int nx, int nz) {
  int zc = 0;
  for (size_t cap : {x2_smem_budget<T>(kind), kSmemMax}) {
    for (int z : {8, 4, 2, 1}) {
      if (z > 1 && z > nz) continue;
      if (x2_smem<T, TS>(kind, z, nx) <= cap) {
        zc = z;
        break;
      }
    }
    if (zc) break;
  }
  const int zmin = std::min(nz, 16 / (int)sizeof(TS));
  while (zc && zc < zmin && zc < 8 && x2_smem<T, TS>(kind, 2 * zc, nx) <= kSmemMax) zc *= 2;
  return zc;
}

// bh: the step's half-level buoyancy field (STAGE only)
template <class T>
size_t y2_smem_zc(int zc, int ny) {
  switch (zc) {
    case 1: return y2_smem<T, 1>(ny);
    case 2: return y2_smem<T, 2>(ny);
    case 4: return y2_smem<T, 4>(ny);
    case 8: return y2_smem<T, 8>(ny);
  }
  return ~size_t(0);
}

template <class T>
int pick_y2_zc(int ny, int nz) {
  for (size_t cap : {y2_smem_budget<T>(), kSmemMax})
    for (int zc : {8, 4, 2, 1}) {
      if (zc > 1 && zc > nz) continue;
      if (y2_smem_zc<T>(zc, ny) <= cap) return zc;
    }
  return 0;
}

template <class T, int MODE, class TO>
void fy2(const OraclePlan* q, int zc, const cplx<T>* in0, const cplx<T>* in1, cplx<TO>* out,
         cudaStream_t st) {
  const GridK& g = q->g;
  const cplx<T>* tw = (const cplx<T>*)q->twy;
  switch (zc) {
#define OB_FY2(Z)                                                                             \
  case Z:                                                                                     \
    k_fy2<T, MODE, TO, Z><<<dim3((g.nz + Z - 1) / Z, g.nxh), kPencilThreads, y2_smem<T, Z>(g.ny), \
                           st>>>(g, q->py8, in0, in1, q->ky, tw, out);                        \
    break;
    OB_FY2(1)
    OB_FY2(2)
    OB_FY2(4)
    OB_FY2(8)
#undef OB_FY2
  }
}

template <int ZC>
void yr_launch(const OraclePlan* p, bool inverse, const cplx<float>* in0, const cplx<float>* in1,
               cplx<float>* out0, cplx<float>* out1, cudaStream_t st) {
  const dim3 grid((p->g.nz + ZC - 1) / ZC, p->g.nxh);
  const cplx<float>* tw = (const cplx<float>*)p->twy;
  if (inverse)
    k_iy3<ZC><<<grid, 64 * ZC, YrSize<ZC>::total, st>>>(p->g, in0, p->ky, tw, out0, out1);
  else
    k_fy3<ZC><<<grid, 64 * ZC, YrSize<ZC>::total, st>>>(p->g, in0, in1, p->ky, tw, out0);
}
// the damper's fused y stage (FP32, ny = 512), in place on (S1, S2)
template <int ZC>
void hy_launch(const OraclePlan* p, double scale, cplx<float>* s1, cplx<float>* s2,
               cudaStream_t st) {
  const dim3 grid((p->g.nz + ZC - 1) / ZC, p->g.nxh);
  k_hy3<ZC><<<grid, 64 * ZC, HySize<ZC>::total, st>>>(
      p->g, s1, s2, p->kx, p->ky, (const cplx<float>*)p->twy, scale, s1, s2);
}
void hy(const OraclePlan* p, double scale, cplx<float>* s1, cplx<float>* s2, cudaStream_t st) {
  switch (p->zc3_fy) {
    case 2: hy_launch<2>(p, scale, s1, s2, st); break;
    case 4: hy_launch<4>(p, scale, s1, s2, st); break;
    default: hy_launch<8>(p, scale, s1, s2, st); break;
  }
}

// register-resident FP32 y pencils (ny = 512): FY_DIV forward or the IY_GRAD inverse
void yr(const OraclePlan* p, bool inverse, const cplx<float>* in0, const cplx<float>* in1,
        cplx<float>* out0, cplx<float>* out1, cudaStream_t st) {
  switch (p->zc3_fy) {
    case 2: yr_launch<2>(p, inverse, in0, in1, out0, out1, st); break;
    case 4: yr_launch<4>(p, inverse, in0, in1, out0, out1, st); break;
    default: yr_launch<8>(p, inverse, in0, in1, out0, out1, st); break;
  }
}

template <class T>
void iy2(const OraclePlan* p, int zc, const cplx<T>* in0, cplx<T>* out0, cplx<T>* out1,
         cudaStream_t st) {
  const GridK& g = p->g;
  const cplx<T>* tw = (const cplx<T>*)p->twy;
  switch (zc) {
#define OB_IY2(Z)                                                                             \
  case Z:                                                                                     \
    k_iy2<T, Z><<<dim3((g.nz + Z - 1) / Z, g.nxh), kPencilThreads, y2_smem<T, Z>(g.ny), st>>>( \
        g, p->py8, in0, p->ky, tw, out0, out1);                                               \
    break;
    OB_IY2(1)
    OB_IY2(2)
    OB_IY2(4)
    OB_IY2(8)
#undef OB_IY2
  }
}

template <class T, bool STAGE, class TS, int ZC>
void fx2_launch(const OraclePlan* q, const TS* u, const TS* v, const TS* w, const TS* bh,
                double sdt, cplx<T>* X0, cplx<T>* X1, cudaStream_t st) {
  const dim3 grid((q->g.nz + ZC - 1) / ZC, q->g.ny);
  k_fx2<T, STAGE, TS, ZC><<<grid, kPencilThreads, fx2_layout<T, TS, ZC>(q->g.nx).total,
                            st>>>(q->g, q->px8, u, v, w, bh, sdt, q->rho, q->rhoh, q->kx,
                                  (const cplx<T>*)q->twx, X0, X1);
}

template <class T, bool STAGE, class TS>
void fx2(const OraclePlan* q, int zc, const TS* u, const TS* v, const TS* w, const TS* bh,
         double sdt, cplx<T>* X0, cplx<T>* X1, cudaStream_t st) {
  switch (zc) {
    case 1: fx2_launch<T, STAGE, TS, 1>(q, u, v, w, bh, sdt, X0, X1, st); break;
    case 2: fx2_launch<T, STAGE, TS, 2>(q, u, v, w, bh, sdt, X0, X1, st); break;
    case 4: fx2_launch<T, STAGE, TS, 4>(q, u, v, w, bh, sdt, X0, X1, st); break;
    default: fx2_launch<T, STAGE, TS, 8>(q, u, v, w, bh, sdt, X0, X1, st); break;
  }
}

template <class T, bool STAGE, int ZC>
void fx3_launch(const OraclePlan* q, const float* u, const float* v, const float* w,
                const float* bh, double sdt, cplx<T>* X0, cplx<T>* X1, cudaStream_t st) {
  const dim3 grid((q->g.nz + ZC - 1) / ZC, q->g.ny);
  k_fx3<T, STAGE, ZC><<<grid, 48 * ZC, fx3_smem<T, STAGE, ZC>(), st>>>(
      q->g, u, v, w, bh, sdt, q->rho, q->rhoh, q->kx, (const cplx<T>*)q->twx, X0, X1);
}
// q's twiddles are of type T (the FP64 refiner plan for T = double)
template <class T, bool STAGE>
void fx3(const OraclePlan* q, int zc, const float* u, const float* v, const float* w,
         const float* bh, double sdt, cplx<T>* X0, cplx<T>* X1, cudaStream_t st) {
  if constexpr (sizeof(T) == 8) {
    if (zc == 2) fx3_launch<T, false, 2>(q, u, v, w, bh, sdt, X0, X1, st);
    else fx3_launch<T, false, 4>(q, u, v, w, bh, sdt, X0, X1, st);
  } else {
    switch (zc) {
      case 2: fx3_launch<T, STAGE, 2>(q, u, v, w, bh, sdt, X0, X1, st); break;
      case 4: fx3_launch<T, STAGE, 4>(q, u, v, w, bh, sdt, X0, X1, st); break;
      default: fx3_launch<T, STAGE, 8>(q, u, v, w, bh, sdt, X0, X1, st); break;
    }
  }
}

// the Helmholtz damper's forward x transform (FP32, nx = 512): FFTx(u), FFTx(v)
template <int ZC>
void fx3f_launch(const OraclePlan* p, const float* u, const float* v, cplx<float>* X0,
                 cplx<float>* X1, cudaStream_t st) {
  const dim3 grid((p->g.nz + ZC - 1) / ZC, p->g.ny);
  k_fx3<float, false, ZC, true><<<grid, 48 * ZC, fx3_smem<float, false, ZC>(), st>>>(
      p->g, u, v, nullptr, nullptr, 0.0, p->rho, p->rhoh, p->kx, (const cplx<float>*)p->twx,
      X0, X1);
}
void fx3f(const OraclePlan* p, int zc, const float* u, const float* v, cplx<float>* X0,
          cplx<float>* X1, cudaStream_t st) {
  switch (zc) {
    case 2: fx3f_launch<2>(p, u, v, X0, X1, st); break;
    case 4: fx3f_launch<4>(p, u, v, X0, X1, st); break;
    default: fx3f_launch<8>(p, u, v, X0, X1, st); break;
  }
}

template <int MODE, int ZC>
void ix3_launch(const OraclePlan* p, const cplx<float>* phs, const cplx<float>* psi,
                const float* u, const float* v, const float* w, const float* bh, double sdt,
                float* uo, float* vo, float* wo, float* phio, cudaStream_t st) {
  const dim3 grid((p->g.nz + ZC - 1) / ZC, p->g.ny);
  k_ix3<MODE, ZC><<<grid, 16 * (3 * ZC + 2), Ix3Size<ZC>::total, st>>>(
      p->g, phs, psi, p->kx, (const cplx<float>*)p->twx, u, v, w, bh, sdt, uo, vo, wo, phio);
}
template <int MODE>
void ix3(const OraclePlan* p, int zc, const cplx<float>* phs, const cplx<float>* psi,
         const float* u, const float* v, const float* w, const float* bh, double sdt,
         float* uo, float* vo, float* wo, float* phio, cudaStream_t st) {
  switch (zc) {
    case 2: ix3_launch<MODE, 2>(p, phs, psi, u, v, w, bh, sdt, uo, vo, wo, phio, st); break;
    case 4: ix3_launch<MODE, 4>(p, phs, psi, u, v, w, bh, sdt, uo, vo, wo, phio, st); break;
    default: ix3_launch<MODE, 8>(p, phs, psi, u, v, w, bh, sdt, uo, vo, wo, phio, st); break;
  }
}

template <class T, int MODE, class TS, int ZC>
void ix2_launch(const OraclePlan* p, const cplx<T>* phs, const cplx<T>* psi, const TS* u,
                const TS* v, const TS* w, const TS* bh, double sdt, TS* uo, TS* vo, TS* wo,
                TS* phio, cudaStream_t st) {
  const dim3 grid((p->g.nz + ZC - 1) / ZC, p->g.ny);
  k_ix2<T, MODE, TS, ZC><<<grid, kPencilThreads,
                           ix2_layout<T, ZC>(p->g.nx).total, st>>>(
      p->g, p->px8, phs, psi, p->kx, (const cplx<T>*)p->twx, u, v, w, bh, sdt, uo, vo, wo,
      phio);
}

template <class T, int MODE, class TS>
void ix2(const OraclePlan* p, int zc, const cplx<T>* phs, const cplx<T>* psi, const TS* u,
         const TS* v, const TS* w, const TS* bh, double sdt, TS* uo, TS* vo, TS* wo, TS* phio,
         cudaStream_t st) {
  switch (zc) {
    case 1: ix2_launch<T, MODE, TS, 1>(p, phs, psi, u, v, w, bh, sdt, uo, vo, wo, phio, st); break;
    case 2: ix2_launch<T, MODE, TS, 2>(p, phs, psi, u, v, w, bh, sdt, uo, vo, wo, phio, st); break;
    case 4: ix2_launch<T, MODE, TS, 4>(p, phs, psi, u, v, w, bh, sdt, uo, vo, wo, phio, st); break;
    default: ix2_launch<T, MODE, TS, 8>(p, phs, psi, u, v, w, bh, sdt, uo, vo, wo, phio, st); break;
  }
}

// ---- register-resident pencils of the 1024-point lines (xreg4.cuh) --------
template <class K>
int resident_ctas(K kernel, int threads, size_t smem);

template <class T, bool STAGE, int ZC>
void fx4_launch(const OraclePlan* q, const float* u, const float* v, const float* w,
                const float* bh, double sdt, cplx<T>* X0, cplx<T>* X1, cudaStream_t st) {
  const dim3 grid((q->g.nz + ZC - 1) / ZC, q->g.ny);
  k_fx4<T, STAGE, ZC><<<grid, 96 * ZC, fx4_smem<T, STAGE, ZC>(), st>>>(
      q->g, u, v, w, bh, sdt, q->rho, q->rhoh, q->kx, (const cplx<T>*)q->twx, X0, X1, nullptr);
}
// the three fast stages' shared forward x transforms: S4, S5, S6
template <int ZC>
void fx4sh_launch(const OraclePlan* p, const float* u, const float* v, const float* w,
                  const float* bh, cudaStream_t st) {
  const dim3 grid((p->g.nz + ZC - 1) / ZC, p->g.ny);
  k_fx4<float, true, ZC, 4><<<grid, 128 * ZC, fx4_smem<float, true, ZC, 4>(), st>>>(
      p->g, u, v, w, bh, 0.0, p->rho, p->rhoh, p->kx, (const cplx<float>*)p->twx,
      (cplx<float>*)p->S4, (cplx<float>*)p->S5, (cplx<float>*)p->S6);
}
void fx4sh(const OraclePlan* p, const float* u, const float* v, const float* w,
           const float* bh, cudaStream_t st) {
  switch (p->zc4_fxsh) {
    case 2: fx4sh_launch<2>(p, u, v, w, bh, st); break;
    case 4: fx4sh_launch<4>(p, u, v, w, bh, st); break;
    default: fx4sh_launch<8>(p, u, v, w, bh, st); break;
  }
}
// q's twiddles are of type T (the FP64 refiner plan for T = double)
template <class T, bool STAGE>
void fx4(const OraclePlan* q, int zc, const float* u, const float* v, const float* w,
         const float* bh, double sdt, cplx<T>* X0, cplx<T>* X1, cudaStream_t st) {
  if constexpr (sizeof(T) == 8) {  // the FP64 residual form
    if (zc == 4) fx4_launch<T, false, 4>(q, u, v, w, bh, sdt, X0, X1, st);
    else fx4_launch<T, false, 2>(q, u, v, w, bh, sdt, X0, X1, st);
  } else {
    switch (zc) {
      case 2: fx4_launch<T, STAGE, 2>(q, u, v, w, bh, sdt, X0, X1, st); break;
      case 4: fx4_launch<T, STAGE, 4>(q, u, v, w, bh, sdt, X0, X1, st); break;
      default: fx4_launch<T, STAGE, 8>(q, u, v, w, bh, sdt, X0, X1, st); break;
    }
  }
}
// Resident CTAs of a persistent kernel on the current device (occupancy API x
// SM count), cached per (kernel, device): kernels of one signature share a
// function-pointer type, so the cache is keyed by the pointer itself.
std::mutex g_resident_mu;
std::map<std::pair<const void*, int>, int> g_resident;

template <class K>
int resident_ctas(K kernel, int threads, size_t smem) {
  int dev = 0;
  cudaGetDevice(&dev);
  const auto key = std::make_pair(reinterpret_cast<const void*>(kernel), dev);
  {
    std::lock_guard<std::mutex> lk(g_resident_mu);
    auto it = g_resident.find(key);
    if (it != g_resident.end()) return it->second;
  }
  int nsm = 148, per = 1;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, smem) != cudaSuccess ||
      per < 1) {
    cudaGetLastError();
    per = 1;
  }
  const int n = per * nsm;
  std::lock_guard<std::mutex> lk(g_resident_mu);
  g_resident[key] = n;
  return n;
}

template <int MODE, int ZC>
void ix4_launch(const OraclePlan* p, const cplx<float>* phs, const cplx<float>* psi,
                const float* u, const float* v, const float* w, const float* bh, double sdt,
                float* uo, float* vo, float* wo, float* phio, cudaStream_t st) {
  const dim3 grid((p->g.nz + ZC - 1) / ZC, p->g.ny);
  k_ix4<MODE, ZC><<<grid, 32 * (3 * ZC + 1), Ix4Size<ZC>::total, st>>>(
      p->g, phs, psi, p->kx, (const cplx<float>*)p->twx, u, v, w, bh, sdt, uo, vo, wo, phio);
}
template <int MODE>
void ix4(const OraclePlan* p, int zc, const cplx<float>* phs, const cplx<float>* psi,
         const float* u, const float* v, const float* w, const float* bh, double sdt,
         float* uo, float* vo, float* wo, float* phio, cudaStream_t st) {
  switch (zc) {
    case 2: ix4_launch<MODE, 2>(p, phs, psi, u, v, w, bh, sdt, uo, vo, wo, phio, st); break;
    case 4: ix4_launch<MODE, 4>(p, phs, psi, u, v, w, bh, sdt, uo, vo, wo, phio, st); break;
    default: ix4_launch<MODE, 8>(p, phs, psi, u, v, w, bh, sdt, uo, vo, wo, phio, st); break;
  }
}
template <int ZC>
void yr4_launch(const OraclePlan* p, bool inverse, const cplx<float>* in0,
                const cplx<float>* in1, cplx<float>* out0, cplx<float>* out1, cudaStream_t st) {
  const dim3 grid((p->g.nz + ZC - 1) / ZC, p->g.nxh);
  const cplx<float>* tw = (const cplx<float>*)p->twy;
  if (inverse)
    k_iy4<ZC><<<grid, 64 * ZC, Yr4Size<ZC>::total, st>>>(p->g, in0, p->ky, tw, out0, out1);
  else
    k_fy4<ZC><<<grid, 64 * ZC, Yr4Size<ZC>::total, st>>>(p->g, in0, in1, p->ky, tw, out0,
                                                         nullptr, 0.0f);
}
// a fast stage's forward y transform from the shared x transforms:
// d^ = FFTy(S4 + sdt S6) + i ky' FFTy(S5) into S3
template <int ZC>
void fy4sh_launch(const OraclePlan* p, float sdt, cudaStream_t st) {
  const dim3 grid((p->g.nz + ZC - 1) / ZC, p->g.nxh);
  k_fy4<ZC, true><<<grid, 64 * ZC, Yr4Size<ZC, 3>::total, st>>>(
      p->g, (const cplx<float>*)p->S4, (const cplx<float>*)p->S5, p->ky,
      (const cplx<float>*)p->twy, (cplx<float>*)p->S3, (const cplx<float>*)p->S6, sdt);
}
void fy4sh(const OraclePlan* p, float sdt, cudaStream_t st) {
  switch (p->zc4_fy) {
    case 2: fy4sh_launch<2>(p, sdt, st); break;
    case 4: fy4sh_launch<4>(p, sdt, st); break;
    default: fy4sh_launch<8>(p, sdt, st); break;
  }
}
// register-resident FP32 y pencils (ny = 1024): FY_DIV forward or the IY_GRAD inverse
void yr4(const OraclePlan* p, bool inverse, const cplx<float>* in0, const cplx<float>* in1,
         cplx<float>* out0, cplx<float>* out1, cudaStream_t st) {
  switch (inverse ? p->zc4_iy : p->zc4_fy) {
    case 2: yr4_launch<2>(p, inverse, in0, in1, out0, out1, st); break;
    case 4: yr4_launch<4>(p, inverse, in0, in1, out0, out1, st); break;
    default: yr4_launch<8>(p, inverse, in0, in1, out0, out1, st); break;
  }
}

// The single-precision short-wave launch with a compile-time level count
// (k_thomas_f32); false when nz has no instance.
bool thomas_f32(OraclePlan* p, int cls, cplx<float>* S3, cudaStream_t st) {
  const long ncols = (long)p->g.nxh * p->g.ny;
  const unsigned nb = (unsigned)((ncols + kThomasCols - 1) / kThomasCols);
  const float scale = (float)(1.0 / ((double)p->g.nx * p->g.ny));
  const float4* coef = reinterpret_cast<const float4*>(p->tcoef);
  switch (p->g.nz) {
#define OB_TF32(N)                                                                          \
  case N: {                                                                                 \
    const size_t sm = N * sizeof(float4) + (size_t)kThomasCols * (N + 1) * sizeof(cplx<float>); \
    Launch L_(p, cls, st);                                                                  \
    k_thomas_f32<N, kThomasCols><<<nb, 2 * kThomasCols, sm, st>>>(p->g, coef, p->kx, p->ky, scale, \
                                                             S3, S3, p->lw_flag);           \
    return true;                                                                            \
  }
    OB_TF32(32)
    OB_TF32(48)
    OB_TF32(64)
    OB_TF32(80)
#undef OB_TF32
  }
  return false;
}

// The batched Thomas solve of a projection, in place on S3: FP64 plans in one
// double launch; FP32 plans as a double launch over the blocks holding a
// long-wave mode and a single-precision launch over the rest (k_thomas).
template <class T>
int thomas_solve(OraclePlan* p, int cls, cplx<T>* S3, double* diag, int slot_c, int slot_d,
                 cudaStream_t st) {
  const long ncols = (long)p->g.nxh * p->g.ny;
  const unsigned nb = (unsigned)((ncols + kThomasCols - 1) / kThomasCols);
  if (sizeof(T) == 8 || !p->lw_blocks) {
    { Launch L_(p, cls, st); k_thomas<T, kThomasCols><<<nb, kThomasCols, smem_thomas(p), st>>>(
          p->g, thomas_args(p), S3, S3, diag, slot_c, slot_d); }
    OB_LAUNCHED();
  } else {
    // the two launches touch disjoint columns: the short double launch (a
    // few blocks, among them the serial zero mode) runs on the plan's side
    // stream, beside the single-precision one
    OB_CUDA(cudaEventRecord(p->ev_fork, st));
    OB_CUDA(cudaStreamWaitEvent(p->aux, p->ev_fork, 0));
    // timed as a class of its own: it overlaps the single-precision sweep,
    // so its events span that sweep too, and it moves few bytes
    const int cls_lw = (cls == OB_PROF_THOMAS) ? OB_PROF_THOMAS_LW : cls;
    { Launch L_(p, cls_lw, p->aux); k_thomas<T, kThomasCols, double><<<(unsigned)p->n_lw, kThomasCols, smem_thomas(p, 8), p->aux>>>(
          p->g, thomas_args(p), S3, S3, diag, slot_c, slot_d, p->lw_blocks, nullptr); }
    OB_LAUNCHED();
    // A solve that logs its residuals (every diag_every-th solve, counted
    // from the plan's first) takes them from the generic sweep, writing into
    // S1: no caller holds data there between the forward y transform and the
    // inverse one.  Its solution comes from the same kernel as every other
    // solve, so no result depends on the logging cadence or on how many
    // solves the plan has run before (a run resumed on a new plan continues
    // bit for bit).
    if (diag) {
      { Launch L_(p, cls, st); k_thomas<T, kThomasCols, float><<<nb, kThomasCols, smem_thomas(p, 4), st>>>(
            p->g, thomas_args(p), S3, (cplx<T>*)p->S1, diag, slot_c, slot_d, nullptr, p->lw_flag); }
      OB_LAUNCHED();
    }
    if (!p->thomas_fast || !thomas_f32(p, cls, (cplx<float>*)S3, st))
      { Launch L_(p, cls, st); k_thomas<T, kThomasCols, float><<<nb, kThomasCols, smem_thomas(p, 4), st>>>(
            p->g, thomas_args(p), S3, S3, nullptr, slot_c, slot_d, nullptr, p->lw_flag); }
    OB_LAUNCHED();
    OB_CUDA(cudaEventRecord(p->ev_join, p->aux));
    OB_CUDA(cudaStreamWaitEvent(st, p->ev_join, 0));
  }
  return OB_OK;
}

// ---- projection pipeline -------------------------------------------------
// One launcher per kernel class of the projection; each runs the variant the
// plan's choice fields select (register-resident > compile-time-chunk pencils
// > shared-memory Stockham), so that project_impl and the autotuner run the
// same code.  stage: the inputs are the anchor state and the provisional
// stage w + sdt * b_half (bh) is formed on the fly.

template <class T>
int proj_fx(OraclePlan* p, bool stage, const T* u, const T* v, const T* w, const T* th,
            const T* bh, double sdt, cudaStream_t st) {
  using C = cplx<T>;
  const GridK g = p->g;
  C* S1 = (C*)p->S1;
  C* S2 = (C*)p->S2;
  Launch L_(p, 0, st);
  if constexpr (sizeof(T) == 4) {
    if (stage && bh && p->zc4_fxs) {
      fx4<float, true>(p, p->zc4_fxs, u, v, w, bh, sdt, S1, S2, st);
      OB_LAUNCHED();
      return OB_OK;
    }
    if (!stage && p->zc4_fx) {
      fx4<float, false>(p, p->zc4_fx, u, v, w, th, 0.0, S1, S2, st);
      OB_LAUNCHED();
      return OB_OK;
    }
    if (stage && bh && p->zc3_fxs) {
      fx3<float, true>(p, p->zc3_fxs, u, v, w, bh, sdt, S1, S2, st);
      OB_LAUNCHED();
      return OB_OK;
    }
    if (!stage && p->zc3_fx) {
      fx3<float, false>(p, p->zc3_fx, u, v, w, th, 0.0, S1, S2, st);
      OB_LAUNCHED();
      return OB_OK;
    }
  }
  if (stage && bh && p->zc2_fxs)
    fx2<T, true, T>(p, p->zc2_fxs, u, v, w, bh, sdt, S1, S2, st);
  else if (!stage && p->zc2_fx)
    fx2<T, false, T>(p, p->zc2_fx, u, v, w, th, 0.0, S1, S2, st);
  else if (stage)
    k_fx<T, FX_DIV_STAGE><<<grid_x(p, p->zc_fx), kFftThreads, smem_fx(p, 3), st>>>(
        g, p->pxf, p->zc_fx, 3, u, v, w, th, sdt, p->rho, p->rhoh, p->theta0, p->kx,
        (const C*)p->twx, S1, S2, nullptr);
  else
    k_fx<T, FX_DIV><<<grid_x(p, p->zc_fx), kFftThreads, smem_fx(p, 3), st>>>(
        g, p->pxf, p->zc_fx, 3, u, v, w, th, 0.0, p->rho, p->rhoh, p->theta0, p->kx,
        (const C*)p->twx, S1, S2, nullptr);
  OB_LAUNCHED();
  return OB_OK;
}

// forward y: (S1, S2) -> S3
template <class T>
int proj_fy(OraclePlan* p, cudaStream_t st) {
  using C = cplx<T>;
  const GridK g = p->g;
  C* S1 = (C*)p->S1;
  C* S2 = (C*)p->S2;
  C* S3 = (C*)p->S3;
  Launch L_(p, 1, st);
  if (sizeof(T) == 4 && p->zc4_fy)
    yr4(p, false, (const cplx<float>*)S1, (const cplx<float>*)S2, (cplx<float>*)S3, nullptr, st);
  else if (sizeof(T) == 4 && p->zc3_fy)
    yr(p, false, (const cplx<float>*)S1, (const cplx<float>*)S2, (cplx<float>*)S3, nullptr, st);
  else if (p->zc2_fy)
    fy2<T, FY_DIV, T>(p, p->zc2_fy, S1, S2, S3, st);
  else
    k_fy<T, FY_DIV><<<grid_y(p, p->zc_fy), kFftThreads, smem_fy(p, 2, p->zc_fy), st>>>(
        g, p->pyf, p->zc_fy, 2, S1, S2, p->kx, p->ky, (const C*)p->twy, 1.0, S3, nullptr);
  OB_LAUNCHED();
  return OB_OK;
}

// inverse y: S3 -> (S1, S2); cls: the profile class the launch is counted in
template <class T>
int proj_iy(OraclePlan* p, int cls, cudaStream_t st) {
  using C = cplx<T>;
  const GridK g = p->g;
  C* S1 = (C*)p->S1;
  C* S2 = (C*)p->S2;
  C* S3 = (C*)p->S3;
  Launch L_(p, cls, st);
  if (sizeof(T) == 4 && p->zc4_iy)
    yr4(p, true, (const cplx<float>*)S3, nullptr, (cplx<float>*)S1, (cplx<float>*)S2, st);
  else if (sizeof(T) == 4 && p->zc3_fy)
    yr(p, true, (const cplx<float>*)S3, nullptr, (cplx<float>*)S1, (cplx<float>*)S2, st);
  else if (p->zc2_iy)
    iy2<T>(p, p->zc2_iy, S3, S1, S2, st);
  else
    k_iy<T, IY_GRAD><<<grid_y(p, p->zc_iy), kFftThreads, smem_fy(p, 2, p->zc_iy), st>>>(
        g, p->py, p->zc_iy, 2, S3, nullptr, p->ky, (const C*)p->twy, 1.0, S1, S2);
  OB_LAUNCHED();
  return OB_OK;
}

// inverse x with the velocity correction: (S1, S2) and the state -> outputs
template <class T>
int proj_ix(OraclePlan* p, bool stage, const T* u, const T* v, const T* w, const T* th,
            const T* bh, double sdt, T* uo, T* vo, T* wo, T* phio, cudaStream_t st) {
  using C = cplx<T>;
  const GridK g = p->g;
  C* S1 = (C*)p->S1;
  C* S2 = (C*)p->S2;
  Launch L_(p, 4, st);
  if constexpr (sizeof(T) == 4) {
    if (p->zc4_ix && (bh || !stage)) {
      if (stage) ix4<IX_STAGE>(p, p->zc4_ix, S1, S2, u, v, w, bh, sdt, uo, vo, wo, phio, st);
      else ix4<IX_CORRECT>(p, p->zc4_ix, S1, S2, u, v, w, nullptr, 0.0, uo, vo, wo, phio, st);
      OB_LAUNCHED();
      return OB_OK;
    }
    if (p->zc3_ix && (bh || !stage)) {
      if (stage) ix3<IX_STAGE>(p, p->zc3_ix, S1, S2, u, v, w, bh, sdt, uo, vo, wo, phio, st);
      else ix3<IX_CORRECT>(p, p->zc3_ix, S1, S2, u, v, w, nullptr, 0.0, uo, vo, wo, phio, st);
      OB_LAUNCHED();
      return OB_OK;
    }
  }
  const size_t sx = smem_ix(p, 3 * p->zc_ix + 1);
  if (p->zc2_ix && stage && bh)
    ix2<T, IX_STAGE, T>(p, p->zc2_ix, S1, S2, u, v, w, bh, sdt, uo, vo, wo, phio, st);
  else if (p->zc2_ix && !stage)
    ix2<T, IX_CORRECT, T>(p, p->zc2_ix, S1, S2, u, v, w, nullptr, 0.0, uo, vo, wo, phio, st);
  else if (stage)
    k_ix<T, IX_STAGE><<<grid_x(p, p->zc_ix), kFftThreads, sx, st>>>(
        g, p->px, p->zc_ix, 0, S1, S2, nullptr, p->kx, (const C*)p->twx, u, v, w, th, sdt,
        p->theta0, uo, vo, wo, phio);
  else
    k_ix<T, IX_CORRECT><<<grid_x(p, p->zc_ix), kFftThreads, sx, st>>>(
        g, p->px, p->zc_ix, 0, S1, S2, nullptr, p->kx, (const C*)p->twx, u, v, w, th, 0.0,
        p->theta0, uo, vo, wo, phio);
  OB_LAUNCHED();
  return OB_OK;
}

// stage_sdt < 0: in-place projection of (u, v, w) with phi output.
// stage_sdt >= 0: inputs are the anchor state (u, v, w, th); the provisional
// stage state w + sdt * b_half is formed on the fly and the projected result
// goes to (uo, vo, wo, phio).
// shared: a fast stage whose forward x transforms are in S4..S6 (fx4sh ran
// on the anchor state): the y pencils form the stage's spectrum from them.
template <class T>
int project_impl(OraclePlan* p, const T* u, const T* v, const T* w, const T* th,
                 double stage_sdt, T* uo, T* vo, T* wo, T* phio, int slot_c, int slot_d,
                 cudaStream_t st, const T* bh = nullptr, bool shared = false) {
  // a stage projection reads the half-level buoyancy in every form but the
  // generic one; without it a selected form would silently fall back
  if (stage_sdt >= 0.0 && !bh && (p->zc2_fxs || p->zc2_ix || p->zc3_fxs || p->zc3_ix || p->zc4_fxs ||
                    p->zc4_ix))
    return fail(OB_ERR_CUDA, "stage projection without the half-level buoyancy its "
                "kernel forms read");
  p->solve_count += 1;
  const int de = p->diag_every < 1 ? 1 : p->diag_every;
  const bool log = !p->capturing && ((de == 1) || (p->solve_count % de == 1));
  double* diag = nullptr;
  if (log) {
    diag = p->diag;
    OB_CUDA(cudaMemsetAsync(p->diag + slot_d, 0, sizeof(double), st));
  } else {
    OB_CUDA(cudaMemsetAsync(p->diag + slot_c, 0, sizeof(double), st));
    OB_CUDA(cudaMemsetAsync(p->diag + slot_d, 0, sizeof(double), st));
  }
  const bool stage = stage_sdt >= 0.0;
  if (shared && sizeof(T) == 4 && stage) {
    { Launch L_(p, 1, st); fy4sh(p, (float)stage_sdt, st); }
    OB_LAUNCHED();
  } else {
    RC(proj_fx<T>(p, stage, u, v, w, th, bh, stage_sdt, st));
    RC(proj_fy<T>(p, st));
  }
  RC(thomas_solve<T>(p, 2, (cplx<T>*)p->S3, diag, slot_c, slot_d, st));
  RC(proj_iy<T>(p, 3, st));
  RC(proj_ix<T>(p, stage, u, v, w, th, bh, stage_sdt, uo, vo, wo, phio, st));
  return OB_OK;
}

// Defect correction of a projected single-precision state (in place).  The
// residual -- the anelastic divergence of the stored (u, v, w) outside the
// Nyquist rows -- is formed in double (x and y transforms of the FP32 fields
// in FP64, tendency.py:717-790 operator order) and rounded to float only once
// the cancellation between its terms has happened; the correction potential
// is then solved and applied in single precision (it is small, so its
// relative FP32 error is negligible against the state):
// u, v, w -= grad(dphi), phi += dphi.
// The residual's x transform (FP32 state in, FP64 half-spectra R1, R2 out).
int refine_fx(OraclePlan* p, const float* u, const float* v, const float* w, cudaStream_t st) {
  OraclePlan* q = p->dbl;
  using Cd = cplx<double>;
  const GridK g = p->g;
  Cd* R1 = (Cd*)q->S1;
  Cd* R2 = (Cd*)q->S2;
  Launch L_(p, OB_PROF_REFINE, st);
  if (p->zc4_fxd)
    fx4<double, false>(q, p->zc4_fxd, u, v, w, nullptr, 0.0, R1, R2, st);
  else if (p->zc3_fxd)
    fx3<double, false>(q, p->zc3_fxd, u, v, w, nullptr, 0.0, R1, R2, st);
  else if (q->zc2_fx)
    fx2<double, false, float>(q, q->zc2_fx, u, v, w, nullptr, 0.0, R1, R2, st);
  else
    k_fx<double, FX_DIV, float><<<grid_x(q, q->zc_fx), kFftThreads, smem_fx(q, 3), st>>>(
        g, q->pxf, q->zc_fx, 3, u, v, w, nullptr, 0.0, q->rho, q->rhoh, q->theta0, q->kx,
        (const Cd*)q->twx, R1, R2, nullptr);
  OB_LAUNCHED();
  return OB_OK;
}

// The residual's y transform (R1, R2 -> the FP32 residual in S3).
int refine_fy(OraclePlan* p, cudaStream_t st) {
  OraclePlan* q = p->dbl;
  using Cd = cplx<double>;
  const GridK g = p->g;
  Cd* R1 = (Cd*)q->S1;
  Cd* R2 = (Cd*)q->S2;
  cplx<float>* S3 = (cplx<float>*)p->S3;
  Launch L_(p, OB_PROF_REFINE, st);
  if (p->zc4_fyd) {
    const int items = ((g.nz + 1) / 2) * g.nxh;
    const int grid = std::min(items, resident_ctas(k_fy4d, 128, Yr4dSize::total));
    k_fy4d<<<grid, 128, Yr4dSize::total, st>>>(g, R1, R2, q->ky, (const Cd*)q->twy, S3);
  } else if (p->zc3_fyd)
    k_fy3<2, double, FY_RESID, float><<<dim3((g.nz + 1) / 2, g.nxh), 128,
                                        YrSize<2, double>::total, st>>>(
        g, R1, R2, q->ky, (const Cd*)q->twy, S3);
  else if (q->zc2_fy)
    fy2<double, FY_RESID, float>(q, q->zc2_fy, R1, R2, S3, st);
  else
    k_fy<double, FY_RESID, float><<<grid_y(q, q->zc_fy), kFftThreads, smem_fy(q, 2, q->zc_fy), st>>>(
        g, q->pyf, q->zc_fy, 2, R1, R2, q->kx, q->ky, (const Cd*)q->twy, 1.0, S3, nullptr);
  OB_LAUNCHED();
  return OB_OK;
}

int refine_impl(OraclePlan* p, float* u, float* v, float* w, float* phi, cudaStream_t st) {
  OraclePlan* q = p->dbl;
  if (!q) return fail(OB_ERR_UNSUPPORTED, "defect correction needs a single-precision plan");
  using Cf = cplx<float>;
  const GridK g = p->g;
  Cf* S1 = (Cf*)p->S1;
  Cf* S2 = (Cf*)p->S2;
  Cf* S3 = (Cf*)p->S3;
  RC(refine_fx(p, u, v, w, st));
  RC(refine_fy(p, st));
  RC(thomas_solve<float>(p, OB_PROF_REFINE, S3, nullptr, 0, 0, st));
  RC(proj_iy<float>(p, OB_PROF_REFINE, st));
  if (p->zc4_ix)
    { Launch L_(p, OB_PROF_REFINE, st); ix4<IX_REFINE>(p, p->zc4_ix, S1, S2, u, v, w, nullptr, 0.0, u, v, w, phi, st); }
  else if (p->zc3_ix)
    { Launch L_(p, OB_PROF_REFINE, st); ix3<IX_REFINE>(p, p->zc3_ix, S1, S2, u, v, w, nullptr, 0.0, u, v, w, phi, st); }
  else if (p->zc2_ix)
    { Launch L_(p, OB_PROF_REFINE, st); ix2<float, IX_REFINE, float>(p, p->zc2_ix, S1, S2, u, v, w, nullptr, 0.0, u, v, w, phi, st); }
  else
    { Launch L_(p, OB_PROF_REFINE, st); k_ix<float, IX_REFINE><<<grid_x(p, p->zc_ix), kFftThreads, smem_ix(p, 3 * p->zc_ix + 1), st>>>(
        g, p->px, p->zc_ix, 0, S1, S2, nullptr, p->kx, (const Cf*)p->twx, u, v, w, nullptr, 0.0,
        p->theta0, u, v, w, phi); }
  OB_LAUNCHED();
  return OB_OK;
}

// Double-precision companion of a single-precision plan for the residual
// transforms: FP64 twiddles and two FP64 half-spectrum buffers; the FFT
// plans, wavenumbers and reference profiles are shared with the plan.
int make_refiner(OraclePlan* p) {
  OraclePlan* q = new OraclePlan();
  p->dbl = q;
  q->prec = OB_PREC_F64;
  q->esz = 8;
  q->g = p->g;
  q->px = p->px;
  q->py = p->py;
  q->pxf = p->pxf;
  q->pyf = p->pyf;
  q->px8 = p->px8;
  q->py8 = p->py8;
  q->kx = p->kx;
  q->ky = p->ky;
  q->rho = p->rho;
  q->rhoh = p->rhoh;
  q->theta0 = p->theta0;
  const int nx = p->g.nx, ny = p->g.ny, nz = p->g.nz;
  const size_t ce = 16;
  q->zc_fx = pick_zc(nz, 2ull * (q->g.M + 1) * 3 * ce, tw_bytes(q, nx));
  q->zc_fy = pick_zc(nz, 2ull * ny * 2 * ce, tw_bytes(q, ny));
  q->zc2_fx = pick_x2_zc<double, float>(0, nx, nz);
  q->zc2_fy = p->zc2_fy ? pick_y2_zc<double>(ny, nz) : 0;
  if (smem_fx(q, 3) > kSmemMax || smem_fy(q, 2, q->zc_fy) > kSmemMax)
    return fail(OB_ERR_ARG, "grid too large for the FP64 residual kernels");
  auto tx = twiddles<double>(nx), ty = twiddles<double>(ny);
  int rc;
  if ((rc = dalloc(p, &q->twx, nx * sizeof(cplx<double>))) ||
      (rc = dalloc(p, &q->twy, ny * sizeof(cplx<double>))))
    return rc;
  OB_CUDA(cudaMemcpyAsync(q->twx, tx.data(), nx * sizeof(cplx<double>), cudaMemcpyHostToDevice,
                          p->astream));
  OB_CUDA(cudaMemcpyAsync(q->twy, ty.data(), ny * sizeof(cplx<double>), cudaMemcpyHostToDevice,
                          p->astream));
  const size_t ns = (size_t)p->g.nxh * ny * nz;
  if ((rc = dalloc(p, &q->S1, ns * ce)) || (rc = dalloc(p, &q->S2, ns * ce))) return rc;
  return set_smem_attrs_once<double>();
}

// Helmholtz divergence damping tendency (tendency.py:1800-1839) into Du, Dv.
template <class T>
int damper_impl(OraclePlan* p, const T* u, const T* v, double dt_slow, cudaStream_t st) {
  using C = cplx<T>;
  const GridK g = p->g;
  C* S1 = (C*)p->S1;
  C* S2 = (C*)p->S2;
  if (sizeof(T) == 4 && p->zc3_fx)
    { Launch L_(p, 0, st); fx3f(p, p->zc3_fx, (const float*)u, (const float*)v, (cplx<float>*)S1,
                               (cplx<float>*)S2, st); }
  else
    { Launch L_(p, 0, st); k_fx<T, FX_FIELDS><<<grid_x(p, p->zc_fx), kFftThreads, smem_fx(p, 2), st>>>(
        g, p->pxf, p->zc_fx, 2, u, v, nullptr, nullptr, 0.0, p->rho, p->rhoh, p->theta0, p->kx,
        (const C*)p->twx, S1, S2, nullptr); }
  OB_LAUNCHED();
  const double scale = -(p->epsilon / dt_slow) / ((double)g.nx * (double)g.ny);
  if (sizeof(T) == 4 && p->zc3_fy) {
    // forward y, multipliers and inverse y in one register-resident pass
    { Launch L_(p, 1, st); hy(p, scale, (cplx<float>*)S1, (cplx<float>*)S2, st); }
    OB_LAUNCHED();
  } else {
  { Launch L_(p, 1, st); k_fy<T, FY_HELM><<<grid_y(p, p->zc_fy), kFftThreads, smem_fy(p, 2, p->zc_fy), st>>>(
      g, p->pyf, p->zc_fy, 2, S1, S2, p->kx, p->ky, (const C*)p->twy, scale, S1, S2); }
  OB_LAUNCHED();
  { Launch L_(p, 3, st); k_iy<T, IY_FIELDS><<<grid_y(p, p->zc_iy), kFftThreads, smem_fy(p, 2, p->zc_iy), st>>>(
      g, p->py, p->zc_iy, 2, S1, S2, p->ky, (const C*)p->twy, 1.0, S1, S2); }
  OB_LAUNCHED();
  }
  if (sizeof(T) == 4 && p->zc3_ix)
    { Launch L_(p, 4, st); ix3<IX_FIELDS>(p, p->zc3_ix, (const cplx<float>*)S1,
                                          (const cplx<float>*)S2, nullptr, nullptr, nullptr,
                                          nullptr, 0.0, (float*)p->Du, (float*)p->Dv, nullptr,
                                          nullptr, st); }
  else
    { Launch L_(p, 4, st); k_ix<T, IX_FIELDS><<<grid_x(p, p->zc_ix), kFftThreads, smem_ix(p, 2 * p->zc_ix), st>>>(
        g, p->px, p->zc_ix, 2, S1, S2, nullptr, p->kx, (const C*)p->twx, nullptr, nullptr,
        nullptr, nullptr, 0.0, p->theta0, (T*)p->Du, (T*)p->Dv, nullptr, nullptr); }
  OB_LAUNCHED();
  return OB_OK;
}

SlowK slow_args(const OraclePlan* p) {
  SlowK s;
  s.adv = p->advection;
  s.cor = p->coriolis;
  s.heat = p->heating;
  s.damp = p->damping;
  s.f0 = p->f0;
  s.u_env = p->u_env;
  s.v_env = p->v_env;
  s.fy = p->fy;
  s.dth0 = p->dth0;
  s.heat_r = p->heat_r;
  s.heat_z = p->heat_z;
  s.inv2dx = 1.0 / (2.0 * p->g.dx);
  s.inv2dy = 1.0 / (2.0 * p->g.dy);
  s.inv60dx = 1.0 / (60.0 * p->g.dx);
  s.inv60dy = 1.0 / (60.0 * p->g.dy);
  s.inv2dz = 1.0 / (2.0 * p->g.dz);
  s.invdz = 1.0 / p->g.dz;
  s.drag = p->drag;
  s.sponge = p->sponge;
  s.diff = p->diffusion;
  s.cool = p->cooling;
  s.drag_cd = p->drag_cd;
  s.drag_dz = p->drag_dz;
  s.drag_u_env = p->drag_u_env;
  s.drag_v_env = p->drag_v_env;
  s.drag_w = p->drag_w;
  s.sp_u_env = p->sponge_u_env;
  s.sp_v_env = p->sponge_v_env;
  s.sp_a = p->sp_a;
  s.sp_ah = p->sp_ah;
  s.diff_nu = p->diff_nu;
  s.diff_dx2 = p->diff_dx2;
  s.diff_dy2 = p->diff_dy2;
  s.lap_u = p->Lu;
  s.lap_v = p->Lv;
  s.cool_alpha = p->cool_alpha;
  return s;
}

// ---- x-marching slow tendency over bulk-copied planes (slowx.cuh) ---------
// The plan's slow_xw value v selects k_slow_xt with R = v % 10 rows per CTA
// and KC = v / 10 cells per thread (4, 8: one cell; 24, 28: two).  Plans with
// production components or centred advection run its production form, which
// has one cell per thread.
bool slow_xt_prod(const OraclePlan* p) {
  return p->drag || p->sponge || p->diffusion || p->cooling ||
         p->advection != OB_ADV_UPWIND5H;
}
bool slow_xt_grid(const OraclePlan* p, int v) {
  const int nz = p->g.nz, r = v % 10;
  const bool adv = p->advection == OB_ADV_UPWIND5H || p->advection == OB_ADV_CENTERED2;
  return p->prec == OB_PREC_F32 && adv && (nz == 32 || nz == 48 || nz == 64 || nz == 80) &&
         (v == 4 || v == 8 || ((v == 24 || v == 28) && !slow_xt_prod(p))) &&
         p->g.ny % r == 0 && p->g.ny >= r + 6 && p->g.nx >= 7 &&
         (long long)p->g.nx * p->g.ny * (p->g.nz + 1) < (1ll << 31);  // 32-bit offsets
}
template <int NZ, int R, int KC, bool PROD = false>
int slow_xt_attr() {
  OB_CUDA(cudaFuncSetAttribute(k_slow_xt<0, NZ, R, KC, PROD>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)SlowXt<NZ, R, KC, PROD>::smem));
  OB_CUDA(cudaFuncSetAttribute(k_slow_xt<1, NZ, R, KC, PROD>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)SlowXt<NZ, R, KC, PROD>::smem));
  return OB_OK;
}
template <int NZ>
int slow_xt_attrs_nz() {
  int rc;
  if ((rc = slow_xt_attr<NZ, 4, 1>()) || (rc = slow_xt_attr<NZ, 8, 1>()) ||
      (rc = slow_xt_attr<NZ, 4, 2>()) || (rc = slow_xt_attr<NZ, 8, 2>()) ||
      (rc = slow_xt_attr<NZ, 4, 1, true>()) || (rc = slow_xt_attr<NZ, 8, 1, true>()))
    return rc;
  return OB_OK;
}
int slow_xt_attrs(int nz) {
  switch (nz) {
    case 32: return slow_xt_attrs_nz<32>();
    case 48: return slow_xt_attrs_nz<48>();
    case 64: return slow_xt_attrs_nz<64>();
    case 80: return slow_xt_attrs_nz<80>();
  }
  return OB_OK;
}
// x-segment of one CTA: a multiple of 7 steps, short enough that the grid
// holds about eight CTAs per SM (each segment re-reads 6 planes of its
// neighbours' columns, from L2)
int slow_xt_seg(const OraclePlan* p, int r) {
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int nrow = p->g.ny / r;
  const int nseg = std::max(1, (8 * nsm + nrow - 1) / nrow);
  int seg = (p->g.nx + nseg - 1) / nseg;
  seg = std::max(21, (seg + 6) / 7 * 7);
  return std::min(seg, (p->g.nx + 6) / 7 * 7);
}
template <int OUT, int NZ, int R, int KC, bool PROD = false>
void slow_xt_launch(OraclePlan* p, int mask, double dts, const float* u, const float* v,
                    const float* w, const float* th, float* uo, float* vo, float* wo,
                    float* tho, cudaStream_t st) {
  const int seg = slow_xt_seg(p, R);
  const dim3 grid(p->g.ny / R, (p->g.nx + seg - 1) / seg);
  k_slow_xt<OUT, NZ, R, KC, PROD><<<grid, R * NZ / KC, SlowXt<NZ, R, KC, PROD>::smem, st>>>(
      p->g, slow_args(p), mask, dts, seg, u, v, w, th, (const float*)p->Du, (const float*)p->Dv,
      uo, vo, wo, tho, p->diag + OB_DIAG_STALL);
}
// k_slow_xt for this call, if the plan selected it and the call allows it:
// advection on and 16-byte aligned fields (the bulk copies' rule)
bool slow_xt_call(const OraclePlan* p, int mask, const void* u, const void* v, const void* w,
                  const void* th) {
  return (mask & OB_TEND_ADVECTION) && slow_xt_grid(p, p->slow_xw) &&
         !((reinterpret_cast<size_t>(u) | reinterpret_cast<size_t>(v) |
            reinterpret_cast<size_t>(w) | reinterpret_cast<size_t>(th)) & 15);
}
template <int OUT>
bool slow_xt_launch_any(OraclePlan* p, int mask, double dts, const float* u, const float* v,
                        const float* w, const float* th, float* uo, float* vo, float* wo,
                        float* tho, cudaStream_t st) {
  const int r = p->slow_xw;
  const bool prod = slow_xt_prod(p);
#define OB_XT(NZ)                                                                  \
  case NZ:                                                                         \
    if (prod && r == 4)                                                            \
      slow_xt_launch<OUT, NZ, 4, 1, true>(p, mask, dts, u, v, w, th, uo, vo, wo, tho, st); \
    else if (prod)                                                                 \
      slow_xt_launch<OUT, NZ, 8, 1, true>(p, mask, dts, u, v, w, th, uo, vo, wo, tho, st); \
    else if (r == 4)                                                               \
      slow_xt_launch<OUT, NZ, 4, 1>(p, mask, dts, u, v, w, th, uo, vo, wo, tho, st);  \
    else if (r == 8)                                                               \
      slow_xt_launch<OUT, NZ, 8, 1>(p, mask, dts, u, v, w, th, uo, vo, wo, tho, st);  \
    else if (r == 24)                                                              \
      slow_xt_launch<OUT, NZ, 4, 2>(p, mask, dts, u, v, w, th, uo, vo, wo, tho, st);  \
    else                                                                           \
      slow_xt_launch<OUT, NZ, 8, 2>(p, mask, dts, u, v, w, th, uo, vo, wo, tho, st);  \
    return true;
  switch (p->g.nz) {
    OB_XT(32)
    OB_XT(48)
    OB_XT(64)
    OB_XT(80)
  }
#undef OB_XT
  return false;
}

template <class T, int OUT>
int slow_impl(OraclePlan* p, int mask, double dts, const T* u, const T* v, const T* w,
              const T* th, T* uo, T* vo, T* wo, T* tho, cudaStream_t st) {
  dim3 blk(32, 8);
  dim3 grd((p->g.ny + 7) / 8, p->g.nx);
  // the biharmonic diffusion's inner Laplacians of this slow half's u, v
  if ((mask & OB_TEND_DIFFUSION) && p->diffusion == OB_DIFF_BIHARMONIC) {
    const dim3 lg((unsigned)((p->g.ny * p->g.nz + 255) / 256), (unsigned)p->g.nx);
    { Launch L_(p, 5, st); k_lap2<T><<<lg, 256, 0, st>>>(
          p->g, u, v, p->diff_dx2, p->diff_dy2, (T*)p->Lu, (T*)p->Lv); }
    OB_LAUNCHED();
  }
  // production components run in the gather kernels
  const bool extra = (mask & (OB_TEND_DRAG | OB_TEND_SPONGE | OB_TEND_DIFFUSION | OB_TEND_COOLING)) &&
                     (p->drag || p->sponge || p->diffusion || p->cooling);
  if constexpr (sizeof(T) == 4) {
    // the x-marching form where the grid tiles it; the gather form otherwise
    if (slow_xt_call(p, mask, u, v, w, th))
      { Launch L_(p, 5, st); slow_xt_launch_any<OUT>(p, mask, dts, u, v, w, th, uo, vo, wo, tho, st); }
    else if (p->slow_xw && !extra && p->g.ny % 8 == 0 && p->g.nx % KXW == 0)
      { Launch L_(p, 5, st); k_slow_xw<OUT><<<dim3(p->g.ny / 8, p->g.nx / KXW), blk, 0, st>>>(
            p->g, slow_args(p), mask, dts, u, v, w, th, (const T*)p->Du, (const T*)p->Dv, uo, vo, wo, tho); }
    else if (extra)
      { Launch L_(p, 5, st); k_slow_f32<OUT, true><<<grd, blk, 0, st>>>(p->g, slow_args(p), mask, dts, u, v, w, th, (const T*)p->Du,
                                                  (const T*)p->Dv, uo, vo, wo, tho); }
    else
      { Launch L_(p, 5, st); k_slow_f32<OUT><<<grd, blk, 0, st>>>(p->g, slow_args(p), mask, dts, u, v, w, th, (const T*)p->Du,
                                            (const T*)p->Dv, uo, vo, wo, tho); }
  } else if (extra) {
    { Launch L_(p, 5, st); k_slow<T, OUT, true><<<grd, blk, 0, st>>>(p->g, slow_args(p), mask, dts, u, v, w, th, (const T*)p->Du,
                                              (const T*)p->Dv, uo, vo, wo, tho); }
  } else {
    { Launch L_(p, 5, st); k_slow<T, OUT><<<grd, blk, 0, st>>>(p->g, slow_args(p), mask, dts, u, v, w, th, (const T*)p->Du,
                                        (const T*)p->Dv, uo, vo, wo, tho); }
  }
  OB_LAUNCHED();
  return OB_OK;
}

template <class T>
int copy_field(void* dst, const void* src, size_t n, cudaStream_t st) {
  if (dst == src) return OB_OK;
  OB_CUDA(cudaMemcpyAsync(dst, src, n * sizeof(T), cudaMemcpyDeviceToDevice, st));
  return OB_OK;
}

template <class T>
int diag_impl(OraclePlan* p, const T* u, const T* v, const T* w, const T* th, const T* phi,
              cudaStream_t st) {
  { Launch L_(p, 6, st); k_diag_partial<T><<<p->nparts, 256, 0, st>>>(p->g, u, v, w, th, phi, p->parts); }
  OB_LAUNCHED();
  { Launch L_(p, 6, st); k_diag_final<<<1, 32, 0, st>>>(p->parts, p->nparts,
                                 (double)p->g.nx * p->g.ny * p->g.nz, p->blowup_u, p->diag); }
  OB_LAUNCHED();
  return OB_OK;
}


template <class T>
int step_impl(OraclePlan* p, const OracleStatePtrs* in, const OracleStatePtrs* out, double dt,
              int want_diag, cudaStream_t st) {
  const size_t n = (size_t)p->g.nx * p->g.ny * p->g.nz;
  const size_t nw = (size_t)p->g.nx * p->g.ny * (p->g.nz + 1);
  const double dts = dt * 0.5;
  const bool slow = p->advection || p->coriolis || p->damping || p->heating || p->drag ||
                    p->sponge || p->diffusion || p->cooling;
  const bool mom = p->advection || p->coriolis || p->damping || p->drag || p->sponge ||
                   p->diffusion;
  const int all = OB_TEND_ADVECTION | OB_TEND_CORIOLIS | OB_TEND_DAMPING | OB_TEND_HEATING |
                  OB_TEND_DRAG | OB_TEND_SPONGE | OB_TEND_DIFFUSION | OB_TEND_COOLING;
  // anchor state y^n after the first slow half step
  const T *au = (const T*)in->u, *av = (const T*)in->v, *aw = (const T*)in->w,
          *ath = (const T*)in->theta_prime, *aphi = (const T*)in->phi;
  if (slow) {
    if (p->damping) RC(damper_impl<T>(p, (const T*)in->u, (const T*)in->v, dts, st));
    RC((slow_impl<T, 0>(p, all, dts, (const T*)in->u, (const T*)in->v, (const T*)in->w,
                        (const T*)in->theta_prime, (T*)p->Au, (T*)p->Av, (T*)p->Aw,
                        (T*)p->Ath, st)));
    // its potential is never read: the fast stages (or, without buoyancy,
    // the projection of y^n below) write the potential the step reports
    if (mom && p->projection)
      RC(project_impl<T>(p, (T*)p->Au, (T*)p->Av, (T*)p->Aw, nullptr, -1.0, (T*)p->Au,
                         (T*)p->Av, (T*)p->Aw, (T*)nullptr, OB_DIAG_LAST_COMPAT,
                         OB_DIAG_LAST_DISC, st));
    else
      RC(copy_field<T>(p->Aphi, in->phi, n, st));
    au = (const T*)p->Au;
    av = (const T*)p->Av;
    aw = (const T*)p->Aw;
    ath = (const T*)p->Ath;
    aphi = (const T*)p->Aphi;
  }
  // fast stages (integrator.py:232-258)
  const T *su = au, *sv = av, *sw = aw, *sphi = aphi;
  if (p->buoyancy && p->projection) {
    const double alphas[3] = {1.0 / 3.0, 1.0 / 2.0, 1.0};
    // the three stages share the buoyancy of the anchor theta', formed once
    // on half levels for every stage form that reads it (all but the generic
    // shared-memory kernels, which form it on the fly; whichever form the
    // autotuner kept, the stage projections must not fall back to those)
    const T* bh = nullptr;
    if (p->Bh) {
      const long ncol = (long)p->g.nx * p->g.ny;
      { Launch L_(p, 7, st); k_bhalf<T><<<(unsigned)std::min<long>((ncol + 7) / 8, 65535), 256, 0, st>>>(
          p->g, ath, p->theta0, p->gth, (T*)p->Bh); }
      OB_LAUNCHED();
      bh = (const T*)p->Bh;
    }
    // the stages' divergence is linear in their sdt: with the shared form
    // one forward x launch serves all three (each stage still projects in
    // full: its own y transforms, solve, inverse transforms and correction)
    const bool shared = sizeof(T) == 4 && bh && p->zc4_fxsh && p->zc4_fy && p->S4;
    if (shared) {
      { Launch L_(p, 0, st); fx4sh(p, (const float*)au, (const float*)av, (const float*)aw,
                                   (const float*)bh, st); }
      OB_LAUNCHED();
    }
    // every stage starts from the anchor state, so only the last stage's
    // potential is read (by the diagnostics and as the reported potential)
    for (int s = 0; s < 3; ++s) {
      const double sdt = alphas[s] * dt;
      RC(project_impl<T>(p, au, av, aw, ath, sdt, (T*)p->Su, (T*)p->Sv, (T*)p->Sw,
                         s == 2 ? (T*)p->Sphi : (T*)nullptr, OB_DIAG_COMPAT0 + s,
                         OB_DIAG_DISC0 + s, st, bh, shared));
    }
    su = (const T*)p->Su;
    sv = (const T*)p->Sv;
    sw = (const T*)p->Sw;
    sphi = (const T*)p->Sphi;
  } else if (p->buoyancy) {
    return fail(OB_ERR_UNSUPPORTED, "buoyancy without a projection is not supported");
  } else if (p->projection) {
    // no fast physics: one projection of y^n (integrator.py:242-258)
    T* tu = slow ? (T*)p->Au : (T*)p->Su;
    T* tv = slow ? (T*)p->Av : (T*)p->Sv;
    T* tw = slow ? (T*)p->Aw : (T*)p->Sw;
    T* tp = slow ? (T*)p->Aphi : (T*)p->Sphi;
    if (!slow) {
      RC(copy_field<T>(tu, in->u, n, st));
      RC(copy_field<T>(tv, in->v, n, st));
      RC(copy_field<T>(tw, in->w, nw, st));
    }
    RC(project_impl<T>(p, tu, tv, tw, nullptr, -1.0, tu, tv, tw, tp, OB_DIAG_LAST_COMPAT,
                       OB_DIAG_LAST_DISC, st));
    su = tu;
    sv = tv;
    sw = tw;
    sphi = tp;
  }
  // second slow half step (integrator.py:261-276)
  if (slow) {
    if (p->damping) RC(damper_impl<T>(p, su, sv, dts, st));
    RC((slow_impl<T, 0>(p, all, dts, su, sv, sw, ath, (T*)out->u, (T*)out->v, (T*)out->w,
                        (T*)out->theta_prime, st)));
    if (mom && p->projection)
      RC(project_impl<T>(p, (T*)out->u, (T*)out->v, (T*)out->w, nullptr, -1.0, (T*)out->u,
                         (T*)out->v, (T*)out->w, (T*)out->phi, OB_DIAG_LAST_COMPAT,
                         OB_DIAG_LAST_DISC, st));
    else
      RC(copy_field<T>(out->phi, sphi, n, st));
  } else {
    RC(copy_field<T>(out->u, su, n, st));
    RC(copy_field<T>(out->v, sv, n, st));
    RC(copy_field<T>(out->w, sw, nw, st));
    RC(copy_field<T>(out->theta_prime, ath, n, st));
    RC(copy_field<T>(out->phi, sphi, n, st));
  }
  // FP64 defect correction of the step's final projection (single precision)
  if constexpr (sizeof(T) == 4) {
    if (p->projection && p->refine_passes > 0 && p->step_count % p->refine_every == 0)
      for (int r = 0; r < p->refine_passes; ++r)
        RC(refine_impl(p, (float*)out->u, (float*)out->v, (float*)out->w, (float*)out->phi, st));
  }
  p->step_count += 1;
  if (want_diag)
    RC(diag_impl<T>(p, (const T*)out->u, (const T*)out->v, (const T*)out->w,
                    (const T*)out->theta_prime, sphi, st));
  return OB_OK;
}

template <class T>
int divergence_impl(OraclePlan* p, const T* u, const T* v, const T* w, T* d, cudaStream_t st) {
  using C = cplx<T>;
  const GridK g = p->g;
  C* S1 = (C*)p->S1;
  C* S2 = (C*)p->S2;
  C* S3 = (C*)p->S3;
  { Launch L_(p, 0, st); k_fx<T, FX_DIV><<<grid_x(p, p->zc_fx), kFftThreads, smem_fx(p, 3), st>>>(
      g, p->pxf, p->zc_fx, 3, u, v, w, nullptr, 0.0, p->rho, p->rhoh, p->theta0, p->kx,
      (const C*)p->twx, S1, S2, nullptr); }
  OB_LAUNCHED();
  { Launch L_(p, 1, st); k_fy<T, FY_DIV><<<grid_y(p, p->zc_fy), kFftThreads, smem_fy(p, 2, p->zc_fy), st>>>(
      g, p->pyf, p->zc_fy, 2, S1, S2, p->kx, p->ky, (const C*)p->twy, 1.0, S3, nullptr); }
  OB_LAUNCHED();
  { Launch L_(p, 3, st); k_iy<T, IY_FIELDS><<<grid_y(p, p->zc_iy), kFftThreads, smem_fy(p, 2, p->zc_iy), st>>>(
      g, p->py, p->zc_iy, 1, S3, nullptr, p->ky, (const C*)p->twy,
      1.0 / ((double)g.nx * (double)g.ny), S1, nullptr); }
  OB_LAUNCHED();
  { Launch L_(p, 4, st); k_ix<T, IX_FIELDS><<<grid_x(p, p->zc_ix), kFftThreads, smem_ix(p, 2 * p->zc_ix), st>>>(
      g, p->px, p->zc_ix, 1, S1, nullptr, nullptr, p->kx, (const C*)p->twx, nullptr, nullptr,
      nullptr, nullptr, 0.0, p->theta0, d, nullptr, nullptr, nullptr); }
  OB_LAUNCHED();
  return OB_OK;
}

// forward 2-D real FFT of one field into S3 (unnormalised)
template <class T>
int fwd_scalar(OraclePlan* p, const T* f, cudaStream_t st) {
  using C = cplx<T>;
  const GridK g = p->g;
  { Launch L_(p, 0, st); k_fx<T, FX_FIELDS><<<grid_x(p, p->zc_fx), kFftThreads, smem_fx(p, 2), st>>>(
      g, p->pxf, p->zc_fx, 1, f, nullptr, nullptr, nullptr, 0.0, p->rho, p->rhoh, p->theta0,
      p->kx, (const C*)p->twx, (C*)p->S1, nullptr, nullptr); }
  OB_LAUNCHED();
  { Launch L_(p, 1, st); k_fy<T, FY_FIELDS><<<grid_y(p, p->zc_fy), kFftThreads, smem_fy(p, 2, p->zc_fy), st>>>(
      g, p->pyf, p->zc_fy, 1, (C*)p->S1, nullptr, p->kx, p->ky, (const C*)p->twy, 1.0,
      (C*)p->S3, nullptr); }
  OB_LAUNCHED();
  return OB_OK;
}

// inverse 2-D real FFT of S3 (scaled) into out
template <class T>
int inv_scalar(OraclePlan* p, double scale, T* out, cudaStream_t st) {
  using C = cplx<T>;
  const GridK g = p->g;
  { Launch L_(p, 3, st); k_iy<T, IY_FIELDS><<<grid_y(p, p->zc_iy), kFftThreads, smem_fy(p, 2, p->zc_iy), st>>>(
      g, p->py, p->zc_iy, 1, (C*)p->S3, nullptr, p->ky, (const C*)p->twy, scale, (C*)p->S1,
      nullptr); }
  OB_LAUNCHED();
  { Launch L_(p, 4, st); k_ix<T, IX_FIELDS><<<grid_x(p, p->zc_ix), kFftThreads, smem_ix(p, 2 * p->zc_ix), st>>>(
      g, p->px, p->zc_ix, 1, (C*)p->S1, nullptr, nullptr, p->kx, (const C*)p->twx, nullptr,
      nullptr, nullptr, nullptr, 0.0, p->theta0, out, nullptr, nullptr, nullptr); }
  OB_LAUNCHED();
  return OB_OK;
}

template <class T>
int gradient_impl(OraclePlan* p, const T* phi, T* gx, T* gy, T* gz, cudaStream_t st) {
  using C = cplx<T>;
  const GridK g = p->g;
  RC(fwd_scalar<T>(p, phi, st));
  { Launch L_(p, 3, st); k_iy<T, IY_GRAD><<<grid_y(p, p->zc_iy), kFftThreads, smem_fy(p, 2, p->zc_iy), st>>>(
      g, p->py, p->zc_iy, 2, (C*)p->S3, nullptr, p->ky, (const C*)p->twy,
      1.0 / ((double)g.nx * (double)g.ny), (C*)p->S1, (C*)p->S2); }
  OB_LAUNCHED();
  { Launch L_(p, 4, st); k_ix<T, IX_GRAD><<<grid_x(p, p->zc_ix), kFftThreads, smem_ix(p, 3 * p->zc_ix + 1), st>>>(
      g, p->px, p->zc_ix, 0, (C*)p->S1, (C*)p->S2, nullptr, p->kx, (const C*)p->twx, nullptr,
      nullptr, nullptr, nullptr, 0.0, p->theta0, gx, gy, gz, nullptr); }
  OB_LAUNCHED();
  return OB_OK;
}

template <class T>
int solve_impl(OraclePlan* p, const T* d, T* phi, int log_diag, cudaStream_t st) {
  using C = cplx<T>;
  const GridK g = p->g;
  RC(fwd_scalar<T>(p, d, st));
  double* diag = nullptr;
  if (log_diag) {
    diag = p->diag;
    OB_CUDA(cudaMemsetAsync(p->diag + OB_DIAG_LAST_DISC, 0, sizeof(double), st));
  }
  const long ncols = (long)g.nxh * g.ny;
  { Launch L_(p, 2, st); k_thomas<T, kThomasCols><<<(unsigned)((ncols + kThomasCols - 1) / kThomasCols), kThomasCols,
                             smem_thomas(p), st>>>(g, thomas_args(p), (C*)p->S3, (C*)p->S3,
                                                   diag, OB_DIAG_LAST_COMPAT, OB_DIAG_LAST_DISC); }
  OB_LAUNCHED();
  return inv_scalar<T>(p, 1.0, phi, st);
}

template <class T>
int apply_op_impl(OraclePlan* p, const T* phi, T* out, cudaStream_t st) {
  using C = cplx<T>;
  const GridK g = p->g;
  RC(fwd_scalar<T>(p, phi, st));
  const size_t ns = (size_t)g.nxh * g.ny * g.nz;
  { Launch L_(p, 7, st); k_neg_ksq<T><<<(unsigned)std::min<size_t>((ns + 255) / 256, 65535), 256, 0, st>>>(
      g, (C*)p->S3, p->kx, p->ky, (C*)p->S3); }
  OB_LAUNCHED();
  RC(inv_scalar<T>(p, 1.0 / ((double)g.nx * (double)g.ny), (T*)p->Du, st));
  const size_t n = (size_t)g.nx * g.ny * g.nz;
  { Launch L_(p, 7, st); k_apply_vert<T><<<(unsigned)std::min<size_t>((n + 255) / 256, 65535), 256, 0, st>>>(
      g, phi, (const T*)p->Du, p->rho, p->rhoh, out); }
  OB_LAUNCHED();
  return OB_OK;
}

template <class T>
int buoyancy_impl(OraclePlan* p, const T* th, T* dw, cudaStream_t st) {
  const size_t n = (size_t)p->g.nx * p->g.ny * (p->g.nz + 1);
  { Launch L_(p, 7, st); k_buoyancy<T><<<(unsigned)std::min<size_t>((n + 255) / 256, 65535), 256, 0, st>>>(
      p->g, th, p->theta0, dw); }
  OB_LAUNCHED();
  return OB_OK;
}

template <class T>
int tendency_impl(OraclePlan* p, int mask, const OracleStatePtrs* s, T* du, T* dv, T* dw,
                  T* dth, double dt_slow, cudaStream_t st) {
  if ((mask & OB_TEND_DAMPING) && p->damping)
    RC(damper_impl<T>(p, (const T*)s->u, (const T*)s->v, dt_slow, st));
  return slow_impl<T, 1>(p, mask, 0.0, (const T*)s->u, (const T*)s->v, (const T*)s->w,
                         (const T*)s->theta_prime, du, dv, dw, dth, st);
}

int check_plan(const OraclePlan* p) {
  if (!p) return fail(OB_ERR_ARG, "plan is NULL");
  return OB_OK;
}

// ---- kernel variants and the autotuner ---------------------------------------
// The plan field behind each OB_VAR_* index (the refiner's compile-time
// chunks live on its FP64 companion); nullptr where the plan has none.
int* var_field(OraclePlan* p, int i) {
  OraclePlan* q = p->dbl;
  switch (i) {
    case OB_VAR_ZC2_FX: return &p->zc2_fx;
    case OB_VAR_ZC2_FXS: return &p->zc2_fxs;
    case OB_VAR_ZC2_IX: return &p->zc2_ix;
    case OB_VAR_ZC2_FY: return &p->zc2_fy;
    case OB_VAR_ZC2_IY: return &p->zc2_iy;
    case OB_VAR_ZC3_FX: return &p->zc3_fx;
    case OB_VAR_ZC3_FXS: return &p->zc3_fxs;
    case OB_VAR_ZC3_IX: return &p->zc3_ix;
    case OB_VAR_ZC3_FXD: return &p->zc3_fxd;
    case OB_VAR_ZC3_FY: return &p->zc3_fy;
    case OB_VAR_ZC3_FYD: return &p->zc3_fyd;
    case OB_VAR_ZC4_FX: return &p->zc4_fx;
    case OB_VAR_ZC4_FXS: return &p->zc4_fxs;
    case OB_VAR_ZC4_IX: return &p->zc4_ix;
    case OB_VAR_ZC4_FXD: return &p->zc4_fxd;
    case OB_VAR_ZC4_FY: return &p->zc4_fy;
    case OB_VAR_ZC4_IY: return &p->zc4_iy;
    case OB_VAR_SLOW_XW: return &p->slow_xw;
    case OB_VAR_THOMAS_FAST: return &p->thomas_fast;
    case OB_VAR_RZC2_FX: return q ? &q->zc2_fx : nullptr;
    case OB_VAR_RZC2_FY: return q ? &q->zc2_fy : nullptr;
    case OB_VAR_ZC4_FYD: return &p->zc4_fyd;
    case OB_VAR_ZC4_FXSH: return &p->zc4_fxsh;
  }
  return nullptr;
}

// The values variant i may take on this plan: 0 (the form off) and the
// z-chunks whose kernels exist for the plan's grid and precision and whose
// tiles fit in shared memory.
std::vector<int> var_values(const OraclePlan* p, int i) {
  const int nx = p->g.nx, ny = p->g.ny, nz = p->g.nz;
  const bool f32 = p->prec == OB_PREC_F32;
  std::vector<int> v{0};
  auto x2 = [&](int kind) {
    if (!p->px8_ok) return;
    for (int z : {1, 2, 4, 8}) {
      if (z > 1 && z > nz) continue;
      const size_t sm = f32 ? x2_smem<float, float>(kind, z, nx) : x2_smem<double, double>(kind, z, nx);
      if (sm <= kSmemMax) v.push_back(z);
    }
  };
  auto y2 = [&](bool dbl) {
    if (!p->py8_ok) return;
    for (int z : {1, 2, 4, 8}) {
      if (z > 1 && z > nz) continue;
      const size_t sm = dbl ? y2_smem_zc<double>(z, ny) : y2_smem_zc<float>(z, ny);
      if (sm <= kSmemMax) v.push_back(z);
    }
  };
  auto list = [&](bool ok, std::initializer_list<int> zs) {
    if (ok)
      for (int z : zs) v.push_back(z);
  };
  switch (i) {
    case OB_VAR_ZC2_FX: x2(0); break;
    case OB_VAR_ZC2_FXS: x2(1); break;
    case OB_VAR_ZC2_IX: x2(2); break;
    case OB_VAR_ZC2_FY:
    case OB_VAR_ZC2_IY: y2(!f32); break;
    case OB_VAR_ZC3_FX:
    case OB_VAR_ZC3_FXS:
    case OB_VAR_ZC3_IX: list(f32 && nx == kXrN, {2, 4, 8}); break;
    case OB_VAR_ZC3_FXD: list(f32 && nx == kXrN, {2, 4}); break;
    case OB_VAR_ZC3_FY: list(f32 && ny == kYrN, {2, 4, 8}); break;
    case OB_VAR_ZC3_FYD: list(f32 && ny == kYrN && p->dbl, {2}); break;
    case OB_VAR_ZC4_FX:
    case OB_VAR_ZC4_FXS:
    case OB_VAR_ZC4_IX: list(f32 && nx == kX4N, {2, 4, 8}); break;
    case OB_VAR_ZC4_FXD: list(f32 && nx == kX4N && p->dbl, {2, 4}); break;
    case OB_VAR_ZC4_FY:
    case OB_VAR_ZC4_IY: list(f32 && ny == kY4N, {2, 4, 8}); break;
    case OB_VAR_SLOW_XW:
      list(true, {1});
      for (int v : {4, 8, 24, 28}) list(slow_xt_grid(p, v), {v});
      break;
    case OB_VAR_THOMAS_FAST: list(true, {1}); break;
    case OB_VAR_RZC2_FX:
      if (f32 && p->dbl && p->px8_ok)
        for (int z : {1, 2, 4, 8})
          if ((z == 1 || z <= nz) && x2_smem<double, float>(0, z, nx) <= kSmemMax) v.push_back(z);
      break;
    case OB_VAR_RZC2_FY:
      if (f32 && p->dbl) y2(true);
      break;
    case OB_VAR_ZC4_FYD: list(f32 && ny == kY4N && p->dbl, {2}); break;
    case OB_VAR_ZC4_FXSH: list(f32 && p->S4 != nullptr, {2, 4, 8}); break;
  }
  return v;
}

bool var_allowed(const OraclePlan* p, int i, int value) {
  for (int z : var_values(p, i))
    if (z == value) return true;
  return false;
}

// Best device time (ms) of three launches of `f` after a warm-up one, with
// CUDA events on st; +inf when a launch fails.
template <class F>
float time_launch(cudaStream_t st, F&& f) {
  const float inf = INFINITY;
  if (f() != OB_OK) return inf;
  cudaEvent_t a = nullptr, b = nullptr;
  if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) return inf;
  float best = inf;
  for (int r = 0; r < 3; ++r) {
    cudaEventRecord(a, st);
    if (f() != OB_OK) break;
    cudaEventRecord(b, st);
    if (cudaEventSynchronize(b) != cudaSuccess) break;
    float ms = inf;
    cudaEventElapsedTime(&ms, a, b);
    best = std::min(best, ms);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (cudaGetLastError() != cudaSuccess) return inf;
  return best;
}

// One tuning group: variants that select among the forms of one kernel
// class; a candidate turns one form on (one variant at one value) with the
// group's other variants off, or every form off.
template <class T>
int tune_group(OraclePlan* p, std::initializer_list<int> vars, cudaStream_t st,
               const std::function<int()>& launch) {
  std::vector<std::pair<int, int>> cands{{-1, 0}};
  for (int i : vars)
    for (int z : var_values(p, i))
      if (z) cands.push_back({i, z});
  if (cands.size() == 1) return OB_OK;
  float best = INFINITY;
  std::pair<int, int> win{-1, 0};
  for (const auto& c : cands) {
    for (int i : vars)
      if (int* f = var_field(p, i)) *f = (i == c.first) ? c.second : 0;
    const float ms = time_launch(st, launch);
    if (ms < best) {
      best = ms;
      win = c;
    }
  }
  for (int i : vars)
    if (int* f = var_field(p, i)) *f = (i == win.first) ? win.second : 0;
  return OB_OK;
}

template <class T>
int tune_impl(OraclePlan* p, cudaStream_t st) {
  const size_t n = (size_t)p->g.nx * p->g.ny * p->g.nz;
  const size_t nw = (size_t)p->g.nx * p->g.ny * (p->g.nz + 1);
  const size_t e = p->esz;
  // finite inputs: zero every buffer a candidate reads
  for (void* b : {p->Au, p->Av, p->Ath, p->Aphi, p->Su, p->Sv, p->Sphi, p->Du, p->Dv})
    OB_CUDA(cudaMemsetAsync(b, 0, n * e, st));
  for (void* b : {p->Aw, p->Sw}) OB_CUDA(cudaMemsetAsync(b, 0, nw * e, st));
  if (p->Bh) OB_CUDA(cudaMemsetAsync(p->Bh, 0, nw * e, st));
  const T *u = (const T*)p->Au, *v = (const T*)p->Av, *w = (const T*)p->Aw,
          *th = (const T*)p->Ath, *bh = (const T*)p->Bh;
  T *uo = (T*)p->Su, *vo = (T*)p->Sv, *wo = (T*)p->Sw, *po = (T*)p->Sphi;
  const bool stage = p->Bh && p->buoyancy && p->projection;
  const double sdt = 10.0;
  RC(tune_group<T>(p, {OB_VAR_ZC4_FX, OB_VAR_ZC3_FX, OB_VAR_ZC2_FX}, st,
                   [&] { return proj_fx<T>(p, false, u, v, w, th, nullptr, 0.0, st); }));
  if (stage)
    RC(tune_group<T>(p, {OB_VAR_ZC4_FXS, OB_VAR_ZC3_FXS, OB_VAR_ZC2_FXS}, st,
                     [&] { return proj_fx<T>(p, true, u, v, w, th, bh, sdt, st); }));
  RC(tune_group<T>(p, {OB_VAR_ZC4_IX, OB_VAR_ZC3_IX, OB_VAR_ZC2_IX}, st, [&] {
    return stage ? proj_ix<T>(p, true, u, v, w, th, bh, sdt, uo, vo, wo, po, st)
                 : proj_ix<T>(p, false, u, v, w, th, nullptr, 0.0, uo, vo, wo, po, st);
  }));
  // forward and inverse y share the 512-point register form's chunk: time
  // the two together for it, and each alone for the others
  {
    const int fy4 = p->zc4_fy, iy4 = p->zc4_iy;
    std::vector<std::array<int, 5>> cands;  // zc4_fy, zc4_iy, zc3_fy, zc2_fy, zc2_iy
    cands.push_back({0, 0, 0, 0, 0});
    auto vals = [&](int i) {
      std::vector<int> r;
      for (int z : var_values(p, i))
        if (z) r.push_back(z);
      return r;
    };
    const auto f4 = vals(OB_VAR_ZC4_FY), i4 = vals(OB_VAR_ZC4_IY), y3 = vals(OB_VAR_ZC3_FY),
               f2 = vals(OB_VAR_ZC2_FY), i2 = vals(OB_VAR_ZC2_IY);
    for (int a : f4)
      for (int b : i4) cands.push_back({a, b, 0, 0, 0});
    for (int a : y3) cands.push_back({0, 0, a, 0, 0});
    for (int a : f2)
      for (int b : i2) cands.push_back({0, 0, 0, a, b});
    (void)fy4;
    (void)iy4;
    if (cands.size() > 1) {
      // time each forward and inverse form once, then pick the best pair
      auto apply = [&](const std::array<int, 5>& c) {
        p->zc4_fy = c[0];
        p->zc4_iy = c[1];
        p->zc3_fy = c[2];
        p->zc2_fy = c[3];
        p->zc2_iy = c[4];
      };
      float best = INFINITY;
      std::array<int, 5> win = cands[0];
      for (const auto& c : cands) {
        apply(c);
        const float t = time_launch(st, [&] { return proj_fy<T>(p, st); }) +
                        time_launch(st, [&] { return proj_iy<T>(p, 3, st); });
        if (t < best) {
          best = t;
          win = c;
        }
      }
      apply(win);
    }
  }
  if constexpr (sizeof(T) == 4) {
    RC(tune_group<T>(p, {OB_VAR_THOMAS_FAST}, st, [&] {
      return thomas_solve<T>(p, 2, (cplx<T>*)p->S3, nullptr, 0, 0, st);
    }));
    if (p->dbl) {
      RC(tune_group<T>(p, {OB_VAR_ZC4_FXD, OB_VAR_ZC3_FXD, OB_VAR_RZC2_FX}, st,
                       [&] { return refine_fx(p, (const float*)u, (const float*)v,
                                              (const float*)w, st); }));
      RC(tune_group<T>(p, {OB_VAR_ZC4_FYD, OB_VAR_ZC3_FYD, OB_VAR_RZC2_FY}, st,
                       [&] { return refine_fy(p, st); }));
    }
    const bool slow = p->advection || p->coriolis || p->heating;
    const bool extra = p->drag || p->sponge || p->diffusion || p->cooling;
    const int all = OB_TEND_ADVECTION | OB_TEND_CORIOLIS | OB_TEND_HEATING |
                    (extra ? (OB_TEND_DRAG | OB_TEND_SPONGE | OB_TEND_DIFFUSION |
                              OB_TEND_COOLING) : 0);
    if (slow && var_values(p, OB_VAR_SLOW_XW).size() > 1)
      RC(tune_group<T>(p, {OB_VAR_SLOW_XW}, st, [&] {
        return slow_impl<T, 0>(p, all, 1.0, u, v, w, th, uo, vo, wo, (T*)p->Sphi, st);
      }));
    // the fast stages' forward transforms, shared or one x launch per stage:
    // timed as the three stages' x and y launches together
    if (stage && p->zc4_fy && var_values(p, OB_VAR_ZC4_FXSH).size() > 1)
      RC(tune_group<T>(p, {OB_VAR_ZC4_FXSH}, st, [&] {
        if (p->zc4_fxsh) {
          fx4sh(p, (const float*)u, (const float*)v, (const float*)w, (const float*)bh, st);
          for (int s = 0; s < 3; ++s) fy4sh(p, (float)(sdt * (s + 1) / 3.0), st);
          OB_LAUNCHED();
          return OB_OK;
        }
        for (int s = 0; s < 3; ++s) {
          RC(proj_fx<T>(p, true, u, v, w, th, bh, sdt * (s + 1) / 3.0, st));
          RC(proj_fy<T>(p, st));
        }
        return OB_OK;
      }));
  }
  OB_CUDA(cudaStreamSynchronize(st));
  return OB_OK;
}

// Tuned choices per (grid, precision, component set, device), for the life
// of the process and optionally in a text file (ORACLE_B200_TUNE_CACHE):
// one line "key | v0 v1 ..." per entry.
std::mutex g_tune_mu;
std::map<std::string, std::vector<int>> g_tune;
bool g_tune_loaded = false;

std::string tune_key(const OraclePlan* p) {
  int dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  cudaDeviceProp prop{};
  cudaGetDeviceProperties(&prop, dev);
  char buf[512];
  snprintf(buf, sizeof buf, "v1 %dx%dx%d prec%d stage%d slow%d%d%d%d prod%d%d%d%d damp%d sm%d %s",
           p->g.nx, p->g.ny, p->g.nz, p->prec, (int)(p->buoyancy && p->projection),
           p->advection, p->coriolis, p->heating, p->damping, p->drag, p->sponge, p->diffusion,
           p->cooling, p->damping, nsm, prop.name);
  std::string k = buf;
  for (char& c : k)
    if (c == '|' || c == '\n') c = '_';
  return k;
}

void tune_cache_load() {
  if (g_tune_loaded) return;
  g_tune_loaded = true;
  const char* path = getenv("ORACLE_B200_TUNE_CACHE");
  if (!path || !*path) return;
  FILE* f = fopen(path, "r");
  if (!f) return;
  char line[1024];
  while (fgets(line, sizeof line, f)) {
    char* bar = strchr(line, '|');
    if (!bar) continue;
    std::string key(line, bar - line);
    while (!key.empty() && key.back() == ' ') key.pop_back();
    std::vector<int> vals;
    char* s = bar + 1;
    char* end = nullptr;
    for (long x = strtol(s, &end, 10); end != s; x = strtol(s, &end, 10)) {
      vals.push_back((int)x);
      s = end;
    }
    if (vals.size() == OB_VAR_COUNT) g_tune[key] = vals;
  }
  fclose(f);
}

void tune_cache_store(const std::string& key, const std::vector<int>& vals) {
  g_tune[key] = vals;
  const char* path = getenv("ORACLE_B200_TUNE_CACHE");
  if (!path || !*path) return;
  FILE* f = fopen(path, "a");
  if (!f) return;
  fprintf(f, "%s |", key.c_str());
  for (int x : vals) fprintf(f, " %d", x);
  fprintf(f, "\n");
  fclose(f);
}

}  // namespace

// ===========================================================================
// extern "C"
// ===========================================================================

extern "C" {

// ---- storm tracker --------------------------------------------------------
struct OracleTracker {
  int nx = 0, ny = 0, nz = 0;
  int npsfc = 1, nmin = 1;  // CTAs of the two grid-wide kernels
  double *z = nullptr, *rho0 = nullptr, *theta0 = nullptr;
  double *p = nullptr, *part = nullptr, *zcol = nullptr;
  TrackPart* parts = nullptr;
  TrackFixD* fix = nullptr;
  std::vector<void*> allocs;
};

namespace {

int tracker_alloc(OracleTracker* t, void** out, size_t bytes) {
  void* q = nullptr;
  OB_CUDA(cudaMalloc(&q, bytes));
  t->allocs.push_back(q);
  *out = q;
  return OB_OK;
}

void tracker_free(OracleTracker* t) {
  for (void* q : t->allocs) cudaFree(q);
  delete t;
}

int check_tracker_call(const OracleTracker* t, int precision, const void* a, const void* b) {
  if (!t) return fail(OB_ERR_ARG, "tracker is NULL");
  if (!a || !b) return fail(OB_ERR_ARG, "tracker: NULL pointer");
  if (precision != OB_PREC_F64 && precision != OB_PREC_F32)
    return fail(OB_ERR_ARG, "tracker: precision must be OB_PREC_F64 or OB_PREC_F32");
  return OB_OK;
}

}  // namespace

int oracle_b200_vortex_fill(int nx, int ny, int nz, int precision, const double* col,
                            const double* S, const double* rr, const double* tab, int nr,
                            double u_env, double v_env, const OracleStatePtrs* out, void* stream) {
  if (nx < 1 || ny < 1 || nz < 1 || nr < 2 || (long long)nx * ny > (1LL << 30))
    return fail(OB_ERR_ARG, "vortex_fill: bad sizes (%d, %d, %d, nr %d)", nx, ny, nz, nr);
  if (!col || !S || !rr || !tab || !out || !out->u || !out->v || !out->w ||
      !out->theta_prime || !out->phi)
    return fail(OB_ERR_ARG, "vortex_fill: NULL pointer");
  if (precision != OB_PREC_F64 && precision != OB_PREC_F32)
    return fail(OB_ERR_ARG, "vortex_fill: precision must be OB_PREC_F64 or OB_PREC_F32");
  const int ncol = nx * ny;
  int dev = 0, nsm = 148;
  OB_CUDA(cudaGetDevice(&dev));
  OB_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const int blocks = (int)std::min<long long>((ncol + 7) / 8, 16LL * nsm);
  cudaStream_t st = (cudaStream_t)stream;
  if (precision == OB_PREC_F64)
    k_vortex_fill<double><<<blocks, 256, 0, st>>>(
        ncol, nz, nr, col, S, rr, tab, u_env, v_env, (double*)out->u, (double*)out->v,
        (double*)out->w, (double*)out->theta_prime, (double*)out->phi);
  else
    k_vortex_fill<float><<<blocks, 256, 0, st>>>(
        ncol, nz, nr, col, S, rr, tab, u_env, v_env, (float*)out->u, (float*)out->v,
        (float*)out->w, (float*)out->theta_prime, (float*)out->phi);
  OB_LAUNCHED();
  return OB_OK;
}

int oracle_b200_tracker_create(int nx, int ny, int nz, const double* z, const double* rho0,
                               const double* theta0, OracleTracker** out) {
  if (!out) return fail(OB_ERR_ARG, "tracker_create: out is NULL");
  *out = nullptr;
  if (nx < 3 || ny < 3 || nz < 2 || (long long)nx * ny > (1LL << 30))
    return fail(OB_ERR_ARG, "tracker_create: need nx, ny >= 3, nz >= 2 (got %d, %d, %d)", nx,
                ny, nz);
  if (!z || !rho0 || !theta0) return fail(OB_ERR_ARG, "tracker_create: NULL profile");
  OracleTracker* t = new OracleTracker();
  t->nx = nx;
  t->ny = ny;
  t->nz = nz;
  int dev = 0, nsm = 148;
  OB_CUDA(cudaGetDevice(&dev));
  OB_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const long long ncol = (long long)nx * ny;
  t->npsfc = (int)std::min<long long>((ncol + 7) / 8, 8LL * nsm);
  t->nmin = (int)std::min<long long>((ncol + kTrackThreads - 1) / kTrackThreads, 2LL * nsm);
  int rc;
  auto A = [&](void** q, size_t bytes) { return tracker_alloc(t, q, bytes); };
  if ((rc = A((void**)&t->z, nz * sizeof(double))) || (rc = A((void**)&t->rho0, nz * sizeof(double))) ||
      (rc = A((void**)&t->theta0, nz * sizeof(double))) ||
      (rc = A((void**)&t->p, ncol * sizeof(double))) ||
      (rc = A((void**)&t->zcol, ncol * sizeof(double))) ||
      (rc = A((void**)&t->part, t->npsfc * sizeof(double))) ||
      (rc = A((void**)&t->parts, t->nmin * sizeof(TrackPart))) ||
      (rc = A((void**)&t->fix, sizeof(TrackFixD)))) {
    tracker_free(t);
    return rc;
  }
  cudaError_t e = cudaMemcpy(t->z, z, nz * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(t->rho0, rho0, nz * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(t->theta0, theta0, nz * sizeof(double), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    tracker_free(t);
    return fail(OB_ERR_CUDA, "tracker_create: copy of the profiles failed: %s", cudaGetErrorString(e));
  }
  *out = t;
  return OB_OK;
}

int oracle_b200_tracker_destroy(OracleTracker* t) {
  if (t) tracker_free(t);
  return OB_OK;
}

int oracle_b200_track_theta(OracleTracker* t, const void* th, int precision, int margin,
                            int has_last, double last_ix, double last_iy, double r0_cells,
                            OracleTrackFix* out, void* stream) {
  if (int rc = check_tracker_call(t, precision, th, out)) return rc;
  if (margin < 0) return fail(OB_ERR_ARG, "track_theta: margin must be >= 0");
  if (has_last && !(r0_cells > 0.0))
    return fail(OB_ERR_ARG, "track_theta: r0_cells must be > 0");
  static_assert(sizeof(TrackFixD) == sizeof(OracleTrackFix), "TrackFixD layout");
  cudaStream_t st = (cudaStream_t)stream;
  const int ncol = t->nx * t->ny;
  if (precision == OB_PREC_F64)
    k_track_psfc<double><<<t->npsfc, kTrackThreads, 0, st>>>(
        ncol, t->nz, (const double*)th, t->z, t->rho0, t->theta0, t->p, t->part);
  else
    k_track_psfc<float><<<t->npsfc, kTrackThreads, 0, st>>>(
        ncol, t->nz, (const float*)th, t->z, t->rho0, t->theta0, t->p, t->part);
  OB_LAUNCHED();
  TrackWin win{has_last ? 1 : 0, last_ix, last_iy, r0_cells};
  k_track_min<<<t->nmin, kTrackThreads, 0, st>>>(t->nx, t->ny, margin, win, t->p, t->part,
                                                  t->npsfc, t->parts);
  OB_LAUNCHED();
  k_track_final<<<1, kTrackThreads, 0, st>>>(t->nx, t->ny, win, t->p, t->part, t->npsfc,
                                              t->parts, t->nmin, t->fix);
  OB_LAUNCHED();
  OB_CUDA(cudaMemcpyAsync(out, t->fix, sizeof(TrackFixD), cudaMemcpyDeviceToHost, st));
  OB_CUDA(cudaStreamSynchronize(st));
  return OB_OK;
}

int oracle_b200_track_vorticity(OracleTracker* t, const void* u, const void* v, int precision,
                                double dx, double* zcol_host, void* stream) {
  if (int rc = check_tracker_call(t, precision, u, v)) return rc;
  if (!zcol_host || !(dx > 0.0)) return fail(OB_ERR_ARG, "track_vorticity: bad output or dx");
  if (t->nz < 2) return fail(OB_ERR_ARG, "track_vorticity: need nz >= 2");
  cudaStream_t st = (cudaStream_t)stream;
  if (precision == OB_PREC_F64)
    k_track_zcol<double><<<t->npsfc, kTrackThreads, 0, st>>>(t->nx, t->ny, t->nz,
                                                           (const double*)u, (const double*)v,
                                                           dx, t->zcol);
  else
    k_track_zcol<float><<<t->npsfc, kTrackThreads, 0, st>>>(t->nx, t->ny, t->nz,
                                                          (const float*)u, (const float*)v,
                                                          dx, t->zcol);
  OB_LAUNCHED();
  OB_CUDA(cudaMemcpyAsync(zcol_host, t->zcol, (size_t)t->nx * t->ny * sizeof(double),
                          cudaMemcpyDeviceToHost, st));
  OB_CUDA(cudaStreamSynchronize(st));
  return OB_OK;
}

/* ---- vortex diagnostics ------------------------------------------------- */

struct OracleVortexDiag {
  int nx = 0, ny = 0, nz = 0;
  int nblk = 1;  // CTAs of the grid-wide reductions
  int* lev = nullptr;
  double *um = nullptr, *vm = nullptr, *zeta = nullptr, *zp = nullptr, *zs = nullptr;
  double *sq = nullptr, *dsum = nullptr, *ring = nullptr, *edges = nullptr, *cen = nullptr;
  VdMax *part = nullptr, *best = nullptr;
  std::vector<void*> allocs;
};

namespace {

constexpr int kVdMaxBins = 64;

void vdiag_free(OracleVortexDiag* d) {
  for (void* q : d->allocs) cudaFree(q);
  delete d;
}

int vdiag_call(const OracleVortexDiag* d, int precision, const void* u, const void* v) {
  if (!d) return fail(OB_ERR_ARG, "vdiag: workspace is NULL");
  if (!u || !v) return fail(OB_ERR_ARG, "vdiag: NULL field");
  if (precision != OB_PREC_F64 && precision != OB_PREC_F32)
    return fail(OB_ERR_ARG, "vdiag: precision must be OB_PREC_F64 or OB_PREC_F32");
  return OB_OK;
}

// Uploads the level list after checking it is ascending inside [0, nz).
int vdiag_levels(OracleVortexDiag* d, const int* lev, int nlev, cudaStream_t st) {
  if (!lev || nlev < 1 || nlev > d->nz) return fail(OB_ERR_ARG, "vdiag: bad level list");
  for (int l = 0; l < nlev; ++l)
    if (lev[l] < 0 || lev[l] >= d->nz || (l > 0 && lev[l] <= lev[l - 1]))
      return fail(OB_ERR_ARG, "vdiag: levels must ascend inside [0, nz)");
  OB_CUDA(cudaMemcpyAsync(d->lev, lev, nlev * sizeof(int), cudaMemcpyHostToDevice, st));
  return OB_OK;
}

int vdiag_mean_winds(OracleVortexDiag* d, const void* u, const void* v, int precision, int nlev,
                     cudaStream_t st) {
  const long long ncol = (long long)d->nx * d->ny;
  if (precision == OB_PREC_F64)
    k_vd_band_mean<double><<<d->nblk, kVdThreads, 0, st>>>(
        (const double*)u, (const double*)v, ncol, d->nz, d->lev, nlev, d->um, d->vm);
  else
    k_vd_band_mean<float><<<d->nblk, kVdThreads, 0, st>>>(
        (const float*)u, (const float*)v, ncol, d->nz, d->lev, nlev, d->um, d->vm);
  OB_LAUNCHED();
  return OB_OK;
}

}  // namespace

int oracle_b200_vdiag_create(int nx, int ny, int nz, OracleVortexDiag** out) {
  if (!out) return fail(OB_ERR_ARG, "vdiag_create: out is NULL");
  *out = nullptr;
  if (nx < 3 || ny < 3 || nz < 1 || (long long)nx * ny > (1LL << 30) ||
      (long long)nx * ny * nz > (1LL << 40))
    return fail(OB_ERR_ARG, "vdiag_create: need nx, ny >= 3 and nz >= 1 (got %d, %d, %d)", nx,
                ny, nz);
  int dev = 0, nsm = 148;
  OB_CUDA(cudaGetDevice(&dev));
  OB_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  OracleVortexDiag* d = new OracleVortexDiag();
  d->nx = nx;
  d->ny = ny;
  d->nz = nz;
  const long long ncol = (long long)nx * ny;
  d->nblk = (int)std::min<long long>((ncol + kVdThreads - 1) / kVdThreads, 2LL * nsm);
  auto A = [&](void** q, size_t bytes) {
    void* p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) return fail(OB_ERR_CUDA, "vdiag_create: cudaMalloc");
    d->allocs.push_back(p);
    *q = p;
    return (int)OB_OK;
  };
  int rc;
  if ((rc = A((void**)&d->lev, nz * sizeof(int))) || (rc = A((void**)&d->um, ncol * 8)) ||
      (rc = A((void**)&d->vm, ncol * 8)) || (rc = A((void**)&d->zeta, ncol * 8)) ||
      (rc = A((void**)&d->zp, ncol * 8)) || (rc = A((void**)&d->zs, ncol * 8)) ||
      (rc = A((void**)&d->sq, d->nblk * 8)) || (rc = A((void**)&d->dsum, 8)) ||
      (rc = A((void**)&d->ring, 3 * (kVdMaxBins + 1) * 8)) ||
      (rc = A((void**)&d->edges, (kVdMaxBins + 1) * 8)) || (rc = A((void**)&d->cen, 3 * 8)) ||
      (rc = A((void**)&d->part, d->nblk * sizeof(VdMax))) ||
      (rc = A((void**)&d->best, sizeof(VdMax)))) {
    vdiag_free(d);
    return rc;
  }
  *out = d;
  return OB_OK;
}

int oracle_b200_vdiag_destroy(OracleVortexDiag* d) {
  if (d) vdiag_free(d);
  return OB_OK;
}

int oracle_b200_vdiag_speed_max(OracleVortexDiag* d, const void* u, const void* v,
                                int precision, const int* levels, int nlev, double u_env,
                                double v_env, OracleVdMax* out, void* stream) {
  if (int rc = vdiag_call(d, precision, u, v)) return rc;
  if (!out) return fail(OB_ERR_ARG, "vdiag_speed_max: out is NULL");
  static_assert(sizeof(VdMax) == sizeof(OracleVdMax), "VdMax layout");
  cudaStream_t st = (cudaStream_t)stream;
  if (int rc = vdiag_levels(d, levels, nlev, st)) return rc;
  const long long ncol = (long long)d->nx * d->ny;
  if (precision == OB_PREC_F64)
    k_vd_speed_max<double><<<d->nblk, kVdThreads, 0, st>>>(
        (const double*)u, (const double*)v, ncol, d->nz, d->lev, nlev, u_env, v_env, d->part);
  else
    k_vd_speed_max<float><<<d->nblk, kVdThreads, 0, st>>>(
        (const float*)u, (const float*)v, ncol, d->nz, d->lev, nlev, u_env, v_env, d->part);
  OB_LAUNCHED();
  k_vd_max_final<<<1, kVdThreads, 0, st>>>(d->part, d->nblk, d->best);
  OB_LAUNCHED();
  OB_CUDA(cudaMemcpyAsync(out, d->best, sizeof(VdMax), cudaMemcpyDeviceToHost, st));
  OB_CUDA(cudaStreamSynchronize(st));
  return OB_OK;
}

int oracle_b200_vdiag_vorticity(OracleVortexDiag* d, const void* u, const void* v,
                                int precision, const int* levels, int nlev, double dx,
                                double dy, double cx_m, double cy_m, double window_m,
                                OracleVdMax* center, double* zeta_sq_sum, void* stream) {
  if (int rc = vdiag_call(d, precision, u, v)) return rc;
  if (!center || !zeta_sq_sum || !(dx > 0.0) || !(dy > 0.0))
    return fail(OB_ERR_ARG, "vdiag_vorticity: bad output or spacing");
  cudaStream_t st = (cudaStream_t)stream;
  if (int rc = vdiag_levels(d, levels, nlev, st)) return rc;
  if (int rc = vdiag_mean_winds(d, u, v, precision, nlev, st)) return rc;
  k_vd_zeta<<<d->nblk, kVdThreads, 0, st>>>(d->um, d->vm, d->nx, d->ny, dx, dy, cx_m, cy_m,
                                            window_m, d->zeta, d->part, d->sq);
  OB_LAUNCHED();
  k_vd_max_final<<<1, kVdThreads, 0, st>>>(d->part, d->nblk, d->best);
  OB_LAUNCHED();
  k_vd_sum_final<<<1, kVdThreads, 0, st>>>(d->sq, d->nblk, d->dsum);
  OB_LAUNCHED();
  OB_CUDA(cudaMemcpyAsync(center, d->best, sizeof(VdMax), cudaMemcpyDeviceToHost, st));
  OB_CUDA(cudaMemcpyAsync(zeta_sq_sum, d->dsum, sizeof(double), cudaMemcpyDeviceToHost, st));
  OB_CUDA(cudaStreamSynchronize(st));
  return OB_OK;
}

int oracle_b200_vdiag_ke(OracleVortexDiag* d, const void* u, const void* v, int precision,
                         double u_env, double v_env, double* sum, void* stream) {
  if (int rc = vdiag_call(d, precision, u, v)) return rc;
  if (!sum) return fail(OB_ERR_ARG, "vdiag_ke: out is NULL");
  cudaStream_t st = (cudaStream_t)stream;
  const long long n = (long long)d->nx * d->ny * d->nz;
  if (precision == OB_PREC_F64)
    k_vd_ke<double><<<d->nblk, kVdThreads, 0, st>>>((const double*)u, (const double*)v, n,
                                                    u_env, v_env, d->sq);
  else
    k_vd_ke<float><<<d->nblk, kVdThreads, 0, st>>>((const float*)u, (const float*)v, n, u_env,
                                                   v_env, d->sq);
  OB_LAUNCHED();
  k_vd_sum_final<<<1, kVdThreads, 0, st>>>(d->sq, d->nblk, d->dsum);
  OB_LAUNCHED();
  OB_CUDA(cudaMemcpyAsync(sum, d->dsum, sizeof(double), cudaMemcpyDeviceToHost, st));
  OB_CUDA(cudaStreamSynchronize(st));
  return OB_OK;
}

int oracle_b200_vdiag_rings(OracleVortexDiag* d, const void* u, const void* v,
                            int precision, const int* levels, int nlev, double dx, double dy,
                            double cx_m, double cy_m, const double* edges, int n_bins,
                            double r_vent_m, double* out, void* stream) {
  if (int rc = vdiag_call(d, precision, u, v)) return rc;
  if (!out || !edges || n_bins < 1 || n_bins > kVdMaxBins || !(dx > 0.0) || !(dy > 0.0))
    return fail(OB_ERR_ARG, "vdiag_rings: bad output, edges, bin count (1..%d) or spacing",
                kVdMaxBins);
  cudaStream_t st = (cudaStream_t)stream;
  if (int rc = vdiag_levels(d, levels, nlev, st)) return rc;
  if (int rc = vdiag_mean_winds(d, u, v, precision, nlev, st)) return rc;
  // bounding box of the disk, one cell of margin each side (every cell with
  // r < r_vent lies inside it); empty for a non-finite centre or radius
  double rmax = r_vent_m;
  for (int b = 0; b <= n_bins; ++b) rmax = std::fmax(rmax, edges[b]);
  int i0 = 0, i1 = 0, j0 = 0, j1 = 0;
  if (std::isfinite(cx_m) && std::isfinite(cy_m) && std::isfinite(rmax)) {
    auto clampi = [](double a, int n) { return (int)std::fmin(std::fmax(a, 0.0), (double)n); };
    i0 = clampi(std::floor((cx_m - rmax) / dx - 0.5) - 1.0, d->nx);
    i1 = clampi(std::ceil((cx_m + rmax) / dx - 0.5) + 2.0, d->nx);
    j0 = clampi(std::floor((cy_m - rmax) / dy - 0.5) - 1.0, d->ny);
    j1 = clampi(std::ceil((cy_m + rmax) / dy - 0.5) + 2.0, d->ny);
  }
  if (i1 <= i0 || j1 <= j0) {
    i0 = i1 = 0;
    j0 = j1 = 0;
  }
  OB_CUDA(cudaMemcpyAsync(d->edges, edges, (n_bins + 1) * sizeof(double),
                          cudaMemcpyHostToDevice, st));
  k_vd_rings<<<1, kVdThreads, 0, st>>>(d->um, d->vm, d->ny, i0, i1, j0, j1, dx, dy, cx_m, cy_m,
                                       d->edges, n_bins, r_vent_m, d->ring);
  OB_LAUNCHED();
  OB_CUDA(cudaMemcpyAsync(out, d->ring, 3 * (n_bins + 1) * sizeof(double),
                          cudaMemcpyDeviceToHost, st));
  OB_CUDA(cudaStreamSynchronize(st));
  return OB_OK;
}

int oracle_b200_vdiag_zpos(OracleVortexDiag* d, const void* u, const void* v, int precision,
                           double dx, void* stream) {
  if (int rc = vdiag_call(d, precision, u, v)) return rc;
  if (!(dx > 0.0)) return fail(OB_ERR_ARG, "vdiag_zpos: dx must be > 0");
  if (d->nz < 2 || d->nz / 2 > kVdMaxPairwise)
    return fail(OB_ERR_ARG, "vdiag_zpos: need 2 <= nz and nz / 2 <= %d", kVdMaxPairwise);
  cudaStream_t st = (cudaStream_t)stream;
  if (precision == OB_PREC_F64)
    k_vd_zpos<double><<<d->nblk, kVdThreads, 0, st>>>((const double*)u, (const double*)v,
                                                      d->nx, d->ny, d->nz, dx, d->zp);
  else
    k_vd_zpos<float><<<d->nblk, kVdThreads, 0, st>>>((const float*)u, (const float*)v, d->nx,
                                                     d->ny, d->nz, dx, d->zp);
  OB_LAUNCHED();
  k_vd_smooth<<<d->nblk, kVdThreads, 0, st>>>(d->zp, d->nx, d->ny, d->zs);
  OB_LAUNCHED();
  OB_CUDA(cudaStreamSynchronize(st));
  return OB_OK;
}

int oracle_b200_vdiag_centroid(OracleVortexDiag* d, int i0, int i1, int j0, int j1,
                               double* out, void* stream) {
  if (!d || !out) return fail(OB_ERR_ARG, "vdiag_centroid: NULL argument");
  if (i0 < 0 || j0 < 0 || i1 > d->nx || j1 > d->ny || i1 < i0 || j1 < j0)
    return fail(OB_ERR_ARG, "vdiag_centroid: patch outside the grid");
  cudaStream_t st = (cudaStream_t)stream;
  k_vd_centroid<<<1, kVdThreads, 0, st>>>(d->zs, d->ny, i0, i1, j0, j1, d->cen);
  OB_LAUNCHED();
  OB_CUDA(cudaMemcpyAsync(out, d->cen, 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
  OB_CUDA(cudaStreamSynchronize(st));
  return OB_OK;
}

const char* oracle_b200_last_error(void) { return g_err.c_str(); }

int oracle_b200_version(void) { return OB_ABI_VERSION; }

size_t oracle_b200_plan_scratch_bytes(const OraclePlan* p) { return p ? p->scratch_bytes : 0; }

int oracle_b200_plan_destroy(OraclePlan* p) {
  if (!p) return OB_OK;
  // wait for all device work, as cudaFree would, so that no queued kernel
  // still uses the memory when the pool hands it out again
  cudaDeviceSynchronize();
  release_plan(p, p->astream);
  return OB_OK;
}

int oracle_b200_plan_release(OraclePlan* p, void* stream) {
  if (!p) return OB_OK;
  release_plan(p, (cudaStream_t)stream);
  return OB_OK;
}

int oracle_b200_plan_create(const OracleGridDesc* grid, const OracleComponentDesc* comp,
                            OraclePlan** out) {
  if (!grid || !comp || !out) return fail(OB_ERR_ARG, "NULL argument to plan_create");
  *out = nullptr;
  const int nx = grid->nx, ny = grid->ny, nz = grid->nz;
  if (nx < 4 || ny < 4 || (nx & 1) || (ny & 1))
    return fail(OB_ERR_ARG, "nx and ny must be even and >= 4 (got %d, %d)", nx, ny);
  if (nz < 3) return fail(OB_ERR_ARG, "nz must be >= 3 (got %d)", nz);
  if (!(grid->Lx > 0 && grid->Ly > 0 && grid->Lz > 0))
    return fail(OB_ERR_ARG, "domain lengths must be positive");
  if (grid->precision != OB_PREC_F64 && grid->precision != OB_PREC_F32)
    return fail(OB_ERR_ARG, "unknown precision %d", grid->precision);
  if (!comp->rho0 || !comp->theta0) return fail(OB_ERR_ARG, "rho0 and theta0 are required");
  if (comp->advection < 0 || comp->advection > 2)
    return fail(OB_ERR_ARG, "unknown advection scheme %d", comp->advection);
  if (comp->coriolis < 0 || comp->coriolis > 2)
    return fail(OB_ERR_ARG, "unknown coriolis mode %d", comp->coriolis);
  if (comp->coriolis == OB_COR_BETA && !comp->f_y)
    return fail(OB_ERR_ARG, "beta-plane Coriolis needs f_y");
  if (comp->heating && (!comp->heat_r || !comp->heat_z))
    return fail(OB_ERR_ARG, "heating needs heat_r and heat_z");
  if (comp->drag && (!comp->drag_weight || !(comp->drag_dz > 0)))
    return fail(OB_ERR_ARG, "surface drag needs drag_weight and a positive drag_dz");
  if (comp->sponge && (!comp->sponge_alpha || !comp->sponge_alpha_h))
    return fail(OB_ERR_ARG, "sponge damping needs sponge_alpha and sponge_alpha_h");
  if (comp->diffusion < OB_DIFF_NONE || comp->diffusion > OB_DIFF_BIHARMONIC)
    return fail(OB_ERR_ARG, "unknown horizontal diffusion %d", comp->diffusion);
  if (comp->diffusion && !(comp->diff_dx2 > 0 && comp->diff_dy2 > 0))
    return fail(OB_ERR_ARG, "horizontal diffusion needs positive diff_dx2 and diff_dy2");
  if ((long)nx * ny * (nz + 1) > (1L << 31))
    return fail(OB_ERR_ARG, "grid too large for 32-bit launch geometry");

  OraclePlan* p = new OraclePlan();
  auto bail = [&](int rc) {
    oracle_b200_plan_destroy(p);
    return rc;
  };
  if (int rc = plan_pool(&p->pool)) return bail(rc);
  if (cudaStreamCreateWithFlags(&p->astream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&p->aux, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&p->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&p->ev_join, cudaEventDisableTiming) != cudaSuccess)
    return bail(fail(OB_ERR_CUDA, "plan_create: stream or event creation failed"));
  p->prec = grid->precision;
  p->esz = p->prec == OB_PREC_F64 ? 8 : 4;
  p->g.nx = nx;
  p->g.ny = ny;
  p->g.nz = nz;
  p->g.M = nx / 2;
  p->g.nxh = nx / 2 + 1;
  p->g.dx = grid->Lx / nx;
  p->g.dy = grid->Ly / ny;
  p->g.dz = grid->Lz / nz;
  p->buoyancy = comp->buoyancy != 0;
  p->projection = comp->projection != 0;
  p->advection = comp->advection;
  p->coriolis = comp->coriolis;
  p->damping = comp->damping != 0;
  p->heating = comp->heating != 0;
  p->drag = comp->drag != 0;
  p->sponge = comp->sponge != 0;
  p->diffusion = comp->diffusion;
  p->cooling = comp->cooling != 0;
  p->drag_cd = comp->drag_cd;
  p->drag_dz = comp->drag_dz > 0 ? comp->drag_dz : 1.0;
  p->drag_u_env = comp->drag_u_env;
  p->drag_v_env = comp->drag_v_env;
  p->sponge_u_env = comp->sponge_u_env;
  p->sponge_v_env = comp->sponge_v_env;
  p->diff_nu = comp->diff_nu;
  p->diff_dx2 = comp->diffusion ? comp->diff_dx2 : 1.0;
  p->diff_dy2 = comp->diffusion ? comp->diff_dy2 : 1.0;
  p->cool_alpha = comp->cool_alpha;
  if (!(comp->blowup_u_max >= 0.0))
    return bail(fail(OB_ERR_ARG, "blowup_u_max must be >= 0 (got %g)", comp->blowup_u_max));
  p->blowup_u = comp->blowup_u_max;
  p->f0 = comp->f0;
  p->u_env = comp->u_env;
  p->v_env = comp->v_env;
  p->epsilon = comp->epsilon;
  p->diag_every = comp->poisson_diag_every;
  if (!factorize(nx / 2, p->px) || !factorize(ny, p->py) || !factorize(nx / 2, p->pxf, false) ||
      !factorize(ny, p->pyf, false))
    return bail(fail(OB_ERR_ARG, "nx/2=%d and ny=%d must factor into 2, 3, 5", nx / 2, ny));

  const double dz = p->g.dz;
  const double* rf = comp->rho0;
  // rho on half levels and the Thomas tables
  const int n0 = nz - 1;
  std::vector<double> rh(nz + 1), a(nz), c(nz), negs(nz), a0(n0), inv0(n0), cp0(n0);
  fill_solver_tables(nz, dz, rf,
                     SolverTables{rh.data(), a.data(), c.data(), negs.data(), a0.data(),
                                  cp0.data(), inv0.data()});
  // d theta0 / dz (tendency.py:1013-1016)
  const double* t0 = comp->theta0;
  std::vector<double> dth0(nz);
  for (int k = 1; k < nz - 1; ++k) dth0[k] = (t0[k + 1] - t0[k - 1]) / (2.0 * dz);
  dth0[0] = (t0[1] - t0[0]) / dz;
  dth0[nz - 1] = (t0[nz - 1] - t0[nz - 2]) / dz;

  std::vector<double> kx = wavenumbers(nx, grid->Lx), ky = wavenumbers(ny, grid->Ly);
  int rc;
  if ((rc = upload(p, &p->kx, kx.data(), nx))) return bail(rc);
  if ((rc = upload(p, &p->ky, ky.data(), ny))) return bail(rc);
  if ((rc = upload(p, &p->rho, rf, nz))) return bail(rc);
  if ((rc = upload(p, &p->rhoh, rh.data(), nz + 1))) return bail(rc);
  if ((rc = upload(p, &p->theta0, t0, nz))) return bail(rc);
  if ((rc = upload(p, &p->dth0, dth0.data(), nz))) return bail(rc);
  if ((rc = upload(p, &p->ta, a.data(), nz))) return bail(rc);
  if ((rc = upload(p, &p->tc, c.data(), nz))) return bail(rc);
  if ((rc = upload(p, &p->tnegs, negs.data(), nz))) return bail(rc);
  if ((rc = upload(p, &p->ta0, a0.data(), n0))) return bail(rc);
  if ((rc = upload(p, &p->tcp0, cp0.data(), n0))) return bail(rc);
  if ((rc = upload(p, &p->tinv0, inv0.data(), n0))) return bail(rc);
  if (p->coriolis == OB_COR_BETA)
    if ((rc = upload(p, &p->fy, comp->f_y, ny))) return bail(rc);
  if (p->heating) {
    if ((rc = upload(p, &p->heat_r, comp->heat_r, (size_t)nx * ny))) return bail(rc);
    if ((rc = upload(p, &p->heat_z, comp->heat_z, nz))) return bail(rc);
  }
  if (p->drag && (rc = upload(p, &p->drag_w, comp->drag_weight, nz))) return bail(rc);
  if (p->sponge && ((rc = upload(p, &p->sp_a, comp->sponge_alpha, nz)) ||
                    (rc = upload(p, &p->sp_ah, comp->sponge_alpha_h, nz + 1))))
    return bail(rc);
  if (p->prec == OB_PREC_F64) {
    auto tx = twiddles<double>(nx), ty = twiddles<double>(ny);
    if ((rc = dalloc(p, &p->twx, nx * sizeof(cplx<double>)))) return bail(rc);
    if ((rc = dalloc(p, &p->twy, ny * sizeof(cplx<double>)))) return bail(rc);
    if (cudaMemcpyAsync(p->twx, tx.data(), nx * sizeof(cplx<double>), cudaMemcpyHostToDevice,
                        p->astream) ||
        cudaMemcpyAsync(p->twy, ty.data(), ny * sizeof(cplx<double>), cudaMemcpyHostToDevice,
                        p->astream))
      return bail(fail(OB_ERR_CUDA, "twiddle upload failed"));
    if ((rc = set_smem_attrs_once<double>())) return bail(rc);
  } else {
    auto tx = twiddles<float>(nx), ty = twiddles<float>(ny);
    if ((rc = dalloc(p, &p->twx, nx * sizeof(cplx<float>)))) return bail(rc);
    if ((rc = dalloc(p, &p->twy, ny * sizeof(cplx<float>)))) return bail(rc);
    if (cudaMemcpyAsync(p->twx, tx.data(), nx * sizeof(cplx<float>), cudaMemcpyHostToDevice,
                        p->astream) ||
        cudaMemcpyAsync(p->twy, ty.data(), ny * sizeof(cplx<float>), cudaMemcpyHostToDevice,
                        p->astream))
      return bail(fail(OB_ERR_CUDA, "twiddle upload failed"));
    if ((rc = set_smem_attrs_once<float>())) return bail(rc);
  }

  // chunk sizes: largest z-chunk whose shared-memory footprint allows two CTAs/SM
  const size_t ce = 2 * p->esz;  // complex element
  p->zc_fx = pick_zc(nz, 2ull * (p->g.M + 1) * 3 * ce, tw_bytes(p, nx));
  p->zc_fy = pick_zc(nz, 2ull * ny * 2 * ce, tw_bytes(p, ny));
  p->zc_iy = p->zc_fy;
  p->zc_ix = pick_zc(nz, (size_t)(2 * p->g.M + 1) * 3 * ce,
                     tw_bytes(p, nx) + (size_t)(2 * p->g.M + 1) * ce);
  if (smem_fx(p, 3) > kSmemMax || smem_fy(p, 2, p->zc_fy) > kSmemMax ||
      smem_ix(p, 3 * p->zc_ix + 1) > kSmemMax || smem_thomas(p) > kSmemMax)
    return bail(fail(OB_ERR_ARG, "grid (%d, %d, %d) exceeds shared-memory tiling limits", nx,
                     ny, nz));
  // compile-time-chunk x-pencil kernels where their tiles fit
  p->py8_ok = factorize8(ny, p->py8);
  p->px8_ok = factorize8(nx / 2, p->px8);
  if (p->py8_ok) {
    p->zc2_fy = p->prec == OB_PREC_F64 ? pick_y2_zc<double>(ny, nz) : pick_y2_zc<float>(ny, nz);
    p->zc2_iy = p->zc2_fy;
  }
  if (p->prec == OB_PREC_F32 && ny == kY4N) {
    p->zc4_fy = p->zc4_iy = nz >= 4 ? 4 : 2;
    p->zc4_fyd = 2;
  }
  if (slow_xt_grid(p, 4)) p->slow_xw = 4;
  if (p->prec == OB_PREC_F32 && ny == kYrN) {
    p->zc3_fy = nz >= 4 ? 4 : 2;
    p->zc3_fyd = p->zc3_fy ? 2 : 0;
  }
  if (p->px8_ok) {
    if (p->prec == OB_PREC_F64) {
      p->zc2_fx = pick_x2_zc<double, double>(0, nx, nz);
      p->zc2_fxs = pick_x2_zc<double, double>(1, nx, nz);
      p->zc2_ix = pick_x2_zc<double, double>(2, nx, nz);
    } else {
      p->zc2_fx = pick_x2_zc<float, float>(0, nx, nz);
      p->zc2_fxs = pick_x2_zc<float, float>(1, nx, nz);
      p->zc2_ix = pick_x2_zc<float, float>(2, nx, nz);
      if (nx == kXrN) {
        p->zc3_fx = p->zc3_fxs = p->zc3_ix = nz >= 8 ? 8 : (nz >= 4 ? 4 : 2);
        p->zc3_fxd = nz >= 4 ? 4 : 2;
      }
      if (nx == kX4N) {
        p->zc4_fxs = p->zc4_fx = p->zc4_ix = nz >= 4 ? 4 : 2;
        p->zc4_fxd = 2;
      }
    }
  }

  const size_t n = (size_t)nx * ny * nz, nw = (size_t)nx * ny * (nz + 1);
  const size_t ns = (size_t)p->g.nxh * ny * nz;
  const size_t e = p->esz;
  if ((rc = dalloc(p, &p->S1, ns * 2 * e)) || (rc = dalloc(p, &p->S2, ns * 2 * e)) ||
      (rc = dalloc(p, &p->S3, ns * 2 * e)) || (rc = dalloc(p, &p->Au, n * e)) ||
      (rc = dalloc(p, &p->Av, n * e)) || (rc = dalloc(p, &p->Aw, nw * e)) ||
      (rc = dalloc(p, &p->Ath, n * e)) || (rc = dalloc(p, &p->Aphi, n * e)) ||
      (rc = dalloc(p, &p->Su, n * e)) || (rc = dalloc(p, &p->Sv, n * e)) ||
      (rc = dalloc(p, &p->Sw, nw * e)) || (rc = dalloc(p, &p->Sphi, n * e)) ||
      (rc = dalloc(p, &p->Du, n * e)) || (rc = dalloc(p, &p->Dv, n * e)))
    return bail(rc);
  if (p->diffusion == OB_DIFF_BIHARMONIC &&
      ((rc = dalloc(p, &p->Lu, n * e)) || (rc = dalloc(p, &p->Lv, n * e))))
    return bail(rc);
  if (p->buoyancy && p->projection && (rc = dalloc(p, &p->Bh, nw * e))) return bail(rc);
  // the shared stage transforms: FP32 1024 x 1024 grids with fast stages
  if (p->buoyancy && p->projection && p->prec == OB_PREC_F32 && nx == kX4N && ny == kY4N &&
      p->px8_ok &&
      ((rc = dalloc(p, &p->S4, ns * 2 * e)) || (rc = dalloc(p, &p->S5, ns * 2 * e)) ||
       (rc = dalloc(p, &p->S6, ns * 2 * e))))
    return bail(rc);
  if (p->prec == OB_PREC_F32) {
    const long ncols = (long)p->g.nxh * ny;
    const long nblk = (ncols + kThomasCols - 1) / kThomasCols;
    std::vector<unsigned char> flag(nblk, 0);
    std::vector<int> lw;
    const double Lz = grid->Lz;
    for (long col = 0; col < ncols; ++col) {
      const int ix = (int)(col / ny), iy = (int)(col - (long)ix * ny);
      if ((kx[ix] * kx[ix] + ky[iy] * ky[iy]) * (Lz * Lz) < 1.0) flag[col / kThomasCols] = 1;
    }
    for (long b = 0; b < nblk; ++b)
      if (flag[b]) lw.push_back((int)b);
    p->n_lw = (int)lw.size();  // >= 1: the zero mode's block
    if ((rc = dalloc(p, &p->lw_flag, nblk)) || (rc = dalloc(p, &p->lw_blocks, lw.size() * sizeof(int))))
      return bail(rc);
    OB_CUDA(cudaMemcpyAsync(p->lw_flag, flag.data(), nblk, cudaMemcpyHostToDevice, p->astream));
    OB_CUDA(cudaMemcpyAsync(p->lw_blocks, lw.data(), lw.size() * sizeof(int),
                            cudaMemcpyHostToDevice, p->astream));
    std::vector<float> coef(4 * (size_t)nz);
    for (int k = 0; k < nz; ++k) {
      coef[4 * k + 0] = (float)negs[k];
      coef[4 * k + 1] = (float)rf[k];
      coef[4 * k + 2] = (float)a[k];
      coef[4 * k + 3] = (float)c[k];
    }
    if ((rc = dalloc(p, &p->tcoef, coef.size() * sizeof(float)))) return bail(rc);
    OB_CUDA(cudaMemcpyAsync(p->tcoef, coef.data(), coef.size() * sizeof(float),
                            cudaMemcpyHostToDevice, p->astream));
    std::vector<float> gth(nz);
    for (int k = 0; k < nz; ++k) gth[k] = (float)(kGravity / comp->theta0[k]);
    if ((rc = dalloc(p, &p->gth, gth.size() * sizeof(float)))) return bail(rc);
    OB_CUDA(cudaMemcpyAsync(p->gth, gth.data(), gth.size() * sizeof(float),
                            cudaMemcpyHostToDevice, p->astream));
    // the vectors must outlive the copies: pageable copies are staged before
    // the call returns
  }
  if ((rc = dalloc(p, &p->diag, 64 * sizeof(double)))) return bail(rc);
  // ordered after the allocation on the set-up stream
  OB_CUDA(cudaMemsetAsync(p->diag, 0, 64 * sizeof(double), p->astream));
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  p->nparts = nsm * 4;
  if ((rc = dalloc(p, &p->parts, p->nparts * sizeof(DiagPart)))) return bail(rc);
  if (p->prec == OB_PREC_F32 && (rc = make_refiner(p))) return bail(rc);
  // allocations and table copies complete: the memory is usable on any stream
  if (cudaStreamSynchronize(p->astream) != cudaSuccess)
    return bail(fail(OB_ERR_CUDA, "plan_create: set-up stream failed"));
  *out = p;
  return OB_OK;
}

#define DISPATCH(P, CALL_F64, CALL_F32) ((P)->prec == OB_PREC_F64 ? (CALL_F64) : (CALL_F32))

int oracle_b200_step(OraclePlan* p, const OracleStatePtrs* in, const OracleStatePtrs* out,
                     double dt, int want_diag, void* stream) {
  if (int rc = check_plan(p)) return rc;
  if (!in || !out || !in->u || !in->v || !in->w || !in->theta_prime || !in->phi || !out->u ||
      !out->v || !out->w || !out->theta_prime || !out->phi)
    return fail(OB_ERR_ARG, "step: NULL state pointer");
  if (!std::isfinite(dt)) return fail(OB_ERR_ARG, "step: dt must be finite");
  cudaStream_t st = (cudaStream_t)stream;
  return DISPATCH(p, step_impl<double>(p, in, out, dt, want_diag, st),
                  step_impl<float>(p, in, out, dt, want_diag, st));
}

struct OracleStepGraph {
  OraclePlan* plan = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  long kernels = 0;  // kernel launches recorded in the graph
};

int oracle_b200_step_graph_create(OraclePlan* p, const OracleStatePtrs* state, double dt,
                                  int nsteps, OracleStepGraph** out) {
  if (int rc = check_plan(p)) return rc;
  if (!out) return fail(OB_ERR_ARG, "step_graph_create: out is NULL");
  *out = nullptr;
  if (!state || !state->u || !state->v || !state->w || !state->theta_prime || !state->phi)
    return fail(OB_ERR_ARG, "step_graph_create: NULL state pointer");
  if (!std::isfinite(dt)) return fail(OB_ERR_ARG, "step_graph_create: dt must be finite");
  if (nsteps < 1 || nsteps > 4096)
    return fail(OB_ERR_ARG, "step_graph_create: need 1 <= nsteps <= 4096");
  if (p->profiling) return fail(OB_ERR_ARG, "step_graph_create: switch profiling off first");
  // record on a private stream: nothing executes while capturing, and the
  // graph can then be launched on any stream
  cudaStream_t cs = nullptr;
  OB_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) {
    cudaStreamDestroy(cs);
    return fail(OB_ERR_CUDA, "step_graph_create: begin capture failed: %s", cudaGetErrorString(e));
  }
  const long l0 = p->launches;
  p->capturing = 1;
  int rc = OB_OK;
  // the last step of the graph also runs the diagnostics reductions, so the
  // plan's blow-up flag is updated once per graph launch
  for (int s = 0; s < nsteps && rc == OB_OK; ++s) {
    const int dg = s == nsteps - 1;
    rc = DISPATCH(p, step_impl<double>(p, state, state, dt, dg, cs),
                  step_impl<float>(p, state, state, dt, dg, cs));
  }
  p->capturing = 0;
  cudaGraph_t graph = nullptr;
  e = cudaStreamEndCapture(cs, &graph);
  cudaStreamDestroy(cs);
  if (rc != OB_OK || e != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    return rc != OB_OK ? rc
                       : fail(OB_ERR_CUDA, "step_graph_create: capture failed: %s",
                              cudaGetErrorString(e));
  }
  cudaGraphExec_t exec = nullptr;
  e = cudaGraphInstantiate(&exec, graph, 0);
  if (e != cudaSuccess) {
    cudaGraphDestroy(graph);
    return fail(OB_ERR_CUDA, "step_graph_create: instantiate failed: %s", cudaGetErrorString(e));
  }
  OracleStepGraph* gr = new OracleStepGraph();
  gr->plan = p;
  gr->graph = graph;
  gr->exec = exec;
  gr->kernels = p->launches - l0;
  p->launches = l0;  // counted when the graph is launched
  *out = gr;
  return OB_OK;
}

int oracle_b200_step_graph_launch(OracleStepGraph* g, void* stream) {
  if (!g) return fail(OB_ERR_ARG, "step_graph_launch: graph is NULL");
  OB_CUDA(cudaGraphLaunch(g->exec, (cudaStream_t)stream));
  g->plan->launches += g->kernels;
  return OB_OK;
}

long oracle_b200_step_graph_kernels(const OracleStepGraph* g) { return g ? g->kernels : -1; }

int oracle_b200_step_graph_destroy(OracleStepGraph* g) {
  if (!g) return OB_OK;
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  delete g;
  return OB_OK;
}

int oracle_b200_project(OraclePlan* p, void* u, void* v, void* w, void* phi, int log_diag,
                        void* stream) {
  if (int rc = check_plan(p)) return rc;
  if (!u || !v || !w || !phi) return fail(OB_ERR_ARG, "project: NULL pointer");
  cudaStream_t st = (cudaStream_t)stream;
  const int de = p->diag_every;
  if (log_diag) p->diag_every = 1;
  int rc = DISPATCH(p,
                    project_impl<double>(p, (double*)u, (double*)v, (double*)w, nullptr, -1.0,
                                         (double*)u, (double*)v, (double*)w, (double*)phi,
                                         OB_DIAG_LAST_COMPAT, OB_DIAG_LAST_DISC, st),
                    project_impl<float>(p, (float*)u, (float*)v, (float*)w, nullptr, -1.0,
                                        (float*)u, (float*)v, (float*)w, (float*)phi,
                                        OB_DIAG_LAST_COMPAT, OB_DIAG_LAST_DISC, st));
  p->diag_every = de;
  return rc;
}

int oracle_b200_divergence(OraclePlan* p, const void* u, const void* v, const void* w, void* d,
                           void* stream) {
  if (int rc = check_plan(p)) return rc;
  if (!u || !v || !w || !d) return fail(OB_ERR_ARG, "divergence: NULL pointer");
  cudaStream_t st = (cudaStream_t)stream;
  return DISPATCH(p,
                  divergence_impl<double>(p, (const double*)u, (const double*)v,
                                          (const double*)w, (double*)d, st),
                  divergence_impl<float>(p, (const float*)u, (const float*)v, (const float*)w,
                                         (float*)d, st));
}

int oracle_b200_phi_gradient(OraclePlan* p, const void* phi, void* gx, void* gy, void* gz,
                             void* stream) {
  if (int rc = check_plan(p)) return rc;
  if (!phi || !gx || !gy || !gz) return fail(OB_ERR_ARG, "phi_gradient: NULL pointer");
  cudaStream_t st = (cudaStream_t)stream;
  return DISPATCH(p,
                  gradient_impl<double>(p, (const double*)phi, (double*)gx, (double*)gy,
                                        (double*)gz, st),
                  gradient_impl<float>(p, (const float*)phi, (float*)gx, (float*)gy,
                                       (float*)gz, st));
}

int oracle_b200_poisson_solve(OraclePlan* p, const void* d, void* phi, int log_diag,
                              void* stream) {
  if (int rc = check_plan(p)) return rc;
  if (!d || !phi) return fail(OB_ERR_ARG, "poisson_solve: NULL pointer");
  cudaStream_t st = (cudaStream_t)stream;
  return DISPATCH(p, solve_impl<double>(p, (const double*)d, (double*)phi, log_diag, st),
                  solve_impl<float>(p, (const float*)d, (float*)phi, log_diag, st));
}

int oracle_b200_apply_operator(OraclePlan* p, const void* phi, void* out, void* stream) {
  if (int rc = check_plan(p)) return rc;
  if (!phi || !out) return fail(OB_ERR_ARG, "apply_operator: NULL pointer");
  cudaStream_t st = (cudaStream_t)stream;
  return DISPATCH(p, apply_op_impl<double>(p, (const double*)phi, (double*)out, st),
                  apply_op_impl<float>(p, (const float*)phi, (float*)out, st));
}

int oracle_b200_buoyancy(OraclePlan* p, const void* th, void* dw, void* stream) {
  if (int rc = check_plan(p)) return rc;
  if (!th || !dw) return fail(OB_ERR_ARG, "buoyancy: NULL pointer");
  cudaStream_t st = (cudaStream_t)stream;
  return DISPATCH(p, buoyancy_impl<double>(p, (const double*)th, (double*)dw, st),
                  buoyancy_impl<float>(p, (const float*)th, (float*)dw, st));
}

int oracle_b200_tendency(OraclePlan* p, int mask, const OracleStatePtrs* s, void* du, void* dv,
                         void* dw, void* dth, double dt_slow, void* stream) {
  if (int rc = check_plan(p)) return rc;
  if (!s || !s->u || !s->v || !s->w || !s->theta_prime || !du || !dv || !dw || !dth)
    return fail(OB_ERR_ARG, "tendency: NULL pointer");
  if ((mask & OB_TEND_DAMPING) && p->damping && !(dt_slow != 0.0))
    return fail(OB_ERR_ARG, "tendency: damping needs a non-zero dt_slow");
  cudaStream_t st = (cudaStream_t)stream;
  return DISPATCH(p,
                  tendency_impl<double>(p, mask, s, (double*)du, (double*)dv, (double*)dw,
                                        (double*)dth, dt_slow, st),
                  tendency_impl<float>(p, mask, s, (float*)du, (float*)dv, (float*)dw,
                                       (float*)dth, dt_slow, st));
}

int oracle_b200_intensity_cap(const void* u, const void* v, int precision, long n,
                              double v_cap, double tau, double u_env, double v_env, void* du,
                              void* dv, void* stream) {
  if (!u || !v || !du || !dv) return fail(OB_ERR_ARG, "intensity_cap: NULL pointer");
  if (n < 0) return fail(OB_ERR_ARG, "intensity_cap: negative size");
  if (!(tau > 0)) return fail(OB_ERR_ARG, "intensity_cap: tau must be positive");
  if (n == 0) return OB_OK;
  cudaStream_t st = (cudaStream_t)stream;
  const unsigned nb = (unsigned)std::min<long>((n + 255) / 256, 148L * 32);
  if (precision == OB_PREC_F64)
    k_intensity_cap<double><<<nb, 256, 0, st>>>((const double*)u, (const double*)v, n, v_cap,
                                                tau, u_env, v_env, (double*)du, (double*)dv);
  else if (precision == OB_PREC_F32)
    k_intensity_cap<float><<<nb, 256, 0, st>>>((const float*)u, (const float*)v, n, v_cap, tau,
                                               u_env, v_env, (float*)du, (float*)dv);
  else
    return fail(OB_ERR_ARG, "intensity_cap: unknown precision %d", precision);
  OB_CUDA(cudaGetLastError());
  return OB_OK;
}

long oracle_b200_launch_count(const OraclePlan* p) { return p ? p->launches : -1; }

int oracle_b200_set_refinement(OraclePlan* p, int passes, int every) {
  if (int rc = check_plan(p)) return rc;
  if (passes < 0 || passes > 4 || every < 1)
    return fail(OB_ERR_ARG, "set_refinement: need 0 <= passes <= 4 and every >= 1");
  if (passes > 0 && p->prec != OB_PREC_F32)
    return fail(OB_ERR_ARG, "set_refinement: defect correction applies to single-precision plans");
  p->refine_passes = passes;
  p->refine_every = every;
  return OB_OK;
}

int oracle_b200_refine(OraclePlan* p, void* u, void* v, void* w, void* phi, void* stream) {
  if (int rc = check_plan(p)) return rc;
  if (!u || !v || !w || !phi) return fail(OB_ERR_ARG, "refine: NULL pointer");
  if (p->prec != OB_PREC_F32)
    return fail(OB_ERR_ARG, "refine: defect correction applies to single-precision plans");
  return refine_impl(p, (float*)u, (float*)v, (float*)w, (float*)phi, (cudaStream_t)stream);
}

int oracle_b200_profile(OraclePlan* p, int enable) {
  if (int rc = check_plan(p)) return rc;
  // the previous marks' events may still be pending on the GPU
  for (auto& m : p->marks) OB_CUDA(cudaEventSynchronize(m.b));
  p->marks.clear();
  p->ev_next = 0;
  // events for a few hundred steps' launches, created before any timing
  constexpr size_t kPoolUpFront = 16384;
  while (enable && p->ev_pool.size() < kPoolUpFront) {
    cudaEvent_t e = nullptr;
    OB_CUDA(cudaEventCreate(&e));
    p->ev_pool.push_back(e);
  }
  p->profiling = enable ? 1 : 0;
  return OB_OK;
}

int oracle_b200_profile_read(OraclePlan* p, double* ms, long* counts, int ncls) {
  if (int rc = check_plan(p)) return rc;
  if (!ms || !counts || ncls < OB_PROF_CLASSES) return fail(OB_ERR_ARG, "profile_read: bad buffers");
  for (int c = 0; c < ncls; ++c) {
    ms[c] = 0.0;
    counts[c] = 0;
  }
  for (auto& m : p->marks) {
    OB_CUDA(cudaEventSynchronize(m.b));
    float t = 0.f;
    OB_CUDA(cudaEventElapsedTime(&t, m.a, m.b));
    ms[m.cls] += t;
    counts[m.cls] += 1;
  }
  return OB_OK;
}

int oracle_b200_read_diag(OraclePlan* p, double* host_out, int n, void* stream) {
  if (int rc = check_plan(p)) return rc;
  if (!host_out || n < 0) return fail(OB_ERR_ARG, "read_diag: bad output");
  if (n > OB_DIAG_COUNT) n = OB_DIAG_COUNT;
  cudaStream_t st = (cudaStream_t)stream;
  double buf[OB_DIAG_COUNT];
  OB_CUDA(cudaMemcpyAsync(buf, p->diag, sizeof buf, cudaMemcpyDeviceToHost, st));
  OB_CUDA(cudaStreamSynchronize(st));
  // discrete residual slots hold sum(w |r^|^2); rms = sqrt(sum / ((nx ny)^2 nz))
  const double nxy = (double)p->g.nx * p->g.ny;
  const double norm = nxy * nxy * p->g.nz;
  for (int s : {OB_DIAG_DISC0, OB_DIAG_DISC0 + 1, OB_DIAG_DISC0 + 2, OB_DIAG_LAST_DISC})
    buf[s] = std::sqrt(std::fmax(buf[s], 0.0) / norm);
  std::memcpy(host_out, buf, n * sizeof(double));
  if (buf[OB_DIAG_STALL] != 0.0)
    return fail(OB_ERR_CUDA, "a kernel's bounded wait for its staged copies ran out: the "
                "results of the steps since are incomplete");
  if (buf[OB_DIAG_BLOWUP] >= 2.0)
    return fail(OB_ERR_NONFINITE, "blow-up: max|u| exceeded %g m/s in a diagnosed step",
                p->blowup_u);
  if (buf[OB_DIAG_BLOWUP] >= 1.0)
    return fail(OB_ERR_NONFINITE, "blow-up: a diagnosed state held a non-finite value");
  return OB_OK;
}

int oracle_b200_read_diag_async(OraclePlan* p, double* host_out, int n, void* stream) {
  if (int rc = check_plan(p)) return rc;
  if (!host_out || n < 0) return fail(OB_ERR_ARG, "read_diag_async: bad output");
  if (n > OB_DIAG_COUNT) n = OB_DIAG_COUNT;
  OB_CUDA(cudaMemcpyAsync(host_out, p->diag, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost,
                          (cudaStream_t)stream));
  return OB_OK;
}

int oracle_b200_plan_get_variants(const OraclePlan* p, int* out, int n) {
  if (int rc = check_plan(p)) return rc;
  if (!out || n < 0) return fail(OB_ERR_ARG, "plan_get_variants: bad output");
  OraclePlan* q = const_cast<OraclePlan*>(p);
  for (int i = 0; i < n && i < OB_VAR_COUNT; ++i) {
    const int* f = var_field(q, i);
    out[i] = f ? *f : 0;
  }
  return OB_OK;
}

int oracle_b200_plan_set_variants(OraclePlan* p, const int* in, int n) {
  if (int rc = check_plan(p)) return rc;
  if (!in || n < 0 || n > OB_VAR_COUNT) return fail(OB_ERR_ARG, "plan_set_variants: bad input");
  for (int i = 0; i < n; ++i)
    if (!var_allowed(p, i, in[i]))
      return fail(OB_ERR_ARG, "plan_set_variants: variant %d cannot be %d on this plan", i, in[i]);
  for (int i = 0; i < n; ++i)
    if (int* f = var_field(p, i)) *f = in[i];
  return OB_OK;
}

int oracle_b200_plan_tune(OraclePlan* p, int flags, void* stream) {
  if (int rc = check_plan(p)) return rc;
  if (flags & ~OB_TUNE_FORCE) return fail(OB_ERR_ARG, "plan_tune: unknown flags %d", flags);
  if (p->capturing) return fail(OB_ERR_ARG, "plan_tune: not while a step graph is recorded");
  const bool prof = p->profiling;
  if (prof) return fail(OB_ERR_ARG, "plan_tune: switch profiling off first");
  std::lock_guard<std::mutex> lk(g_tune_mu);
  tune_cache_load();
  const std::string key = tune_key(p);
  auto it = g_tune.find(key);
  if (it != g_tune.end() && !(flags & OB_TUNE_FORCE)) {
    bool ok = true;
    for (int i = 0; i < OB_VAR_COUNT; ++i) ok = ok && var_allowed(p, i, it->second[i]);
    if (ok) {
      for (int i = 0; i < OB_VAR_COUNT; ++i)
        if (int* f = var_field(p, i)) *f = it->second[i];
      return OB_OK;
    }
  }
  // run after the caller's queued work, on the plan's private stream
  OB_CUDA(cudaEventRecord(p->ev_fork, (cudaStream_t)stream));
  OB_CUDA(cudaStreamWaitEvent(p->astream, p->ev_fork, 0));
  const long l0 = p->launches;
  const int rc = DISPATCH(p, tune_impl<double>(p, p->astream), tune_impl<float>(p, p->astream));
  p->launches = l0;
  if (rc) return rc;
  std::vector<int> vals(OB_VAR_COUNT);
  for (int i = 0; i < OB_VAR_COUNT; ++i) {
    const int* f = var_field(p, i);
    vals[i] = f ? *f : 0;
  }
  tune_cache_store(key, vals);
  return OB_OK;
}

}  // extern "C"

// ===========================================================================
// Poisson solve that allocates nothing
// ===========================================================================
//
// Some callers cannot call cudaMalloc when they need a solve: a host program
// whose own allocator has already reserved the GPU's memory, code that runs
// inside a framework whose memory pool must stay the only owner of device
// memory, or a caller on a latency-critical path where cudaMalloc's implicit
// device synchronisation is not acceptable.  oracle_b200_poisson_solve_noalloc
// serves them: it performs the same FFT + Thomas solve as
// oracle_b200_poisson_solve, but every byte of working memory (spectral
// buffers, wavenumber / twiddle / Thomas tables) lives in the fixed array
// below.  The array belongs to this library's CUDA module: it is reserved on a
// device when the module is loaded there (with CUDA's lazy module loading, at
// the first call of this entry point or the first plan created on that
// device) and stays reserved until the process exits.  Hosts that hand the
// GPU's memory to their own allocator make that first call beforehand.

namespace {

constexpr size_t kNoAllocScratchBytes = 32ull << 20;  // 32 MiB per device
constexpr int kNoAllocMaxDevices = 64;
constexpr int kNoAllocMaxN = 2048;  // nx, ny limit (table sizes)
constexpr int kNoAllocMaxNz = 512;

}  // namespace

// File-scope device scratch.  In host code this name is only a host-side
// stand-in: its device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {

std::mutex g_noalloc_mu;
unsigned char* g_noalloc_dev_base[kNoAllocMaxDevices] = {};
// host staging of the tables (guarded by g_noalloc_mu)
alignas(256) unsigned char g_noalloc_host[512 * 1024];

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// Once per device, with that device current: look up the array's device
// address and raise the kernels' shared-memory limits.
int noalloc_base(unsigned char** out) {
  int dev = 0;
  OB_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoAllocMaxDevices)
    return fail(OB_ERR_ARG, "poisson_solve_noalloc: device index %d out of range", dev);
  if (!g_noalloc_dev_base[dev]) {
    void* ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || ptr == nullptr)
      return fail(OB_ERR_CUDA, "cudaGetSymbolAddress(no-alloc scratch) failed: %s",
                  cudaGetErrorString(e));
    int rc = set_smem_attrs<double>();
    if (rc) return rc;
    rc = set_smem_attrs<float>();
    if (rc) return rc;
    g_noalloc_dev_base[dev] = static_cast<unsigned char*>(ptr);
  }
  *out = g_noalloc_dev_base[dev];
  return OB_OK;
}

template <class T>
int noalloc_solve(const OracleGridDesc* grid, const double* rho0, const T* d, T* phi,
                  cudaStream_t st) {
  const int nx = grid->nx, ny = grid->ny, nz = grid->nz;
  OraclePlan p;  // stack descriptor; every pointer below aims into the fixed array
  p.prec = grid->precision;
  p.esz = sizeof(T);
  p.g.nx = nx;
  p.g.ny = ny;
  p.g.nz = nz;
  p.g.M = nx / 2;
  p.g.nxh = nx / 2 + 1;
  p.g.dx = grid->Lx / nx;
  p.g.dy = grid->Ly / ny;
  p.g.dz = grid->Lz / nz;
  if (!factorize(nx / 2, p.px) || !factorize(ny, p.py) || !factorize(nx / 2, p.pxf, false) ||
      !factorize(ny, p.pyf, false))
    return fail(OB_ERR_ARG, "nx/2=%d and ny=%d must factor into 2, 3, 5", nx / 2, ny);
  const size_t ce = 2 * sizeof(T);
  p.zc_fx = pick_zc(nz, 2ull * (p.g.M + 1) * 3 * ce, tw_bytes(&p, nx));
  p.zc_fy = pick_zc(nz, 2ull * ny * 2 * ce, tw_bytes(&p, ny));
  p.zc_iy = p.zc_fy;
  p.zc_ix = pick_zc(nz, (size_t)(2 * p.g.M + 1) * 3 * ce,
                    tw_bytes(&p, nx) + (size_t)(2 * p.g.M + 1) * ce);
  if (smem_fx(&p, 3) > kSmemMax || smem_fy(&p, 2, p.zc_fy) > kSmemMax ||
      smem_ix(&p, 3 * p.zc_ix + 1) > kSmemMax || smem_thomas(&p) > kSmemMax)
    return fail(OB_ERR_ARG, "grid (%d, %d, %d) exceeds shared-memory tiling limits", nx, ny, nz);

  // carve: [tables | twiddles | S1 | S3]
  const size_t ns = (size_t)p.g.nxh * ny * nz;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t o = off;
    off += align256(bytes);
    return o;
  };
  const size_t o_kx = take(nx * 8), o_ky = take(ny * 8), o_rho = take(nz * 8),
               o_rhoh = take((nz + 1) * 8), o_a = take(nz * 8), o_c = take(nz * 8),
               o_negs = take(nz * 8), o_a0 = take(nz * 8), o_cp0 = take(nz * 8),
               o_inv0 = take(nz * 8), o_twx = take(nx * ce), o_twy = take(ny * ce);
  const size_t table_bytes = off;
  const size_t o_s1 = take(ns * ce), o_s3 = take(ns * ce);
  if (off > kNoAllocScratchBytes)
    return fail(OB_ERR_ARG,
                "poisson_solve_noalloc: grid (%d, %d, %d) needs %zu bytes of scratch; the "
                "no-allocation entry point holds at most %zu bytes (use oracle_b200_poisson_solve)",
                nx, ny, nz, off, kNoAllocScratchBytes);
  if (table_bytes > sizeof(g_noalloc_host))
    return fail(OB_ERR_ARG, "poisson_solve_noalloc: tables exceed the host staging buffer");

  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  unsigned char* base = nullptr;
  if (int rc = noalloc_base(&base)) return rc;

  // host tables, built as oracle_b200_plan_create builds them (poisson.py:286-325)
  unsigned char* h = g_noalloc_host;
  std::memset(h, 0, table_bytes);
  double* kx = (double*)(h + o_kx);
  double* ky = (double*)(h + o_ky);
  double* rf = (double*)(h + o_rho);
  double* rh = (double*)(h + o_rhoh);
  double* a = (double*)(h + o_a);
  double* c = (double*)(h + o_c);
  double* negs = (double*)(h + o_negs);
  double* a0 = (double*)(h + o_a0);
  double* cp0 = (double*)(h + o_cp0);
  double* inv0 = (double*)(h + o_inv0);
  fill_wavenumbers(kx, nx, grid->Lx);
  fill_wavenumbers(ky, ny, grid->Ly);
  for (int k = 0; k < nz; ++k) rf[k] = rho0[k];
  fill_solver_tables(nz, p.g.dz, rf, SolverTables{rh, a, c, negs, a0, cp0, inv0});
  fill_twiddles<T>((cplx<T>*)(h + o_twx), nx);
  fill_twiddles<T>((cplx<T>*)(h + o_twy), ny);
  // pageable source: the call returns once the bytes are staged, so the host
  // buffer may be rewritten by the next call
  OB_CUDA(cudaMemcpyAsync(base, h, table_bytes, cudaMemcpyHostToDevice, st));

  p.kx = (double*)(base + o_kx);
  p.ky = (double*)(base + o_ky);
  p.rho = (double*)(base + o_rho);
  p.rhoh = (double*)(base + o_rhoh);
  p.ta = (double*)(base + o_a);
  p.tc = (double*)(base + o_c);
  p.tnegs = (double*)(base + o_negs);
  p.ta0 = (double*)(base + o_a0);
  p.tcp0 = (double*)(base + o_cp0);
  p.tinv0 = (double*)(base + o_inv0);
  p.theta0 = p.rho;  // not read by the solve kernels
  p.twx = base + o_twx;
  p.twy = base + o_twy;
  p.S1 = base + o_s1;
  p.S3 = base + o_s3;
  return solve_impl<T>(&p, d, phi, 0, st);
}

}  // namespace

extern "C" int oracle_b200_poisson_solve_noalloc(const OracleGridDesc* grid, const double* rho0,
                                                 const void* d, void* phi, void* stream) {
  if (!grid || !rho0 || !d || !phi) return fail(OB_ERR_ARG, "poisson_solve_noalloc: NULL argument");
  const int nx = grid->nx, ny = grid->ny, nz = grid->nz;
  if (nx < 4 || ny < 4 || (nx & 1) || (ny & 1) || nz < 3)
    return fail(OB_ERR_ARG, "poisson_solve_noalloc: need even nx, ny >= 4 and nz >= 3 (got %d, %d, %d)",
                nx, ny, nz);
  if (nx > kNoAllocMaxN || ny > kNoAllocMaxN || nz > kNoAllocMaxNz)
    return fail(OB_ERR_ARG, "poisson_solve_noalloc: grid (%d, %d, %d) exceeds the limits "
                "nx, ny <= %d, nz <= %d", nx, ny, nz, kNoAllocMaxN, kNoAllocMaxNz);
  if (!(grid->Lx > 0 && grid->Ly > 0 && grid->Lz > 0))
    return fail(OB_ERR_ARG, "poisson_solve_noalloc: domain lengths must be positive");
  cudaStream_t st = (cudaStream_t)stream;
  // Never inside a stream capture: the tables are copied from the shared host
  // staging buffer, and a captured copy would read that buffer when the graph
  // is replayed, after later calls may have rewritten it with another grid's
  // tables.  The check comes before anything is enqueued, so a refused call
  // leaves the caller's capture valid.
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  const cudaError_t ce = cudaStreamIsCapturing(st, &cap);
  if (ce != cudaSuccess)
    return fail(OB_ERR_CUDA, "poisson_solve_noalloc: cudaStreamIsCapturing failed: %s",
                cudaGetErrorString(ce));
  if (cap != cudaStreamCaptureStatusNone)
    return fail(OB_ERR_ARG, "poisson_solve_noalloc cannot be captured into a CUDA graph: the "
                "stream is capturing; call it outside the capture");
  if (grid->precision == OB_PREC_F64)
    return noalloc_solve<double>(grid, rho0, (const double*)d, (double*)phi, st);
  if (grid->precision == OB_PREC_F32)
    return noalloc_solve<float>(grid, rho0, (const float*)d, (float*)phi, st);
  return fail(OB_ERR_ARG, "poisson_solve_noalloc: unknown precision %d", grid->precision);
}
