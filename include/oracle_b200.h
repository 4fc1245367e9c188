/*
 * oracle_b200.h — C ABI of the B200 (sm_100a) LH82 anelastic dynamical-core step.
 *
 * The reference (justingwatford-dev/Oraclev8) is a Python/NumPy code whose
 * array seam is oracle_v8/backend.py; this library is the compiled engine a
 * backend shim binds with ctypes.  Every entry point below names the reference
 * function whose semantics it implements (path:line inside the reference).
 *
 * Conventions
 *  - State fields are C-order (nx, ny, nz) with z contiguous; w is
 *    (nx, ny, nz+1) with index 0 the surface and nz the lid
 *    (oracle_v8/solver/tendency.py:119-172).
 *  - Field pointers are DEVICE pointers owned by the caller (e.g. torch
 *    tensors); the library borrows them for the duration of a call and never
 *    frees them.  Their element type is double for OB_PREC_F64 plans and
 *    float for OB_PREC_F32 plans.
 *  - Plan-owned scratch (spectral buffers, stage buffers, constants) is
 *    allocated once in oracle_b200_plan_create and released by
 *    oracle_b200_plan_destroy.
 *  - All work is enqueued on the caller's stream; nothing synchronises except
 *    oracle_b200_read_diag.
 *  - Every function returns an OB_* status; oracle_b200_last_error() gives the
 *    message of the last failure on the calling thread.  The Python layer maps
 *    OB_ERR_ARG to ValueError and the others to RuntimeError, matching the
 *    reference's exception types (tendency.py:539-545, operator_config.py:126-138).
 */
#ifndef ORACLE_B200_H
#define ORACLE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OB_OK 0
#define OB_ERR_ARG 1       /* bad argument / shape contract */
#define OB_ERR_CUDA 2      /* a CUDA runtime call failed */
#define OB_ERR_NONFINITE 3 /* non-finite value detected by a device check */
#define OB_ERR_UNSUPPORTED 4

#define OB_PREC_F64 0
#define OB_PREC_F32 1

#define OB_ADV_NONE 0
#define OB_ADV_CENTERED2 1
#define OB_ADV_UPWIND5H 2

#define OB_COR_NONE 0
#define OB_COR_FPLANE 1
#define OB_COR_BETA 2

/* Slow-component selection masks for oracle_b200_tendency. */
#define OB_TEND_ADVECTION 1
#define OB_TEND_CORIOLIS 2
#define OB_TEND_DAMPING 4
#define OB_TEND_HEATING 8
#define OB_TEND_DRAG 16       /* SurfaceDragComponent */
#define OB_TEND_SPONGE 32     /* SpongeDampingComponent */
#define OB_TEND_DIFFUSION 64  /* HorizontalDiffusion / HyperDiffusionComponent */
#define OB_TEND_COOLING 128   /* NewtonianCoolingComponent */

/* horizontal diffusion kinds (OperatorConfig.horiz_diffusion) */
#define OB_DIFF_NONE 0
#define OB_DIFF_LAPLACIAN 1   /* HorizontalDiffusionComponent (tendency.py:1517-1566) */
#define OB_DIFF_BIHARMONIC 2  /* HyperDiffusionComponent (tendency.py:1569-1627) */

/* Layout of the diagnostics block read by oracle_b200_read_diag
 * (StepDiagnostics, oracle_v8/solver/integrator.py:83-132). */
#define OB_DIAG_MAX_U 0
#define OB_DIAG_MAX_V 1
#define OB_DIAG_MAX_W 2
#define OB_DIAG_MAX_TH 3
#define OB_DIAG_PHI_MIN 4      /* min of (phi_fast - mean(phi_fast)) at k=0 */
#define OB_DIAG_PHI_MAX 5
#define OB_DIAG_COMPAT0 6      /* compat residual of the 3 fast-stage solves */
#define OB_DIAG_DISC0 9        /* discrete-operator residual of the 3 stages */
#define OB_DIAG_LAST_COMPAT 12 /* last solve's compat residual */
#define OB_DIAG_LAST_DISC 13   /* last solve's discrete residual */
/* Blow-up flag, sticky over the plan's life: 1 once a diagnosed state held a
 * non-finite value, 2 once max|u| exceeded the plan's blowup_u_max (the
 * blow-up test of oracle_v8/measure_lh82_phase3.py:129-130).  The maxima in
 * slots 0-3 propagate NaN as NumPy's max does. */
#define OB_DIAG_BLOWUP 14
/* Non-zero once a kernel's bounded wait for its own staged copies ran out (it
 * then stops early and its outputs are incomplete); oracle_b200_read_diag
 * reports it as OB_ERR_CUDA.  It cannot happen with in-bounds copies. */
#define OB_DIAG_STALL 15
#define OB_DIAG_COUNT 16

/* Kernel-variant choices of a plan, in this order (oracle_b200_plan_get_variants,
 * oracle_b200_plan_set_variants, oracle_b200_plan_tune).  Each pencil entry is
 * the z-chunk (levels per CTA) of one kernel form, 0 = that form off; a class
 * runs the first form that is on, in the order register-resident 1024-point
 * (ZC4), register-resident 512-point (ZC3), compile-time-chunk Stockham (ZC2),
 * and otherwise the runtime-chunk Stockham kernels.  _FXS: the stage forward
 * x transform; _FX: the correction one; _FXD / _FYD and RZC2_*: the FP64
 * residual transforms of the defect correction. */
#define OB_VAR_ZC2_FX 0
#define OB_VAR_ZC2_FXS 1
#define OB_VAR_ZC2_IX 2
#define OB_VAR_ZC2_FY 3
#define OB_VAR_ZC2_IY 4
#define OB_VAR_ZC3_FX 5
#define OB_VAR_ZC3_FXS 6
#define OB_VAR_ZC3_IX 7
#define OB_VAR_ZC3_FXD 8
#define OB_VAR_ZC3_FY 9     /* forward and inverse y at ny = 512 */
#define OB_VAR_ZC3_FYD 10
#define OB_VAR_ZC4_FX 11
#define OB_VAR_ZC4_FXS 12
#define OB_VAR_ZC4_IX 13
#define OB_VAR_ZC4_FXD 14
#define OB_VAR_ZC4_FY 15
#define OB_VAR_ZC4_IY 16
#define OB_VAR_SLOW_XW 17   /* FP32 slow tendency: 0 gathering, 1 marching along x with rows
                               loaded per step, 4 / 8 marching over bulk-copied planes of 4 / 8
                               rows (one cell per thread), 24 / 28 the same with two cells per
                               thread (nz in {32, 48, 64, 80}, WS5 advection) */
#define OB_VAR_THOMAS_FAST 18 /* FP32 sweep with a compile-time level count (1) */
#define OB_VAR_RZC2_FX 19
#define OB_VAR_RZC2_FY 20
#define OB_VAR_ZC4_FYD 21   /* FP64 residual y at ny = 1024 (register form, 0 or 2) */
#define OB_VAR_ZC4_FXSH 22  /* FP32 1024 x 1024 plans with fast stages: the three stages'
                             * forward x transforms in one launch of the anchor state
                             * (their divergence is linear in the stage's sdt), each
                             * stage's y pencils forming its spectrum; z-chunk, 0 = off;
                             * takes effect with the 1024-point y pencils (zc4_fy) */
#define OB_VAR_COUNT 23

#define OB_TUNE_FORCE 1  /* time the candidates even when a choice is cached */

typedef struct OracleGridDesc {
    int nx, ny, nz;      /* even nx, ny; nz >= 3 */
    double Lx, Ly, Lz;   /* metres */
    int precision;       /* OB_PREC_* */
} OracleGridDesc;

/* Active components, mirroring the OperatorConfig slots
 * (oracle_v8/solver/operator_config.py:91-105).  Host arrays are copied into
 * plan-owned device memory at creation; the caller may free them afterwards. */
typedef struct OracleComponentDesc {
    int buoyancy;               /* BuoyancyComponent (tendency.py:508-552) */
    int projection;             /* AnelasticProjection (tendency.py:677-832) */
    int advection;              /* OB_ADV_*; AdvectionComponent (tendency.py:835-1068) */
    int coriolis;               /* OB_COR_*; CoriolisComponent (tendency.py:1071-1256) */
    double f0, u_env, v_env;    /* Coriolis f0 and geostrophic background */
    const double *f_y;          /* (ny) f(y) for OB_COR_BETA (tendency.py:1168-1200) */
    int damping;                /* HelmholtzDivergenceDampingComponent (tendency.py:1741-1845) */
    double epsilon;
    int heating;                /* DiabaticHeatingComponent (tendency.py:1671-1738) */
    const double *heat_r;       /* (nx*ny) Q_max * f_r(x, y) */
    const double *heat_z;       /* (nz) f_z(z) */
    const double *rho0;         /* (nz) base-state density, full levels */
    const double *theta0;       /* (nz) base-state potential temperature */
    int poisson_diag_every;     /* ORACLE_POISSON_DIAG_EVERY (tendency.py:769-774) */
    /* production slow components (operator_config.py:100-103), summed in slot
     * order after Coriolis and before the divergence damper */
    int drag;                   /* SurfaceDragComponent (tendency.py:1259-1357) */
    double drag_cd;             /* Cd */
    double drag_dz;             /* z[1] - z[0] of the base state */
    double drag_u_env, drag_v_env;
    const double *drag_weight;  /* (nz) max(0, 1 - z / H_bl) */
    int sponge;                 /* SpongeDampingComponent (tendency.py:1417-1514) */
    double sponge_u_env, sponge_v_env;
    const double *sponge_alpha;   /* (nz) damping rate on full levels */
    const double *sponge_alpha_h; /* (nz+1) on half levels */
    int diffusion;              /* OB_DIFF_* */
    double diff_nu;             /* nu_H (Laplacian) or nu4 (biharmonic) */
    double diff_dx2, diff_dy2;  /* (Lx/nx)^2, (Ly/ny)^2 */
    int cooling;                /* NewtonianCoolingComponent (tendency.py:1630-1668) */
    double cool_alpha;          /* 1 / tau */
    /* blow-up limit of max|u| in m/s for OB_DIAG_BLOWUP (0: non-finite values
     * only); no OperatorConfig slot, the reference's harnesses test it after
     * each step (measure_lh82_phase3.py:129-130) */
    double blowup_u_max;
} OracleComponentDesc;

typedef struct OracleStatePtrs {
    void *u, *v, *w, *theta_prime, *phi;
} OracleStatePtrs;

typedef struct OraclePlan OraclePlan;

/* Build a plan: validates the grid, uploads constants, builds FFT and Thomas
 * tables and allocates scratch.  Replaces the constructors of
 * VariableCoefficientPoissonSolver (poisson.py:112-137), AnelasticProjection
 * (tendency.py:700-715) and RK3Integrator (integrator.py:179-183). */
int oracle_b200_plan_create(const OracleGridDesc *grid, const OracleComponentDesc *comp,
                            OraclePlan **out);
int oracle_b200_plan_destroy(OraclePlan *plan);
/* Plans draw their device memory from a per-device pool that keeps released
 * blocks for the next plan.  plan_destroy waits for all device work first
 * (as cudaFree would); plan_release instead returns the memory in the order
 * of `stream`, without synchronising: every kernel that uses the plan must
 * have been queued on `stream` or have completed.  No reference counterpart
 * (the reference's solvers are garbage-collected Python objects). */
int oracle_b200_plan_release(OraclePlan *plan, void *stream);

/* ---- captured steps --------------------------------------------------------
 * A CUDA graph of `nsteps` consecutive in-place steps of one state: the kernel
 * sequence of oracle_b200_step (want_diag = 0) recorded once, then replayed
 * with a single launch per call, so a run's whole step costs one host call.
 * No reference counterpart (the reference steps from Python, integrator.py:
 * 189-311).  The graph holds the state pointers, dt and the plan's scratch:
 * replays of graphs of one plan must not overlap, and the plan must outlive
 * its graphs.  Solver-residual logging is off inside graphs; with a
 * refinement cadence `every` > 1, nsteps should be a multiple of it. */
typedef struct OracleStepGraph OracleStepGraph;
int oracle_b200_step_graph_create(OraclePlan *plan, const OracleStatePtrs *state, double dt,
                                  int nsteps, OracleStepGraph **out);
int oracle_b200_step_graph_launch(OracleStepGraph *graph, void *stream);
long oracle_b200_step_graph_kernels(const OracleStepGraph *graph);
int oracle_b200_step_graph_destroy(OracleStepGraph *graph);

/* Bytes of device scratch the plan holds. */
size_t oracle_b200_plan_scratch_bytes(const OraclePlan *plan);

/* One full WS-RK3 step with Strang-split slow terms: RK3Integrator.step
 * (integrator.py:189-311).  `in` and `out` may alias (in-place step).
 * want_diag != 0 computes the six StepDiagnostics reductions on the device
 * (integrator.py:287-295); read them with oracle_b200_read_diag. */
int oracle_b200_step(OraclePlan *plan, const OracleStatePtrs *in, const OracleStatePtrs *out,
                     double dt, int want_diag, void *stream);

/* AnelasticProjection.apply_projection (tendency.py:717-790), in place on
 * u, v, w; phi receives the projection potential.  log_diag != 0 records the
 * compatibility and discrete residuals of this solve. */
int oracle_b200_project(OraclePlan *plan, void *u, void *v, void *w, void *phi,
                        int log_diag, void *stream);

/* anelastic_divergence (tendency.py:393-437): d = div(rho u). */
int oracle_b200_divergence(OraclePlan *plan, const void *u, const void *v, const void *w,
                           void *d, void *stream);

/* _phi_gradient (tendency.py:440-500). gz has nz+1 levels, zero at the ends. */
int oracle_b200_phi_gradient(OraclePlan *plan, const void *phi, void *gx, void *gy, void *gz,
                             void *stream);

/* VariableCoefficientPoissonSolver.solve (poisson.py:202-277). */
int oracle_b200_poisson_solve(OraclePlan *plan, const void *d, void *phi, int log_diag,
                              void *stream);

/* VariableCoefficientPoissonSolver.apply_operator (poisson.py:139-200). */
int oracle_b200_apply_operator(OraclePlan *plan, const void *phi, void *out, void *stream);

/* BuoyancyComponent.compute_tendency (tendency.py:513-546): dw_dt, nz+1 levels. */
int oracle_b200_buoyancy(OraclePlan *plan, const void *theta_prime, void *dw_dt, void *stream);

/* Sum of the selected SLOW tendencies (OB_TEND_* mask) in OperatorConfig slot
 * order, as _apply_slow accumulates them (integrator.py:346-357).  dt_slow is
 * the dt the components receive (the damper divides by it).  Outputs that no
 * selected component writes are set to zero. */
int oracle_b200_tendency(OraclePlan *plan, int mask, const OracleStatePtrs *state,
                         void *du, void *dv, void *dw, void *dth, double dt_slow,
                         void *stream);

/* IntensityCapComponent.compute_tendency (tendency.py:1396-1403) on n cells:
 * du = -alpha (u - u_env), dv = -alpha (v - v_env), alpha = max(0, |V'| - v_cap)
 * / (tau max(|V'|, 1e-6)).  The reference's run loop adds dt times it to the
 * state after every step (run_storm.py:168-172).  precision: OB_PREC_*; the
 * outputs may alias nothing. */
int oracle_b200_intensity_cap(const void *u, const void *v, int precision, long n,
                              double v_cap, double tau, double u_env, double v_env,
                              void *du, void *dv, void *stream);

/* Enqueue a copy of the first n raw diagnostics slots (the residual slots
 * not yet normalised) into host_out on `stream`, without waiting.  No
 * counterpart in the reference: the serving loop polls the blow-up flag
 * (OB_DIAG_BLOWUP) this way while a run's later steps are already queued.
 * host_out should be page-locked memory, or the copy waits for the stream. */
int oracle_b200_read_diag_async(OraclePlan *plan, double *host_out, int n, void *stream);

/* Kernel variants (OB_VAR_*).  No counterpart in the reference, which leaves
 * its transforms to the array library: these choose among this library's
 * kernel forms for the same operations.  get: the n first choices of the plan.
 * set: validates every value against the forms the plan's grid and precision
 * allow (OB_ERR_ARG otherwise, nothing changed).  tune: for each kernel
 * class, times every allowed form on the plan's own buffers (a warm-up launch
 * and the best of three, CUDA events, after the work queued on `stream`) and
 * keeps the fastest; the choice is cached per grid, precision, component set
 * and device for the life of the process, and also in the file named by
 * ORACLE_B200_TUNE_CACHE when that variable is set.  A later plan of the same
 * key takes the cached choice without timing (unless flags has
 * OB_TUNE_FORCE).  Tuning overwrites the plan's scratch and stage buffers:
 * call it before the plan holds state.  Synchronises. */
int oracle_b200_plan_get_variants(const OraclePlan *plan, int *out, int n);
int oracle_b200_plan_set_variants(OraclePlan *plan, const int *values, int n);
int oracle_b200_plan_tune(OraclePlan *plan, int flags, void *stream);

/* Copy the OB_DIAG_COUNT diagnostics doubles to host (synchronises `stream`).
 * Returns OB_ERR_NONFINITE, with host_out filled all the same, when the plan's
 * blow-up flag (OB_DIAG_BLOWUP) is set. */
int oracle_b200_read_diag(OraclePlan *plan, double *host_out, int n, void *stream);

/* FP64 defect correction of single-precision plans (the FP32-refined
 * scheme; no counterpart in the reference, which is FP64 throughout).  After
 * the final projection of every `every`-th step, `passes` correction passes
 * run: the divergence of the stored FP32 velocity is formed in FP64, the
 * correction potential solved with the FP64 Thomas sweep, and u, v, w -=
 * grad(dphi), phi += dphi.  passes = 0 (the default) gives the plain FP32 step. */
int oracle_b200_set_refinement(OraclePlan *plan, int passes, int every);

/* One defect-correction pass on a projected FP32 state, in place. */
int oracle_b200_refine(OraclePlan *plan, void *u, void *v, void *w, void *phi, void *stream);

/* Number of kernels this plan has launched since creation (launch accounting
 * for benchmarks).  No counterpart in the reference (it launches through CuPy). */
long oracle_b200_launch_count(const OraclePlan *plan);

/* Per-kernel-class device timing for benchmarks (no counterpart in the
 * reference, whose ORACLE_PROF timers are host wall clocks,
 * integrator.py:59-69).  oracle_b200_profile(plan, 1) clears previous marks
 * and brackets every later launch with CUDA events on its stream;
 * oracle_b200_profile_read synchronises on them and returns the summed
 * milliseconds and launch counts per class, index OB_PROF_*. */
#define OB_PROF_FX 0      /* x-pencil forward FFT + divergence assembly */
#define OB_PROF_FY 1      /* y-pencil forward FFT */
#define OB_PROF_THOMAS 2  /* batched tridiagonal solve */
#define OB_PROF_IY 3      /* y-pencil inverse FFT + d/dy */
#define OB_PROF_IX 4      /* x-pencil inverse FFT + velocity correction */
#define OB_PROF_SLOW 5    /* fused slow tendency + forward Euler */
#define OB_PROF_DIAG 6    /* step diagnostics reductions */
#define OB_PROF_OTHER 7
#define OB_PROF_REFINE 8  /* defect-correction passes of single-precision plans */
#define OB_PROF_THOMAS_LW 9  /* long-wave FP64 columns of a single-precision solve: a few
                              * CTAs on the plan's side stream, concurrent with the
                              * OB_PROF_THOMAS sweep of every other column */
#define OB_PROF_CLASSES 10
int oracle_b200_profile(OraclePlan *plan, int enable);
int oracle_b200_profile_read(OraclePlan *plan, double *ms, long *counts, int nclasses);

/* ---- vortex initial state (oracle_v8/vortex_init.py) --------------------- */
/* Per-cell part of HollandVortexInit.build_state (vortex_init.py:330-370) on
 * the device, from tables the host computes once (all device pointers, FP64):
 * col: 4 * nx * ny values (r, V_t(r), sin phi, cos phi) per (x, y) column in
 * C order; S: nz wind-structure factors; rr: nr increasing radii; tab: nr x nz
 * theta' radial profiles.  Writes theta' = numpy.interp(r, rr, tab[:, k]),
 * u = -V_t S sin + u_env, v = V_t S cos + v_env and w = phi = 0 into `out`
 * (device fields of `precision`), with numpy's rounding. */
int oracle_b200_vortex_fill(int nx, int ny, int nz, int precision, const double *col,
                            const double *S, const double *rr, const double *tab, int nr,
                            double u_env, double v_env, const OracleStatePtrs *out,
                            void *stream);

/* ---- storm tracker reductions (oracle_v8/storm_tracker.py) -------------- */
/* Device half of find_storm_centre (storm_tracker.py:232-394): the theta'
 * surface-pressure proxy and its masked argmin run on the GPU; the scalar
 * decisions (parabolic refine, continuity gate, fall-backs) stay on the host. */
typedef struct OracleTracker OracleTracker;

/* Result of one theta' fix.  Indices are C-order cell indices ix * ny + iy, as
 * numpy's argmin returns them; the *_nb arrays hold the field at (ix, iy),
 * (ix-1, iy), (ix+1, iy), (ix, iy-1), (ix, iy+1) (0 outside the grid). */
typedef struct OracleTrackFix {
  double mean;             /* domain mean of p_sfc (storm_tracker.py:72) */
  double raw_min, raw_max; /* interior minimum / field maximum of the anomaly */
  long long raw_idx;       /* masked argmin of the anomaly (:191-203) */
  double raw_nb[5];
  double win_min, win_max; /* the same for the Gaussian-windowed anomaly (:76-98) */
  long long win_idx;       /* == raw_idx when there is no previous fix */
  double win_nb[5];
} OracleTrackFix;

/* z, rho0, theta0: host arrays of nz values (the base state's levels and
 * profiles, storm_tracker.py:69-71).  Replaces the per-call profile reads of
 * _theta_prime_proxy (storm_tracker.py:64-73). */
int oracle_b200_tracker_create(int nx, int ny, int nz, const double *z, const double *rho0,
                               const double *theta0, OracleTracker **out);
int oracle_b200_tracker_destroy(OracleTracker *tracker);

/* theta_prime: device (nx, ny, nz) field of `precision` (OB_PREC_*).
 * margin: cells masked at every edge.  has_last != 0 applies the window
 * exp(-r^2 / (2 r0^2)) about (last_ix, last_iy) in cells.  Blocks until
 * `out` (host) holds the result.  Replaces _theta_prime_proxy,
 * _gaussian_weight and _masked_argmin (storm_tracker.py:64-98,191-203). */
int oracle_b200_track_theta(OracleTracker *tracker, const void *theta_prime, int precision,
                            int margin, int has_last, double last_ix, double last_iy,
                            double r0_cells, OracleTrackFix *out, void *stream);

/* Column mean over the lower nz/2 levels of max(dv/dx - du/dy, 0) (periodic
 * centred differences, spacing dx on both axes) into zcol_host (nx * ny
 * doubles, C order).  Blocks until it is copied.  Replaces the field part of
 * _vorticity_centre (storm_tracker.py:115-139). */
int oracle_b200_track_vorticity(OracleTracker *tracker, const void *u, const void *v,
                                int precision, double dx, double *zcol_host, void *stream);

/* ---- vortex diagnostics read-outs (oracle_v8/diagnostics.py) ------------ */
/* Device reductions behind diagnostics.low_level_vmax, vmax_3d,
 * ventilation_flow, vorticity_center, perturbation_ke and enstrophy
 * (diagnostics.py:65-220) and the sub-cell centre refinement
 * (run_translation_test.py:115-161).  u, v: device (nx, ny, nz) fields of
 * `precision`; arithmetic in double.  levels: HOST array of nlev ascending
 * level indices (the level band).  Every call blocks until its host outputs
 * hold the result. */
typedef struct OracleVortexDiag OracleVortexDiag;

/* numpy.argmax result: value and C-order flat index. */
typedef struct OracleVdMax {
  double value;
  long long index;
} OracleVdMax;

int oracle_b200_vdiag_create(int nx, int ny, int nz, OracleVortexDiag **out);
int oracle_b200_vdiag_destroy(OracleVortexDiag *diag);

/* argmax over the listed levels of |(u - u_env, v - v_env)|; index
 * (ix * ny + iy) * nz + iz (low_level_vmax :65-98 with its band, vmax_3d
 * :101-112 with every level). */
int oracle_b200_vdiag_speed_max(OracleVortexDiag *diag, const void *u, const void *v,
                                int precision, const int *levels, int nlev, double u_env,
                                double v_env, OracleVdMax *out, void *stream);

/* Band-mean winds, their periodic centred vorticity, its argmax inside
 * r < window_m about (cx_m, cy_m) (index ix * ny + iy; 0 when the window holds
 * no cell) and the sum of zeta^2 over the plane (vorticity_center :172-191,
 * enstrophy :210-220). */
int oracle_b200_vdiag_vorticity(OracleVortexDiag *diag, const void *u, const void *v,
                                int precision, const int *levels, int nlev, double dx,
                                double dy, double cx_m, double cy_m, double window_m,
                                OracleVdMax *center, double *zeta_sq_sum, void *stream);

/* Sum over every cell of (u - u_env)^2 + (v - v_env)^2 (perturbation_ke :203-207). */
int oracle_b200_vdiag_ke(OracleVortexDiag *diag, const void *u, const void *v, int precision,
                         double u_env, double v_env, double *sum, void *stream);

/* Band-mean winds summed over the rings edges[b] <= r < edges[b+1]
 * (b < n_bins, 1 <= n_bins <= 64) and over the disk r < r_vent_m:
 * out[3 b + 0..2] = (cells, sum u, sum v), the disk at b = n_bins
 * (ventilation_flow :150-166). */
int oracle_b200_vdiag_rings(OracleVortexDiag *diag, const void *u, const void *v,
                            int precision, const int *levels, int nlev, double dx, double dy,
                            double cx_m, double cy_m, const double *edges, int n_bins,
                            double r_vent_m, double *out, void *stream);

/* The refinement's field: positive vorticity mean over levels [0, nz/2)
 * (nz/2 <= 128), spacing dx on both axes, [1,2,1] smoothed in x then y; kept
 * in the workspace for oracle_b200_vdiag_centroid. */
int oracle_b200_vdiag_zpos(OracleVortexDiag *diag, const void *u, const void *v, int precision,
                           double dx, void *stream);

/* (sum w, sum ix w, sum iy w), w = field^2, over [i0, i1) x [j0, j1) of the
 * last oracle_b200_vdiag_zpos field: one centroid iteration. */
int oracle_b200_vdiag_centroid(OracleVortexDiag *diag, int i0, int i1, int j0, int j1,
                               double *out, void *stream);

/* Poisson solve that allocates no device memory.  No counterpart in the
 * reference: it is an extra entry point for callers that cannot call
 * cudaMalloc when they need a solve (a process whose own allocator already
 * holds the GPU's memory, a framework whose pool must remain the only owner of
 * device memory, or a latency-critical caller that cannot afford cudaMalloc's
 * device synchronisation).  Same result as oracle_b200_poisson_solve on a plan
 * of the same grid and rho0 (host array, nz values), without a plan.
 *  - Working memory is one fixed 32 MiB array per device.  It needs the
 *    tables (under 0.2 MiB) plus 2 (nx/2 + 1) ny nz 2 sizeof(T) bytes for two
 *    half-spectrum buffers; grids beyond that, or with nx, ny > 2048 or
 *    nz > 512, are rejected with OB_ERR_ARG.  FP64: 192x192x32 fits (19 MB),
 *    256x256x32 does not (33.8 MB).  FP32: 256x256x48 fits (25 MB),
 *    256x256x64 does not.
 *  - The array is part of this library's CUDA module and is reserved on a
 *    device when the module loads there: under CUDA's lazy module loading, at
 *    the first call of this function or the first plan created on that
 *    device.  It stays reserved until the process exits.  A host that gives
 *    the GPU's free memory to its own allocator makes that first call before
 *    doing so; later calls allocate nothing.
 *  - The first call on each device also looks up the array's address and
 *    sets kernel attributes.
 *  - It cannot be captured into a CUDA graph: on a capturing stream it returns
 *    OB_ERR_ARG before enqueuing anything, and the capture stays valid.  The
 *    tables are copied from a shared host staging buffer, so the call returns
 *    after they are staged; the solve itself is enqueued on `stream`.
 *  - Every call shares the array and overwrites all of it that it reads, so
 *    nothing carries over between calls; calls whose GPU work overlaps (other
 *    streams, other host threads on the same device) race on it. */
int oracle_b200_poisson_solve_noalloc(const OracleGridDesc *grid, const double *rho0,
                                      const void *d, void *phi, void *stream);

const char *oracle_b200_last_error(void);
/* The ABI version of the library (no counterpart in the reference): raised
 * whenever a constant, an array length or a struct of this header changes, so
 * that bindings can refuse a library built from another header.  2: the
 * shared stage transforms (OB_VAR_ZC4_FXSH, OB_VAR_COUNT 23) and the
 * long-wave Thomas profile class (OB_PROF_THOMAS_LW, OB_PROF_CLASSES 10). */
#define OB_ABI_VERSION 2
int oracle_b200_version(void);

#ifdef __cplusplus
}
#endif
#endif /* ORACLE_B200_H */
