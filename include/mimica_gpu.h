/*
 * mimica_gpu.h -- C ABI of the B200 (sm_100a) implementation of MIMICA's
 * dynamical-core hot path: flux-form scalar advection (WENO3-switch, PPM, MUSCL),
 * FD2/FD4 momentum advection with artificial viscosity, the Heun stage update and
 * the anelastic pressure projection (horizontal FFT, vertical tridiagonal per
 * wavenumber, inverse FFT, correction).
 *
 * Plain C types only (pointers, sizes, doubles); no CUDA or torch types cross this
 * boundary.  Every entry point returns an int status (MG_OK == 0) and never exits,
 * traps or aborts; mg_error_string() names a code.
 *
 * Array convention: the reference's own.  A 3-D field is real(8) x(1:nx,1:ny,1:nz)
 * in Fortran (column-major) order with nx = MAXX+5, ny = MAXY+5: three ghost cells
 * on the low side and two on the high side of x and y, no ghost cells in z.  Host
 * buffers passed to this library use exactly that layout, so a Fortran caller
 * passes its arrays through ISO_C_BINDING (c_loc) unchanged.
 *
 * Each entry point names the reference routine it replaces (paths relative to the
 * MIMICA source tree).
 */
#ifndef MIMICA_GPU_H
#define MIMICA_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
enum {
    MG_OK = 0,
    MG_ERR_PARAM = 1,        /* invalid or unsupported parameter */
    MG_ERR_CUDA = 2,         /* a CUDA runtime call failed */
    MG_ERR_NAN = 3,          /* non-finite value detected in a field */
    MG_ERR_PIVOT = 4,        /* zero pivot in the vertical tridiagonal solve (TRIDAG2 CODE 1/2) */
    MG_ERR_TIMEOUT = 5,      /* a bounded device-side wait gave up */
    MG_ERR_NOMEM = 6,        /* device or host allocation failed */
    MG_ERR_STATE = 7         /* call out of order (e.g. step before upload) */
};

/* ---- scheme selectors (src/TOOLS/advection.f90:603-614, advq_muscl.f90:367-380) ----
 * MG_LW is the dispatcher's `case default` (advq_lw.f90) with the module's 'MC'
 * limiter (lwlimiter, advq_lw.f90:50, is in no namelist); MG_QUICK is advq_quick.f90. */
enum { MG_WENO = 0, MG_PPM = 1, MG_MUSCL = 2, MG_LW = 3, MG_QUICK = 4 };
enum { MG_LIM_MINMOD = 0, MG_LIM_VL = 1, MG_LIM_MC = 2, MG_LIM_DEFAULT = 3 };
/* arithmetic forms */
enum {
    MG_PREC_FP64 = 0,        /* plain form: FP64 everywhere, matches the reference routines */
    MG_PREC_MIXED = 1        /* FP32 fluxes and FP32 spectra, FP64 state, tendencies, tridiagonal,
                                divergence residual; FP64-residual refinement of the Poisson solve */
};

/*
 * Run parameters: the reference's module globals for this path
 * (src/TYPES/shared_data.f90, INCLUDE/default.h).  Profile pointers are host
 * arrays of length nz, copied at mg_create.
 */
typedef struct mg_params {
    int maxx, maxy, nz;        /* interior sizes (MAXX, MAXY, MAXZ); nx = maxx+5, ny = maxy+5 */
    int nscal;                 /* density-weighted scalars advected besides density:
                                  scal[0] = es (potential temperature), then qt (if iqt >= 0),
                                  then passive scalars */
    int iqt;                   /* index of qt in scal[], or -1 (dry) */
    int scal_adv;              /* MG_WENO / MG_PPM / MG_MUSCL / MG_LW / MG_QUICK
                                  (scal_adv, sorder=2, limit=.true.) */
    int muscl_limiter;         /* MG_LIM_* (module default 'minmod') */
    int mom_ord;               /* 2 or 4 (windadv.f90:515-519); 3 is rejected */
    int lavisc;                /* artificial viscosity (lavisc) */
    int nsubp;                 /* pressure sub-iterations (nsubp >= 1) */
    int with_buoy;             /* buoyancy (with_buoy, imp_buoy=.true.) */
    int precision;             /* MG_PREC_* */
    int refine_iters;          /* mixed form: max refinement passes per pressure solve, each on the
                                  FP64 residual r = b - A dp of the Poisson system; nsubp*(1+refine_iters) <= 64 */
    double dx, dy, dz, dt0;
    double lim_tol;            /* flux-limiter tolerance of MUSCL, lw and QUICK (lim_tol) */
    double u0shift, v0shift;   /* Galilean shift of the advective velocity */
    double refine_tol;         /* mixed form: skip further refinement once max|r|*dt0 < tol [1/s]
                                  (r in the units of b = div(rho0 u)/(dt0 rho0)) */
    const double *fdz0, *dzw, *dz1w, *dz1;              /* grid metrics, define_grid.f90:179-187 */
    const double *den0, *avden0, *stab0, *pt0, *qv0;     /* base state, initial.f90:500-558 */
} mg_params;

typedef struct mg_ctx mg_ctx;

const char *mg_error_string(int code);
int mg_version(void);

/* ---- host precompute: the reference's once-per-run init routines ---- */
/* src/TOOLS/define_grid.f90:179-187 */
int mg_grid_metrics(int nz, double dz, const double *fdz, double *dzw, double *dz1w, double *dz1);
/* src/IO/initial.f90:473-558 (dry cp/cv, with_t=.false.); p0 and den0 by the hydrostatic recurrence */
int mg_base_state(int nz, double dz, double psurf, const double *fdz0, const double *dz1,
                  const double *pt0, const double *qv0,
                  double *p0, double *den0, double *avden0, double *stab0);
/* src/PRESSURE/fft_tools.f90:46-112: wv(1:maxx,1:maxy), l fastest */
int mg_get_wv(int maxx, int maxy, double dx, double dy, double *wv);

/* ---- context: device-resident fields of one domain, one CUDA stream ----
 * Replaces the reference's allocations of the shared_* modules for this path
 * (src/TOOLS/alloc.f90) and get_wv at init (src/MAIN/modelctl.f90:172-174). */
int mg_create(const mg_params *params, int device, mg_ctx **out);
int mg_destroy(mg_ctx *ctx);
/* bytes of device memory held by the context */
size_t mg_device_bytes(const mg_ctx *ctx);

/* ---- resident state (time level n, natural variables) ----
 * u, v, w: velocities; p: pressure perturbation; dens: prognostic density;
 * scal[s]: natural scalars (es = theta first).  Host pointers, reference layout.
 * Replaces the wind2/pressure2/state2 hand-over of time_step.f90:172-194,447-503. */
int mg_upload_state(mg_ctx *ctx, const double *u, const double *v, const double *w,
                    const double *p, const double *dens, const double *const *scal);
int mg_download_state(mg_ctx *ctx, double *u, double *v, double *w, double *p,
                      double *dens, double *const *scal);
/* One field at a time, for callers that cannot hold every field on the host at once
 * (the 1024 x 1024 x 256 capacity case has 2.2 GB per field).  field: MG_FIELD_U, _V,
 * _W, _P, _DENS, or MG_FIELD_SCAL + s for scal[s].  Host pointers, reference layout,
 * natural values, as mg_upload_state / mg_download_state take them.  A fresh context
 * holds a state once every field has been uploaded; afterwards an upload replaces its
 * field between steps (as the host physics' hand-over of one field would). */
enum { MG_FIELD_U = 0, MG_FIELD_V = 1, MG_FIELD_W = 2, MG_FIELD_P = 3, MG_FIELD_DENS = 4, MG_FIELD_SCAL = 5 };
int mg_upload_field(mg_ctx *ctx, int field, const double *src);
int mg_download_field(mg_ctx *ctx, int field, double *dst);
/* Device-pointer variants (pointers into device memory, same layout) */
int mg_upload_state_device(mg_ctx *ctx, const double *u, const double *v, const double *w,
                           const double *p, const double *dens, const double *const *scal);
int mg_download_state_device(mg_ctx *ctx, double *u, double *v, double *w, double *p,
                             double *dens, double *const *scal);

/* ---- integration ----
 * nsteps calls of `stepping` (src/INTEG/time_step.f90:76-334, dynamics subset):
 * two Heun stages, each = scalar advection + momentum + stage update + projection.
 * ntime0 is the reference's step counter of the first step (it sets the direction
 * order of momentum advection, windadv.f90:103,158).  maxdiv (optional) receives
 * the signed max of the post-projection divergence of the last stage
 * (pressure_solver.f90:125), p1 (optional, nz) the hydrostatic correction. */
int mg_step(mg_ctx *ctx, int nsteps, int ntime0, double *maxdiv, double *p1);
/* Same, recorded once in a CUDA graph per (nsteps parity) and replayed. */
int mg_step_graph(mg_ctx *ctx, int nsteps, int ntime0, double *maxdiv, double *p1);
/* wait for all work queued on the context's stream */
int mg_synchronize(mg_ctx *ctx);
/* most recent kernel-launch count of mg_step (kernels launched per call) */
int mg_last_launch_count(const mg_ctx *ctx);

/* ---- ensembles of independent domains (no counterpart in the reference, which runs one
 * domain per job) ----
 * The members are contexts from mg_create on one device, each with its own sizes and
 * parameters and already holding a state (mg_upload_state).  mg_ensemble_step advances
 * every member by nsteps steps: a pair of steps of all members is recorded once per step
 * parity into one CUDA graph that forks to the members' streams and joins back, so the
 * launches of small members run concurrently.  The members stay owned by the caller and
 * must outlive the ensemble; their states are read with mg_download_state. */
typedef struct mg_ens mg_ens;
int mg_ensemble_create(mg_ctx *const *members, int n, mg_ens **out);
int mg_ensemble_destroy(mg_ens *ens);
int mg_ensemble_step(mg_ens *ens, int nsteps, int ntime0);
/* device time of nsteps ensemble steps (CUDA events on the ensemble's stream) */
int mg_ensemble_time_steps(mg_ens *ens, int nsteps, int ntime0, double *ms);
/* kernels launched per ensemble step (all members) */
int mg_ensemble_launch_count(const mg_ens *ens);
/* How a step pair of all members is recorded into its CUDA graph:
 *   MG_ENS_GROUPED  each kernel of a stage is one launch over the blocks of every member
 *                   (a (member, block) work table, largest blocks first); members must
 *                   share the arithmetic form, scheme, field count and projection passes
 *                   and run without SGS (MG_ERR_PARAM otherwise, here and at the step);
 *   MG_ENS_STREAMS  each member's own launches, on its own stream, forked and joined.
 * The default is MG_ENS_GROUPED when the members allow it.  The results are identical. */
enum { MG_ENS_GROUPED = 1, MG_ENS_STREAMS = 2 };
int mg_ensemble_set_mode(mg_ens *ens, int mode);
int mg_ensemble_get_mode(const mg_ens *ens);

/* ---- timing and profiling (no counterpart in the reference, whose only timer is the
 * per-step wall clock of src/MAIN/modelctl.f90:395-397) ---- */
/* device time of nsteps steps, CUDA events recorded on the context's stream */
int mg_time_steps(mg_ctx *ctx, int nsteps, int ntime0, int use_graph, double *ms);
/* per-kernel event timing of subsequent eager steps (on != 0); resets the totals */
int mg_profile_enable(mg_ctx *ctx, int on);
/* text report, one line per kernel group: "<name> <launches> <total ms>" */
int mg_profile_report(mg_ctx *ctx, char *buf, size_t len);

/* ---- autotuner (no counterpart in the reference, whose transforms take FFTW's plans) ----
 * The projection's plan: the radix sequence of the x and of the y transforms
 * (shared-memory Stockham stages of radix 2, 3, 4, 5 or 8 whose product is maxx resp.
 * maxy) and the launch shapes of the x transforms, the y transforms and the vertical
 * tridiagonal solve; and the work split of the scalar advection (k segments per column
 * tile).  Plans differ in rounding only (FP64 projection: ~1e-15; the segments not at
 * all).
 *   mg_autotune:  times candidate plans on the context's own grid (the projection of
 *                 copies of the resident momentum, or of zeros before an upload; the
 *                 state is left unchanged), one coordinate at a time, and keeps the
 *                 fastest (a change must gain more than 1 %); reps projections per
 *                 candidate.  Step graphs recorded earlier are dropped.
 *   mg_tune_get / mg_tune_set: the plan in force; mg_tune_set rejects a plan that does
 *                 not fit the grid with MG_ERR_PARAM (and drops recorded step graphs).
 *   mg_radix_candidates: the radix sequences mg_autotune tries for a transform of length
 *                 n (host only, no device needed); returns their number (<= maxc),
 *                 sequence q in radix[16 q ..], its length in nstage[q]. */
typedef struct mg_tune {
    int x_nstage, x_radix[16];
    int y_nstage, y_radix[16];
    int x_threads;      /* threads per packed pair of rows, x transforms: a multiple of 8 in [8, 64] */
    int y_threads;      /* threads per row, y transforms: a multiple of 8 in [16, 128] */
    int tri_block;      /* threads per block, tridiagonal solve: 64, 128, 256 */
    int k1_segments;    /* scalar advection: k segments per 32 x 8 column tile (0: chosen per
                           launch from the grid by a wave model; PPM keeps whole columns) */
    int k2_segments;    /* momentum: k segments per 32 x 8 column tile (0: the wave model) */
    int candidates;     /* plans timed by mg_autotune */
    double ms_default;  /* one projection with the plan in force before mg_autotune */
    double ms_tuned;    /* one projection with the plan it chose */
    double k1_ms_default, k1_ms_tuned;   /* one stage-1 scalar-advection launch, likewise */
    double k2_ms_default, k2_ms_tuned;   /* one stage-1 momentum launch, likewise */
} mg_tune;
int mg_autotune(mg_ctx *ctx, int reps, mg_tune *result);
int mg_tune_get(mg_ctx *ctx, mg_tune *t);
int mg_tune_set(mg_ctx *ctx, const mg_tune *t);
int mg_radix_candidates(int n, int *radix, int *nstage, int maxc);

/* ---- unit-level entry points (host buffers, reference layout) ---- */
/* advection_ac (src/TOOLS/advection.f90:801-915) of one density-weighted field x with
 * the advective velocity derived from momentum (mu,mv,mw) as get_advective does
 * (funcpack.f90:65-94): xs := ((xs - Tx) - Ty) - Tz. */
int mg_advection_ac(mg_ctx *ctx, const double *x, const double *mu, const double *mv,
                    const double *mw, double *xs);
/* qnadv_uvw (src/INTEG/windadv.f90:46-79): momentum advection tendency of (mu,mv,mw)
 * with the advective velocity derived from them; positive sign convention (winda). */
int mg_qnadv_uvw(mg_ctx *ctx, int ntime, const double *mu, const double *mv, const double *mw,
                 double *au, double *av, double *aw);
/* fft_solve (src/PRESSURE/pressure_solver.f90:462-538 -> fft_interface.f90:543-666):
 * out(interior) = the unnormalised solution of the per-wavenumber vertical system
 * for right-hand side tend; mode (0,0) is returned as the reference leaves it
 * (the horizontal sum of tend per level). */
int mg_fft_solve(mg_ctx *ctx, const double *tend, double *out);
/* anelastic_pressure (src/PRESSURE/pressure_solver.f90:73-140): nsubp passes of
 * solve + correction, cal_p1, residual.  mu,mv,mw,p in/out; wold = momentum w at the
 * start of the stage. */
int mg_anelastic_pressure(mg_ctx *ctx, double *mu, double *mv, double *mw, double *p,
                          const double *wold, double *maxdiv, double *p1);

/* ---- the compressible model's acoustic sub-steps ----
 * prognostic_pressure (src/INTEG/prognostic_pressure.f90:64-259), the step the
 * compressible build (no ANELASTIC) runs in place of the projection: ntau sub-steps of
 * dtau = dt0/ntau at integrator stage im, for the dry ISENTROPIC CONSERVATIVE build
 * (es = density-weighted potential temperature, div_pressure compiled out, no
 * hydrometeors, the two-stage scheme, sponge off).  Each sub-step advects density and
 * es with the unlimited Lax-Wendroff faces (advq_lw_nolim.f90) on wind_adv, integrates
 * every scalar with its slow tendency (integ_scal), evaluates the equation of state
 * (thermodynamics.f90:74-294) and integrates the momentum with the pressure gradient,
 * the density buoyancy and the divergence damping 0.2 dtau <cs2>_k grad(div m)
 * (integ_mom).  The tendency accumulators tu..tqt, tscal (integpack's tend) are read
 * and updated.  All arrays are nx*ny*nz host arrays of the reference layout with their
 * ghost cells; the grid, dt0, den0 and the metrics are the context's.  The context's
 * scheme selects the faces (advection.f90:582-592): quick its own unlimited ones
 * (advq_quick_nolim.f90, nz >= 6, else MG_ERR_PARAM), every other scheme the
 * Lax-Wendroff ones (advq_lw_nolim.f90). */
typedef struct mg_acoustic {
    int im;                          /* integrator stage: 1 or 2 */
    int ntau;                        /* sub-steps, >= 1 */
    int cst_cp;                      /* 1: cp_a, cv_a; 0: moist-air cp, cv from qt */
    int nscal;                       /* passive scalars, 0 .. 12 */
    const double *p0;                /* base-state pressure, nz */
    const double *su, *sv, *sw;      /* winds: the step's slow momentum tendencies */
    const double *sdens, *ses, *sqt; /* pressures%dens, states%es, states%qt */
    const double *const *sscal;      /* states%scal, nscal arrays */
    const double *uadv, *vadv, *wadv;/* wind_adv */
    double *dens, *p;                /* in/out: pressure%dens, pressure%p (p is overwritten) */
    double *u, *v, *w;               /* in/out: momentum */
    double *es, *qt;                 /* in/out: density-weighted es, qt */
    double *const *scal;             /* in/out: density-weighted passive scalars */
    double *tu, *tv, *tw;            /* in/out: tendency accumulators (interior cells written) */
    double *tdens, *tes, *tqt;
    double *const *tscal;
    double *cs2;                     /* out: thermo_prop%cs2 */
} mg_acoustic;
int mg_prognostic_pressure(mg_ctx *ctx, const mg_acoustic *a);
/* the same call, then `warmup` (>= 0) untimed and `reps` (>= 1) timed calls on the
 * uploaded fields; ms = device time of one call of ntau sub-steps (CUDA events, the mean
 * over the timed calls); the fields written back are those after all calls */
int mg_time_prognostic_pressure(mg_ctx *ctx, const mg_acoustic *a, int warmup, int reps, double *ms);

/* ---- per-step checks and time-step control: checkall (src/IO/check.f90:59-95) ----
 * checkx (:341-417) of es (theta) and qt, then checkwind (:102-337, ANELASTIC: the
 * advective CFL only) on the resident level-n state, as the time loop calls it after
 * each step (modelctl.f90:369).  Locations are absolute 1-based (i, j, k) of the first
 * occurrence in the reference's loop order; the CFL location is (0, 0, 0) when every
 * CFL number is 0.  stop reports what makes the reference call stop_mimica(1): the
 * library itself never stops.  A NaN or Inf in u, v, w, es or qt returns MG_ERR_NAN
 * with nonfinite = 1 and the first such cell in nonfinite_ijk (no dt decision is made;
 * the reference has no such check). */
enum { MG_STOP_NONE = 0, MG_STOP_ES = 1, MG_STOP_QT = 2, MG_STOP_CFL = 3, MG_STOP_DT = 4 };
typedef struct mg_check_params {
    double cfl_max, cfl_min;   /* cfl_max, cfl_min (namelist defaults 0.5, 0.4) */
    double dt0_i;              /* dt0_i: the run's initial time step */
    double limit_ts;           /* limit_ts (default 20): stop when dt0 <= dt0_i/limit_ts */
    double es_min, es_max;     /* checkx bounds of es (200, 4000 K) */
    double qt_min, qt_max;     /* checkx bounds of qt (1e-15, 1); unused without qt */
    int ldtfix;                /* ldtfix: 1 keeps dt0 */
    int apply;                 /* 1: a new dt0 becomes the context's time step (mg_set_dt) */
} mg_check_params;
typedef struct mg_check_result {
    double maxcfl;             /* maxcfl */
    int cfl_ijk[3];            /* local_value of checkwind */
    int stop;                  /* MG_STOP_*: the first check that stops the reference's run */
    double dt0_old, dt0_new;   /* dt0 before and after the CFL rule */
    double es_min, es_max, qt_min, qt_max;
    int es_min_ijk[3], es_max_ijk[3], qt_min_ijk[3], qt_max_ijk[3];
    int nonfinite;             /* 1: a NaN or Inf in u, v, w, es or qt (the call returns MG_ERR_NAN) */
    int nonfinite_ijk[3];      /* its first location in the loop order above */
} mg_check_result;
int mg_checkall(mg_ctx *ctx, const mg_check_params *p, mg_check_result *r);
/* the advective time-step rule of checkwind (:193-264; no microphysics time scale):
 * host only, no context */
int mg_cfl_dt(const mg_check_params *p, double maxcfl, double dt0, double *dt0_new, int *stop);
/* change the time step dt0 of a context (recorded step graphs are re-recorded) */
int mg_set_dt(mg_ctx *ctx, double dt0);
/* Failure-path check of the bounded device waits (no counterpart in the reference, which
 * has no device code): one kernel arms an mbarrier for bytes that no copy delivers and
 * waits for it with the same bounded wait the TMA pipelines use, limited to limit_cycles
 * SM clock cycles (0 .. the library's own limit).  The wait runs out, the context's error
 * flag is raised and read back, and the call returns MG_ERR_TIMEOUT with the flag
 * cleared, so the next call on the context proceeds normally. */
int mg_selftest_wait(mg_ctx *ctx, long long limit_cycles);

/* ---- SGS turbulence diffusion (src/PHYS/subgrid.f90) ----
 * The Smagorinsky-Lilly closure of the build without TKE: calc_subgrid (cal_dij,
 * stability, calc_smago with the 'Lilly' stability correction, :87-145, :793-866,
 * :909-1001), the momentum stresses efud (:187-456) and the scalar fluxes eff0/effs/eff
 * (:459-789, grad_quick).  Scope: diff_ord = 2, nl_sgs = .false., no microphysics
 * (the dry N2 branch; ptv = theta (1 + epsm qt)), CONSERVATIVE, ISENTROPIC, periodic
 * lateral and rigid ('nnf') vertical boundaries, CHANNEL off.
 * With with_dif set, every mg_step / mg_step_graph evaluates the three once per step
 * from the level-n state (the reference's subgrid_interface before the dynamics loop
 * and efud/eff0/effs on wind2/state2/pressure2, time_step.f90:222, momentum.f90:104,
 * scalars.f90:106, tracers.f90:81-85) and adds them in both Heun stages. */
typedef struct mg_sgs_params {
    int with_dif;              /* with_dif: 0 = off (the default of a new context) */
    int anis_k;                /* anis_k: anisotropic viscosity, f_an = (sqrt(dx dy)/dz(k))**2 */
    int momsf;                 /* momsf > 0: surface momentum flux from mg_set_surface_fluxes' mflux */
    int reserved;              /* must be 0 */
    double diff;               /* diff: 0 = Smagorinsky-Lilly; otherwise constant viscosity |diff| */
    double pran;               /* pran (!= 0); < 0: diffusion damped above zdec, scalars by 1/|pran| */
    double zdec;               /* zdec [m] (> 0) */
    double zrough;             /* zrough [m], in the length scale vk (z + zrough) */
    double min_w;              /* min_w [m/s] (> 0), floor of the surface wind in the momentum flux */
    const double *qt0;         /* diff != 0: base-state qt profile (nz, host), NULL = qv0; copied */
} mg_sgs_params;
int mg_set_sgs(mg_ctx *ctx, const mg_sgs_params *sgs);
/* surface fluxes of the reference's surf%esflux, surf%qvflux, surf%mflux (host arrays
 * nx*ny, i fastest, the reference's 2-D layout; NULL = 0).  The SGS step reads them on
 * the device; call again whenever the caller's surface layer updates them. */
int mg_set_surface_fluxes(mg_ctx *ctx, const double *esflux, const double *qvflux, const double *mflux);
/* per-level factors (host, prof[q*nz + k-1], 11*nz values): q = 0 z0, 1 (C_s delta)**2,
 * 2 pran < 0 damping, 3 f_an, 4 N2 coefficient, 5 N2 denominator, 6..9 the d/dz
 * denominators of grad_wind_3d (gradients.f90:884-905) for u, v, w and w at nz-1,
 * 10 the length scale delta (length_scale, subgrid.f90:1183-1232). */
int mg_sgs_profiles(const mg_params *p, const mg_sgs_params *sgs, double *prof);
/* unit entries, host arrays in the reference layout with periodic ghosts:
 *   mg_calc_subgrid: fkv := turbu%fkv from natural u, v, w, es (theta), qt (NULL = dry)
 *   mg_efud: su, sv, sw := (s + eh) + ev (winds%u ... in efud) for dens and fkv = turbu%fkv
 *   mg_eff: ec := the eff tendency on levels 1..nz-1 (other cells unchanged);
 *           kind 1 = es (x0 = pt0), 2 = qt (x0 = qt0), 3 = a tracer (effs, x0 = 0);
 *           flux_s: eff's surface flux argument (nx*ny), NULL = 0 */
int mg_calc_subgrid(mg_ctx *ctx, const double *u, const double *v, const double *w, const double *es,
                    const double *qt, double *fkv);
int mg_efud(mg_ctx *ctx, const double *u, const double *v, const double *w, const double *dens,
            const double *fkv, double *su, double *sv, double *sw);
int mg_eff(mg_ctx *ctx, int kind, const double *dens, const double *fkv, const double *x,
           const double *flux_s, double *ec);
/* turbu%ksgs = (turbu%fkv/(C_k delta))**2 (calc_smago, subgrid.f90:860) of the viscosity of
 * the last step's level n, as savedata writes it when with_dif (restarting.f90:876-880);
 * host array nx*ny*nz.  MG_ERR_STATE before the first step with SGS diffusion on. */
int mg_download_ksgs(mg_ctx *ctx, double *ksgs);

/* ---- tangent linear and adjoint of the scalar advection operator (WENO; no counterpart
 * in the reference, whose adjoint does not exist) ----
 * The operator is the advective tendency A(x, m) = -(Tx + Ty + Tz) that mg_advection_ac
 * adds to xs, as a function of the density-weighted field x and of the momentum
 * (mu, mv, mw) that carries the face velocities.  The face Jacobians include the
 * differentiated smoothness weights and positivity limiter, along the branches the FP64
 * form takes.  Host arrays, reference layout, periodic ghosts filled by the caller.
 *   mg_advection_tl: dA = dA/dx . dx + dA/dm . dm     (interior; ghosts of dA are 0)
 *   mg_advection_ad: xbar = (dA/dx)^T Abar, mbar = (dA/dm)^T Abar (outputs overwritten;
 *                    the adjoints of the periodic ghost images are folded onto the
 *                    interior cells they copy, so ghost entries are 0) */
int mg_advection_tl(mg_ctx *ctx, const double *x, const double *mu, const double *mv, const double *mw,
                    const double *dx, const double *dmu, const double *dmv, const double *dmw, double *dA);
int mg_advection_ad(mg_ctx *ctx, const double *x, const double *mu, const double *mv, const double *mw,
                    const double *Abar, double *xbar, double *mubar, double *mvbar, double *mwbar);

/* ---- tangent linear and adjoint of qnadv_uvw (windadv.f90:46-1127; no counterpart in the
 * reference) ----  The momentum advection tendency (au, av, aw) = qnadv(m) of
 * mg_qnadv_uvw as a function of the momentum, its advective velocities m/rho0 - shift
 * included; the artificial viscosity's |u| is differentiated along its sign.
 *   mg_qnadv_tl: (dau, dav, daw) = dqnadv/dm . dm (interior); au, av, aw (may be NULL)
 *                receive the operator itself from the same per-cell form.
 *   mg_qnadv_ad: mbar = (dqnadv/dm)^T abar (overwritten; ghost adjoints folded onto the
 *                interior cells they copy, so ghost entries are 0). */
int mg_qnadv_tl(mg_ctx *ctx, int ntime, const double *mu, const double *mv, const double *mw,
                const double *dmu, const double *dmv, const double *dmw, double *au, double *av, double *aw,
                double *dau, double *dav, double *daw);
int mg_qnadv_ad(mg_ctx *ctx, int ntime, const double *mu, const double *mv, const double *mw,
                const double *aubar, const double *avbar, const double *awbar, double *mubar, double *mvbar,
                double *mwbar);

/* ---- trajectory tangent linear and adjoint (no counterpart in the reference) ----
 * The integrator step of mg_step written as the composition its linearisation follows:
 * the advection tendencies of all scalar fields (K1 unit mode), qnadv (K2 unit mode),
 * the stage assembly (pressure gradient, implicit buoyancy, Heun update) and the
 * projection, with the natural <-> stage variables at the ends of the step.  FP64
 * contexts, WENO scalars, SGS diffusion off.  State arrays: 5 + nscal host pointers in
 * the order u, v, w, p, dens, scal[0..nscal-1], reference layout.
 *   mg_traj_forward: the resident state advanced nsteps by that composition.
 *   mg_traj_tl:      dxT = (dx(T)/dx(0)) dx0 from the resident state x(0) (unchanged);
 *                    dx0 with periodic ghost cells.
 *   mg_traj_adjoint: g0 = (dx(T)/dx(0))^T lamT, the gradient of J = <lamT, x(T)> (interior
 *                    inner product) with respect to x(0); the forward sweep keeps a state
 *                    every ckpt steps and each segment is recomputed before its backward
 *                    sweep: (nsteps/ckpt + 1) checkpoints (on the device or on the host,
 *                    mg_traj_checkpoints) and ckpt + 3 states of 4 + nf fields (nf = nscal
 *                    + 1) and ~8 nf + 30 work fields, plus the segment's stage records,
 *                    2 (2 nf + 3) fields per step, when they fit in half the free device
 *                    memory and in mg_traj_record_limit (else each backward step
 *                    recomputes its stages); with the records, the last segment keeps
 *                    those of the forward sweep and is not recomputed (ckpt >= nsteps:
 *                    one forward pass in all).  Ghost entries of g0 are 0. */
int mg_traj_forward(mg_ctx *ctx, int nsteps, int ntime0);
int mg_traj_tl(mg_ctx *ctx, int nsteps, int ntime0, const double *const *dx0, double *const *dxT);
int mg_traj_adjoint(mg_ctx *ctx, int nsteps, int ntime0, int ckpt, const double *const *lamT, double *const *g0);
/* Cap on the device bytes mg_traj_adjoint may hold for a segment's stage records
 * (bytes < 0: half the free device memory, the default; 0: never keep them, so that
 * every backward step recomputes its stages). */
int mg_traj_record_limit(mg_ctx *ctx, double bytes);
/* Where mg_traj_adjoint keeps its checkpoints (the nsteps/ckpt + 1 states of 4 + nf
 * fields): MG_CKPT_DEVICE, MG_CKPT_HOST (page-locked host memory, copied in and out on
 * the context stream), or MG_CKPT_AUTO (the default: on the host when on the device they
 * would take more than a quarter of the free memory).  The gradient does not depend on
 * the choice. */
enum { MG_CKPT_AUTO = -1, MG_CKPT_DEVICE = 0, MG_CKPT_HOST = 1 };
int mg_traj_checkpoints(mg_ctx *ctx, int where);
/* Device times (ms) of nsteps of mg_traj_forward's composition (out4[0]), of the tangent
 * linear (out4[1]) and of the checkpointed adjoint, forward sweep and recomputation
 * included (out4[2]), from the resident state, which is left unchanged; out4[3] = device
 * bytes the adjoint held. */
int mg_time_traj(mg_ctx *ctx, int nsteps, int ntime0, int ckpt, double *out4);

/* Adjoint of anelastic_pressure (pressure_solver.f90:73-140: nsubp passes of solve +
 * correction, then the level-mean removal of w) as a map of the momentum and pressure;
 * the map is affine (linear in m), so its tangent linear is mg_anelastic_pressure itself.
 * In place: (mubar, mvbar, mwbar, pbar) := adjoint applied to them (interior values;
 * ghosts 0).  FP64 contexts only. */
int mg_anelastic_pressure_ad(mg_ctx *ctx, double *mubar, double *mvbar, double *mwbar, double *pbar);

/* device time (ms per call) of, on copies of the resident state: [0] the advection
 * operator, [1] its tangent linear, [2] its adjoint, [3] anelastic_pressure, [4] its
 * adjoint; averaged over reps.  FP64 contexts, WENO.  No counterpart in the reference. */
int mg_time_adjoint(mg_ctx *ctx, int reps, double *out5);

/* ---- allocation-free entry (no counterpart in the reference) ----
 * The projection residual of pressure_solver.f90:121-130 (signed max of the
 * divergence over the interior, k = 2..nz-1), computed without a context and without
 * allocating: its block partials live in a fixed 8 KiB device array of the library.
 * mu, mv, mw: device pointers to momentum in the reference layout (nx = maxx+5,
 * ny = maxy+5, nz); dz1w: device pointer (nz); maxdiv: device pointer receiving the
 * result; stream: a cudaStream_t (or NULL for the legacy default stream).
 * Limits: maxx, maxy <= 4096, 3 <= nz <= 4096 (MG_ERR_PARAM beyond).  A call outside
 * a stream capture resolves the scratch address of the current device; a call inside
 * a capture uses the address of that device's last call outside one, so make one call
 * outside any capture first (again after a cudaDeviceReset of the device).  Calls in
 * flight together on one device race on the scratch. */
int mg_maxdiv_noalloc(int maxx, int maxy, int nz, double dx, double dy, const double *dz1w,
                      const double *mu, const double *mv, const double *mw, double *maxdiv,
                      void *stream);

#ifdef __cplusplus
}
#endif
#endif
