/*
 * mimica_oracle.h -- CPU FP64 restatement of MIMICA's dynamical-core hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path: only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it.
 * It is never the thing measured on the GPU arm and never a fallback of the
 * product library.
 *
 * Parity status: the reference (Fortran 90, CPU only) has no compiler, no FFTW and
 * no golden vectors for this path in this environment, so the Fortran routines are
 * "parity unpinned" against a reference binary; they are restated line by line
 * (each function cites the reference file:line it follows).  The FFT step is
 * pinned against the reference's own KISS FFT (src/fftmpi/src/kissfft.h) compiled
 * from its sources by oracle/build_ref.sh, and against numpy.fft.
 *
 * Array convention (identical to the reference): a 3-D field is
 * real(8) x(1:nx,1:ny,1:nz), column-major, nx = MAXX+5, ny = MAXY+5, interior
 * i in [4, nx-2], j in [4, ny-2]; C index ((k-1)*ny + (j-1))*nx + (i-1).
 * Lateral boundaries periodic (bcl(1:4) = 'per'), bottom/top rigid (bcl(5:6) = 'nnf').
 */
#ifndef MIMICA_ORACLE_H
#define MIMICA_ORACLE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { MO_WENO = 0, MO_PPM = 1, MO_MUSCL = 2, MO_LW = 3, MO_QUICK = 4 };
/* the unlimited faces of the acoustic sub-steps: Lax-Wendroff (advq_lw_nolim.f90) and
 * QUICK (advq_quick_nolim.f90) */
enum { MO_LW_NL = 16, MO_QUICK_NL = 17 };
enum { MO_LIM_MINMOD = 0, MO_LIM_VL = 1, MO_LIM_MC = 2, MO_LIM_DEFAULT = 3 };

/* SGS turbulence switches (src/TYPES/shared_data.f90, INCLUDE/default.h), the
 * Smagorinsky-Lilly build (TKE undefined), nl_sgs=.false., diff_ord=2, lmicro=0. */
typedef struct mo_sgs {
    int with_dif;                /* with_dif */
    int anis_k;                  /* anis_k */
    int momsf;                   /* momsf > 0: surface momentum flux from mflux */
    int pad;
    double diff;                 /* 0: Smagorinsky-Lilly; otherwise constant viscosity |diff| */
    double pran;                 /* Prandtl number; < 0: viscosity damped above zdec */
    double zdec, zrough, min_w;
    const double *qt0;           /* diff != 0: base-state qt profile (nz), NULL = qv0 */
    const double *esflux, *qvflux, *mflux;   /* surface fluxes (nx*ny) or NULL = 0 */
} mo_sgs;

typedef struct mo_grid {
    int nx, ny, nz;              /* full sizes incl. ghost cells */
    int scal_adv;                /* MO_WENO / MO_PPM / MO_MUSCL / MO_LW / MO_QUICK */
    int muscl_limiter;           /* MO_LIM_* (module default 'minmod') */
    int mom_ord;                 /* 2 or 4 */
    int lavisc;                  /* artificial viscosity on momentum */
    int nsubp;                   /* pressure sub-iterations */
    int with_buoy;
    double dx, dy, dz, dt0;
    double lim_tol;
    double u0shift, v0shift;
    /* 1-D profiles, length nz */
    const double *fdz0, *dzw, *dz1w, *dz1;
    const double *den0, *avden0, *stab0, *pt0, *qv0;
    /* horizontal eigenvalues wv(1:nx-5, 1:ny-5), l fastest */
    const double *wv;
    const mo_sgs *sgs;           /* SGS diffusion, or NULL (with_dif = .false.) */
} mo_grid;

/* ---- host precompute (define_grid, initial, get_wv) ---- */
void mo_grid_metrics(int nz, double dz, const double *fdz, double *dzw, double *dz1w, double *dz1);
void mo_base_state(int nz, double dz, double psurf, const double *fdz0, const double *dz1,
                   const double *pt0, const double *qv0,
                   double *p0, double *den0, double *avden0, double *stab0);
void mo_get_wv(int nxp, int nyp, double dx, double dy, double *wv);

/* ---- halo maps (bc.f90) ---- */
void mo_statebc(const mo_grid *g, double *x);

/* ---- per-pencil schemes (advq_*.f90), 1-based semantics, arrays of length n ---- */
void mo_advs_h(const mo_grid *g, int scheme, int n, int i1, int i2, double d,
               const double *x, const double *u, double *xa, int adv);
void mo_advs_z(const mo_grid *g, int scheme, const double *x, const double *w, double *xa, int adv);

/* ---- 3-D operators ---- */
/* advection_x/y/z: xs := xs - xx, with xx the tendency of one direction */
void mo_advection_dir(const mo_grid *g, int dir, const double *xtmp, const double *uadv,
                      double *xs, int adv);
/* advection of one field in all three directions: xs := ((xs - Tx) - Ty) - Tz */
void mo_advection_ac(const mo_grid *g, const double *x, const double *ua, const double *va,
                     const double *wa, double *xs, int adv);
/* get_advective: wind_adv = m/rho0 - shift over all cells */
void mo_get_advective(const mo_grid *g, const double *mu, const double *mv, const double *mw,
                      double *ua, double *va, double *wa);
/* qnadv_uvw: winda = momentum advection tendency (positive sign convention) */
void mo_qnadv_uvw(const mo_grid *g, int ntime, const double *mu, const double *mv, const double *mw,
                  const double *ua, const double *va, const double *wa,
                  double *au, double *av, double *aw);
void mo_caldiv(const mo_grid *g, double *mu, double *mv, double *mw, double *div);
void mo_gradp(const mo_grid *g, double *p, const double *w, double *gpx, double *gpy, double *gpz);
/* buoyancy (thermodynamics.f90:472-534), ANELASTIC, ISENTROPIC, nhydro=0 */
void mo_buoyancy(const mo_grid *g, const double *dens, const double *es, const double *qt, double *buoy);

/* ---- pressure ---- */
void mo_fft2d(int nxp, int nyp, double *re, double *im, int inverse);   /* unnormalised DFT */
int  mo_tridiag(const mo_grid *g, int m, int nxp, int nzp, const double *wvl,
                double *s1re, double *s1im, size_t stride_l, size_t stride_k);
int  mo_fft_solve(const mo_grid *g, const double *tend, double *out);
void mo_rescale_pressure(const mo_grid *g, double *pp);
void mo_horav(const mo_grid *g, const double *x, double *xav);
int  mo_anelastic_pressure(const mo_grid *g, double *mu, double *mv, double *mw, double *p,
                           const double *wold, double *maxdiv, double *p1);

/* ---- SGS turbulence (src/PHYS/subgrid.f90, src/TOOLS/gradients.f90) ----
 * Per-level profiles, prof[q*nz + k-1] for q = 0..MO_SGS_NPROF-1:
 * 0 z0, 1 (C_s*delta)**2, 2 damping func, 3 anisotropy f_an, 4 N2 coefficient,
 * 5 N2 denominator, 6..9 denominators of the 4th-order d/dz of u, v, w and w at
 * nz-1, 10 the length scale delta. */
#define MO_SGS_NPROF 11
void mo_sgs_profiles(const mo_grid *g, double *prof);
/* cal_dij: d[0..5] = d11, d22, d33, d12, d13, d23 (cell centred, full arrays) */
void mo_cal_dij(const mo_grid *g, const double *u, const double *v, const double *w, double *const *d);
/* calc_subgrid: turbu%fkv from natural level-n winds, es (theta) and qt (NULL = dry) */
void mo_calc_subgrid(const mo_grid *g, const double *u, const double *v, const double *w,
                     const double *es, const double *qt, double *fkv);
/* efud: su/sv/sw := (s + eh) + ev on the interior (the reference's winds%u etc.) */
void mo_efud(const mo_grid *g, const double *u, const double *v, const double *w, const double *dens,
             const double *fkv, double *su, double *sv, double *sw);
/* eff: kind 1 = es (flux -esflux, x0 = pt0), 2 = qt (-qvflux, qt0), 3 = tracer (effs: 0, 0);
 * ec := SGS tendency on the interior levels 1..nz-1 (conservative form) */
void mo_eff(const mo_grid *g, int kind, const double *dens, const double *fkv, const double *x, double *ec);

/* ---- per-step checks (src/IO/check.f90 checkwind, checkx) ---- */
void mo_checkwind(const mo_grid *g, const double *u, const double *v, const double *w, double *maxcfl, int *loc);
void mo_checkx(const mo_grid *g, const double *x, double *mn, double *mx, int *locmin, int *locmax);

/* ---- one full integrator step (time_step.f90 stepping, dynamics subset) ----
 * State at time level n, natural variables, all arrays nx*ny*nz with valid halos:
 *   u, v, w (velocities), p, dens, scal[0..nsc)  (es = theta first, then qt if
 *   with_qt, then passive scalars).  Updated in place to level n+1.
 * iqt: index of qt among scal (or -1); buoyancy uses scal[0] as es.
 */
int mo_step(const mo_grid *g, int ntime, double *u, double *v, double *w, double *p,
            double *dens, int nsc, double **scal, int iqt, double *maxdiv, double *p1);

/* ---- the compressible model's acoustic sub-steps (src/INTEG/prognostic_pressure.f90) ----
 * Dry ISENTROPIC CONSERVATIVE build: es is density-weighted potential temperature,
 * div_pressure is compiled out, nhydro = 0, sorder = 2 (Heun coefficients of stage im),
 * sponge off.  All arrays nx*ny*nz. */
typedef struct mo_acoustic {
    int im;                        /* integrator stage: a_lm, b_lm (INCLUDE/integ.h) */
    int ntau;                      /* acoustic sub-steps per dt0 */
    int cst_cp;                    /* 1: cp_a, cv_a; 0: cp, cv of moist air from qt */
    int nscal;                     /* passive scalars */
    const double *p0;              /* base-state pressure (nz) */
    const double *su, *sv, *sw;    /* winds: the step's slow momentum tendencies */
    const double *sdens, *ses, *sqt;   /* pressures%dens, states%es, states%qt */
    const double *const *sscal;    /* states%scal */
    const double *uadv, *vadv, *wadv;  /* wind_adv */
} mo_acoustic;
typedef struct mo_acoustic_state {
    double *dens, *p;              /* pressure%dens, pressure%p */
    double *u, *v, *w;             /* wind (momentum) */
    double *es, *qt;               /* state (density-weighted) */
    double **scal;
    double *tu, *tv, *tw;          /* the integrator's tendency accumulators (integpack tend) */
    double *tdens, *tes, *tqt;
    double **tscal;
    double *cs2;                   /* out: thermo_prop%cs2 */
} mo_acoustic_state;
/* returns 0, or 1 for scal_adv = quick with nz < 6 (its bottom face reads x(nz-5)) */
int mo_prognostic_pressure(const mo_grid *g, const mo_acoustic *a, const mo_acoustic_state *s);

#ifdef __cplusplus
}
#endif
#endif
