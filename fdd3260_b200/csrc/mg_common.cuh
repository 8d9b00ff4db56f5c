// mg_common.cuh -- shared definitions of the sm_100a kernels of the MIMICA
// dynamical-core path (internal; the public boundary is include/mimica_gpu.h).
//
// Device layout of a 3-D field: the reference's halo'd Fortran layout
// x(1:nx,1:ny,1:nz), nx = MAXX+5, ny = MAXY+5, with the x pitch padded to a
// multiple of 8 doubles (64 B) so that rows are 16-B aligned for TMA.
// Element (i,j,k) (1-based, as in the reference) sits at
//   ((k-1)*ny + (j-1))*px + (i-1).
// Ghost cells hold periodic images of the interior after every producer kernel
// (the reference's windbc/statebc invariant, src/TOOLS/bc.f90:81-502).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "mimica_gpu.h"
#ifndef __CUDACC_RTC__
#include <string.h>
#include <algorithm>
#include <functional>
#include <numeric>
#include <vector>
#endif

#define MG_MAXF 16   // max fields handled by one scalar-advection launch

struct DevGrid {
    int nx, ny, nz, px;   // full sizes incl. ghost cells; padded x pitch
    int maxx, maxy;       // interior sizes
    long long ps;         // plane stride = px*ny
    double dx, dy, dz, dt0, lim_tol, u0shift, v0shift;
    int scal_adv, muscl_lim, mom_ord, lavisc, with_buoy;
    const double *fdz0, *dzw, *dz1w, *dz1, *den0, *avden0, *stab0, *pt0, *qv0;  // device, nz each
    const double *rden0, *ravden0;   // 1/den0, 1/avden0 (the linearised operators multiply by them)
};

__host__ __device__ inline long long gidx(const DevGrid &g, int i, int j, int k) {
    return ((long long)(k - 1) * g.ny + (j - 1)) * (long long)g.px + (i - 1);
}

// Level-n representation of the resident state.
//   REP_NAT : buffers hold natural variables (after an upload):  value = x * w
//   REP_CONS: buffers hold density-weighted values from the previous step; the
//             reference divides by the weight at the end of a step and multiplies
//             again at the start of the next one, so value = (x / w) * w.
enum { REP_NAT = 0, REP_CONS = 1 };

// 1/x for the mixed form's kernels: the FP32 hardware reciprocal refined by two Newton
// steps r <- r (2 - x r) in FP64, which square the FP32 estimate's relative error
// (about 2^-23) twice, to within a few ulps of the quotient 1/x; for x in FP32's normal
// range (densities, reference temperatures).  The FP64 form divides.
__device__ __forceinline__ double rcp_nr(double x)
{
    const float xf = (float)x;
    float rf;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(rf) : "f"(xf));
    double r = (double)rf;
    r = r * (2. - x * r);
    r = r * (2. - x * r);
    return r;
}

__device__ __forceinline__ double rep_value(int rep, double x, double w) {
    return rep == REP_NAT ? x * w : (x / w) * w;
}

// ---- scalar advection + stage update (K1) ----
struct K1Args {
    int nf;                        // number of fields (field 0 = density when dens_first)
    int dens_first;                // field 0 is the density (unweighted, adv=.false.)
    int stage;                     // 1 or 2 (0: unit mode, inputs used as given)
    double a_dt;                   // a_lm*dt0
    double b;                      // b_lm
    const double *xin[MG_MAXF];    // stencil input (stage 1: level-n natural; stage 2: working)
    double *xold[MG_MAXF];         // level-n natural buffer (pointwise; stage 2 writes it in place)
    double *xout[MG_MAXF];         // stage 1: working buffers; stage 2: the level-n buffers
    double *tend[MG_MAXF];         // tendency accumulator (stage 1 writes, stage 2 reads)
    double *fst[MG_MAXF];          // optional: this stage's tendency (for buoyancy), or null
    const double *mw;              // momentum w (stage 1: natural w) for the vertical face velocity
    int mode;                      // 0: stage update; 1: unit mode: xout := ((xout - Tx) - Ty) - Tz
    int *err;                      // device error flag (bounded waits)
    int xold_is_xin;               // xold[f] == xin[f]: the level-n value is the plane's own cell
    // SGS tendency of field f (level-n, equal in both stages), or null.  Bit f of
    // sgs_post set: T = advection + S (es, qt: scalars.f90:146-150); clear: S is the
    // initial tendency that advection_ac then updates (tracers: tracers.f90:81-106).
    const double *sgs[MG_MAXF];
    unsigned sgs_post;
    int nseg;                      // k segments per column tile (0: launch_k1 chooses for the grid alone)
};
// TMA descriptors of the K1 inputs: haloed planes (38 x 14) of every field, momentum boxes (34 x 9)
struct alignas(64) K1Maps {
    CUtensorMap x[MG_MAXF];
    CUtensorMap mu, mv;
};

// ---- grouped launches: one launch over the blocks of several domains ----
// Work item of a grouped launch: the domain (member) and the block of that domain's own
// grid that one block of the launch runs.  The items are ordered heaviest first.
struct GItem {
    int m, b;
};
// A recorded sequence of grouped launches: the member and item tables of every launch
// in one host image (uploaded once to `dev`), and per launch a closure that issues it
// given the device image.  Recorded once, issued (captured into a graph) many times.
struct GroupProgram {
    std::vector<unsigned char> host;
    std::vector<std::function<cudaError_t(const unsigned char *dev, cudaStream_t s)>> ops;
    int launches = 0;
    template <class T> size_t put(const std::vector<T> &v)
    {
        const size_t o = (host.size() + 127) / 128 * 128;
        host.resize(o + v.size() * sizeof(T));
        if (!v.empty()) memcpy(host.data() + o, v.data(), v.size() * sizeof(T));
        return o;
    }
};
// The work items of a grouped launch: every block of every member, the members with the
// costliest blocks first (largest-first list scheduling over the GPU's CTA slots), each
// member's blocks in order.
inline std::vector<GItem> group_items(const std::vector<int> &nblk, const std::vector<double> &cost)
{
    std::vector<int> ord(nblk.size());
    std::iota(ord.begin(), ord.end(), 0);
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return cost[a] > cost[b]; });
    std::vector<GItem> it;
    for (int m : ord)
        for (int b = 0; b < nblk[m]; b++) it.push_back(GItem{m, b});
    return it;
}
// K1 arguments of one member, in global memory (the maps 64-byte aligned)
struct alignas(64) K1Member {
    K1Maps M;
    DevGrid G;
    K1Args A;
};
// ---- momentum advection + pgf + buoyancy + stage update (K2) ----
struct K2Args {
    int stage;
    int rep;                       // REP_* of level-n momentum buffers
    int ntime;                     // reference step counter (direction order)
    double a_dt, b;
    const double *mu, *mv, *mw;    // stencil momentum (stage 1: level-n buffers; stage 2: working)
    int in_is_leveln;              // stencil momentum is the level-n buffer (apply rep conversion)
    const double *mu_n, *mv_n, *mw_n;  // level-n buffers (pointwise old values)
    const double *p;               // pressure (working)
    const double *dens, *es, *qt;  // working density and density-weighted es, qt (qt may be null)
    int dens_is_leveln;            // stage 1: dens/es/qt are level-n buffers (rep conversion of es,qt)
    const double *fes, *fqt;       // this stage's tendencies of es and qt (qt may be null)
    double *ou, *ov, *ow;          // new momentum
    double *tu, *tv, *tw;          // tendency accumulators
    int mode;                      // 0: full stage; 1: unit mode: ou/ov/ow := advection tendency only
    int *err;                      // device error flag (bounded waits)
    const double *su, *sv, *sw;    // SGS momentum tendencies (efud), or null: winds starts at S
    int nseg;                      // k segments per column tile (0: launch_k2 chooses for the grid alone)
};
// TMA descriptors of the K2 stencil momentum (boxes of 38 x 12 doubles)
struct alignas(64) K2Maps {
    CUtensorMap m[3];
};

// K2 arguments of the members of one grouped launch, passed as the kernel parameter
// (64 x 440 bytes, inside the 32 KB parameter limit); more members take more launches
constexpr int K2G_MAX = 64;
struct K2GroupArgs {
    DevGrid G;
    K2Args A;
};
struct K2GroupParams {
    K2GroupArgs a[K2G_MAX];
};
// launch wrappers (implemented in the .cu files)
cudaError_t launch_k1(const DevGrid &g, const K1Args &a, const K1Maps &maps, cudaStream_t s);
cudaError_t k1_init();
cudaError_t launch_k1_mixed(const DevGrid &g, const K1Args &a, const K1Maps &maps, cudaStream_t s);
cudaError_t k1_mixed_init();
size_t k1_smem_bytes(int scheme, int nf);
// K1 over the blocks of several members: same scheme, stage (1 or 2) and field count, no SGS
cudaError_t launch_k1_group(int scheme, int stage, int nf, const K1Member *mem, const GItem *items, int nitems,
                            cudaStream_t s);
cudaError_t launch_k1_group_mixed(int scheme, int stage, int nf, const K1Member *mem, const GItem *items, int nitems,
                                  cudaStream_t s);
// TMA descriptor of one field buffer (box in doubles)
int make_field_map(const DevGrid &g, const double *base, int boxx, int boxy, CUtensorMap *map);
cudaError_t launch_k2(const DevGrid &g, const K2Args &a, const K2Maps &maps, cudaStream_t s);
cudaError_t launch_k2_mixed(const DevGrid &g, const K2Args &a, const K2Maps &maps, cudaStream_t s);
// K2 over the blocks of up to K2G_MAX members at one ntime parity (even: ntime % 2 == 0);
// maps[m]: member m's tensor maps in device memory
cudaError_t launch_k2_group(int even, const K2GroupParams &P, const K2Maps *maps, const GItem *items, int nitems,
                            cudaStream_t s);
cudaError_t launch_k2_group_mixed(int even, const K2GroupParams &P, const K2Maps *maps, const GItem *items, int nitems,
                                  cudaStream_t s);
cudaError_t launch_halo_fill(const DevGrid &g, double *const *fields, int nf, cudaStream_t s);

// ---- SGS turbulence diffusion (k_sgs.cu) ----
#define SGS_NPROF 11   // per-level factors: z0, (C_s delta)^2, func, f_an, N2 coef., N2 den., d/dz den. u, v, w, w(nz-1), delta
struct SgsDev {
    int anis_k, momsf, diff_on;
    double diff, pran, min_w;
    const double *cs2d, *func, *fan, *n2c, *n2d, *du, *dv, *dw, *dwt;   // device, nz each
};
struct SgsDij {
    double *d[6];   // d11, d22, d33, d12, d13, d23 (cell centred, periodic ghosts)
};
struct SgsVisc {
    double *fkv;   // turbu%fkv (interior), or null
    double *fe;    // dens*fkv (times func(k) when pran < 0), or null (then nut null too)
    double *nut;   // fe/|pran|, the scalar diffusivity
};
struct SgsScal {
    int nf;
    const double *x[MG_MAXF];      // natural level-n scalar
    const double *x0[MG_MAXF];     // diff != 0: base profile subtracted (pt0, qt0), or null
    const double *fs[MG_MAXF];     // surface flux (nx*ny), or null
    int fs_neg[MG_MAXF];           // flux_s = -fs (eff0 passes -surf%esflux, -surf%qvflux)
    double *out[MG_MAXF];          // SGS tendency (levels 1..nz-1 written)
};
__host__ __device__ __forceinline__ double fmax_ref(double a, double b) { return a > b ? a : b; }
cudaError_t launch_sgs_visc(const DevGrid &g, const SgsDev &s, const double *u, const double *v, const double *w,
                            const double *es, const double *qt, const double *dens, const SgsDij &d,
                            const SgsVisc &o, cudaStream_t st);
cudaError_t launch_sgs_prep(const DevGrid &g, const SgsDev &s, const double *dens, const double *fkv, double *fe,
                            double *nut, cudaStream_t st);
cudaError_t launch_sgs_mom(const DevGrid &g, const SgsDev &s, const double *u, const double *v, const double *fe,
                           const SgsDij &d, const double *mflux, const double *in_u, const double *in_v,
                           const double *in_w, double *out_u, double *out_v, double *out_w, cudaStream_t st);
cudaError_t launch_sgs_scal(const DevGrid &g, const SgsDev &s, const double *nut, const SgsScal &a, cudaStream_t st);
void sgs_host_profiles(int nz, double dx, double dy, double dz, const double *fdz0, const double *pt0,
                       const double *qv0, int anis_k, double zdec, double zrough, double *prof);

// ---- per-step checks (k_check.cu) ----
size_t check_scratch_bytes();
cudaError_t launch_check(const DevGrid &g, const double *u, const double *v, const double *w, const double *es,
                         const double *qt, void *scratch, cudaStream_t s);
// a bounded mbarrier wait that runs out after `limit` cycles and raises *err
cudaError_t launch_selftest_wait(long long limit, int *err, cudaStream_t s);

// ---- one integrator stage for the trajectory tangent linear / adjoint (k_traj.cu) ----
enum { TM_P, TM_MW, TM_RHO, TM_ES, TM_AES, TM_QT, TM_AQT, TM_AU, TM_AV, TM_AW, TM_TU, TM_TV, TM_TW, TM_UN, TM_VN,
       TM_WN, TM_N };
struct TrajMomArgs {
    const double *v[TM_N], *d[TM_N];   // values and (tangent mode) tangents of the inputs
    double *out[6], *dout[6];          // tu, tv, tw, mu, mv, mw (values may be null in tangent mode)
    double a_dt, b;
};
struct TrajScalArgs {
    int nf;                             // field 0: the density
    const double *adv[MG_MAXF], *dadv[MG_MAXF], *tprev[MG_MAXF], *dtprev[MG_MAXF], *sn[MG_MAXF], *dsn[MG_MAXF];
    const double *rhon, *drhon;
    double *tout[MG_MAXF], *dtout[MG_MAXF], *out[MG_MAXF], *dout[MG_MAXF];
    double a_dt, b;
};
struct TrajConv {
    int dir, ns;                        // 0: natural -> stage variables; 1: back; ns scalars besides density
    const double *in[3 + MG_MAXF], *din[3 + MG_MAXF];
    double *out[3 + MG_MAXF], *dout[3 + MG_MAXF];
    const double *rho, *drho;
};
struct TrajMomAd {
    const double *mbar[3], *tcarry[3];
    double *tprev_bar[3], *abar[3], *mnbar[3];
    double *pbar, *mwin_bar;
    const double *rho, *es, *aes, *qt, *aqt;
    double *rho_bar, *es_bar, *aes_bar, *qt_bar, *aqt_bar;
    double a_dt, b;
};
struct TrajScalAd {
    int nf;
    const double *psibar[MG_MAXF], *tcarry[MG_MAXF], *sn[MG_MAXF];
    double *advbar[MG_MAXF], *tprev_bar[MG_MAXF], *snbar[MG_MAXF];
    const double *rhon;
    double a_dt, b;
};
struct TrajConvAd {
    int dir, ns;
    const double *outbar[3 + MG_MAXF], *in[3 + MG_MAXF];
    double *inbar[3 + MG_MAXF];
    const double *rho;
    double *rhobar;
};
cudaError_t launch_stage_mom(const DevGrid &g, const TrajMomArgs &a, int tangent, cudaStream_t s);
cudaError_t launch_stage_scal(const DevGrid &g, const TrajScalArgs &a, int tangent, cudaStream_t s);
cudaError_t launch_convert(const DevGrid &g, const TrajConv &a, int tangent, cudaStream_t s);
cudaError_t launch_stage_mom_ad(const DevGrid &g, const TrajMomAd &a, cudaStream_t s);
cudaError_t launch_stage_scal_ad(const DevGrid &g, const TrajScalAd &a, cudaStream_t s);
cudaError_t launch_convert_ad(const DevGrid &g, const TrajConvAd &a, cudaStream_t s);
cudaError_t launch_axpy(const DevGrid &g, double *y, const double *x, double alpha, cudaStream_t s);

// tangent linear / adjoint of the momentum advection operator (k_momadj.cu)
cudaError_t launch_qnadv_tl(const DevGrid &g, int ntime, const double *mu, const double *mv, const double *mw,
                            const double *dmu, const double *dmv, const double *dmw, double *au, double *av, double *aw,
                            double *dau, double *dav, double *daw, cudaStream_t s);
cudaError_t launch_qnadv_ad(const DevGrid &g, const double *mu, const double *mv, const double *mw, double *aubar,
                            double *avbar, double *awbar, double *mubar, double *mvbar, double *mwbar, cudaStream_t s);

// tangent linear / adjoint of the scalar advection operator (k_adjoint.cu)
cudaError_t launch_advection_tl(const DevGrid &g, const double *x, const double *mu, const double *mv, const double *mw,
                                const double *dx, const double *dmu, const double *dmv, const double *dmw, double *dA,
                                double *scratch, cudaStream_t s);
// accumulate = 0: xbar, mubar, mvbar, mwbar are overwritten; 1: added to (their ghost
// cells must be zero on entry, and are zero on exit)
cudaError_t launch_advection_ad(const DevGrid &g, const double *x, const double *mu, const double *mv, const double *mw,
                                const double *Abar, double *xbar, double *mubar, double *mvbar, double *mwbar,
                                cudaStream_t s, int accumulate = 0);

// projection
struct PressurePlan;
cudaError_t pressure_plan_create(const DevGrid &g, const double *wv_host, int mixed, PressurePlan **out,
                                 int *pivot_error);
void pressure_plan_destroy(PressurePlan *pp);
size_t pressure_plan_bytes(const PressurePlan *pp);
// the projection's tunable plan: radix sequences of the x and y transforms (radix of
// stage s in bits [4s, 4s+4)) and launch shapes
struct PressureKnobs {
    unsigned long long xr, yr;
    int xst, yst;   // stages
    int xt;         // threads per packed row pair of the x transforms: 8 .. 64, power of 2
    int yt;         // threads per row of the y transforms: 16 .. 128, power of 2
    int tb;         // threads per block of the tridiagonal solve: 64, 128, 256
};
void pressure_get_knobs(const PressurePlan *pp, PressureKnobs *k);
bool pressure_knobs_valid(const DevGrid &g, const PressureKnobs &k);
bool pressure_set_knobs(PressurePlan *pp, const DevGrid &g, const PressureKnobs &k);
int pressure_radix_candidates(int n, unsigned long long *pk, int *nst, int maxc);
// Refinement control of one projection pass.  The mixed form solves the Poisson system
// A dp = b of the reference (b = div(m)/(dt0*rho0); A: periodic 5-point horizontal
// Laplacian plus the vertical tridiagonal rows) with FP32 transforms, then refines:
// r = (b - <b>_k) - A dp in FP64, solve A e = r with FP32 transforms, dp += e.  The plan
// keeps, per pass, the residual max|rhs|*dt0 [1/s] seen by that pass (as the bit pattern
// of a non-negative double).  A refinement pass is skipped on the device -- its kernels
// return at entry -- once that residual is below tol, so a captured graph keeps a fixed
// launch sequence while the work stops at convergence.
struct PassCtl {
    int slot;        // residual slot of this pass, or -1 (no bookkeeping)
    int refine;      // refinement pass (residual rhs, dp += solution, skipped once converged)
    int skip_prev;   // refinement pass after another: skip entirely once that one had converged
    int store_b;     // first pass of a refined projection: keep b and its level sums
    double tol;
};
constexpr PassCtl kNoPassCtl = {-1, 0, 0, 0, 0.};
constexpr int MG_MAXPASS = 64;
// ---- grouped projection and halo refresh over several members (k_pressure.cu) ----
struct GroupHaloIn {
    const DevGrid *G;
    int nf;
    double *f[MG_MAXF];
};
// the ghost-cell refresh of every member's fields as one launch
void group_halo(GroupProgram &P, const std::vector<GroupHaloIn> &m);
struct GroupProjIn {
    const DevGrid *G;
    PressurePlan *pp;
    double *mu, *mv, *mw, *p;   // momentum and pressure of the stage
    const double *wold;         // w of the stage's input (cal_p1), with its representation
    int wold_rep;
};
// One projection of every member as grouped launches, the same passes as the
// single-domain path (nsub passes, nref refinement passes each in the mixed form, the
// correction with its ghost refresh, cal_p1 without p1; finalize: the last correction and
// cal_p1 leave natural velocities).  All members share the arithmetic form.  The x
// transforms are launched once per distinct threads-per-row-pair plan knob (the block
// sums of the refined form's right-hand side follow that thread layout); every other
// launch covers all members.
void group_projection(GroupProgram &P, const std::vector<GroupProjIn> &m, int finalize, int nsub, int nref, double tol);
// ---- the compressible model's acoustic sub-steps (k_acoustic.cu) ----
// device fields (halo'd layout) of prognostic_pressure; dens2 and es2 are work fields
// of the same size, div a work field
struct AcousticFields {
    int nscal;
    const double *p0;
    const double *su, *sv, *sw, *sdens, *ses, *sqt;
    const double *sscal[MG_MAXF];
    const double *uadv, *vadv, *wadv;
    double *dens, *dens2, *es, *es2, *p, *u, *v, *w, *qt;
    double *scal[MG_MAXF];
    double *tu, *tv, *tw, *tdens, *tes, *tqt;
    double *tscal[MG_MAXF];
    double *cs2, *div;
};
// ntau sub-steps of stage im (lvl: nz doubles of device scratch)
cudaError_t launch_acoustic(const DevGrid &g, const AcousticFields &f, int im, int ntau, int cst_cp, double *lvl,
                            cudaStream_t s);
// the level means of a field over the interior (horav), into nz doubles
cudaError_t launch_level_mean(const DevGrid &g, const double *x, double *mean, cudaStream_t s);
// zero the residual slots before a projection
cudaError_t pressure_resid_reset(PressurePlan *pp, cudaStream_t s);
const unsigned long long *pressure_resid_dev(const PressurePlan *pp);
// refinement pass right-hand side: r = (b - <b>_k) - A dp into the spectrum (FP64 residual)
cudaError_t launch_resid_rhs(const DevGrid &g, PressurePlan *pp, const PassCtl &pc, cudaStream_t s);
// rhs = div(m)/(dt0*rho0) into the plan's real buffer (interior)
cudaError_t launch_div_rhs(const DevGrid &g, PressurePlan *pp, const double *mu, const double *mv,
                           const double *mw, const PassCtl &pc, cudaStream_t s);
// external rhs (unit entry): copy interior of a halo'd field into the real buffer
cudaError_t launch_load_rhs(const DevGrid &g, PressurePlan *pp, const double *tend, cudaStream_t s);
// forward FFT -> tridiagonal -> inverse FFT on the plan's buffers; out real buffer = unnormalised
// solution (scale = 1) or rescaled solution (scale = 1/N_h); keep00: keep mode (0,0) untouched
cudaError_t pressure_solve(const DevGrid &g, PressurePlan *pp, double scale, int keep00, const PassCtl &pc,
                           cudaStream_t s);
// copy the plan's real solution into the interior of a halo'd field
cudaError_t launch_store_solution(const DevGrid &g, PressurePlan *pp, double *out, cudaStream_t s);
// correction: p += rho0*dp; m -= dt0*rho0*grad(dp); ghost cells refreshed
cudaError_t launch_correction(const DevGrid &g, PressurePlan *pp, double *mu, double *mv, double *mw,
                              double *p, int natural_uv, cudaStream_t s);
// cal_p1 (+ optional p1), residual max of div
cudaError_t launch_cal_p1(const DevGrid &g, PressurePlan *pp, double *mw, const double *wold, int wold_rep,
                          int want_p1, int natural_w, cudaStream_t s);
// momentum -> natural velocities over all cells (get_velocities, funcpack.f90:265-344)
cudaError_t launch_to_velocity(const DevGrid &g, double *mu, double *mv, double *mw, cudaStream_t s);
cudaError_t launch_maxdiv(const DevGrid &g, PressurePlan *pp, const double *mu, const double *mv,
                          const double *mw, cudaStream_t s, int natural = 0);
// results of the last cal_p1 / maxdiv (device pointers inside the plan)
const double *pressure_p1_dev(const PressurePlan *pp);
const double *pressure_maxdiv_dev(const PressurePlan *pp);

// adjoint of anelastic_pressure (nsubp passes + cal_p1) on interior adjoints, in place
cudaError_t pressure_adjoint(const DevGrid &g, PressurePlan *pp, int nsubp, double *mub, double *mvb, double *mwb,
                             double *pb, cudaStream_t s);

// host-layout transfers: the natural value of a resident field into a packed nx*ny*nz
// array (download); packed nx*ny*nz -> device layout (upload)
cudaError_t launch_to_natural_packed(const DevGrid &g, const double *src, const double *w, int weight_kind, int rep,
                                     double *dst, cudaStream_t s);
cudaError_t launch_unpack(const DevGrid &g, const double *src, double *dst, cudaStream_t s);
// copy with pitch change: halo'd host layout (nx) <-> device layout (px)

