// capi.cu -- the C ABI of include/mimica_gpu.h: context, resident state, the Heun
// step driver and the unit-level entry points.
//
// Step structure (src/INTEG/time_step.f90 stepping :76-334, dynamics subset):
//   for each of the two stages (a,b) = (1,0), (1/2,1)  (INCLUDE/integ.h):
//     K1  scalars + density: advection, tend = F + b*tend, psi = psi_n + a*dt*tend
//     K2  momentum: -grad p, buoyancy, advection, tend, m = m_n + a*dt*tend
//     projection: nsubp x (rhs -> FFT -> tridiagonal -> inverse FFT -> correction),
//                 cal_p1
// Buffers: level n (A, natural variables between steps), stage working (B, density
// weighted), tendencies.  Stage 2 writes the new level-n values into A in place.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <new>
#include <memory>
#include <vector>

#include <climits>
#include <cmath>

#include "mg_common.cuh"
#include "mimica_gpu.h"

struct mg_ctx {
    mg_params prm;
    int device = 0;
    cudaStream_t stream = nullptr;
    DevGrid G{};
    int nf = 0;                          // 1 (density) + nscal
    double *prof = nullptr;              // 11 profiles x nz
    std::vector<double> wv;
    size_t fbytes = 0;                   // bytes per field
    double *mA[3] = {}, *mB[3] = {}, *tm[3] = {};
    double *p = nullptr;
    double *sA[MG_MAXF] = {}, *sB[MG_MAXF] = {}, *ts[MG_MAXF] = {};
    double *dens3 = nullptr;
    double *fes = nullptr, *fqt = nullptr;
    double *unit[16] = {};               // scratch of the unit-level entry points
    PressurePlan *pp = nullptr;
    K1Maps maps1, maps2;                 // TMA descriptors: stage-1 inputs (level n), stage-2 inputs (working)
    K2Maps mmaps1, mmaps2;               // TMA descriptors of the K2 stencil momentum, per stage
    int *derr = nullptr;                 // device error flag of bounded waits
    int rep = REP_NAT;
    int k1_nseg = 0;                     // K1 k segments per tile (0: chosen per launch for this grid alone)
    int k2_nseg = 0;                     // K2 likewise
    double traj_rec_limit = -1.;         // bytes the trajectory adjoint's stage records may take (< 0: half the free memory)
    int traj_ck_where = MG_CKPT_AUTO;    // where the trajectory adjoint keeps its checkpoints (MG_CKPT_*)
    int have_state = 0;
    unsigned up_mask = 0;                // fields uploaded one at a time (bit = MG_FIELD_*) before a full state
    int launches = 0;
    size_t bytes = 0;
    cudaGraphExec_t gexec[2] = {nullptr, nullptr};
    int gsteps[2] = {0, 0};
    long long gen = 0;                   // bumped whenever recorded step graphs go stale
    void *chk = nullptr;                 // scratch of the per-step checks
    // SGS diffusion (mg_set_sgs): per-level factors + qt0 on the device, the
    // deformation tensor and eddy viscosity of level n, the stored tendencies
    mg_sgs_params sgsp{};
    std::vector<double> sgs_qt0;
    int sgs_on = 0;
    double *sgs_prof = nullptr;          // SGS_NPROF*nz factors, then qt0 (nz)
    double *dij[6] = {}, *fkv = nullptr, *sfe = nullptr, *snut = nullptr, *sgm[3] = {}, *sgsc[MG_MAXF] = {};
    double *sfc[3] = {};                 // esflux, qvflux, mflux (nx*ny), zero until set
    int have_fkv = 0;                    // fkv holds the viscosity of the last step's level n
    // per-kernel profiling (CUDA events on the context stream)
    int prof_on = 0;
    struct Ev { const char *name; cudaEvent_t a, b; };
    std::vector<Ev> evs;
    std::vector<cudaEvent_t> pool;
    struct Acc { const char *name; double ms; long long n; };
    std::vector<Acc> acc;
};

static cudaEvent_t ev_get(mg_ctx *c)
{
    if (!c->pool.empty()) { cudaEvent_t e = c->pool.back(); c->pool.pop_back(); return e; }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}
// wrap one launch: records events around it when profiling is on
#define PROF(c, nm, call) do {                                              \
        cudaEvent_t ea_ = nullptr, eb_ = nullptr;                          \
        if ((c)->prof_on) { ea_ = ev_get(c); cudaEventRecord(ea_, (c)->stream); } \
        cudaError_t pe_ = (call);                                          \
        if ((c)->prof_on) { eb_ = ev_get(c); cudaEventRecord(eb_, (c)->stream); \
                            (c)->evs.push_back({nm, ea_, eb_}); }          \
        if (pe_ != cudaSuccess) return pe_;                                \
    } while (0)

static void prof_collect(mg_ctx *c)
{
    if (c->evs.empty()) return;
    cudaStreamSynchronize(c->stream);
    for (auto &e : c->evs) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e.a, e.b);
        bool found = false;
        for (auto &a : c->acc)
            if (!strcmp(a.name, e.name)) { a.ms += ms; a.n++; found = true; break; }
        if (!found) c->acc.push_back({e.name, (double)ms, 1});
        c->pool.push_back(e.a);
        c->pool.push_back(e.b);
    }
    c->evs.clear();
}

static int cuerr(cudaError_t e) { return e == cudaSuccess ? MG_OK : (e == cudaErrorMemoryAllocation ? MG_ERR_NOMEM : MG_ERR_CUDA); }
#define CKR(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) return cuerr(e_); } while (0)

extern "C" const char *mg_error_string(int code)
{
    switch (code) {
    case MG_OK: return "ok";
    case MG_ERR_PARAM: return "invalid or unsupported parameter";
    case MG_ERR_CUDA: return "CUDA runtime error";
    case MG_ERR_NAN: return "non-finite value detected";
    case MG_ERR_PIVOT: return "zero pivot in the vertical tridiagonal solve";
    case MG_ERR_TIMEOUT: return "bounded device wait timed out";
    case MG_ERR_NOMEM: return "out of memory";
    case MG_ERR_STATE: return "call out of order (no state uploaded)";
    default: return "unknown error";
    }
}

extern "C" int mg_version(void) { return 1; }

// ---------------- host precompute ----------------
extern "C" int mg_grid_metrics(int nz, double dz, const double *fdz, double *dzw, double *dz1w, double *dz1)
{
    if (nz < 2 || !fdz || !dzw || !dz1w || !dz1) return MG_ERR_PARAM;
    for (int k = 0; k < nz; k++) {
        dzw[k] = dz * fdz[k];
        dz1w[k] = 1. / (dz * fdz[k]);
    }
    for (int k = 0; k < nz - 1; k++) dz1[k] = 1. / ((dz * 0.5) * (fdz[k] + fdz[k + 1]));
    dz1[nz - 1] = dz1[nz - 2];
    return MG_OK;
}

extern "C" int mg_base_state(int nz, double dz, double psurf, const double *fdz0, const double *dz1,
                             const double *pt0, const double *qv0, double *p0, double *den0, double *avden0, double *stab0)
{
    if (nz < 3) return MG_ERR_PARAM;
    (void)qv0;
    const double g = 9.81, pref = 100000., cp_a = 1004., cv_a = 716.;
    const double cpm = cp_a, cvm = cv_a, ex = (cp_a - cv_a) / cp_a;
    double dsurf;
    p0[0] = psurf;
    for (int l = 0; l < 10; l++) {
        den0[0] = p0[0] / ((cpm - cvm) * pt0[0] * pow(p0[0] / pref, ex));
        dsurf = psurf / ((cpm - cvm) * pt0[0] * pow(psurf / pref, ex));
        p0[0] = psurf - g * 0.5 * (dsurf + den0[0]) * 0.5 * dz * fdz0[0];
    }
    for (int k = 1; k < nz; k++) {
        p0[k] = p0[k - 1] - g * den0[k - 1] / dz1[k - 1];
        for (int l = 0; l < 10; l++) {
            den0[k] = p0[k] / ((cpm - cvm) * pt0[k] * pow(p0[k] / pref, ex));
            p0[k] = p0[k - 1] - g * 0.5 * (den0[k - 1] + den0[k]) / dz1[k - 1];
        }
    }
    for (int k = 1; k < nz; k++) avden0[k] = (fdz0[k] * den0[k] + fdz0[k - 1] * den0[k - 1]) / (fdz0[k] + fdz0[k - 1]);
    avden0[0] = den0[0];
    for (int k = 1; k < nz - 1; k++)
        stab0[k] = (den0[k + 1] - den0[k - 1]) / (den0[k] * dz * (0.5 * fdz0[k + 1] + fdz0[k] + 0.5 * fdz0[k - 1]));
    stab0[0] = (den0[1] - den0[0]) / (den0[0] * 0.5 * dz * (fdz0[1] + fdz0[0]));
    stab0[nz - 1] = (den0[nz - 1] - den0[nz - 2]) / (den0[nz - 1] * 0.5 * dz * (fdz0[nz - 1] + fdz0[nz - 2]));
    return MG_OK;
}

extern "C" int mg_get_wv(int maxx, int maxy, double dx, double dy, double *wv)
{
    if (maxx < 1 || maxy < 1 || !wv) return MG_ERR_PARAM;
    const double pi = 3.14159265;   // the reference's constant, src/TYPES/shared_data.f90:147
    const int nl = maxx, nm = maxy;
    for (int l = 1; l <= maxx; l++) {
        double xl = (l <= nl / 2) ? (double)(l - 1) : (double)(l - nl - 1);
        for (int m = 1; m <= maxy; m++) {
            double xm = (m <= nm / 2) ? (double)(m - 1) : (double)(m - nm - 1);
            double sx = sin(pi * xl / (double)nl), sy = sin(pi * xm / (double)nm);
            wv[(size_t)(m - 1) * maxx + (l - 1)] = -4. * (sx * sx / (dx * dx) + sy * sy / (dy * dy));
        }
    }
    wv[0] = 1.;
    return MG_OK;
}

// ---------------- TMA descriptors ----------------
#include "tma.cuh"
int make_field_map(const DevGrid &g, const double *base, int boxx, int boxy, CUtensorMap *map)
{
    CUresult r = mg_encode_field_map(map, base, g.nx, g.ny, g.nz, g.px, boxx, boxy);
    return r == CUDA_SUCCESS ? MG_OK : MG_ERR_CUDA;
}

static int build_mom_maps(mg_ctx *c, const double *const *m3, K2Maps *m)
{
    for (int q = 0; q < 3; q++)
        if (make_field_map(c->G, m3[q], 38, 12, &m->m[q])) return MG_ERR_CUDA;
    return MG_OK;
}

static int build_maps(mg_ctx *c, const double *const *x, int nf, const double *mu, const double *mv, K1Maps *m)
{
    memset(m, 0, sizeof(*m));
    for (int f = 0; f < nf; f++)
        if (make_field_map(c->G, x[f], 38, 14, &m->x[f])) return MG_ERR_CUDA;
    if (make_field_map(c->G, mu, 34, 9, &m->mu)) return MG_ERR_CUDA;
    if (make_field_map(c->G, mv, 34, 9, &m->mv)) return MG_ERR_CUDA;
    return MG_OK;
}

// ---------------- context ----------------
static bool good_len(int n)
{
    int m = n;
    for (int r : {2, 3, 5}) while (m % r == 0) m /= r;
    return m == 1;
}

static int validate(const mg_params *p)
{
    if (!p) return MG_ERR_PARAM;
    if (p->maxx < 8 || p->maxy < 8 || p->nz < 8) return MG_ERR_PARAM;
    if (p->maxx % 2 || p->maxy % 2 || !good_len(p->maxx) || !good_len(p->maxy)) return MG_ERR_PARAM;
    if (p->maxx > 4096 || p->maxy > 4096) return MG_ERR_PARAM;
    if (p->nscal < 1 || p->nscal + 1 > MG_MAXF) return MG_ERR_PARAM;
    if (p->iqt >= p->nscal || p->iqt == 0) return MG_ERR_PARAM;
    if (p->scal_adv < MG_WENO || p->scal_adv > MG_QUICK) return MG_ERR_PARAM;
    if (p->muscl_limiter < MG_LIM_MINMOD || p->muscl_limiter > MG_LIM_DEFAULT) return MG_ERR_PARAM;
    if (p->mom_ord != 2 && p->mom_ord != 4) return MG_ERR_PARAM;
    if (p->nsubp < 1 || p->nsubp > 16) return MG_ERR_PARAM;
    if (p->precision != MG_PREC_FP64 && p->precision != MG_PREC_MIXED) return MG_ERR_PARAM;
    if (p->precision == MG_PREC_MIXED &&
        (p->refine_iters < 0 || p->nsubp * (1 + p->refine_iters) > MG_MAXPASS || !(p->refine_tol >= 0.)))
        return MG_ERR_PARAM;
    if (!(p->dx > 0) || !(p->dy > 0) || !(p->dz > 0) || !(p->dt0 > 0)) return MG_ERR_PARAM;
    if (!p->fdz0 || !p->dzw || !p->dz1w || !p->dz1 || !p->den0 || !p->avden0 || !p->stab0 || !p->pt0 || !p->qv0)
        return MG_ERR_PARAM;
    return MG_OK;
}

static void free_ctx(mg_ctx *c)
{
    if (!c) return;
    for (int i = 0; i < 2; i++) if (c->gexec[i]) cudaGraphExecDestroy(c->gexec[i]);
    for (int i = 0; i < 3; i++) { cudaFree(c->mA[i]); cudaFree(c->mB[i]); cudaFree(c->tm[i]); }
    for (int f = 0; f < MG_MAXF; f++) { cudaFree(c->sA[f]); cudaFree(c->sB[f]); cudaFree(c->ts[f]); }
    for (int i = 0; i < 16; i++) cudaFree(c->unit[i]);
    cudaFree(c->sgs_prof); cudaFree(c->fkv); cudaFree(c->sfe); cudaFree(c->snut); cudaFree(c->chk);
    for (int q = 0; q < 6; q++) cudaFree(c->dij[q]);
    for (int q = 0; q < 3; q++) { cudaFree(c->sgm[q]); cudaFree(c->sfc[q]); }
    for (int f = 0; f < MG_MAXF; f++) cudaFree(c->sgsc[f]);
    cudaFree(c->p); cudaFree(c->dens3); cudaFree(c->fes); cudaFree(c->fqt); cudaFree(c->prof); cudaFree(c->derr);
    pressure_plan_destroy(c->pp);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

extern "C" int mg_create(const mg_params *params, int device, mg_ctx **out)
{
    if (!out) return MG_ERR_PARAM;
    *out = nullptr;
    int v = validate(params);
    if (v) return v;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) return MG_ERR_CUDA;
    if (device < 0 || device >= ndev) return MG_ERR_PARAM;
    CKR(cudaSetDevice(device));
    mg_ctx *c = new (std::nothrow) mg_ctx();
    if (!c) return MG_ERR_NOMEM;
    c->prm = *params;
    c->device = device;
    // SGS switches: off, with the reference's namelist defaults (INCLUDE/default.h)
    c->sgsp.with_dif = 0; c->sgsp.anis_k = 0; c->sgsp.momsf = 0; c->sgsp.reserved = 0;
    c->sgsp.diff = 0.; c->sgsp.pran = 0.4; c->sgsp.zdec = 2000.; c->sgsp.zrough = 0.01; c->sgsp.min_w = 0.1;
    c->sgsp.qt0 = nullptr;
    const int nz = params->nz;
    DevGrid &G = c->G;
    G.maxx = params->maxx; G.maxy = params->maxy; G.nz = nz;
    G.nx = params->maxx + 5; G.ny = params->maxy + 5;
    G.px = (G.nx + 7) / 8 * 8;
    G.ps = (long long)G.px * G.ny;
    G.dx = params->dx; G.dy = params->dy; G.dz = params->dz; G.dt0 = params->dt0;
    G.lim_tol = params->lim_tol; G.u0shift = params->u0shift; G.v0shift = params->v0shift;
    G.scal_adv = params->scal_adv; G.muscl_lim = params->muscl_limiter; G.mom_ord = params->mom_ord;
    G.lavisc = params->lavisc; G.with_buoy = params->with_buoy;
    c->nf = 1 + params->nscal;
    c->fbytes = (size_t)G.ps * nz * sizeof(double);
    int rc = MG_OK;
    auto fail = [&](int code) { free_ctx(c); return code; };
    cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return fail(cuerr(e));
    // profiles
    e = cudaMalloc(&c->prof, 11 * nz * sizeof(double));
    if (e != cudaSuccess) return fail(cuerr(e));
    std::vector<double> rden(2 * (size_t)nz);
    for (int k = 0; k < nz; k++) { rden[k] = 1. / params->den0[k]; rden[nz + k] = 1. / params->avden0[k]; }
    const double *src[11] = {params->fdz0, params->dzw, params->dz1w, params->dz1, params->den0, params->avden0,
                             params->stab0, params->pt0, params->qv0, rden.data(), rden.data() + nz};
    for (int q = 0; q < 11; q++) {
        e = cudaMemcpy(c->prof + q * nz, src[q], nz * sizeof(double), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return fail(cuerr(e));
    }
    G.fdz0 = c->prof; G.dzw = c->prof + nz; G.dz1w = c->prof + 2 * nz; G.dz1 = c->prof + 3 * nz;
    G.den0 = c->prof + 4 * nz; G.avden0 = c->prof + 5 * nz; G.stab0 = c->prof + 6 * nz;
    G.pt0 = c->prof + 7 * nz; G.qv0 = c->prof + 8 * nz; G.rden0 = c->prof + 9 * nz; G.ravden0 = c->prof + 10 * nz;
    // fields
    auto alloc = [&](double **p) -> int {
        cudaError_t ee = cudaMalloc(p, c->fbytes);
        if (ee != cudaSuccess) return cuerr(ee);
        c->bytes += c->fbytes;
        return cudaMemset(*p, 0, c->fbytes) == cudaSuccess ? MG_OK : MG_ERR_CUDA;
    };
    for (int i = 0; i < 3 && !rc; i++) {
        rc = alloc(&c->mA[i]);
        if (!rc) rc = alloc(&c->mB[i]);
        if (!rc) rc = alloc(&c->tm[i]);
    }
    for (int f = 0; f < c->nf && !rc; f++) {
        rc = alloc(&c->sA[f]);
        if (!rc) rc = alloc(&c->sB[f]);
        if (!rc) rc = alloc(&c->ts[f]);
    }
    if (!rc) rc = alloc(&c->p);
    if (!rc) rc = alloc(&c->fes);
    if (!rc) rc = alloc(&c->fqt);
    if (rc) return fail(rc);
    e = cudaMalloc(&c->derr, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(c->derr, 0, sizeof(int));
    if (e == cudaSuccess) e = k1_init();
    if (e == cudaSuccess) e = k1_mixed_init();
    if (e != cudaSuccess) return fail(cuerr(e));
    if (build_maps(c, c->sA, c->nf, c->mA[0], c->mA[1], &c->maps1) ||
        build_maps(c, c->sB, c->nf, c->mB[0], c->mB[1], &c->maps2) ||
        build_mom_maps(c, c->mA, &c->mmaps1) || build_mom_maps(c, c->mB, &c->mmaps2))
        return fail(MG_ERR_CUDA);
    // horizontal eigenvalues (get_wv) and the projection plan
    c->wv.resize((size_t)G.maxx * G.maxy);
    mg_get_wv(G.maxx, G.maxy, G.dx, G.dy, c->wv.data());
    int piv = 0;
    e = pressure_plan_create(G, c->wv.data(), params->precision == MG_PREC_MIXED, &c->pp, &piv);
    if (e != cudaSuccess) return fail(cuerr(e));
    c->bytes += pressure_plan_bytes(c->pp);
    if (piv) return fail(MG_ERR_PIVOT);
    *out = c;
    return MG_OK;
}

extern "C" int mg_destroy(mg_ctx *ctx)
{
    if (!ctx) return MG_ERR_PARAM;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    free_ctx(ctx);
    return MG_OK;
}

extern "C" size_t mg_device_bytes(const mg_ctx *ctx) { return ctx ? ctx->bytes : 0; }
extern "C" int mg_last_launch_count(const mg_ctx *ctx) { return ctx ? ctx->launches : -1; }

// host (dense nx) <-> device (pitched px)
static cudaError_t h2d(mg_ctx *c, double *dst, const double *src, cudaMemcpyKind kind)
{
    const DevGrid &G = c->G;
    return cudaMemcpy2DAsync(dst, (size_t)G.px * 8, src, (size_t)G.nx * 8, (size_t)G.nx * 8, (size_t)G.ny * G.nz, kind,
                             c->stream);
}
static cudaError_t d2h(mg_ctx *c, double *dst, const double *src, cudaMemcpyKind kind)
{
    const DevGrid &G = c->G;
    return cudaMemcpy2DAsync(dst, (size_t)G.nx * 8, src, (size_t)G.px * 8, (size_t)G.nx * 8, (size_t)G.ny * G.nz, kind,
                             c->stream);
}

static int upload_impl(mg_ctx *c, const double *u, const double *v, const double *w, const double *p,
                       const double *dens, const double *const *scal, cudaMemcpyKind kind)
{
    if (!c || !u || !v || !w || !p || !dens || !scal) return MG_ERR_PARAM;
    for (int s = 0; s < c->prm.nscal; s++)
        if (!scal[s]) return MG_ERR_PARAM;
    CKR(cudaSetDevice(c->device));
    // host sources: one linear copy per field into a staging buffer (a stage buffer, free
    // between steps), then unpacked into the padded layout; device sources are unpacked
    // directly
    const size_t packed = (size_t)c->G.nx * c->G.ny * c->G.nz * sizeof(double);
    double *stage = c->sB[0];
    auto put = [&](double *dst, const double *src) -> cudaError_t {
        if (kind == cudaMemcpyDeviceToDevice) return launch_unpack(c->G, src, dst, c->stream);
        cudaError_t e = cudaMemcpyAsync(stage, src, packed, kind, c->stream);
        return e == cudaSuccess ? launch_unpack(c->G, stage, dst, c->stream) : e;
    };
    CKR(put(c->mA[0], u));
    CKR(put(c->mA[1], v));
    CKR(put(c->mA[2], w));
    CKR(put(c->p, p));
    CKR(put(c->sA[0], dens));
    for (int s = 0; s < c->prm.nscal; s++) CKR(put(c->sA[1 + s], scal[s]));
    // ghost cells from the interior (the reference's state after update_prognostic)
    std::vector<double *> f = {c->mA[0], c->mA[1], c->mA[2], c->p};
    for (int q = 0; q < c->nf; q++) f.push_back(c->sA[q]);
    CKR(launch_halo_fill(c->G, f.data(), (int)f.size(), c->stream));
    c->rep = REP_NAT;
    c->have_state = 1;
    return cuerr(cudaStreamSynchronize(c->stream));
}

extern "C" int mg_upload_state(mg_ctx *c, const double *u, const double *v, const double *w, const double *p,
                               const double *dens, const double *const *scal)
{
    return upload_impl(c, u, v, w, p, dens, scal, cudaMemcpyHostToDevice);
}
extern "C" int mg_upload_state_device(mg_ctx *c, const double *u, const double *v, const double *w, const double *p,
                                      const double *dens, const double *const *scal)
{
    return upload_impl(c, u, v, w, p, dens, scal, cudaMemcpyDeviceToDevice);
}

// one field of the level-n state (natural values) from host memory: a linear copy into a
// stage buffer (free between steps), unpacked into the padded layout, ghosts refreshed
extern "C" int mg_upload_field(mg_ctx *c, int field, const double *src)
{
    if (!c || !src || field < MG_FIELD_U || field >= MG_FIELD_SCAL + c->prm.nscal) return MG_ERR_PARAM;
    if (c->have_state && c->rep != REP_NAT) return MG_ERR_STATE;
    CKR(cudaSetDevice(c->device));
    double *dst = field == MG_FIELD_U ? c->mA[0] : field == MG_FIELD_V ? c->mA[1] : field == MG_FIELD_W ? c->mA[2]
                : field == MG_FIELD_P ? c->p : c->sA[field - MG_FIELD_DENS];
    const size_t packed = (size_t)c->G.nx * c->G.ny * c->G.nz * sizeof(double);
    double *stage = c->sB[0];
    CKR(cudaMemcpyAsync(stage, src, packed, cudaMemcpyHostToDevice, c->stream));
    CKR(launch_unpack(c->G, stage, dst, c->stream));
    CKR(launch_halo_fill(c->G, &dst, 1, c->stream));
    CKR(cudaStreamSynchronize(c->stream));
    if (!c->have_state) {
        c->up_mask |= 1u << field;
        const unsigned all = (1u << (MG_FIELD_SCAL + c->prm.nscal)) - 1u;   // nscal < MG_MAXF: fits 32 bits
        if (c->up_mask == all) {
            c->rep = REP_NAT;
            c->have_state = 1;
        }
    }
    return MG_OK;
}

static int download_impl(mg_ctx *c, double *u, double *v, double *w, double *p, double *dens, double *const *scal,
                         cudaMemcpyKind kind)
{
    if (!c) return MG_ERR_PARAM;
    if (!c->have_state) return MG_ERR_STATE;
    CKR(cudaSetDevice(c->device));
    const DevGrid &G = c->G;
    double *tmp = c->sB[0];   // stage buffer reused as scratch between steps
    struct Item { double *dst; const double *src; const double *w; int kind; };
    std::vector<Item> items;
    if (u) items.push_back({u, c->mA[0], nullptr, 1});
    if (v) items.push_back({v, c->mA[1], nullptr, 1});
    if (w) items.push_back({w, c->mA[2], nullptr, 2});
    if (p) items.push_back({p, c->p, nullptr, 0});
    if (dens) items.push_back({dens, c->sA[0], nullptr, 0});
    if (scal)
        for (int s = 0; s < c->prm.nscal; s++)
            if (scal[s]) items.push_back({scal[s], c->sA[1 + s], c->sA[0], 3});
    // natural values written packed (nx*ny*nz), then one linear copy per field; device
    // destinations receive them directly
    const size_t packed = (size_t)G.nx * G.ny * G.nz * sizeof(double);
    for (auto &it : items) {
        if (kind == cudaMemcpyDeviceToDevice) {
            CKR(launch_to_natural_packed(G, it.src, it.w, it.kind, c->rep, it.dst, c->stream));
            continue;
        }
        CKR(launch_to_natural_packed(G, it.src, it.w, it.kind, c->rep, tmp, c->stream));
        CKR(cudaMemcpyAsync(it.dst, tmp, packed, kind, c->stream));
    }
    return cuerr(cudaStreamSynchronize(c->stream));
}

extern "C" int mg_download_state(mg_ctx *c, double *u, double *v, double *w, double *p, double *dens, double *const *scal)
{
    return download_impl(c, u, v, w, p, dens, scal, cudaMemcpyDeviceToHost);
}
extern "C" int mg_download_field(mg_ctx *c, int field, double *dst)
{
    if (!c || !dst || field < MG_FIELD_U || field >= MG_FIELD_SCAL + c->prm.nscal) return MG_ERR_PARAM;
    std::vector<double *> sc(c->prm.nscal > 0 ? c->prm.nscal : 1, nullptr);
    if (field >= MG_FIELD_SCAL) sc[field - MG_FIELD_SCAL] = dst;
    return download_impl(c, field == MG_FIELD_U ? dst : nullptr, field == MG_FIELD_V ? dst : nullptr,
                         field == MG_FIELD_W ? dst : nullptr, field == MG_FIELD_P ? dst : nullptr,
                         field == MG_FIELD_DENS ? dst : nullptr, field >= MG_FIELD_SCAL ? sc.data() : nullptr,
                         cudaMemcpyDeviceToHost);
}
extern "C" int mg_download_state_device(mg_ctx *c, double *u, double *v, double *w, double *p, double *dens,
                                        double *const *scal)
{
    return download_impl(c, u, v, w, p, dens, scal, cudaMemcpyDeviceToDevice);
}

// ---------------- projection ----------------
// nsubp x (solve + correction), cal_p1; wold: momentum w at stage start.
// finalize: end of a step -- leave natural velocities (get_velocities) in mu, mv, mw.
static cudaError_t project(mg_ctx *c, double *mu, double *mv, double *mw, const double *wold, int wold_rep,
                           int want_p1, int want_maxdiv, int finalize, int *launches)
{
    const DevGrid &G = c->G;
    const int fuse = finalize && !want_maxdiv;   // maxdiv needs the momentum after cal_p1
    // each of the nsubp sub-iterations: solve (+ in the mixed form up to refine_iters
    // refinement passes on the FP64 residual of the Poisson system), then the correction
    const int nsub = c->prm.nsubp;
    const int nref = c->prm.precision == MG_PREC_MIXED ? c->prm.refine_iters : 0;
    cudaError_t er = pressure_resid_reset(c->pp, c->stream);
    if (er != cudaSuccess) return er;
    for (int ip = 0; ip < nsub; ip++) {
        const int last = ip == nsub - 1;
        const int slot0 = ip * (1 + nref);
        const PassCtl p0 = {slot0, 0, 0, nref > 0, c->prm.refine_tol};
        PROF(c, "fft_x_fwd_div", launch_div_rhs(G, c->pp, mu, mv, mw, p0, c->stream));
        PROF(c, "fft_y_tridiag_fft_y_fft_x_inv", pressure_solve(G, c->pp, 0., 0, p0, c->stream));
        *launches += 5;
        for (int r = 0; r < nref; r++) {
            const PassCtl pr = {slot0 + 1 + r, 1, r > 0, 0, c->prm.refine_tol};
            PROF(c, "refine_residual_fft_x", launch_resid_rhs(G, c->pp, pr, c->stream));
            PROF(c, "refine_solve", pressure_solve(G, c->pp, 0., 0, pr, c->stream));
            *launches += 5;
        }
        PROF(c, "correction_halo", launch_correction(G, c->pp, mu, mv, mw, c->p, fuse && last, c->stream));
        *launches += 2;
    }
    PROF(c, "cal_p1", launch_cal_p1(G, c->pp, mw, wold, wold_rep, want_p1, fuse, c->stream));
    *launches += want_p1 ? 3 : 2;
    if (want_maxdiv) {
        PROF(c, "maxdiv", launch_maxdiv(G, c->pp, mu, mv, mw, c->stream));
        *launches += 2;
        if (finalize) {
            PROF(c, "to_velocity", launch_to_velocity(G, mu, mv, mw, c->stream));
            *launches += 1;
        }
    }
    return cudaSuccess;
}

// ---------------- one step ----------------
// step graphs recorded before a change of the step (time step, SGS switches) no longer
// describe it: drop the context's own, and make ensembles that hold it re-record
static void drop_graphs(mg_ctx *c)
{
    for (int i = 0; i < 2; i++)
        if (c->gexec[i]) { cudaGraphExecDestroy(c->gexec[i]); c->gexec[i] = nullptr; }
    c->gen++;
}

// ---------------- SGS diffusion ----------------
static SgsDev sgs_dev(const mg_ctx *c)
{
    const int nz = c->G.nz;
    const double *P = c->sgs_prof;
    SgsDev S{};
    S.anis_k = c->sgsp.anis_k; S.momsf = c->sgsp.momsf; S.diff_on = c->sgsp.diff != 0.;
    S.diff = c->sgsp.diff; S.pran = c->sgsp.pran; S.min_w = c->sgsp.min_w;
    S.cs2d = P + nz; S.func = P + 2 * nz; S.fan = P + 3 * nz; S.n2c = P + 4 * nz; S.n2d = P + 5 * nz;
    S.du = P + 6 * nz; S.dv = P + 7 * nz; S.dw = P + 8 * nz; S.dwt = P + 9 * nz;
    return S;
}
static const double *sgs_qt0_dev(const mg_ctx *c) { return c->sgs_prof + SGS_NPROF * c->G.nz; }

// allocate the SGS work fields (first use) and upload the per-level factors of sgsp
static int ensure_sgs(mg_ctx *c)
{
    const DevGrid &G = c->G;
    const int nz = G.nz;
    auto field = [&](double **p, size_t bytes) -> int {
        if (*p) return MG_OK;
        cudaError_t e = cudaMalloc(p, bytes);
        if (e != cudaSuccess) return cuerr(e);
        c->bytes += bytes;
        return cudaMemset(*p, 0, bytes) == cudaSuccess ? MG_OK : MG_ERR_CUDA;
    };
    int rc = field(&c->sgs_prof, (size_t)(SGS_NPROF + 1) * nz * sizeof(double));
    for (int q = 0; q < 6 && !rc; q++) rc = field(&c->dij[q], c->fbytes);
    if (!rc) rc = field(&c->fkv, c->fbytes);
    if (!rc) rc = field(&c->sfe, c->fbytes);
    if (!rc) rc = field(&c->snut, c->fbytes);
    for (int q = 0; q < 3 && !rc; q++) rc = field(&c->sgm[q], c->fbytes);
    for (int q = 0; q < 3 && !rc; q++) rc = field(&c->sfc[q], (size_t)G.nx * G.ny * sizeof(double));
    if (rc) return rc;
    const mg_params &P = c->prm;
    std::vector<double> h((size_t)(SGS_NPROF + 1) * nz);
    sgs_host_profiles(nz, P.dx, P.dy, P.dz, P.fdz0, P.pt0, P.qv0, c->sgsp.anis_k, c->sgsp.zdec, c->sgsp.zrough, h.data());
    for (int k = 0; k < nz; k++) h[(size_t)SGS_NPROF * nz + k] = c->sgs_qt0.empty() ? P.qv0[k] : c->sgs_qt0[k];
    CKR(cudaMemcpyAsync(c->sgs_prof, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    return cuerr(cudaStreamSynchronize(c->stream));
}

// calc_subgrid, efud and eff0/effs of level n (once per step)
static cudaError_t sgs_tendencies(mg_ctx *c, int *launches)
{
    const DevGrid &G = c->G;
    const int ies = 1, iqt = c->prm.iqt >= 0 ? 1 + c->prm.iqt : -1;
    const SgsDev S = sgs_dev(c);
    SgsDij D{};
    for (int q = 0; q < 6; q++) D.d[q] = c->dij[q];
    const SgsVisc O{c->fkv, c->sfe, c->snut};
    PROF(c, "sgs_viscosity", launch_sgs_visc(G, S, c->mA[0], c->mA[1], c->mA[2], c->sA[ies], iqt >= 0 ? c->sA[iqt] : nullptr,
                                             c->sA[0], D, O, c->stream));
    double *hf[9] = {c->dij[0], c->dij[1], c->dij[2], c->dij[3], c->dij[4], c->dij[5], c->sfe, c->snut, c->fkv};
    PROF(c, "sgs_halo", launch_halo_fill(G, hf, 9, c->stream));
    c->have_fkv = 1;
    PROF(c, "sgs_momentum", launch_sgs_mom(G, S, c->mA[0], c->mA[1], c->sfe, D, c->sfc[2], nullptr, nullptr, nullptr,
                                           c->sgm[0], c->sgm[1], c->sgm[2], c->stream));
    SgsScal A{};
    A.nf = c->nf - 1;
    for (int f = 1; f < c->nf; f++) {
        const int q = f - 1;
        A.x[q] = c->sA[f];
        A.out[q] = c->sgsc[f];
        A.x0[q] = f == ies ? G.pt0 : (f == iqt ? sgs_qt0_dev(c) : nullptr);
        A.fs[q] = f == ies ? c->sfc[0] : (f == iqt ? c->sfc[1] : nullptr);
        A.fs_neg[q] = 1;
    }
    if (A.nf > 0) PROF(c, "sgs_scalars", launch_sgs_scal(G, S, c->snut, A, c->stream));
    *launches += A.nf > 0 ? 4 : 3;
    return cudaSuccess;
}

// K1's arguments for one stage of the step (stage 1 writes only the stage buffers)
static void k1_stage_args(mg_ctx *c, int stage, K1Args &a1)
{
    const DevGrid &G = c->G;
    const int nf = c->nf;
    const int ies = 1, iqt = c->prm.iqt >= 0 ? 1 + c->prm.iqt : -1;
    a1.nf = nf; a1.dens_first = 1; a1.stage = stage; a1.mode = 0;
    a1.a_dt = (stage == 1 ? 1. : 0.5) * G.dt0;
    a1.b = stage == 1 ? 0. : 1.;
    a1.nseg = c->k1_nseg;
    a1.err = c->derr;
    for (int f = 0; f < nf; f++) {
        a1.xin[f] = stage == 1 ? c->sA[f] : c->sB[f];
        a1.xold[f] = c->sA[f];
        a1.xold_is_xin = stage == 1;
        a1.xout[f] = stage == 1 ? c->sB[f] : c->sA[f];
        a1.tend[f] = c->ts[f];
        a1.fst[f] = (f == ies && G.with_buoy) ? c->fes : ((f == iqt && G.with_buoy) ? c->fqt : nullptr);
        a1.sgs[f] = (c->sgs_on && f >= 1) ? c->sgsc[f] : nullptr;
    }
    a1.sgs_post = c->sgs_on ? ((1u << ies) | (iqt >= 0 ? 1u << iqt : 0u)) : 0u;
    a1.mw = (stage == 1 ? c->mA : c->mB)[2];
}

static void k2_stage_args(mg_ctx *c, int stage, int ntime, K2Args &a2)
{
    const DevGrid &G = c->G;
    const int ies = 1, iqt = c->prm.iqt >= 0 ? 1 + c->prm.iqt : -1;
    const double *const *mom = stage == 1 ? c->mA : c->mB;
    a2.stage = stage; a2.rep = REP_NAT; a2.ntime = ntime;
    a2.a_dt = (stage == 1 ? 1. : 0.5) * G.dt0;
    a2.b = stage == 1 ? 0. : 1.;
    a2.nseg = c->k2_nseg;
    a2.mu = mom[0]; a2.mv = mom[1]; a2.mw = mom[2];
    a2.in_is_leveln = stage == 1;
    a2.mu_n = c->mA[0]; a2.mv_n = c->mA[1]; a2.mw_n = c->mA[2];
    a2.p = c->p;
    // buoyancy reads the stage's input density and scalars: level n in stage 1 (natural,
    // unchanged by K1 stage 1), the working values in stage 2
    a2.dens = stage == 1 ? c->sA[0] : c->sB[0];
    a2.es = stage == 1 ? c->sA[ies] : c->sB[ies];
    a2.qt = iqt >= 0 ? (stage == 1 ? c->sA[iqt] : c->sB[iqt]) : nullptr;
    a2.dens_is_leveln = stage == 1;
    a2.fes = c->fes; a2.fqt = iqt >= 0 ? c->fqt : nullptr;
    double **mo = stage == 1 ? c->mB : c->mA;
    a2.ou = mo[0]; a2.ov = mo[1]; a2.ow = mo[2];
    a2.tu = c->tm[0]; a2.tv = c->tm[1]; a2.tw = c->tm[2];
    a2.mode = 0;
    a2.err = c->derr;
    if (c->sgs_on) { a2.su = c->sgm[0]; a2.sv = c->sgm[1]; a2.sw = c->sgm[2]; }
}

static cudaError_t step_once(mg_ctx *c, int ntime, int last, int want_p1, int want_maxdiv, int *launches)
{
    const DevGrid &G = c->G;
    const mg_params &P = c->prm;
    const int nf = c->nf;
    if (c->sgs_on) {
        cudaError_t e = sgs_tendencies(c, launches);
        if (e != cudaSuccess) return e;
    }
    for (int stage = 1; stage <= 2; stage++) {
        // ---- K1: density + scalars (level-n buffers hold natural variables) ----
        K1Args a1{};
        k1_stage_args(c, stage, a1);
        if (P.precision == MG_PREC_MIXED)
            PROF(c, "k1_scalar_advection", launch_k1_mixed(G, a1, stage == 1 ? c->maps1 : c->maps2, c->stream));
        else
            PROF(c, "k1_scalar_advection", launch_k1(G, a1, stage == 1 ? c->maps1 : c->maps2, c->stream));
        {
            std::vector<double *> f;
            for (int q = 0; q < nf; q++) f.push_back(a1.xout[q]);
            PROF(c, "halo_scalars", launch_halo_fill(G, f.data(), nf, c->stream));
        }
        // ---- K2: momentum ----
        K2Args a2{};
        k2_stage_args(c, stage, ntime, a2);
        double **mo = stage == 1 ? c->mB : c->mA;
        const K2Maps &mm = stage == 1 ? c->mmaps1 : c->mmaps2;
        if (P.precision == MG_PREC_MIXED)
            PROF(c, "k2_momentum", launch_k2_mixed(G, a2, mm, c->stream));
        else
            PROF(c, "k2_momentum", launch_k2(G, a2, mm, c->stream));
        PROF(c, "halo_momentum", launch_halo_fill(G, mo, 3, c->stream));
        *launches += 4;
        // ---- projection ----
        const double *wold = stage == 1 ? c->mA[2] : c->mB[2];
        const int wold_rep = stage == 1 ? REP_NAT : -1;
        cudaError_t e = project(c, mo[0], mo[1], mo[2], wold, wold_rep, last && stage == 2 && want_p1,
                                last && stage == 2 && want_maxdiv, stage == 2, launches);
        if (e != cudaSuccess) return e;
    }
    c->rep = REP_NAT;
    return cudaSuccess;
}

static int check_err(mg_ctx *c)
{
    int h = 0;
    cudaError_t e = cudaMemcpyAsync(&h, c->derr, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuerr(e);
    if (h) {
        cudaMemsetAsync(c->derr, 0, sizeof(int), c->stream);
        return MG_ERR_TIMEOUT;
    }
    return MG_OK;
}

extern "C" int mg_step(mg_ctx *c, int nsteps, int ntime0, double *maxdiv, double *p1)
{
    if (!c || nsteps < 0) return MG_ERR_PARAM;
    if (!c->have_state) return MG_ERR_STATE;
    CKR(cudaSetDevice(c->device));
    int launches = 0;
    for (int s = 0; s < nsteps; s++) {
        cudaError_t e = step_once(c, ntime0 + s, s == nsteps - 1, p1 != nullptr, maxdiv != nullptr, &launches);
        if (e != cudaSuccess) return cuerr(e);
    }
    c->launches = launches;
    if (maxdiv && nsteps > 0) CKR(cudaMemcpyAsync(maxdiv, pressure_maxdiv_dev(c->pp), 8, cudaMemcpyDeviceToHost, c->stream));
    if (p1 && nsteps > 0) CKR(cudaMemcpyAsync(p1, pressure_p1_dev(c->pp), c->G.nz * 8, cudaMemcpyDeviceToHost, c->stream));
    return check_err(c);
}

extern "C" int mg_step_graph(mg_ctx *c, int nsteps, int ntime0, double *maxdiv, double *p1)
{
    // The graph covers a pair of steps (the momentum direction order alternates with
    // the step counter's parity); odd remainders run eagerly.
    if (!c || nsteps < 0) return MG_ERR_PARAM;
    if (!c->have_state) return MG_ERR_STATE;
    CKR(cudaSetDevice(c->device));
    int rc = MG_OK;
    int s = 0;
    int par = (ntime0 + s) & 1;
    while (nsteps - s >= 2) {
        if (!c->gexec[par]) {
            cudaGraph_t graph;
            CKR(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
            int launches = 0;
            cudaError_t e = step_once(c, ntime0 + s, 0, 0, 0, &launches);
            if (e == cudaSuccess) e = step_once(c, ntime0 + s + 1, 0, 0, 0, &launches);
            cudaError_t e2 = cudaStreamEndCapture(c->stream, &graph);
            if (e != cudaSuccess) return cuerr(e);
            if (e2 != cudaSuccess) return cuerr(e2);
            e = cudaGraphInstantiate(&c->gexec[par], graph, 0);
            cudaGraphDestroy(graph);
            if (e != cudaSuccess) return cuerr(e);
            c->launches = launches / 2;
        }
        CKR(cudaGraphLaunch(c->gexec[par], c->stream));
        s += 2;
    }
    rc = check_err(c);
    if (rc) return rc;
    if (s < nsteps) {
        rc = mg_step(c, nsteps - s, ntime0 + s, maxdiv, p1);
        if (rc) return rc;
    } else if (maxdiv || p1) {
        // diagnostics of the final state: the level-n buffers hold velocities, whose
        // momentum the residual is the divergence of
        const DevGrid &G = c->G;
        if (maxdiv) {
            CKR(launch_maxdiv(G, c->pp, c->mA[0], c->mA[1], c->mA[2], c->stream, 1));
            CKR(cudaMemcpyAsync(maxdiv, pressure_maxdiv_dev(c->pp), 8, cudaMemcpyDeviceToHost, c->stream));
        }
        if (p1) memset(p1, 0, sizeof(double) * G.nz);
        CKR(cudaStreamSynchronize(c->stream));
    }
    return MG_OK;
}

// ---------------- ensembles of independent domains ----------------
// The members are contexts of their own (sizes, parameters, streams).  A pair of steps
// of all members is recorded once per parity into one CUDA graph, in one of two modes:
//  * MG_ENS_GROUPED: every kernel of a stage is ONE launch over the blocks of all
//    members (a work table of (member, block) items, largest blocks first, with each
//    member's arguments and tensor maps in device memory), so a stage is the same dozen
//    or so launches whatever the member count;
//  * MG_ENS_STREAMS: the graph forks from the ensemble's stream to every member's stream
//    and joins back; each member's launches are its single-domain ones.
// Both run the same kernel bodies on the same data: the results are identical.
struct mg_ens {
    std::vector<mg_ctx *> m;
    int device = 0;
    int mode = MG_ENS_STREAMS;
    cudaStream_t stream = nullptr;
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> join;
    cudaGraphExec_t gexec[2] = {nullptr, nullptr};
    unsigned char *gdev[2] = {nullptr, nullptr};   // grouped mode: device tables of each parity's graph
    long long gen = -1;                  // sum of the members' generations the graphs were recorded at
    int launches = 0;
};

// members that can share grouped launches: one arithmetic form, scheme and field count,
// no SGS, the same projection passes
static bool ens_groupable(const mg_ens *e)
{
    const mg_ctx *a = e->m[0];
    for (const mg_ctx *c : e->m) {
        if (c->sgs_on || c->prm.precision != a->prm.precision || c->G.scal_adv != a->G.scal_adv || c->nf != a->nf ||
            c->prm.nsubp != a->prm.nsubp)
            return false;
        if (a->prm.precision == MG_PREC_MIXED &&
            (c->prm.refine_iters != a->prm.refine_iters || c->prm.refine_tol != a->prm.refine_tol))
            return false;
    }
    return true;
}

static void ens_drop_graphs(mg_ens *e)
{
    for (int i = 0; i < 2; i++) {
        if (e->gexec[i]) { cudaGraphExecDestroy(e->gexec[i]); e->gexec[i] = nullptr; }
        if (e->gdev[i]) { cudaFree(e->gdev[i]); e->gdev[i] = nullptr; }
    }
}

// steps ntime0, ntime0+1 of the members `mem` as grouped launches (the launch sequence
// of step_once without SGS, last = 0)
static void ens_group_record(const std::vector<mg_ctx *> &mem, int ntime0, GroupProgram &P)
{
    const int n = (int)mem.size();
    const mg_ctx *c0 = mem[0];
    const bool mixed = c0->prm.precision == MG_PREC_MIXED;
    const int scheme = c0->G.scal_adv, nf = c0->nf;
    const int nsub = c0->prm.nsubp, nref = mixed ? c0->prm.refine_iters : 0;
    const double tol = c0->prm.refine_tol;
    for (int st = 0; st < 2; st++) {
        const int ntime = ntime0 + st;
        for (int stage = 1; stage <= 2; stage++) {
            std::vector<int> nb(n);
            std::vector<double> cost(n);
            for (int q = 0; q < n; q++) {
                const DevGrid &G = mem[q]->G;
                nb[q] = ((G.maxx + 31) / 32) * ((G.maxy + 7) / 8);   // whole-column tiles of K1 and K2 (32 x 8)
                cost[q] = (double)G.nz;
            }
            const std::vector<GItem> it = group_items(nb, cost);
            const size_t io = P.put(it);
            const int ni = (int)it.size();
            // ---- K1 and the scalars' ghost cells ----
            std::vector<K1Member> k1(n);
            std::vector<GroupHaloIn> hs(n);
            for (int q = 0; q < n; q++) {
                mg_ctx *c = mem[q];
                k1[q].M = stage == 1 ? c->maps1 : c->maps2;
                k1[q].G = c->G;
                k1[q].A = K1Args{};
                k1_stage_args(c, stage, k1[q].A);
                k1[q].A.nseg = 1;
                hs[q].G = &c->G;
                hs[q].nf = nf;
                for (int f = 0; f < nf; f++) hs[q].f[f] = k1[q].A.xout[f];
            }
            const size_t m1 = P.put(k1);
            P.ops.push_back([=](const unsigned char *d, cudaStream_t s) {
                return mixed ? launch_k1_group_mixed(scheme, stage, nf, (const K1Member *)(d + m1), (const GItem *)(d + io), ni, s)
                             : launch_k1_group(scheme, stage, nf, (const K1Member *)(d + m1), (const GItem *)(d + io), ni, s);
            });
            P.launches++;
            group_halo(P, hs);
            // ---- K2 (one launch per K2G_MAX members) and the momentum's ghost cells ----
            std::vector<GroupHaloIn> hm(n);
            std::vector<GroupProjIn> pj(n);
            const int even = (ntime % 2) == 0;
            for (int c0 = 0; c0 < n; c0 += K2G_MAX) {
                const int cn = std::min(K2G_MAX, n - c0);
                auto prm = std::make_shared<K2GroupParams>();
                std::vector<K2Maps> maps(cn);
                for (int q = 0; q < cn; q++) {
                    mg_ctx *c = mem[c0 + q];
                    maps[q] = stage == 1 ? c->mmaps1 : c->mmaps2;
                    prm->a[q].G = c->G;
                    prm->a[q].A = K2Args{};
                    k2_stage_args(c, stage, ntime, prm->a[q].A);
                    prm->a[q].A.nseg = 1;
                }
                const std::vector<GItem> itc =
                    group_items(std::vector<int>(nb.begin() + c0, nb.begin() + c0 + cn),
                                std::vector<double>(cost.begin() + c0, cost.begin() + c0 + cn));
                const size_t mm = P.put(maps), ic = P.put(itc);
                const int nic = (int)itc.size();
                P.ops.push_back([=](const unsigned char *d, cudaStream_t s) {
                    return mixed ? launch_k2_group_mixed(even, *prm, (const K2Maps *)(d + mm), (const GItem *)(d + ic), nic, s)
                                 : launch_k2_group(even, *prm, (const K2Maps *)(d + mm), (const GItem *)(d + ic), nic, s);
                });
                P.launches++;
            }
            for (int q = 0; q < n; q++) {
                mg_ctx *c = mem[q];
                double **mo = stage == 1 ? c->mB : c->mA;
                hm[q].G = &c->G;
                hm[q].nf = 3;
                for (int f = 0; f < 3; f++) hm[q].f[f] = mo[f];
                pj[q] = GroupProjIn{&c->G, c->pp, mo[0], mo[1], mo[2], c->p, stage == 1 ? c->mA[2] : c->mB[2],
                                    stage == 1 ? REP_NAT : -1};
            }
            group_halo(P, hm);
            // ---- projection ----
            group_projection(P, pj, stage == 2, nsub, nref, tol);
        }
    }
}

extern "C" int mg_ensemble_create(mg_ctx *const *members, int n, mg_ens **out)
{
    if (!members || n < 1 || !out) return MG_ERR_PARAM;
    *out = nullptr;
    for (int i = 0; i < n; i++) {
        if (!members[i]) return MG_ERR_PARAM;
        if (members[i]->device != members[0]->device) return MG_ERR_PARAM;
        for (int j = 0; j < i; j++) if (members[j] == members[i]) return MG_ERR_PARAM;
    }
    CKR(cudaSetDevice(members[0]->device));
    mg_ens *e = new mg_ens();
    e->device = members[0]->device;
    e->m.assign(members, members + n);
    e->mode = ens_groupable(e) ? MG_ENS_GROUPED : MG_ENS_STREAMS;
    cudaError_t er = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking);
    if (er == cudaSuccess) er = cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming);
    e->join.resize(n, nullptr);
    for (int i = 0; i < n && er == cudaSuccess; i++) er = cudaEventCreateWithFlags(&e->join[i], cudaEventDisableTiming);
    if (er != cudaSuccess) {
        mg_ensemble_destroy(e);
        return cuerr(er);
    }
    *out = e;
    return MG_OK;
}

extern "C" int mg_ensemble_destroy(mg_ens *e)
{
    if (!e) return MG_ERR_PARAM;
    cudaSetDevice(e->device);
    if (e->stream) cudaStreamSynchronize(e->stream);
    ens_drop_graphs(e);
    for (cudaEvent_t ev : e->join) if (ev) cudaEventDestroy(ev);
    if (e->fork) cudaEventDestroy(e->fork);
    if (e->stream) cudaStreamDestroy(e->stream);
    delete e;
    return MG_OK;
}

// steps [ntime, ntime+nst) of every member, forked from and joined back to e->stream
static cudaError_t ens_issue(mg_ens *e, int ntime, int nst, int *launches)
{
    cudaError_t er = cudaEventRecord(e->fork, e->stream);
    for (size_t i = 0; i < e->m.size() && er == cudaSuccess; i++) {
        mg_ctx *c = e->m[i];
        er = cudaStreamWaitEvent(c->stream, e->fork, 0);
        // the members run side by side and fill the device together: whole columns per CTA
        const int nseg1 = c->k1_nseg, nseg2 = c->k2_nseg;
        c->k1_nseg = 1;
        c->k2_nseg = 1;
        for (int s = 0; s < nst && er == cudaSuccess; s++) er = step_once(c, ntime + s, 0, 0, 0, launches);
        c->k1_nseg = nseg1;
        c->k2_nseg = nseg2;
        if (er == cudaSuccess) er = cudaEventRecord(e->join[i], c->stream);
        if (er == cudaSuccess) er = cudaStreamWaitEvent(e->stream, e->join[i], 0);
    }
    return er;
}

extern "C" int mg_ensemble_step(mg_ens *e, int nsteps, int ntime0)
{
    if (!e || nsteps < 0) return MG_ERR_PARAM;
    for (mg_ctx *c : e->m) {
        if (!c->have_state) return MG_ERR_STATE;
        if (c->prof_on) return MG_ERR_STATE;   // per-kernel events cannot be recorded into the graph
    }
    CKR(cudaSetDevice(e->device));
    long long gsum = 0;
    for (mg_ctx *c : e->m) gsum += c->gen;
    if (gsum != e->gen) {   // a member's step changed since the graphs were recorded
        ens_drop_graphs(e);
        e->gen = gsum;
    }
    if (e->mode == MG_ENS_GROUPED && !ens_groupable(e)) return MG_ERR_PARAM;
    int s = 0;
    while (nsteps - s >= 2) {
        const int par = (ntime0 + s) & 1;
        if (!e->gexec[par]) {
            GroupProgram prog;
            if (e->mode == MG_ENS_GROUPED) {   // tables first: nothing is allocated or copied during the capture
                ens_group_record(e->m, ntime0 + s, prog);
                if (e->gdev[par]) { cudaFree(e->gdev[par]); e->gdev[par] = nullptr; }
                CKR(cudaMalloc(&e->gdev[par], prog.host.size()));
                CKR(cudaMemcpy(e->gdev[par], prog.host.data(), prog.host.size(), cudaMemcpyHostToDevice));
            }
            cudaGraph_t graph;
            CKR(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
            int launches = 0;
            cudaError_t er = cudaSuccess;
            if (e->mode == MG_ENS_GROUPED) {
                for (size_t q = 0; q < prog.ops.size() && er == cudaSuccess; q++) er = prog.ops[q](e->gdev[par], e->stream);
                launches = prog.launches;
            } else {
                er = ens_issue(e, ntime0 + s, 2, &launches);
            }
            cudaError_t er2 = cudaStreamEndCapture(e->stream, &graph);
            if (er2 == cudaSuccess && er != cudaSuccess) cudaGraphDestroy(graph);
            if (er != cudaSuccess) return cuerr(er);
            if (er2 != cudaSuccess) return cuerr(er2);
            er = cudaGraphInstantiate(&e->gexec[par], graph, 0);
            cudaGraphDestroy(graph);
            if (er != cudaSuccess) return cuerr(er);
            e->launches = launches / 2;
        }
        CKR(cudaGraphLaunch(e->gexec[par], e->stream));
        s += 2;
    }
    if (s < nsteps) {
        int launches = 0;
        CKR(ens_issue(e, ntime0 + s, nsteps - s, &launches));
    }
    CKR(cudaStreamSynchronize(e->stream));
    for (mg_ctx *c : e->m) {
        int rc = check_err(c);
        if (rc) return rc;
    }
    return MG_OK;
}

extern "C" int mg_ensemble_time_steps(mg_ens *e, int nsteps, int ntime0, double *ms)
{
    if (!e || nsteps < 0 || !ms) return MG_ERR_PARAM;
    CKR(cudaSetDevice(e->device));
    cudaEvent_t a, b;
    CKR(cudaEventCreate(&a));
    CKR(cudaEventCreate(&b));
    cudaError_t er = cudaEventRecord(a, e->stream);
    int rc = er == cudaSuccess ? mg_ensemble_step(e, nsteps, ntime0) : cuerr(er);
    if (rc == MG_OK) {
        // mg_ensemble_step synchronised its stream; b closes the interval there
        er = cudaEventRecord(b, e->stream);
        if (er == cudaSuccess) er = cudaEventSynchronize(b);
        float f = 0.f;
        if (er == cudaSuccess) er = cudaEventElapsedTime(&f, a, b);
        *ms = f;
        if (er != cudaSuccess) rc = cuerr(er);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return rc;
}

extern "C" int mg_ensemble_launch_count(const mg_ens *e) { return e ? e->launches : -1; }

extern "C" int mg_ensemble_set_mode(mg_ens *e, int mode)
{
    if (!e || (mode != MG_ENS_GROUPED && mode != MG_ENS_STREAMS)) return MG_ERR_PARAM;
    if (mode == MG_ENS_GROUPED && !ens_groupable(e)) return MG_ERR_PARAM;
    if (mode != e->mode) {
        CKR(cudaSetDevice(e->device));
        CKR(cudaStreamSynchronize(e->stream));
        ens_drop_graphs(e);
        e->mode = mode;
    }
    return MG_OK;
}

extern "C" int mg_ensemble_get_mode(const mg_ens *e) { return e ? e->mode : MG_ERR_PARAM; }

extern "C" int mg_synchronize(mg_ctx *c)
{
    if (!c) return MG_ERR_PARAM;
    return cuerr(cudaStreamSynchronize(c->stream));
}

// ---------------- unit-level entry points ----------------
static int ensure_unit(mg_ctx *c, int n)
{
    for (int i = 0; i < n; i++)
        if (!c->unit[i]) {
            cudaError_t e = cudaMalloc(&c->unit[i], c->fbytes);
            if (e != cudaSuccess) return cuerr(e);
            c->bytes += c->fbytes;
        }
    return MG_OK;
}

extern "C" int mg_advection_ac(mg_ctx *c, const double *x, const double *mu, const double *mv, const double *mw, double *xs)
{
    if (!c || !x || !mu || !mv || !mw || !xs) return MG_ERR_PARAM;
    CKR(cudaSetDevice(c->device));
    int rc = ensure_unit(c, 5);
    if (rc) return rc;
    CKR(h2d(c, c->unit[0], x, cudaMemcpyHostToDevice));
    CKR(h2d(c, c->unit[1], mu, cudaMemcpyHostToDevice));
    CKR(h2d(c, c->unit[2], mv, cudaMemcpyHostToDevice));
    CKR(h2d(c, c->unit[3], mw, cudaMemcpyHostToDevice));
    CKR(h2d(c, c->unit[4], xs, cudaMemcpyHostToDevice));
    K1Args a{};
    a.nf = 1; a.dens_first = 0; a.stage = 0; a.mode = 1; a.err = c->derr;
    a.xin[0] = c->unit[0]; a.xold[0] = c->unit[0]; a.xout[0] = c->unit[4];
    a.mw = c->unit[3];
    K1Maps maps;
    const double *xv[1] = {c->unit[0]};
    rc = build_maps(c, xv, 1, c->unit[1], c->unit[2], &maps);
    if (rc) return rc;
    CKR(c->prm.precision == MG_PREC_MIXED ? launch_k1_mixed(c->G, a, maps, c->stream) : launch_k1(c->G, a, maps, c->stream));
    CKR(d2h(c, xs, c->unit[4], cudaMemcpyDeviceToHost));
    return check_err(c);
}

// ---- SGS turbulence diffusion (src/PHYS/subgrid.f90) ----
extern "C" int mg_sgs_profiles(const mg_params *p, const mg_sgs_params *s, double *prof)
{
    if (!p || !s || !prof || p->nz < 5 || !p->fdz0 || !p->pt0 || !p->qv0) return MG_ERR_PARAM;
    sgs_host_profiles(p->nz, p->dx, p->dy, p->dz, p->fdz0, p->pt0, p->qv0, s->anis_k, s->zdec, s->zrough, prof);
    return MG_OK;
}

static int sgs_validate(const mg_sgs_params *s)
{
    if (!s || s->reserved != 0) return MG_ERR_PARAM;
    if (!(std::isfinite(s->diff) && std::isfinite(s->pran) && std::isfinite(s->zdec) && std::isfinite(s->zrough) &&
          std::isfinite(s->min_w)))
        return MG_ERR_PARAM;
    if (s->pran == 0. || s->zdec <= 0. || s->min_w <= 0. || s->zrough < 0.) return MG_ERR_PARAM;
    return MG_OK;
}

extern "C" int mg_set_sgs(mg_ctx *c, const mg_sgs_params *s)
{
    if (!c) return MG_ERR_PARAM;
    int rc = sgs_validate(s);
    if (rc) return rc;
    if (c->G.nz < 5) return MG_ERR_PARAM;
    CKR(cudaSetDevice(c->device));
    c->sgsp = *s;
    c->sgsp.qt0 = nullptr;
    c->sgs_qt0.clear();
    if (s->qt0) c->sgs_qt0.assign(s->qt0, s->qt0 + c->G.nz);
    rc = ensure_sgs(c);
    if (rc) return rc;
    if (s->with_dif)
        for (int f = 1; f < c->nf; f++)
            if (!c->sgsc[f]) {
                CKR(cudaMalloc(&c->sgsc[f], c->fbytes));
                c->bytes += c->fbytes;
                CKR(cudaMemset(c->sgsc[f], 0, c->fbytes));
            }
    c->sgs_on = s->with_dif != 0;
    c->have_fkv = 0;
    drop_graphs(c);
    return MG_OK;
}

extern "C" int mg_set_surface_fluxes(mg_ctx *c, const double *esflux, const double *qvflux, const double *mflux)
{
    if (!c) return MG_ERR_PARAM;
    CKR(cudaSetDevice(c->device));
    int rc = ensure_sgs(c);
    if (rc) return rc;
    const size_t b = (size_t)c->G.nx * c->G.ny * sizeof(double);
    const double *src[3] = {esflux, qvflux, mflux};
    for (int q = 0; q < 3; q++) {
        if (src[q]) CKR(cudaMemcpyAsync(c->sfc[q], src[q], b, cudaMemcpyHostToDevice, c->stream));
        else CKR(cudaMemsetAsync(c->sfc[q], 0, b, c->stream));
    }
    return cuerr(cudaStreamSynchronize(c->stream));
}

// ---- per-step checks and time-step control (src/IO/check.f90) ----
extern "C" int mg_set_dt(mg_ctx *c, double dt0)
{
    if (!c || !std::isfinite(dt0) || !(dt0 > 0.)) return MG_ERR_PARAM;
    if (dt0 == c->G.dt0) return MG_OK;
    CKR(cudaSetDevice(c->device));
    CKR(cudaStreamSynchronize(c->stream));
    c->prm.dt0 = dt0;
    c->G.dt0 = dt0;
    drop_graphs(c);
    return MG_OK;
}

extern "C" int mg_cfl_dt(const mg_check_params *p, double maxcfl, double dt0, double *dt0_new, int *stop)
{
    if (!p || !dt0_new || !stop) return MG_ERR_PARAM;
    *dt0_new = dt0;
    *stop = MG_STOP_NONE;
    if (maxcfl > 2. || maxcfl < 1.e-7) {   // check.f90:191-202
        *stop = MG_STOP_CFL;
        return MG_OK;
    }
    const double dtref = dt0;
    if (maxcfl >= p->cfl_max && p->ldtfix == 0) {   // :208-226
        const double xx = maxcfl / dtref;
        const double fac = 0.95 * p->cfl_max / xx;
        *dt0_new = fac;
        const double lim = p->limit_ts > 1. ? p->limit_ts : 1.;
        if (p->limit_ts > 1. && *dt0_new <= p->dt0_i / lim) *stop = MG_STOP_DT;
    }
    if (maxcfl <= p->cfl_min && maxcfl > 0. && p->ldtfix == 0) {   // :253-264
        const double xx = maxcfl / dtref;
        const double fac = 1.15 * p->cfl_min / xx;
        const double cap = 2. * p->dt0_i;
        *dt0_new = fac < cap ? fac : cap;
    }
    return MG_OK;
}

extern "C" int mg_checkall(mg_ctx *c, const mg_check_params *p, mg_check_result *r)
{
    if (!c || !p || !r) return MG_ERR_PARAM;
    if (!c->have_state) return MG_ERR_STATE;
    CKR(cudaSetDevice(c->device));
    if (!c->chk) {
        CKR(cudaMalloc(&c->chk, check_scratch_bytes()));
        c->bytes += check_scratch_bytes();
    }
    const DevGrid &G = c->G;
    const int iqt = c->prm.iqt >= 0 ? 1 + c->prm.iqt : -1;
    CKR(launch_check(G, c->mA[0], c->mA[1], c->mA[2], c->sA[1], iqt >= 0 ? c->sA[iqt] : nullptr, c->chk, c->stream));
    struct { double v; long long L; } h[6];
    const size_t off = check_scratch_bytes() - sizeof(h);
    CKR(cudaMemcpyAsync(h, (char *)c->chk + off, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
    CKR(cudaStreamSynchronize(c->stream));
    auto ijk = [&](long long L, int *o) {
        if (L == LLONG_MAX) { o[0] = o[1] = o[2] = 0; return; }
        o[0] = 4 + (int)(L % G.maxx);
        const long long rr = L / G.maxx;
        o[1] = 4 + (int)(rr % G.maxy);
        o[2] = 1 + (int)(rr / G.maxy);
    };
    memset(r, 0, sizeof(*r));
    r->maxcfl = h[0].L == LLONG_MAX ? 0. : h[0].v;
    ijk(h[0].L, r->cfl_ijk);
    r->es_max = h[1].v; ijk(h[1].L, r->es_max_ijk);
    r->es_min = h[2].v; ijk(h[2].L, r->es_min_ijk);
    if (iqt >= 0) {
        r->qt_max = h[3].v; ijk(h[3].L, r->qt_max_ijk);
        r->qt_min = h[4].v; ijk(h[4].L, r->qt_min_ijk);
    }
    r->dt0_old = r->dt0_new = G.dt0;
    if (h[5].L != LLONG_MAX) {
        // a non-finite value: reported with its first location, no time-step decision
        r->nonfinite = 1;
        ijk(h[5].L, r->nonfinite_ijk);
        return MG_ERR_NAN;
    }
    // checkall order: checkx(es), checkx(qt), checkwind; the first failing check stops
    if (r->es_max > p->es_max || r->es_min < p->es_min) {
        r->stop = MG_STOP_ES;
    } else if (iqt >= 0 && (r->qt_max > p->qt_max || r->qt_min < p->qt_min)) {
        r->stop = MG_STOP_QT;
    } else {
        int rc = mg_cfl_dt(p, r->maxcfl, G.dt0, &r->dt0_new, &r->stop);
        if (rc) return rc;
        if (p->apply && r->stop == MG_STOP_NONE && r->dt0_new != r->dt0_old) {
            rc = mg_set_dt(c, r->dt0_new);
            if (rc) return rc;
        }
    }
    return MG_OK;
}

extern "C" int mg_selftest_wait(mg_ctx *c, long long limit_cycles)
{
    if (!c || limit_cycles < 0 || limit_cycles > MG_WAIT_CYCLES) return MG_ERR_PARAM;
    CKR(cudaSetDevice(c->device));
    CKR(launch_selftest_wait(limit_cycles, c->derr, c->stream));
    return check_err(c);
}

extern "C" int mg_download_ksgs(mg_ctx *c, double *ksgs)
{
    if (!c || !ksgs) return MG_ERR_PARAM;
    if (!c->sgs_on || !c->have_fkv) return MG_ERR_STATE;
    CKR(cudaSetDevice(c->device));
    CKR(d2h(c, ksgs, c->fkv, cudaMemcpyDeviceToHost));
    CKR(cudaStreamSynchronize(c->stream));
    const DevGrid &G = c->G;
    std::vector<double> prof((size_t)SGS_NPROF * G.nz);
    const mg_params &P = c->prm;
    sgs_host_profiles(G.nz, P.dx, P.dy, P.dz, P.fdz0, P.pt0, P.qv0, c->sgsp.anis_k, c->sgsp.zdec, c->sgsp.zrough,
                      prof.data());
    const double C_k = 0.12;   // shared_turbu.f90:48
    const size_t pl = (size_t)G.nx * G.ny;
    for (int k = 1; k <= G.nz; k++) {
        const double cd = C_k * prof[(size_t)10 * G.nz + k - 1];
        for (size_t q = (size_t)(k - 1) * pl; q < (size_t)k * pl; q++) {
            const double t = ksgs[q] / cd;
            ksgs[q] = t * t;
        }
    }
    return MG_OK;
}

extern "C" int mg_calc_subgrid(mg_ctx *c, const double *u, const double *v, const double *w, const double *es,
                               const double *qt, double *fkv)
{
    if (!c || !u || !v || !w || !es || !fkv) return MG_ERR_PARAM;
    if (c->G.nz < 5) return MG_ERR_PARAM;
    CKR(cudaSetDevice(c->device));
    int rc = ensure_sgs(c);
    if (!rc) rc = ensure_unit(c, 5);
    if (rc) return rc;
    const double *in[5] = {u, v, w, es, qt};
    for (int q = 0; q < 5; q++)
        if (in[q]) CKR(h2d(c, c->unit[q], in[q], cudaMemcpyHostToDevice));
    SgsDij D{};
    for (int q = 0; q < 6; q++) D.d[q] = c->dij[q];
    const SgsVisc O{c->fkv, nullptr, nullptr};
    CKR(launch_sgs_visc(c->G, sgs_dev(c), c->unit[0], c->unit[1], c->unit[2], c->unit[3], qt ? c->unit[4] : nullptr,
                        nullptr, D, O, c->stream));
    double *hf[1] = {c->fkv};
    CKR(launch_halo_fill(c->G, hf, 1, c->stream));
    CKR(d2h(c, fkv, c->fkv, cudaMemcpyDeviceToHost));
    c->have_fkv = 0;   // the buffer no longer holds the step's viscosity
    return cuerr(cudaStreamSynchronize(c->stream));
}

extern "C" int mg_efud(mg_ctx *c, const double *u, const double *v, const double *w, const double *dens,
                       const double *fkv, double *su, double *sv, double *sw)
{
    if (!c || !u || !v || !w || !dens || !fkv || !su || !sv || !sw) return MG_ERR_PARAM;
    if (c->G.nz < 5) return MG_ERR_PARAM;
    CKR(cudaSetDevice(c->device));
    int rc = ensure_sgs(c);
    if (!rc) rc = ensure_unit(c, 8);
    if (rc) return rc;
    const double *in[8] = {u, v, w, dens, fkv, su, sv, sw};
    for (int q = 0; q < 8; q++) CKR(h2d(c, c->unit[q], in[q], cudaMemcpyHostToDevice));
    SgsDij D{};
    for (int q = 0; q < 6; q++) D.d[q] = c->dij[q];
    const SgsDev S = sgs_dev(c);
    CKR(launch_sgs_visc(c->G, S, c->unit[0], c->unit[1], c->unit[2], nullptr, nullptr, nullptr, D, SgsVisc{}, c->stream));
    CKR(launch_halo_fill(c->G, D.d, 6, c->stream));
    CKR(launch_sgs_prep(c->G, S, c->unit[3], c->unit[4], c->sfe, c->snut, c->stream));
    CKR(launch_sgs_mom(c->G, S, c->unit[0], c->unit[1], c->sfe, D, c->sfc[2], c->unit[5], c->unit[6], c->unit[7],
                       c->unit[5], c->unit[6], c->unit[7], c->stream));
    CKR(d2h(c, su, c->unit[5], cudaMemcpyDeviceToHost));
    CKR(d2h(c, sv, c->unit[6], cudaMemcpyDeviceToHost));
    CKR(d2h(c, sw, c->unit[7], cudaMemcpyDeviceToHost));
    return cuerr(cudaStreamSynchronize(c->stream));
}

extern "C" int mg_eff(mg_ctx *c, int kind, const double *dens, const double *fkv, const double *x,
                      const double *flux_s, double *ec)
{
    if (!c || kind < 1 || kind > 3 || !dens || !fkv || !x || !ec) return MG_ERR_PARAM;
    if (c->G.nz < 5) return MG_ERR_PARAM;
    CKR(cudaSetDevice(c->device));
    int rc = ensure_sgs(c);
    if (!rc) rc = ensure_unit(c, 5);
    if (rc) return rc;
    CKR(h2d(c, c->unit[0], dens, cudaMemcpyHostToDevice));
    CKR(h2d(c, c->unit[1], fkv, cudaMemcpyHostToDevice));
    CKR(h2d(c, c->unit[2], x, cudaMemcpyHostToDevice));
    CKR(h2d(c, c->unit[3], ec, cudaMemcpyHostToDevice));
    if (flux_s)
        CKR(cudaMemcpyAsync(c->unit[4], flux_s, (size_t)c->G.nx * c->G.ny * sizeof(double), cudaMemcpyHostToDevice,
                            c->stream));
    SgsScal A{};
    A.nf = 1;
    A.x[0] = c->unit[2];
    A.out[0] = c->unit[3];
    A.x0[0] = kind == 1 ? c->G.pt0 : (kind == 2 ? sgs_qt0_dev(c) : nullptr);
    A.fs[0] = flux_s ? c->unit[4] : nullptr;
    A.fs_neg[0] = 0;
    const SgsDev S = sgs_dev(c);
    CKR(launch_sgs_prep(c->G, S, c->unit[0], c->unit[1], c->sfe, c->snut, c->stream));
    CKR(launch_sgs_scal(c->G, S, c->snut, A, c->stream));
    CKR(d2h(c, ec, c->unit[3], cudaMemcpyDeviceToHost));
    return cuerr(cudaStreamSynchronize(c->stream));
}

// ---- tangent linear and adjoint of the momentum advection operator ----
extern "C" int mg_qnadv_tl(mg_ctx *c, int ntime, const double *mu, const double *mv, const double *mw,
                           const double *dmu, const double *dmv, const double *dmw, double *au, double *av, double *aw,
                           double *dau, double *dav, double *daw)
{
    if (!c || !mu || !mv || !mw || !dmu || !dmv || !dmw || !dau || !dav || !daw) return MG_ERR_PARAM;
    if (c->G.nz < 5) return MG_ERR_PARAM;
    CKR(cudaSetDevice(c->device));
    int rc = ensure_unit(c, 12);
    if (rc) return rc;
    const double *in[6] = {mu, mv, mw, dmu, dmv, dmw};
    for (int q = 0; q < 6; q++) CKR(h2d(c, c->unit[q], in[q], cudaMemcpyHostToDevice));
    for (int q = 6; q < 12; q++) CKR(cudaMemsetAsync(c->unit[q], 0, c->fbytes, c->stream));
    CKR(launch_qnadv_tl(c->G, ntime, c->unit[0], c->unit[1], c->unit[2], c->unit[3], c->unit[4], c->unit[5],
                        au ? c->unit[6] : nullptr, av ? c->unit[7] : nullptr, aw ? c->unit[8] : nullptr, c->unit[9],
                        c->unit[10], c->unit[11], c->stream));
    double *outs[6] = {au, av, aw, dau, dav, daw};
    for (int q = 0; q < 6; q++)
        if (outs[q]) CKR(d2h(c, outs[q], c->unit[6 + q], cudaMemcpyDeviceToHost));
    return cuerr(cudaStreamSynchronize(c->stream));
}

extern "C" int mg_qnadv_ad(mg_ctx *c, int ntime, const double *mu, const double *mv, const double *mw,
                           const double *aubar, const double *avbar, const double *awbar, double *mubar, double *mvbar,
                           double *mwbar)
{
    if (!c || !mu || !mv || !mw || !aubar || !avbar || !awbar || !mubar || !mvbar || !mwbar) return MG_ERR_PARAM;
    if (c->G.nz < 5) return MG_ERR_PARAM;
    CKR(cudaSetDevice(c->device));
    int rc = ensure_unit(c, 9);
    if (rc) return rc;
    const double *in[6] = {mu, mv, mw, aubar, avbar, awbar};
    for (int q = 0; q < 6; q++) CKR(h2d(c, c->unit[q], in[q], cudaMemcpyHostToDevice));
    for (int q = 6; q < 9; q++) CKR(cudaMemsetAsync(c->unit[q], 0, c->fbytes, c->stream));
    (void)ntime;   // the adjoint of the sum of the direction terms does not depend on their order
    CKR(launch_qnadv_ad(c->G, c->unit[0], c->unit[1], c->unit[2], c->unit[3], c->unit[4], c->unit[5], c->unit[6],
                        c->unit[7], c->unit[8], c->stream));
    CKR(d2h(c, mubar, c->unit[6], cudaMemcpyDeviceToHost));
    CKR(d2h(c, mvbar, c->unit[7], cudaMemcpyDeviceToHost));
    CKR(d2h(c, mwbar, c->unit[8], cudaMemcpyDeviceToHost));
    return cuerr(cudaStreamSynchronize(c->stream));
}

// ---------------- trajectory tangent linear and adjoint ----------------
// The FP64 step as a composition the linearisation follows: unit-mode K1 (advection
// tendencies of all scalar fields), unit-mode K2 (qnadv), the stage glue of k_traj.cu
// and the projection; natural <-> stage variables at the ends of the step.  The
// adjoint recomputes each step's two stages from stored step-start states: states are
// checkpointed every ckpt steps, and a segment is recomputed forward before it is
// swept backward.  Scope: FP64 contexts, WENO scalars, SGS diffusion off.
namespace {

struct TrajBufs {
    mg_ctx *c = nullptr;
    std::vector<double *> own;
    cudaError_t err = cudaSuccess;
    double *get()
    {
        double *p = nullptr;
        if (err == cudaSuccess) err = cudaMalloc(&p, c->fbytes);
        if (err == cudaSuccess) err = cudaMemsetAsync(p, 0, c->fbytes, c->stream);
        if (err == cudaSuccess) own.push_back(p);
        return p;
    }
    ~TrajBufs()
    {
        if (c) cudaStreamSynchronize(c->stream);
        for (double *p : own) cudaFree(p);
    }
};

// natural state: m[0..2] = u, v, w; p; s[0] = density, s[1..nf-1] = scalars
struct NatState {
    double *m[3] = {};
    double *p = nullptr;
    double *s[MG_MAXF] = {};
};

// what a stage's tangent linear and adjoint need besides the level-n state
struct StageRec {
    double *xs[MG_MAXF] = {};   // scalar inputs (field 0: density)
    double *xm[3] = {};         // momentum inputs
    double *A[MG_MAXF] = {};    // advection tendencies of the inputs
};

NatState nat_alloc(TrajBufs &B, int nf)
{
    NatState n;
    for (int q = 0; q < 3; q++) n.m[q] = B.get();
    n.p = B.get();
    for (int f = 0; f < nf; f++) n.s[f] = B.get();
    return n;
}

// page-locked host buffers of field size (checkpoints kept off the device)
struct HostBufs {
    size_t bytes = 0;
    std::vector<double *> own;
    cudaError_t err = cudaSuccess;
    double *get()
    {
        double *p = nullptr;
        if (err == cudaSuccess) err = cudaMallocHost(&p, bytes);
        if (err == cudaSuccess) own.push_back(p);
        return p;
    }
    ~HostBufs()
    {
        for (double *p : own) cudaFreeHost(p);
    }
};

NatState nat_alloc_host(HostBufs &H, int nf)
{
    NatState n;
    for (int q = 0; q < 3; q++) n.m[q] = H.get();
    n.p = H.get();
    for (int f = 0; f < nf; f++) n.s[f] = H.get();
    return n;
}

// field-by-field copy on the context stream; either side may be page-locked host memory
// (the direction follows from the unified address space)
cudaError_t nat_copy(mg_ctx *c, const NatState &dst, const NatState &src, int nf)
{
    cudaError_t e = cudaSuccess;
    for (int q = 0; q < 3 && e == cudaSuccess; q++)
        e = cudaMemcpyAsync(dst.m[q], src.m[q], c->fbytes, cudaMemcpyDefault, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dst.p, src.p, c->fbytes, cudaMemcpyDefault, c->stream);
    for (int f = 0; f < nf && e == cudaSuccess; f++)
        e = cudaMemcpyAsync(dst.s[f], src.s[f], c->fbytes, cudaMemcpyDefault, c->stream);
    return e;
}

cudaError_t nat_zero(mg_ctx *c, const NatState &n, int nf)
{
    cudaError_t e = cudaSuccess;
    for (int q = 0; q < 3 && e == cudaSuccess; q++) e = cudaMemsetAsync(n.m[q], 0, c->fbytes, c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(n.p, 0, c->fbytes, c->stream);
    for (int f = 0; f < nf && e == cudaSuccess; f++) e = cudaMemsetAsync(n.s[f], 0, c->fbytes, c->stream);
    return e;
}

}  // namespace

// projection of (mu, mv, mw) with the pressure p, FP64, no diagnostics
static cudaError_t traj_project(mg_ctx *c, double *mu, double *mv, double *mw, double *p)
{
    double *psave = c->p;
    c->p = p;
    int launches = 0;
    cudaError_t e = project(c, mu, mv, mw, mw, -1, 0, 0, 0, &launches);
    c->p = psave;
    return e;
}

// one stage forward from R (xs, xm filled): R.A, tm/ts (in: previous stage's, out: this
// stage's), p (in/out: projected), outputs xs_out, xm_out
static cudaError_t traj_stage_fwd(mg_ctx *c, int ntime, int stage, const NatState &N, StageRec &R, double *const *ts,
                                  double *const *tm, double *p, double *const *xs_out, double *const *xm_out,
                                  double *const *au)
{
    const DevGrid &G = c->G;
    const int nf = c->nf;
    const int iqt = c->prm.iqt >= 0 ? 1 + c->prm.iqt : -1;
    const double a_dt = (stage == 1 ? 1. : 0.5) * G.dt0, b = stage == 1 ? 0. : 1.;
    cudaError_t e = cudaSuccess;
    for (int f = 0; f < nf && e == cudaSuccess; f++) e = cudaMemsetAsync(R.A[f], 0, c->fbytes, c->stream);
    for (int q = 0; q < 3 && e == cudaSuccess; q++) e = cudaMemsetAsync(au[q], 0, c->fbytes, c->stream);
    if (e != cudaSuccess) return e;
    // advection tendencies of every scalar field (K1 unit mode)
    K1Args a1{};
    a1.nf = nf; a1.dens_first = 0; a1.stage = 0; a1.mode = 1; a1.err = c->derr;
    for (int f = 0; f < nf; f++) { a1.xin[f] = R.xs[f]; a1.xold[f] = R.xs[f]; a1.xout[f] = R.A[f]; }
    a1.mw = R.xm[2];
    K1Maps maps;
    const double *xv[MG_MAXF];
    for (int f = 0; f < nf; f++) xv[f] = R.xs[f];
    if (build_maps(c, xv, nf, R.xm[0], R.xm[1], &maps)) return cudaErrorInvalidValue;
    if ((e = launch_k1(G, a1, maps, c->stream)) != cudaSuccess) return e;
    // momentum advection (K2 unit mode)
    K2Args a2{};
    a2.ntime = ntime; a2.mode = 1; a2.in_is_leveln = 0; a2.rep = REP_NAT;
    a2.mu = R.xm[0]; a2.mv = R.xm[1]; a2.mw = R.xm[2];
    a2.ou = au[0]; a2.ov = au[1]; a2.ow = au[2];
    a2.err = c->derr;
    K2Maps mm;
    const double *m3[3] = {R.xm[0], R.xm[1], R.xm[2]};
    if (build_mom_maps(c, m3, &mm)) return cudaErrorInvalidValue;
    if ((e = launch_k2(G, a2, mm, c->stream)) != cudaSuccess) return e;
    // momentum assembly and update
    TrajMomArgs A{};
    A.v[TM_P] = p; A.v[TM_MW] = R.xm[2]; A.v[TM_RHO] = R.xs[0]; A.v[TM_ES] = R.xs[1]; A.v[TM_AES] = R.A[1];
    A.v[TM_QT] = iqt >= 0 ? R.xs[iqt] : nullptr; A.v[TM_AQT] = iqt >= 0 ? R.A[iqt] : nullptr;
    A.v[TM_AU] = au[0]; A.v[TM_AV] = au[1]; A.v[TM_AW] = au[2];
    A.v[TM_TU] = tm[0]; A.v[TM_TV] = tm[1]; A.v[TM_TW] = tm[2];
    A.v[TM_UN] = N.m[0]; A.v[TM_VN] = N.m[1]; A.v[TM_WN] = N.m[2];
    A.out[0] = tm[0]; A.out[1] = tm[1]; A.out[2] = tm[2];
    A.out[3] = xm_out[0]; A.out[4] = xm_out[1]; A.out[5] = xm_out[2];
    A.a_dt = a_dt; A.b = b;
    if ((e = launch_stage_mom(G, A, 0, c->stream)) != cudaSuccess) return e;
    // scalar update
    TrajScalArgs S{};
    S.nf = nf; S.rhon = N.s[0]; S.a_dt = a_dt; S.b = b;
    for (int f = 0; f < nf; f++) {
        S.adv[f] = R.A[f]; S.tprev[f] = ts[f]; S.sn[f] = N.s[f]; S.tout[f] = ts[f]; S.out[f] = xs_out[f];
    }
    if ((e = launch_stage_scal(G, S, 0, c->stream)) != cudaSuccess) return e;
    double *hm[3] = {xm_out[0], xm_out[1], xm_out[2]};
    if ((e = launch_halo_fill(G, hm, 3, c->stream)) != cudaSuccess) return e;
    if ((e = launch_halo_fill(G, xs_out, nf, c->stream)) != cudaSuccess) return e;
    return traj_project(c, xm_out[0], xm_out[1], xm_out[2], p);
}

// natural state -> stage-1 inputs (m = u rho0, psi = s rho; the density itself)
static cudaError_t traj_to_stage(mg_ctx *c, const NatState &N, StageRec &R)
{
    TrajConv V{};
    V.dir = 0; V.ns = c->nf - 1; V.rho = N.s[0];
    for (int q = 0; q < 3; q++) { V.in[q] = N.m[q]; V.out[q] = R.xm[q]; }
    for (int f = 1; f < c->nf; f++) { V.in[2 + f] = N.s[f]; V.out[2 + f] = R.xs[f]; }
    cudaError_t e = launch_convert(c->G, V, 0, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(R.xs[0], N.s[0], c->fbytes, cudaMemcpyDeviceToDevice, c->stream);
    return e;
}

// one step forward: N -> Nout (may alias nothing); R1, R2 receive the stages' records
static cudaError_t traj_step_fwd(mg_ctx *c, int ntime, const NatState &N, const NatState &Nout, StageRec &R1,
                                 StageRec &R2, double *const *ts, double *const *tm, double *const *au)
{
    const int nf = c->nf;
    cudaError_t e = traj_to_stage(c, N, R1);
    if (e == cudaSuccess) e = cudaMemcpyAsync(Nout.p, N.p, c->fbytes, cudaMemcpyDeviceToDevice, c->stream);
    if (e != cudaSuccess) return e;
    if ((e = traj_stage_fwd(c, ntime, 1, N, R1, ts, tm, Nout.p, R2.xs, R2.xm, au)) != cudaSuccess) return e;
    // stage 2 writes its outputs into Nout's buffers (stage variables), converted below
    if ((e = traj_stage_fwd(c, ntime, 2, N, R2, ts, tm, Nout.p, Nout.s, Nout.m, au)) != cudaSuccess) return e;
    TrajConv V{};
    V.dir = 1; V.ns = nf - 1; V.rho = Nout.s[0];
    for (int q = 0; q < 3; q++) { V.in[q] = Nout.m[q]; V.out[q] = Nout.m[q]; }
    for (int f = 1; f < nf; f++) { V.in[2 + f] = Nout.s[f]; V.out[2 + f] = Nout.s[f]; }
    if ((e = launch_convert(c->G, V, 0, c->stream)) != cudaSuccess) return e;
    double *hm[3] = {Nout.m[0], Nout.m[1], Nout.m[2]};
    if ((e = launch_halo_fill(c->G, hm, 3, c->stream)) != cudaSuccess) return e;
    return launch_halo_fill(c->G, Nout.s, nf, c->stream);
}

// tangent of one stage (values of the stage, R and N, computed by traj_stage_fwd first)
static cudaError_t traj_stage_tl(mg_ctx *c, int ntime, int stage, const NatState &N, const NatState &dN,
                                 const StageRec &R, const StageRec &dR, double *const *ts, double *const *dts,
                                 double *const *tm, double *const *dtm, double *p, double *dp,
                                 double *const *dxs_out, double *const *dxm_out, double *const *dau, double *tls)
{
    const DevGrid &G = c->G;
    const int nf = c->nf;
    const int iqt = c->prm.iqt >= 0 ? 1 + c->prm.iqt : -1;
    const double a_dt = (stage == 1 ? 1. : 0.5) * G.dt0, b = stage == 1 ? 0. : 1.;
    cudaError_t e = cudaSuccess;
    for (int f = 0; f < nf && e == cudaSuccess; f++) {
        e = cudaMemsetAsync(dR.A[f], 0, c->fbytes, c->stream);
        if (e == cudaSuccess)
            e = launch_advection_tl(G, R.xs[f], R.xm[0], R.xm[1], R.xm[2], dR.xs[f], dR.xm[0], dR.xm[1], dR.xm[2], dR.A[f], tls,
                                    c->stream);
    }
    for (int q = 0; q < 3 && e == cudaSuccess; q++) e = cudaMemsetAsync(dau[q], 0, c->fbytes, c->stream);
    if (e == cudaSuccess)
        e = launch_qnadv_tl(G, ntime, R.xm[0], R.xm[1], R.xm[2], dR.xm[0], dR.xm[1], dR.xm[2], nullptr, nullptr, nullptr,
                            dau[0], dau[1], dau[2], c->stream);
    if (e != cudaSuccess) return e;
    TrajMomArgs A{};
    A.v[TM_P] = p; A.v[TM_MW] = R.xm[2]; A.v[TM_RHO] = R.xs[0]; A.v[TM_ES] = R.xs[1]; A.v[TM_AES] = R.A[1];
    A.v[TM_QT] = iqt >= 0 ? R.xs[iqt] : nullptr; A.v[TM_AQT] = iqt >= 0 ? R.A[iqt] : nullptr;
    A.v[TM_AU] = dau[0]; A.v[TM_AV] = dau[1]; A.v[TM_AW] = dau[2];   // values unused (linear term)
    A.v[TM_TU] = tm[0]; A.v[TM_TV] = tm[1]; A.v[TM_TW] = tm[2];
    A.v[TM_UN] = N.m[0]; A.v[TM_VN] = N.m[1]; A.v[TM_WN] = N.m[2];
    A.d[TM_P] = dp; A.d[TM_MW] = dR.xm[2]; A.d[TM_RHO] = dR.xs[0]; A.d[TM_ES] = dR.xs[1]; A.d[TM_AES] = dR.A[1];
    A.d[TM_QT] = iqt >= 0 ? dR.xs[iqt] : nullptr; A.d[TM_AQT] = iqt >= 0 ? dR.A[iqt] : nullptr;
    A.d[TM_AU] = dau[0]; A.d[TM_AV] = dau[1]; A.d[TM_AW] = dau[2];
    A.d[TM_TU] = dtm[0]; A.d[TM_TV] = dtm[1]; A.d[TM_TW] = dtm[2];
    A.d[TM_UN] = dN.m[0]; A.d[TM_VN] = dN.m[1]; A.d[TM_WN] = dN.m[2];
    for (int q = 0; q < 3; q++) { A.dout[q] = dtm[q]; A.dout[3 + q] = dxm_out[q]; }
    A.a_dt = a_dt; A.b = b;
    if ((e = launch_stage_mom(G, A, 1, c->stream)) != cudaSuccess) return e;
    TrajScalArgs S{};
    S.nf = nf; S.rhon = N.s[0]; S.drhon = dN.s[0]; S.a_dt = a_dt; S.b = b;
    for (int f = 0; f < nf; f++) {
        S.adv[f] = R.A[f]; S.dadv[f] = dR.A[f]; S.tprev[f] = ts[f]; S.dtprev[f] = dts[f];
        S.sn[f] = N.s[f]; S.dsn[f] = dN.s[f]; S.dtout[f] = dts[f]; S.dout[f] = dxs_out[f];
    }
    if ((e = launch_stage_scal(G, S, 1, c->stream)) != cudaSuccess) return e;
    double *hm[3] = {dxm_out[0], dxm_out[1], dxm_out[2]};
    if ((e = launch_halo_fill(G, hm, 3, c->stream)) != cudaSuccess) return e;
    if ((e = launch_halo_fill(G, dxs_out, nf, c->stream)) != cudaSuccess) return e;
    return traj_project(c, dxm_out[0], dxm_out[1], dxm_out[2], dp);
}

// tangent of one step: (N, dN) -> (Nout, dNout)
static cudaError_t traj_step_tl(mg_ctx *c, int ntime, const NatState &N, const NatState &dN, const NatState &Nout,
                                const NatState &dNout, StageRec &R1, StageRec &R2, StageRec &dR1, StageRec &dR2,
                                double *const *ts, double *const *tm, double *const *dts, double *const *dtm,
                                double *const *au, double *tls)
{
    const int nf = c->nf;
    cudaError_t e = traj_to_stage(c, N, R1);
    if (e != cudaSuccess) return e;
    {
        TrajConv V{};
        V.dir = 0; V.ns = nf - 1; V.rho = N.s[0]; V.drho = dN.s[0];
        for (int q = 0; q < 3; q++) { V.in[q] = N.m[q]; V.din[q] = dN.m[q]; V.dout[q] = dR1.xm[q]; }
        for (int f = 1; f < nf; f++) { V.in[2 + f] = N.s[f]; V.din[2 + f] = dN.s[f]; V.dout[2 + f] = dR1.xs[f]; }
        if ((e = launch_convert(c->G, V, 1, c->stream)) != cudaSuccess) return e;
        if ((e = cudaMemcpyAsync(dR1.xs[0], dN.s[0], c->fbytes, cudaMemcpyDeviceToDevice, c->stream)) != cudaSuccess) return e;
    }
    if ((e = cudaMemcpyAsync(Nout.p, N.p, c->fbytes, cudaMemcpyDeviceToDevice, c->stream)) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(dNout.p, dN.p, c->fbytes, cudaMemcpyDeviceToDevice, c->stream)) != cudaSuccess) return e;
    if ((e = traj_stage_fwd(c, ntime, 1, N, R1, ts, tm, Nout.p, R2.xs, R2.xm, au)) != cudaSuccess) return e;
    if ((e = traj_stage_tl(c, ntime, 1, N, dN, R1, dR1, ts, dts, tm, dtm, Nout.p, dNout.p, dR2.xs, dR2.xm, au, tls)) !=
        cudaSuccess)
        return e;
    if ((e = traj_stage_fwd(c, ntime, 2, N, R2, ts, tm, Nout.p, Nout.s, Nout.m, au)) != cudaSuccess) return e;
    if ((e = traj_stage_tl(c, ntime, 2, N, dN, R2, dR2, ts, dts, tm, dtm, Nout.p, dNout.p, dNout.s, dNout.m, au, tls)) !=
        cudaSuccess)
        return e;
    // natural variables: tangent first (it needs the stage values), then the values
    TrajConv V{};
    V.dir = 1; V.ns = nf - 1; V.rho = Nout.s[0]; V.drho = dNout.s[0];
    for (int q = 0; q < 3; q++) { V.in[q] = Nout.m[q]; V.din[q] = dNout.m[q]; V.dout[q] = dNout.m[q]; }
    for (int f = 1; f < nf; f++) { V.in[2 + f] = Nout.s[f]; V.din[2 + f] = dNout.s[f]; V.dout[2 + f] = dNout.s[f]; }
    if ((e = launch_convert(c->G, V, 1, c->stream)) != cudaSuccess) return e;
    for (int q = 0; q < 3; q++) { V.out[q] = Nout.m[q]; V.dout[q] = nullptr; }
    for (int f = 1; f < nf; f++) { V.out[2 + f] = Nout.s[f]; V.dout[2 + f] = nullptr; }
    TrajConv W{};
    W.dir = 1; W.ns = nf - 1; W.rho = Nout.s[0];
    for (int q = 0; q < 3; q++) { W.in[q] = Nout.m[q]; W.out[q] = Nout.m[q]; }
    for (int f = 1; f < nf; f++) { W.in[2 + f] = Nout.s[f]; W.out[2 + f] = Nout.s[f]; }
    if ((e = launch_convert(c->G, W, 0, c->stream)) != cudaSuccess) return e;
    double *hm[3] = {dNout.m[0], dNout.m[1], dNout.m[2]};
    if ((e = launch_halo_fill(c->G, hm, 3, c->stream)) != cudaSuccess) return e;
    double *hv[3] = {Nout.m[0], Nout.m[1], Nout.m[2]};
    if ((e = launch_halo_fill(c->G, hv, 3, c->stream)) != cudaSuccess) return e;
    if ((e = launch_halo_fill(c->G, dNout.s, nf, c->stream)) != cudaSuccess) return e;
    return launch_halo_fill(c->G, Nout.s, nf, c->stream);
}

// adjoint of one stage; bars of the stage outputs (xm_bar after the projection, xs_bar) and
// p_bar in; bars of the stage inputs (xs_in_bar, xm_in_bar, zeroed here) out, p_bar in place,
// level-n bars Nbar accumulated, carries tcarry_in (from the later stage) / tcarry_out
struct StageAdWork {
    double *abar[3];
    double *Abar[MG_MAXF];
};

static cudaError_t traj_stage_ad(mg_ctx *c, int ntime, int stage, const NatState &N, const NatState &Nbar,
                                 const StageRec &R, double *const *xm_bar, double *const *xs_bar, double *p_bar,
                                 double *const *xm_in_bar, double *const *xs_in_bar, double *const *tm_in,
                                 double *const *ts_in, double *const *tm_out, double *const *ts_out, StageAdWork &W)
{
    const DevGrid &G = c->G;
    const int nf = c->nf;
    const int iqt = c->prm.iqt >= 0 ? 1 + c->prm.iqt : -1;
    const double a_dt = (stage == 1 ? 1. : 0.5) * G.dt0, b = stage == 1 ? 0. : 1.;
    cudaError_t e = pressure_adjoint(G, c->pp, c->prm.nsubp, xm_bar[0], xm_bar[1], xm_bar[2], p_bar, c->stream);
    for (int q = 0; q < 3 && e == cudaSuccess; q++) {
        e = cudaMemsetAsync(W.abar[q], 0, c->fbytes, c->stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(xm_in_bar[q], 0, c->fbytes, c->stream);
    }
    for (int f = 0; f < nf && e == cudaSuccess; f++) {
        e = cudaMemsetAsync(W.Abar[f], 0, c->fbytes, c->stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(xs_in_bar[f], 0, c->fbytes, c->stream);
    }
    if (e != cudaSuccess) return e;
    TrajMomAd M{};
    for (int q = 0; q < 3; q++) {
        M.mbar[q] = xm_bar[q]; M.tcarry[q] = tm_in ? tm_in[q] : nullptr; M.tprev_bar[q] = tm_out ? tm_out[q] : nullptr;
        M.abar[q] = W.abar[q]; M.mnbar[q] = Nbar.m[q];
    }
    M.pbar = p_bar; M.mwin_bar = xm_in_bar[2];
    M.rho = R.xs[0]; M.es = R.xs[1]; M.aes = R.A[1];
    M.qt = iqt >= 0 ? R.xs[iqt] : nullptr; M.aqt = iqt >= 0 ? R.A[iqt] : nullptr;
    M.rho_bar = xs_in_bar[0]; M.es_bar = xs_in_bar[1]; M.aes_bar = W.Abar[1];
    M.qt_bar = iqt >= 0 ? xs_in_bar[iqt] : nullptr; M.aqt_bar = iqt >= 0 ? W.Abar[iqt] : nullptr;
    M.a_dt = a_dt; M.b = b;
    if ((e = launch_stage_mom_ad(G, M, c->stream)) != cudaSuccess) return e;
    if ((e = launch_qnadv_ad(G, R.xm[0], R.xm[1], R.xm[2], W.abar[0], W.abar[1], W.abar[2], xm_in_bar[0], xm_in_bar[1],
                             xm_in_bar[2], c->stream)) != cudaSuccess)
        return e;
    TrajScalAd S{};
    S.nf = nf; S.rhon = N.s[0]; S.a_dt = a_dt; S.b = b;
    for (int f = 0; f < nf; f++) {
        S.psibar[f] = xs_bar[f]; S.tcarry[f] = ts_in ? ts_in[f] : nullptr; S.sn[f] = N.s[f];
        S.advbar[f] = W.Abar[f]; S.tprev_bar[f] = ts_out ? ts_out[f] : nullptr; S.snbar[f] = Nbar.s[f];
    }
    if ((e = launch_stage_scal_ad(G, S, c->stream)) != cudaSuccess) return e;
    // each field's advection adjoint adds onto the stage-input bars directly (their ghost
    // cells are zero: every other contribution above writes the interior only)
    for (int f = 0; f < nf; f++)
        if ((e = launch_advection_ad(G, R.xs[f], R.xm[0], R.xm[1], R.xm[2], W.Abar[f], xs_in_bar[f], xm_in_bar[0],
                                     xm_in_bar[1], xm_in_bar[2], c->stream, 1)) != cudaSuccess)
            return e;
    return cudaSuccess;
}

struct StepAdWork {
    StageAdWork W;
    double *xm2b[3], *xs2b[MG_MAXF], *xm1b[3], *xs1b[MG_MAXF], *xm0b[3], *xs0b[MG_MAXF], *pb;
    double *tmc[3], *tsc[MG_MAXF];
};

// adjoint of one step: bar holds N_out-bar on entry and N-bar on exit; Nout = the step's
// forward result from N (natural), R1/R2 its stage records
static cudaError_t traj_step_ad(mg_ctx *c, int ntime, const NatState &N, const NatState &Nout, const StageRec &R1,
                                const StageRec &R2, const NatState &bar, StepAdWork &S)
{
    const DevGrid &G = c->G;
    const int nf = c->nf;
    cudaError_t e = cudaSuccess;
    // natural outputs -> stage-2 output bars
    for (int q = 0; q < 3 && e == cudaSuccess; q++) e = cudaMemsetAsync(S.xm2b[q], 0, c->fbytes, c->stream);
    for (int f = 1; f < nf && e == cudaSuccess; f++) e = cudaMemsetAsync(S.xs2b[f], 0, c->fbytes, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(S.xs2b[0], bar.s[0], c->fbytes, cudaMemcpyDeviceToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(S.pb, bar.p, c->fbytes, cudaMemcpyDeviceToDevice, c->stream);
    if (e != cudaSuccess) return e;
    {
        TrajConvAd V{};
        V.dir = 1; V.ns = nf - 1; V.rho = Nout.s[0]; V.rhobar = S.xs2b[0];
        for (int q = 0; q < 3; q++) { V.outbar[q] = bar.m[q]; V.inbar[q] = S.xm2b[q]; }
        for (int f = 1; f < nf; f++) { V.outbar[2 + f] = bar.s[f]; V.in[2 + f] = Nout.s[f]; V.inbar[2 + f] = S.xs2b[f]; }
        if ((e = launch_convert_ad(G, V, c->stream)) != cudaSuccess) return e;
    }
    if ((e = nat_zero(c, bar, nf)) != cudaSuccess) return e;
    if ((e = traj_stage_ad(c, ntime, 2, N, bar, R2, S.xm2b, S.xs2b, S.pb, S.xm1b, S.xs1b, nullptr, nullptr, S.tmc, S.tsc,
                           S.W)) != cudaSuccess)
        return e;
    if ((e = traj_stage_ad(c, ntime, 1, N, bar, R1, S.xm1b, S.xs1b, S.pb, S.xm0b, S.xs0b, S.tmc, S.tsc, nullptr, nullptr,
                           S.W)) != cudaSuccess)
        return e;
    // stage-1 inputs from the natural state
    if ((e = launch_axpy(G, bar.s[0], S.xs0b[0], 1., c->stream)) != cudaSuccess) return e;
    {
        TrajConvAd V{};
        V.dir = 0; V.ns = nf - 1; V.rho = N.s[0]; V.rhobar = bar.s[0];
        for (int q = 0; q < 3; q++) { V.outbar[q] = S.xm0b[q]; V.inbar[q] = bar.m[q]; }
        for (int f = 1; f < nf; f++) { V.outbar[2 + f] = S.xs0b[f]; V.in[2 + f] = N.s[f]; V.inbar[2 + f] = bar.s[f]; }
        if ((e = launch_convert_ad(G, V, c->stream)) != cudaSuccess) return e;
    }
    return launch_axpy(G, bar.p, S.pb, 1., c->stream);
}

static int traj_check(mg_ctx *c)
{
    if (!c) return MG_ERR_PARAM;
    if (!c->have_state) return MG_ERR_STATE;
    if (c->prm.precision != MG_PREC_FP64 || c->prm.scal_adv != MG_WENO || c->sgs_on || c->G.nz < 5) return MG_ERR_PARAM;
    return MG_OK;
}

static NatState traj_resident(mg_ctx *c)
{
    NatState n;
    for (int q = 0; q < 3; q++) n.m[q] = c->mA[q];
    n.p = c->p;
    for (int f = 0; f < c->nf; f++) n.s[f] = c->sA[f];
    return n;
}

static cudaError_t nat_h2d(mg_ctx *c, const NatState &n, const double *const *h)
{
    cudaError_t e = cudaSuccess;
    for (int q = 0; q < 3 && e == cudaSuccess; q++) e = h2d(c, n.m[q], h[q], cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = h2d(c, n.p, h[3], cudaMemcpyHostToDevice);
    for (int f = 0; f < c->nf && e == cudaSuccess; f++) e = h2d(c, n.s[f], h[4 + f], cudaMemcpyHostToDevice);
    return e;
}

static cudaError_t nat_d2h(mg_ctx *c, double *const *h, const NatState &n)
{
    cudaError_t e = cudaSuccess;
    for (int q = 0; q < 3 && e == cudaSuccess; q++) e = d2h(c, h[q], n.m[q], cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = d2h(c, h[3], n.p, cudaMemcpyDeviceToHost);
    for (int f = 0; f < c->nf && e == cudaSuccess; f++) e = d2h(c, h[4 + f], n.s[f], cudaMemcpyDeviceToHost);
    return e;
}

struct TrajCtx {
    TrajBufs B;
    StageRec R1, R2, dR1, dR2;
    double *ts[MG_MAXF], *tm[3], *dts[MG_MAXF], *dtm[3], *au[3], *tls = nullptr;
    void init(mg_ctx *c, bool tangent)
    {
        B.c = c;
        const int nf = c->nf;
        for (StageRec *R : {&R1, &R2}) {
            for (int f = 0; f < nf; f++) { R->xs[f] = B.get(); R->A[f] = B.get(); }
            for (int q = 0; q < 3; q++) R->xm[q] = B.get();
        }
        for (int f = 0; f < nf; f++) ts[f] = B.get();
        for (int q = 0; q < 3; q++) { tm[q] = B.get(); au[q] = B.get(); }
        if (tangent) {
            for (StageRec *R : {&dR1, &dR2}) {
                for (int f = 0; f < nf; f++) { R->xs[f] = B.get(); R->A[f] = B.get(); }
                for (int q = 0; q < 3; q++) R->xm[q] = B.get();
            }
            for (int f = 0; f < nf; f++) dts[f] = B.get();
            for (int q = 0; q < 3; q++) dtm[q] = B.get();
            tls = B.get();   // face tangents of the advection TL
        }
    }
};

// CUDA-event timer around a device-resident section (ms stays untouched when null)
struct TrajTimer {
    cudaStream_t s;
    float *ms;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t start()
    {
        if (!ms) return cudaSuccess;
        cudaError_t e = cudaEventCreate(&e0);
        if (e == cudaSuccess) e = cudaEventCreate(&e1);
        if (e == cudaSuccess) e = cudaEventRecord(e0, s);
        return e;
    }
    cudaError_t stop()
    {
        if (!ms) return cudaSuccess;
        cudaError_t e = cudaEventRecord(e1, s);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        if (e == cudaSuccess) e = cudaEventElapsedTime(ms, e0, e1);
        return e;
    }
    ~TrajTimer()
    {
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
    }
};

// nsteps of the composition from the resident state; written back when writeback
static int traj_forward_run(mg_ctx *c, int nsteps, int ntime0, bool writeback, float *ms)
{
    TrajCtx T;
    T.init(c, false);
    const NatState res = traj_resident(c);
    NatState a = nat_alloc(T.B, c->nf), b = nat_alloc(T.B, c->nf);
    CKR(T.B.err);
    CKR(nat_copy(c, a, res, c->nf));
    TrajTimer tm{c->stream, ms};
    CKR(tm.start());
    for (int s = 0; s < nsteps; s++) {
        CKR(traj_step_fwd(c, ntime0 + s, a, b, T.R1, T.R2, T.ts, T.tm, T.au));
        std::swap(a, b);
    }
    CKR(tm.stop());
    if (writeback) {
        CKR(nat_copy(c, res, a, c->nf));
        c->rep = REP_NAT;
    }
    return cuerr(cudaStreamSynchronize(c->stream));
}

// tangent linear of nsteps; dx0 == nullptr starts from a copy of the resident state (timing)
static int traj_tl_run(mg_ctx *c, int nsteps, int ntime0, const double *const *dx0, double *const *dxT, float *ms)
{
    TrajCtx T;
    T.init(c, true);
    NatState a = nat_alloc(T.B, c->nf), b = nat_alloc(T.B, c->nf), da = nat_alloc(T.B, c->nf), db = nat_alloc(T.B, c->nf);
    CKR(T.B.err);
    CKR(nat_copy(c, a, traj_resident(c), c->nf));
    if (dx0) CKR(nat_h2d(c, da, dx0));
    else CKR(nat_copy(c, da, traj_resident(c), c->nf));
    TrajTimer tm{c->stream, ms};
    CKR(tm.start());
    for (int s = 0; s < nsteps; s++) {
        CKR(traj_step_tl(c, ntime0 + s, a, da, b, db, T.R1, T.R2, T.dR1, T.dR2, T.ts, T.tm, T.dts, T.dtm, T.au, T.tls));
        std::swap(a, b);
        std::swap(da, db);
    }
    CKR(tm.stop());
    if (dxT) CKR(nat_d2h(c, dxT, da));
    return cuerr(cudaStreamSynchronize(c->stream));
}

// adjoint of nsteps with checkpoints every ckpt steps; lamT == nullptr seeds the adjoint
// with a copy of the resident state (timing).  bytes: device memory the run held.
static int traj_adjoint_run(mg_ctx *c, int nsteps, int ntime0, int ckpt, const double *const *lamT,
                            double *const *g0, float *ms, double *bytes)
{
    const int nf = c->nf;
    TrajCtx T;
    T.init(c, false);
    StepAdWork S{};
    for (int q = 0; q < 3; q++) {
        S.W.abar[q] = T.B.get(); S.xm2b[q] = T.B.get(); S.xm1b[q] = T.B.get(); S.xm0b[q] = T.B.get(); S.tmc[q] = T.B.get();
    }
    for (int f = 0; f < nf; f++) {
        S.W.Abar[f] = T.B.get(); S.xs2b[f] = T.B.get(); S.xs1b[f] = T.B.get(); S.xs0b[f] = T.B.get(); S.tsc[f] = T.B.get();
    }
    S.pb = T.B.get();
    // checkpoints (natural states every ckpt steps) and the states of one segment; the
    // checkpoints go to page-locked host memory when asked, or (auto) when on the device
    // they would take more than a quarter of the free memory.  Kernels never read them in
    // place: they are copied to and from device work states, so both places give the same
    // gradient bit for bit.
    const int nck = nsteps / ckpt + 1;
    const int nseg = std::max(1, std::min(ckpt, nsteps));   // steps of the longest segment
    size_t mfree = 0, mtot = 0;
    CKR(T.B.err);
    CKR(cudaMemGetInfo(&mfree, &mtot));
    const double ck_bytes = (double)nck * (4 + nf) * (double)c->fbytes;
    const bool ck_host = c->traj_ck_where == MG_CKPT_HOST || (c->traj_ck_where == MG_CKPT_AUTO && ck_bytes > 0.25 * (double)mfree);
    HostBufs H;
    H.bytes = c->fbytes;
    std::vector<NatState> ck(nck), seg(nseg + 1);
    for (int q = 0; q < nck; q++) ck[q] = ck_host ? nat_alloc_host(H, nf) : nat_alloc(T.B, nf);
    if (H.err != cudaSuccess) return cuerr(H.err);
    for (int q = 0; q <= nseg; q++) seg[q] = nat_alloc(T.B, nf);
    NatState bar = nat_alloc(T.B, nf), tmp = nat_alloc(T.B, nf);
    // the stage records of every step of a segment, when they fit in half the free memory:
    // the segment's forward recomputation then leaves them for its backward sweep;
    // otherwise each backward step recomputes its own stages
    CKR(T.B.err);
    CKR(cudaMemGetInfo(&mfree, &mtot));
    const double rec_bytes = (double)nseg * 2 * (2 * nf + 3) * (double)c->fbytes;
    const bool keep = rec_bytes < 0.5 * (double)mfree && (c->traj_rec_limit < 0. || rec_bytes <= c->traj_rec_limit);
    std::vector<StageRec> rec1(keep ? nseg : 0), rec2(keep ? nseg : 0);
    for (int q = 0; keep && q < nseg; q++)
        for (StageRec *R : {&rec1[q], &rec2[q]}) {
            for (int f = 0; f < nf; f++) { R->xs[f] = T.B.get(); R->A[f] = T.B.get(); }
            for (int m = 0; m < 3; m++) R->xm[m] = T.B.get();
        }
    CKR(T.B.err);
    if (bytes) *bytes = (double)T.B.own.size() * (double)c->fbytes;
    CKR(nat_copy(c, ck[0], traj_resident(c), nf));
    if (lamT) CKR(nat_h2d(c, bar, lamT));
    else CKR(nat_copy(c, bar, traj_resident(c), nf));
    TrajTimer tm{c->stream, ms};
    CKR(tm.start());
    // forward sweep: keep every ckpt-th state; with the records kept, the last segment (the
    // first swept backward) keeps its states and records here and is not recomputed.  The
    // steps run between two device work states (tmp, seg[1]), from which each checkpoint
    // is copied out.
    const int s0_last = nsteps > 0 ? ((nsteps - 1) / ckpt) * ckpt : 0;
    NatState cur = tmp, nxt = seg[std::min(1, nseg)];
    CKR(nat_copy(c, cur, ck[0], nf));
    for (int s = 0; s < nsteps; s++) {
        if (keep && s >= s0_last) {
            if (s == s0_last) CKR(nat_copy(c, seg[0], cur, nf));
            CKR(traj_step_fwd(c, ntime0 + s, seg[s - s0_last], seg[s - s0_last + 1], rec1[s - s0_last],
                              rec2[s - s0_last], T.ts, T.tm, T.au));
            continue;
        }
        CKR(traj_step_fwd(c, ntime0 + s, cur, nxt, T.R1, T.R2, T.ts, T.tm, T.au));
        std::swap(cur, nxt);
        if ((s + 1) % ckpt == 0) CKR(nat_copy(c, ck[(s + 1) / ckpt], cur, nf));
    }
    for (int s0 = s0_last; nsteps > 0 && s0 >= 0; s0 -= ckpt) {
        const int s1 = std::min(s0 + ckpt, nsteps);
        if (keep) {
            if (s0 != s0_last) {   // the segment's states and stage records
                CKR(nat_copy(c, seg[0], ck[s0 / ckpt], nf));
                for (int s = s0; s < s1; s++)
                    CKR(traj_step_fwd(c, ntime0 + s, seg[s - s0], seg[s - s0 + 1], rec1[s - s0], rec2[s - s0], T.ts,
                                      T.tm, T.au));
            }
            for (int s = s1 - 1; s >= s0; s--)
                CKR(traj_step_ad(c, ntime0 + s, seg[s - s0], seg[s - s0 + 1], rec1[s - s0], rec2[s - s0], bar, S));
            continue;
        }
        CKR(nat_copy(c, seg[0], ck[s0 / ckpt], nf));
        for (int s = s0; s < s1 - 1; s++)   // states at the starts of the segment's steps
            CKR(traj_step_fwd(c, ntime0 + s, seg[s - s0], seg[s - s0 + 1], T.R1, T.R2, T.ts, T.tm, T.au));
        for (int s = s1 - 1; s >= s0; s--) {
            // this step's stage records and output, then its adjoint
            CKR(traj_step_fwd(c, ntime0 + s, seg[s - s0], tmp, T.R1, T.R2, T.ts, T.tm, T.au));
            CKR(traj_step_ad(c, ntime0 + s, seg[s - s0], tmp, T.R1, T.R2, bar, S));
        }
    }
    CKR(tm.stop());
    if (g0) CKR(nat_d2h(c, g0, bar));
    return cuerr(cudaStreamSynchronize(c->stream));
}

extern "C" int mg_traj_forward(mg_ctx *c, int nsteps, int ntime0)
{
    int rc = traj_check(c);
    if (rc) return rc;
    if (nsteps < 0) return MG_ERR_PARAM;
    CKR(cudaSetDevice(c->device));
    return traj_forward_run(c, nsteps, ntime0, true, nullptr);
}

extern "C" int mg_traj_tl(mg_ctx *c, int nsteps, int ntime0, const double *const *dx0, double *const *dxT)
{
    int rc = traj_check(c);
    if (rc) return rc;
    if (nsteps < 0 || !dx0 || !dxT) return MG_ERR_PARAM;
    CKR(cudaSetDevice(c->device));
    return traj_tl_run(c, nsteps, ntime0, dx0, dxT, nullptr);
}

extern "C" int mg_traj_adjoint(mg_ctx *c, int nsteps, int ntime0, int ckpt, const double *const *lamT, double *const *g0)
{
    int rc = traj_check(c);
    if (rc) return rc;
    if (nsteps < 0 || ckpt < 1 || !lamT || !g0) return MG_ERR_PARAM;
    CKR(cudaSetDevice(c->device));
    return traj_adjoint_run(c, nsteps, ntime0, ckpt, lamT, g0, nullptr, nullptr);
}

extern "C" int mg_traj_checkpoints(mg_ctx *c, int where)
{
    if (!c || where < MG_CKPT_AUTO || where > MG_CKPT_HOST) return MG_ERR_PARAM;
    c->traj_ck_where = where;
    return MG_OK;
}

extern "C" int mg_traj_record_limit(mg_ctx *c, double bytes)
{
    if (!c || bytes != bytes) return MG_ERR_PARAM;
    c->traj_rec_limit = bytes;
    return MG_OK;
}

// device times (ms) of nsteps of the trajectory forward composition, its tangent linear and
// its checkpointed adjoint (forward sweep, segment recomputation and backward sweep), from
// the resident state, which is left unchanged; out[3] = device bytes the adjoint held
extern "C" int mg_time_traj(mg_ctx *c, int nsteps, int ntime0, int ckpt, double *out)
{
    int rc = traj_check(c);
    if (rc) return rc;
    if (nsteps < 1 || ckpt < 1 || !out) return MG_ERR_PARAM;
    CKR(cudaSetDevice(c->device));
    float t[3] = {0.f, 0.f, 0.f};
    if ((rc = traj_forward_run(c, nsteps, ntime0, false, &t[0]))) return rc;
    if ((rc = traj_tl_run(c, nsteps, ntime0, nullptr, nullptr, &t[1]))) return rc;
    if ((rc = traj_adjoint_run(c, nsteps, ntime0, ckpt, nullptr, nullptr, &t[2], &out[3]))) return rc;
    for (int q = 0; q < 3; q++) out[q] = t[q];
    return check_err(c);
}

// ---- tangent linear and adjoint of the scalar advection operator (WENO) ----
extern "C" int mg_advection_tl(mg_ctx *c, const double *x, const double *mu, const double *mv, const double *mw,
                               const double *dx, const double *dmu, const double *dmv, const double *dmw, double *dA)
{
    if (!c || !x || !mu || !mv || !mw || !dx || !dmu || !dmv || !dmw || !dA) return MG_ERR_PARAM;
    if (c->prm.scal_adv != MG_WENO) return MG_ERR_PARAM;
    CKR(cudaSetDevice(c->device));
    int rc = ensure_unit(c, 10);
    if (rc) return rc;
    const double *in[8] = {x, mu, mv, mw, dx, dmu, dmv, dmw};
    for (int q = 0; q < 8; q++) CKR(h2d(c, c->unit[q], in[q], cudaMemcpyHostToDevice));
    CKR(cudaMemsetAsync(c->unit[8], 0, c->fbytes, c->stream));
    CKR(launch_advection_tl(c->G, c->unit[0], c->unit[1], c->unit[2], c->unit[3], c->unit[4], c->unit[5], c->unit[6],
                            c->unit[7], c->unit[8], c->unit[9], c->stream));
    CKR(d2h(c, dA, c->unit[8], cudaMemcpyDeviceToHost));
    return cuerr(cudaStreamSynchronize(c->stream));
}

extern "C" int mg_advection_ad(mg_ctx *c, const double *x, const double *mu, const double *mv, const double *mw,
                               const double *Abar, double *xbar, double *mubar, double *mvbar, double *mwbar)
{
    if (!c || !x || !mu || !mv || !mw || !Abar || !xbar || !mubar || !mvbar || !mwbar) return MG_ERR_PARAM;
    if (c->prm.scal_adv != MG_WENO) return MG_ERR_PARAM;
    CKR(cudaSetDevice(c->device));
    int rc = ensure_unit(c, 9);
    if (rc) return rc;
    const double *in[5] = {x, mu, mv, mw, Abar};
    for (int q = 0; q < 5; q++) CKR(h2d(c, c->unit[q], in[q], cudaMemcpyHostToDevice));
    CKR(launch_advection_ad(c->G, c->unit[0], c->unit[1], c->unit[2], c->unit[3], c->unit[4], c->unit[5], c->unit[6],
                            c->unit[7], c->unit[8], c->stream));
    double *outs[4] = {xbar, mubar, mvbar, mwbar};
    for (int q = 0; q < 4; q++) CKR(d2h(c, outs[q], c->unit[5 + q], cudaMemcpyDeviceToHost));
    return cuerr(cudaStreamSynchronize(c->stream));
}

// ---- adjoint of the projection (anelastic_pressure, FP64 contexts) ----
extern "C" int mg_anelastic_pressure_ad(mg_ctx *c, double *mub, double *mvb, double *mwb, double *pb)
{
    if (!c || !mub || !mvb || !mwb || !pb) return MG_ERR_PARAM;
    if (c->prm.precision != MG_PREC_FP64) return MG_ERR_PARAM;
    CKR(cudaSetDevice(c->device));
    int rc = ensure_unit(c, 4);
    if (rc) return rc;
    double *io[4] = {mub, mvb, mwb, pb};
    for (int q = 0; q < 4; q++) CKR(h2d(c, c->unit[q], io[q], cudaMemcpyHostToDevice));
    CKR(pressure_adjoint(c->G, c->pp, c->prm.nsubp, c->unit[0], c->unit[1], c->unit[2], c->unit[3], c->stream));
    for (int q = 0; q < 4; q++) CKR(d2h(c, io[q], c->unit[q], cudaMemcpyDeviceToHost));
    return cuerr(cudaStreamSynchronize(c->stream));
}

// ---- device time of the operators and their adjoints on the resident state ----
// out[0]: advection (unit K1 on one field), out[1]: its tangent linear, out[2]: its
// adjoint, out[3]: anelastic_pressure (nsubp passes + cal_p1), out[4]: its adjoint; ms per
// call, averaged over reps after one untimed call of each.  The operands are copies of
// the resident state (density-weighted first scalar, momentum); FP64 contexts, WENO.
extern "C" int mg_time_adjoint(mg_ctx *c, int reps, double *out)
{
    if (!c || reps < 1 || !out) return MG_ERR_PARAM;
    if (!c->have_state) return MG_ERR_STATE;
    if (c->prm.precision != MG_PREC_FP64 || c->prm.scal_adv != MG_WENO) return MG_ERR_PARAM;
    CKR(cudaSetDevice(c->device));
    int rc = ensure_unit(c, 10);
    if (rc) return rc;
    const size_t fb = c->fbytes;
    double **u = c->unit;
    // x, mu, mv, mw from the state; dx, dm = the same fields (any perturbation costs the same)
    CKR(cudaMemcpyAsync(u[0], c->sA[c->nf > 1 ? 1 : 0], fb, cudaMemcpyDeviceToDevice, c->stream));
    for (int q = 0; q < 3; q++) CKR(cudaMemcpyAsync(u[1 + q], c->mA[q], fb, cudaMemcpyDeviceToDevice, c->stream));
    for (int q = 0; q < 4; q++) CKR(cudaMemcpyAsync(u[4 + q], u[q], fb, cudaMemcpyDeviceToDevice, c->stream));
    K1Args a{};
    a.nf = 1; a.stage = 0; a.mode = 1; a.err = c->derr;
    a.xin[0] = u[0]; a.xold[0] = u[0]; a.xout[0] = u[8]; a.mw = u[3];
    K1Maps maps;
    const double *xv[1] = {u[0]};
    rc = build_maps(c, xv, 1, u[1], u[2], &maps);
    if (rc) return rc;
    auto run = [&](int which) -> cudaError_t {
        int launches = 0;
        switch (which) {
        case 0: return launch_k1(c->G, a, maps, c->stream);
        case 1: return launch_advection_tl(c->G, u[0], u[1], u[2], u[3], u[4], u[5], u[6], u[7], u[8], u[9], c->stream);
        case 2: return launch_advection_ad(c->G, u[0], u[1], u[2], u[3], u[8], u[4], u[5], u[6], u[7], c->stream);
        case 3: return project(c, u[4], u[5], u[6], u[7], -1, 0, 0, 0, &launches);
        default: return pressure_adjoint(c->G, c->pp, c->prm.nsubp, u[4], u[5], u[6], u[7], c->stream);
        }
    };
    cudaEvent_t e0, e1;
    CKR(cudaEventCreate(&e0));
    CKR(cudaEventCreate(&e1));
    cudaError_t er = cudaSuccess;
    for (int w = 0; w < 5 && er == cudaSuccess; w++) {
        er = run(w);   // untimed (the adjoint of the projection builds its transposed system here)
        if (er == cudaSuccess) er = cudaEventRecord(e0, c->stream);
        for (int r = 0; r < reps && er == cudaSuccess; r++) er = run(w);
        if (er == cudaSuccess) er = cudaEventRecord(e1, c->stream);
        if (er == cudaSuccess) er = cudaEventSynchronize(e1);
        float f = 0.f;
        if (er == cudaSuccess) er = cudaEventElapsedTime(&f, e0, e1);
        out[w] = f / reps;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (er != cudaSuccess) return cuerr(er);
    return check_err(c);
}

extern "C" int mg_qnadv_uvw(mg_ctx *c, int ntime, const double *mu, const double *mv, const double *mw, double *au,
                            double *av, double *aw)
{
    if (!c || !mu || !mv || !mw || !au || !av || !aw) return MG_ERR_PARAM;
    CKR(cudaSetDevice(c->device));
    int rc = ensure_unit(c, 6);
    if (rc) return rc;
    CKR(h2d(c, c->unit[0], mu, cudaMemcpyHostToDevice));
    CKR(h2d(c, c->unit[1], mv, cudaMemcpyHostToDevice));
    CKR(h2d(c, c->unit[2], mw, cudaMemcpyHostToDevice));
    for (int i = 3; i < 6; i++) CKR(cudaMemsetAsync(c->unit[i], 0, c->fbytes, c->stream));
    K2Args a{};
    a.ntime = ntime; a.mode = 1; a.in_is_leveln = 0; a.rep = REP_NAT;
    a.mu = c->unit[0]; a.mv = c->unit[1]; a.mw = c->unit[2];
    a.ou = c->unit[3]; a.ov = c->unit[4]; a.ow = c->unit[5];
    a.err = c->derr;
    K2Maps mm;
    const double *m3[3] = {c->unit[0], c->unit[1], c->unit[2]};
    if (build_mom_maps(c, m3, &mm)) return MG_ERR_CUDA;
    CKR(c->prm.precision == MG_PREC_MIXED ? launch_k2_mixed(c->G, a, mm, c->stream) : launch_k2(c->G, a, mm, c->stream));
    CKR(d2h(c, au, c->unit[3], cudaMemcpyDeviceToHost));
    CKR(d2h(c, av, c->unit[4], cudaMemcpyDeviceToHost));
    CKR(d2h(c, aw, c->unit[5], cudaMemcpyDeviceToHost));
    return cuerr(cudaStreamSynchronize(c->stream));
}

extern "C" int mg_fft_solve(mg_ctx *c, const double *tend, double *out)
{
    if (!c || !tend || !out) return MG_ERR_PARAM;
    CKR(cudaSetDevice(c->device));
    int rc = ensure_unit(c, 2);
    if (rc) return rc;
    CKR(h2d(c, c->unit[0], tend, cudaMemcpyHostToDevice));
    CKR(h2d(c, c->unit[1], out, cudaMemcpyHostToDevice));
    CKR(launch_load_rhs(c->G, c->pp, c->unit[0], c->stream));
    CKR(pressure_solve(c->G, c->pp, 1., 1, kNoPassCtl, c->stream));
    CKR(launch_store_solution(c->G, c->pp, c->unit[1], c->stream));
    CKR(d2h(c, out, c->unit[1], cudaMemcpyDeviceToHost));
    return cuerr(cudaStreamSynchronize(c->stream));
}

// ---- the compressible model's acoustic sub-steps (src/INTEG/prognostic_pressure.f90) ----
// reps > 0: after the first call, `warmup` untimed calls and `reps` calls timed with
// events run on the resident fields (ms: device time of one call of ntau sub-steps)
static int acoustic_impl(mg_ctx *c, const mg_acoustic *a, int warmup, int reps, double *ms)
{
    if (!c || !a) return MG_ERR_PARAM;
    if (a->ntau < 1 || (a->im != 1 && a->im != 2) || a->nscal < 0 || a->nscal > MG_MAXF - 4 ||
        (a->cst_cp != 0 && a->cst_cp != 1))
        return MG_ERR_PARAM;
    if (c->G.scal_adv == MG_QUICK && c->G.nz < 6) return MG_ERR_PARAM;
    const double *in[9] = {a->su, a->sv, a->sw, a->sdens, a->ses, a->sqt, a->uadv, a->vadv, a->wadv};
    double *io[14] = {a->dens, a->p, a->u, a->v, a->w, a->es, a->qt, a->tu, a->tv, a->tw, a->tdens, a->tes, a->tqt,
                      a->cs2};
    if (!a->p0) return MG_ERR_PARAM;
    for (const double *x : in) if (!x) return MG_ERR_PARAM;
    for (double *x : io) if (!x) return MG_ERR_PARAM;
    const int ns = a->nscal;
    if (ns > 0 && (!a->sscal || !a->scal || !a->tscal)) return MG_ERR_PARAM;
    for (int h = 0; h < ns; h++)
        if (!a->sscal[h] || !a->scal[h] || !a->tscal[h]) return MG_ERR_PARAM;
    CKR(cudaSetDevice(c->device));
    const DevGrid &G = c->G;
    const size_t fe = c->fbytes / sizeof(double);
    const int nfield = 9 + 14 + 3 + 3 * ns;   // inputs, in/out, dens2/es2/div, scalar triples
    double *blk = nullptr;
    CKR(cudaMalloc(&blk, (size_t)nfield * c->fbytes + 2 * (size_t)G.nz * sizeof(double)));
    auto fld = [&](int q) { return blk + (size_t)q * fe; };
    double *p0 = fld(nfield), *lvl = p0 + G.nz;
    AcousticFields f{};
    f.nscal = ns;
    f.p0 = p0;
    f.su = fld(0); f.sv = fld(1); f.sw = fld(2); f.sdens = fld(3); f.ses = fld(4); f.sqt = fld(5);
    f.uadv = fld(6); f.vadv = fld(7); f.wadv = fld(8);
    double **iod[14] = {&f.dens, &f.p, &f.u, &f.v, &f.w, &f.es, &f.qt, &f.tu, &f.tv, &f.tw, &f.tdens, &f.tes, &f.tqt,
                        &f.cs2};
    for (int q = 0; q < 14; q++) *iod[q] = fld(9 + q);
    f.dens2 = fld(23); f.es2 = fld(24); f.div = fld(25);
    for (int h = 0; h < ns; h++) {
        f.sscal[h] = fld(26 + 3 * h);
        f.scal[h] = fld(27 + 3 * h);
        f.tscal[h] = fld(28 + 3 * h);
    }
    cudaError_t e = cudaMemsetAsync(blk, 0, (size_t)nfield * c->fbytes, c->stream);
    for (int q = 0; q < 9 && e == cudaSuccess; q++) e = h2d(c, fld(q), in[q], cudaMemcpyHostToDevice);
    for (int q = 0; q < 14 && e == cudaSuccess; q++) e = h2d(c, fld(9 + q), io[q], cudaMemcpyHostToDevice);
    for (int h = 0; h < ns && e == cudaSuccess; h++) {
        e = h2d(c, fld(26 + 3 * h), a->sscal[h], cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = h2d(c, fld(27 + 3 * h), a->scal[h], cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = h2d(c, fld(28 + 3 * h), a->tscal[h], cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(p0, a->p0, G.nz * sizeof(double), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = launch_acoustic(G, f, a->im, a->ntau, a->cst_cp, lvl, c->stream);
    if (reps > 0 && e == cudaSuccess) {
        for (int r = 0; r < warmup && e == cudaSuccess; r++) e = launch_acoustic(G, f, a->im, a->ntau, a->cst_cp, lvl, c->stream);
        cudaEvent_t t0 = nullptr, t1 = nullptr;
        if (e == cudaSuccess) e = cudaEventCreate(&t0);
        if (e == cudaSuccess) e = cudaEventCreate(&t1);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e == cudaSuccess) e = cudaEventRecord(t0, c->stream);
        for (int r = 0; r < reps && e == cudaSuccess; r++) e = launch_acoustic(G, f, a->im, a->ntau, a->cst_cp, lvl, c->stream);
        if (e == cudaSuccess) e = cudaEventRecord(t1, c->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(t1);
        float tm = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&tm, t0, t1);
        if (e == cudaSuccess && ms) *ms = tm / reps;
        if (t0) cudaEventDestroy(t0);
        if (t1) cudaEventDestroy(t1);
    }
    for (int q = 0; q < 14 && e == cudaSuccess; q++) e = d2h(c, io[q], fld(9 + q), cudaMemcpyDeviceToHost);
    for (int h = 0; h < ns && e == cudaSuccess; h++) {
        e = d2h(c, a->scal[h], fld(27 + 3 * h), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = d2h(c, a->tscal[h], fld(28 + 3 * h), cudaMemcpyDeviceToHost);
    }
    const cudaError_t es = cudaStreamSynchronize(c->stream);
    cudaFree(blk);
    if (e == cudaErrorInvalidValue) return MG_ERR_PARAM;
    if (e != cudaSuccess) return cuerr(e);
    return cuerr(es);
}

extern "C" int mg_prognostic_pressure(mg_ctx *c, const mg_acoustic *a) { return acoustic_impl(c, a, 0, 0, nullptr); }

extern "C" int mg_time_prognostic_pressure(mg_ctx *c, const mg_acoustic *a, int warmup, int reps, double *ms)
{
    if (warmup < 0 || reps < 1 || !ms) return MG_ERR_PARAM;
    return acoustic_impl(c, a, warmup, reps, ms);
}

extern "C" int mg_anelastic_pressure(mg_ctx *c, double *mu, double *mv, double *mw, double *p, const double *wold,
                                     double *maxdiv, double *p1)
{
    if (!c || !mu || !mv || !mw || !p || !wold) return MG_ERR_PARAM;
    CKR(cudaSetDevice(c->device));
    int rc = ensure_unit(c, 5);
    if (rc) return rc;
    CKR(h2d(c, c->unit[0], mu, cudaMemcpyHostToDevice));
    CKR(h2d(c, c->unit[1], mv, cudaMemcpyHostToDevice));
    CKR(h2d(c, c->unit[2], mw, cudaMemcpyHostToDevice));
    CKR(h2d(c, c->unit[3], p, cudaMemcpyHostToDevice));
    CKR(h2d(c, c->unit[4], wold, cudaMemcpyHostToDevice));
    double *f[4] = {c->unit[0], c->unit[1], c->unit[2], c->unit[3]};
    CKR(launch_halo_fill(c->G, f, 4, c->stream));
    // the projection updates c->p; route it through the unit pressure buffer
    double *psave = c->p;
    c->p = c->unit[3];
    int launches = 0;
    cudaError_t e = project(c, c->unit[0], c->unit[1], c->unit[2], c->unit[4], -1, p1 != nullptr, 1, 0, &launches);
    c->p = psave;
    if (e != cudaSuccess) return cuerr(e);
    CKR(d2h(c, mu, c->unit[0], cudaMemcpyDeviceToHost));
    CKR(d2h(c, mv, c->unit[1], cudaMemcpyDeviceToHost));
    CKR(d2h(c, mw, c->unit[2], cudaMemcpyDeviceToHost));
    CKR(d2h(c, p, c->unit[3], cudaMemcpyDeviceToHost));
    if (maxdiv) CKR(cudaMemcpyAsync(maxdiv, pressure_maxdiv_dev(c->pp), 8, cudaMemcpyDeviceToHost, c->stream));
    if (p1) CKR(cudaMemcpyAsync(p1, pressure_p1_dev(c->pp), c->G.nz * 8, cudaMemcpyDeviceToHost, c->stream));
    return cuerr(cudaStreamSynchronize(c->stream));
}

// ---------------- timing and profiling ----------------
extern "C" int mg_time_steps(mg_ctx *c, int nsteps, int ntime0, int use_graph, double *ms)
{
    if (!c || nsteps < 0 || !ms) return MG_ERR_PARAM;
    if (!c->have_state) return MG_ERR_STATE;
    CKR(cudaSetDevice(c->device));
    cudaEvent_t a, b;
    CKR(cudaEventCreate(&a));
    CKR(cudaEventCreate(&b));
    CKR(cudaEventRecord(a, c->stream));
    int rc = use_graph ? mg_step_graph(c, nsteps, ntime0, nullptr, nullptr) : mg_step(c, nsteps, ntime0, nullptr, nullptr);
    if (rc == MG_OK) {
        cudaError_t e = cudaEventRecord(b, c->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(b);
        float f = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&f, a, b);
        *ms = f;
        if (e != cudaSuccess) rc = cuerr(e);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return rc;
}

extern "C" int mg_profile_enable(mg_ctx *c, int on)
{
    if (!c) return MG_ERR_PARAM;
    prof_collect(c);
    c->prof_on = on ? 1 : 0;
    c->acc.clear();
    return MG_OK;
}

extern "C" int mg_profile_report(mg_ctx *c, char *buf, size_t len)
{
    if (!c || !buf || len == 0) return MG_ERR_PARAM;
    prof_collect(c);
    size_t off = 0;
    buf[0] = 0;
    for (auto &a : c->acc) {
        int w = snprintf(buf + off, len - off, "%s %lld %.6f\n", a.name, a.n, a.ms);
        if (w < 0 || (size_t)w >= len - off) break;
        off += (size_t)w;
    }
    return MG_OK;
}

// ---------------- autotuner: the projection's plan ----------------
static void knobs_to_tune(const PressureKnobs &k, mg_tune *t)
{
    t->x_nstage = k.xst;
    t->y_nstage = k.yst;
    for (int q = 0; q < 16; q++) {
        t->x_radix[q] = q < k.xst ? (int)((k.xr >> (4 * q)) & 15ull) : 0;
        t->y_radix[q] = q < k.yst ? (int)((k.yr >> (4 * q)) & 15ull) : 0;
    }
    t->x_threads = k.xt;
    t->y_threads = k.yt;
    t->tri_block = k.tb;
}

// mean device time (ms) of one stage-1 K1 launch, which reads the resident state and
// writes only the stage buffers
static int time_k1(mg_ctx *c, int reps, double *ms)
{
    K1Args a{};
    k1_stage_args(c, 1, a);
    cudaEvent_t e0, e1;
    CKR(cudaEventCreate(&e0));
    cudaError_t er = cudaEventCreate(&e1);
    if (er != cudaSuccess) { cudaEventDestroy(e0); return cuerr(er); }
    auto launch = [&]() {
        return c->prm.precision == MG_PREC_MIXED ? launch_k1_mixed(c->G, a, c->maps1, c->stream)
                                                  : launch_k1(c->G, a, c->maps1, c->stream);
    };
    er = launch();   // warm-up
    if (er == cudaSuccess) er = cudaEventRecord(e0, c->stream);
    for (int r = 0; r < reps && er == cudaSuccess; r++) er = launch();
    if (er == cudaSuccess) er = cudaEventRecord(e1, c->stream);
    if (er == cudaSuccess) er = cudaEventSynchronize(e1);
    float f = 0.f;
    if (er == cudaSuccess) er = cudaEventElapsedTime(&f, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (er != cudaSuccess) return cuerr(er);
    *ms = f / reps;
    return check_err(c);
}

// one stage-1 momentum launch (K2 writes the stage buffers only), averaged over reps
static int time_k2(mg_ctx *c, int reps, double *ms)
{
    K2Args a{};
    k2_stage_args(c, 1, 1, a);
    cudaEvent_t e0, e1;
    CKR(cudaEventCreate(&e0));
    cudaError_t er = cudaEventCreate(&e1);
    if (er != cudaSuccess) { cudaEventDestroy(e0); return cuerr(er); }
    auto launch = [&]() {
        return c->prm.precision == MG_PREC_MIXED ? launch_k2_mixed(c->G, a, c->mmaps1, c->stream)
                                                  : launch_k2(c->G, a, c->mmaps1, c->stream);
    };
    er = launch();   // warm-up
    if (er == cudaSuccess) er = cudaEventRecord(e0, c->stream);
    for (int r = 0; r < reps && er == cudaSuccess; r++) er = launch();
    if (er == cudaSuccess) er = cudaEventRecord(e1, c->stream);
    if (er == cudaSuccess) er = cudaEventSynchronize(e1);
    float f = 0.f;
    if (er == cudaSuccess) er = cudaEventElapsedTime(&f, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (er != cudaSuccess) return cuerr(er);
    *ms = f / reps;
    return check_err(c);
}

static bool tune_to_knobs(const mg_tune *t, PressureKnobs *k)
{
    if (t->x_nstage < 1 || t->x_nstage > 16 || t->y_nstage < 1 || t->y_nstage > 16) return false;
    k->xr = k->yr = 0ull;
    for (int q = 0; q < t->x_nstage; q++) {
        if (t->x_radix[q] < 2 || t->x_radix[q] > 8) return false;
        k->xr |= (unsigned long long)t->x_radix[q] << (4 * q);
    }
    for (int q = 0; q < t->y_nstage; q++) {
        if (t->y_radix[q] < 2 || t->y_radix[q] > 8) return false;
        k->yr |= (unsigned long long)t->y_radix[q] << (4 * q);
    }
    k->xst = t->x_nstage;
    k->yst = t->y_nstage;
    k->xt = t->x_threads;
    k->yt = t->y_threads;
    k->tb = t->tri_block;
    return true;
}

extern "C" int mg_tune_get(mg_ctx *c, mg_tune *t)
{
    if (!c || !t) return MG_ERR_PARAM;
    memset(t, 0, sizeof(*t));
    PressureKnobs k;
    pressure_get_knobs(c->pp, &k);
    knobs_to_tune(k, t);
    t->k1_segments = c->k1_nseg;
    t->k2_segments = c->k2_nseg;
    return MG_OK;
}

extern "C" int mg_tune_set(mg_ctx *c, const mg_tune *t)
{
    if (!c || !t) return MG_ERR_PARAM;
    PressureKnobs k;
    if (t->k1_segments < 0 || t->k1_segments > c->G.nz) return MG_ERR_PARAM;
    if (t->k2_segments < 0 || t->k2_segments > c->G.nz) return MG_ERR_PARAM;
    if (!tune_to_knobs(t, &k) || !pressure_set_knobs(c->pp, c->G, k)) return MG_ERR_PARAM;
    c->k1_nseg = t->k1_segments;
    c->k2_nseg = t->k2_segments;
    drop_graphs(c);
    return MG_OK;
}

extern "C" int mg_radix_candidates(int n, int *radix, int *nstage, int maxc)
{
    if (n < 1 || !radix || !nstage || maxc < 1) return MG_ERR_PARAM;
    std::vector<unsigned long long> pk(maxc);
    std::vector<int> ns(maxc);
    const int nc = pressure_radix_candidates(n, pk.data(), ns.data(), maxc);
    for (int q = 0; q < nc; q++) {
        nstage[q] = ns[q];
        for (int s = 0; s < 16; s++) radix[16 * q + s] = s < ns[q] ? (int)((pk[q] >> (4 * s)) & 15ull) : 0;
    }
    return nc;
}

// mean device time (ms) of one projection of copies of the resident momentum and
// pressure (the copies are refreshed before every projection, outside the timed part)
static int time_projection(mg_ctx *c, int reps, double *ms)
{
    int rc = ensure_unit(c, 4);
    if (rc) return rc;
    double *u = c->unit[0], *v = c->unit[1], *w = c->unit[2], *p = c->unit[3];
    cudaEvent_t e0, e1;
    CKR(cudaEventCreate(&e0));
    cudaError_t er = cudaEventCreate(&e1);
    if (er != cudaSuccess) { cudaEventDestroy(e0); return cuerr(er); }
    double tot = 0.;
    for (int r = 0; r <= reps && er == cudaSuccess; r++) {   // r = 0: untimed warm-up
        double *src[4] = {c->mA[0], c->mA[1], c->mA[2], c->p}, *dst[4] = {u, v, w, p};
        for (int q = 0; q < 4 && er == cudaSuccess; q++)
            er = cudaMemcpyAsync(dst[q], src[q], c->fbytes, cudaMemcpyDeviceToDevice, c->stream);
        if (er == cudaSuccess) er = cudaEventRecord(e0, c->stream);
        if (er == cudaSuccess) {
            double *psave = c->p;
            c->p = p;
            int launches = 0;
            er = project(c, u, v, w, w, -1, 0, 0, 0, &launches);
            c->p = psave;
        }
        if (er == cudaSuccess) er = cudaEventRecord(e1, c->stream);
        if (er == cudaSuccess) er = cudaEventSynchronize(e1);
        float f = 0.f;
        if (er == cudaSuccess) er = cudaEventElapsedTime(&f, e0, e1);
        if (r > 0) tot += f;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (er != cudaSuccess) return cuerr(er);
    *ms = tot / reps;
    return check_err(c);
}

extern "C" int mg_autotune(mg_ctx *c, int reps, mg_tune *result)
{
    if (!c || reps < 1 || reps > 1000) return MG_ERR_PARAM;
    CKR(cudaSetDevice(c->device));
    PressureKnobs cur, k;
    pressure_get_knobs(c->pp, &cur);
    double best = 0., t = 0.;
    int rc = time_projection(c, reps, &best);
    if (rc) return rc;
    const double ms_default = best;
    int ncand = 1;
    // one coordinate at a time; a change is kept when it gains more than 1 %
    auto trial = [&](const PressureKnobs &cand) -> int {
        if (!pressure_knobs_valid(c->G, cand)) return MG_OK;
        pressure_set_knobs(c->pp, c->G, cand);
        int r = time_projection(c, reps, &t);
        if (r) { pressure_set_knobs(c->pp, c->G, cur); return r; }
        ncand++;
        if (t < 0.99 * best) { best = t; cur = cand; }
        pressure_set_knobs(c->pp, c->G, cur);
        return MG_OK;
    };
    unsigned long long pk[16];
    int ns[16];
    for (int axis = 0; axis < 2; axis++) {
        const int nc = pressure_radix_candidates(axis == 0 ? c->G.maxx : c->G.maxy, pk, ns, 16);
        for (int q = 0; q < nc; q++) {
            k = cur;
            if (axis == 0) { k.xr = pk[q]; k.xst = ns[q]; } else { k.yr = pk[q]; k.yst = ns[q]; }
            if (axis == 0 ? (k.xr == cur.xr && k.xst == cur.xst) : (k.yr == cur.yr && k.yst == cur.yst)) continue;
            if ((rc = trial(k))) return rc;
        }
    }
    for (int xt = 8; xt <= 64; xt *= 2)
        if (xt != cur.xt) { k = cur; k.xt = xt; if ((rc = trial(k))) return rc; }
    for (int yt = 16; yt <= 128; yt *= 2)
        if (yt != cur.yt) { k = cur; k.yt = yt; if ((rc = trial(k))) return rc; }
    for (int tb = 64; tb <= 256; tb *= 2)
        if (tb != cur.tb) { k = cur; k.tb = tb; if ((rc = trial(k))) return rc; }
    pressure_set_knobs(c->pp, c->G, cur);
    double tuned = 0.;
    if ((rc = time_projection(c, reps, &tuned))) return rc;
    // K1's k segments per column tile (0: the wave model's choice); PPM keeps whole columns
    double k1_def = 0., k1_best = 0., t1 = 0.;
    const int nseg_in = c->k1_nseg;
    int nseg_best = nseg_in;
    if (c->prm.scal_adv != MG_PPM) {
        if ((rc = time_k1(c, reps, &k1_def))) return rc;
        k1_best = k1_def;
        const int cands[9] = {0, 1, 2, 3, 4, 6, 8, 12, 16};
        for (int n : cands) {
            if (n == nseg_in || n * 8 > c->G.nz) continue;
            c->k1_nseg = n;
            rc = time_k1(c, reps, &t1);
            c->k1_nseg = nseg_in;
            if (rc) return rc;
            ncand++;
            if (t1 < 0.99 * k1_best) { k1_best = t1; nseg_best = n; }
        }
        c->k1_nseg = nseg_best;
    }
    // K2's k segments per column tile, the same candidates
    double k2_def = 0., k2_best = 0., t2 = 0.;
    const int nseg2_in = c->k2_nseg;
    int nseg2_best = nseg2_in;
    {
        if ((rc = time_k2(c, reps, &k2_def))) return rc;
        k2_best = k2_def;
        const int cands[9] = {0, 1, 2, 3, 4, 6, 8, 12, 16};
        for (int n : cands) {
            if (n == nseg2_in || n * 8 > c->G.nz) continue;
            c->k2_nseg = n;
            rc = time_k2(c, reps, &t2);
            c->k2_nseg = nseg2_in;
            if (rc) return rc;
            ncand++;
            if (t2 < 0.99 * k2_best) { k2_best = t2; nseg2_best = n; }
        }
        c->k2_nseg = nseg2_best;
    }
    drop_graphs(c);
    if (result) {
        memset(result, 0, sizeof(*result));
        knobs_to_tune(cur, result);
        result->k1_segments = nseg_best;
        result->k2_segments = nseg2_best;
        result->candidates = ncand;
        result->ms_default = ms_default;
        result->ms_tuned = tuned;
        result->k1_ms_default = k1_def;
        result->k1_ms_tuned = k1_best;
        result->k2_ms_default = k2_def;
        result->k2_ms_tuned = k2_best;
    }
    return MG_OK;
}
