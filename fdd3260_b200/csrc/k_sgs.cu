// k_sgs.cu -- SGS turbulence diffusion of the dynamical core (src/PHYS/subgrid.f90):
// the Smagorinsky-Lilly eddy viscosity (calc_subgrid: cal_dij, stability,
// calc_smago), the momentum stresses (efud) and the scalar fluxes (eff0/effs/eff).
//
// All three are evaluated once per step from the level-n natural state: the
// reference calls subgrid_interface before the dynamics loop and efud/eff0/effs
// with wind2/state2/pressure2, which update_prognostic refreshes only after both
// Heun stages (src/INTEG/time_step.f90:222,243-276,337-500).  The stage kernels
// K1/K2 then add the stored tendencies in the reference's order.
//
// FP64, compiled with -fmad=false: each expression keeps the reference's operation
// order, so results are bit-identical with the CPU restatement.  The per-level
// factors with transcendental functions (length scale, damping, anisotropy) are
// evaluated once on the host.
//
// Data: one thread per interior cell, direct loads through L1/L2; the gradients of
// neighbouring cells that a stencil needs are recomputed from the winds, which
// reads less HBM than storing the nine gradient fields.
#include <cmath>
#include <vector>

#include "mg_common.cuh"

namespace {

constexpr double C98 = 9. / 8.;
constexpr double C124 = 1. / 24.;
constexpr double SGS_CS = 0.23, SGS_RIC = 0.25, SGS_VK = 0.41, SGS_G = 9.81, SGS_EPSM = 0.60243;

__device__ __forceinline__ double ld(const double *a, long long q) { return __ldg(a + q); }

// periodic image of a ghost column index (the gradients' gradbc)
__device__ __forceinline__ int wrapx(const DevGrid &G, int i) { return i < 4 ? i + G.maxx : (i > G.nx - 2 ? i - G.maxx : i); }
__device__ __forceinline__ int wrapy(const DevGrid &G, int j) { return j < 4 ? j + G.maxy : (j > G.ny - 2 ? j - G.maxy : j); }

// 4th-order staggered derivative (gradients.f90:835-843)
__device__ __forceinline__ double d4(double am1, double a0, double a1, double a2, double d1)
{
    return C98 * (a1 - a0) * d1 - C124 * (a2 - am1) * d1;
}

struct Grad {
    const DevGrid &G;
    const SgsDev &S;
    double dx1, dy1;
    // d(a)/dx and d(a)/dy at (i, j, k), ghost columns mapped to their periodic images
    __device__ __forceinline__ double gx(const double *a, int i, int j, int k) const
    {
        i = wrapx(G, i); j = wrapy(G, j);
        const long long q = gidx(G, i, j, k);
        return d4(ld(a, q - 1), ld(a, q), ld(a, q + 1), ld(a, q + 2), dx1);
    }
    __device__ __forceinline__ double gy(const double *a, int i, int j, int k) const
    {
        i = wrapx(G, i); j = wrapy(G, j);
        const long long q = gidx(G, i, j, k), p = G.px;
        return d4(ld(a, q - p), ld(a, q), ld(a, q + p), ld(a, q + 2 * p), dy1);
    }
    // d(u)/dz and d(v)/dz (which = 0, 1), grad_wind_3d :884-905 with bcl(6) = 'nnf'
    __device__ __forceinline__ double gz_uv(const double *a, int which, int i, int j, int k) const
    {
        i = wrapx(G, i); j = wrapy(G, j);
        const int nz = G.nz;
        const long long q0 = gidx(G, i, j, 1), ps = G.ps;
        auto A = [&](int kk) { return ld(a, q0 + (long long)(kk - 1) * ps); };
        if (k == 1) return (A(2) - A(1)) * ld(G.dz1, 0);
        if (k >= nz - 1) return (A(nz) - A(nz - 1)) * ld(G.dz1, nz - 2);
        const double den = ld(which == 0 ? S.du : S.dv, k - 1);
        return C98 * (A(k + 1) - A(k)) * ld(G.dz1, k - 1) - 1. / 8. * (A(k + 2) - A(k - 1)) / den;
    }
    __device__ __forceinline__ double gz_w(const double *a, int i, int j, int k) const
    {
        i = wrapx(G, i); j = wrapy(G, j);
        const int nz = G.nz;
        const long long q0 = gidx(G, i, j, 1), ps = G.ps;
        auto A = [&](int kk) { return ld(a, q0 + (long long)(kk - 1) * ps); };
        if (k == 1) return (A(2) - 0.) * ld(G.dz1w, 0);
        if (k == nz) return (0. - A(nz)) * ld(G.dz1w, nz - 1);
        if (k == nz - 1)
            return C98 * (A(nz) - A(nz - 1)) * ld(G.dz1w, nz - 2) - 1. / 8. * (0. - A(nz - 2)) / ld(S.dwt, nz - 2);
        return C98 * (A(k + 1) - A(k)) * ld(G.dz1w, k - 1) - 1. / 8. * (A(k + 2) - A(k - 1)) / ld(S.dw, k - 1);
    }
};

// turbu%fkv of a cell and the two density-weighted forms the flux kernels use:
// fe = dens*fkv, times func(k) when pran < 0 (efud, subgrid.f90:228-239), and
// nut = fe/|pran| (eff0/effs, :489-497: ((dens*fkv)*func)/|pran| = fe/|pran|, the
// product being commutative)
__device__ __forceinline__ void sgs_store_visc(const SgsDev &S, const SgsVisc &O, long long c, int k, double fk,
                                               const double *dens)
{
    if (O.fkv) O.fkv[c] = fk;
    if (O.fe) {
        const double t0 = ld(dens, c) * fk;
        const double t = S.pran < 0. ? ld(S.func, k - 1) * t0 : t0;
        O.fe[c] = t;
        O.nut[c] = t / fabs(S.pran);
    }
}

// calc_subgrid for one interior cell: cal_dij (gradients.f90:476-600), stability
// (subgrid.f90:909-1001, dry branch, ISENTROPIC: ptv = es (1 + epsm qt)) and
// calc_smago (:793-866, 'Lilly').  Writes d11, d22, d33, d12, d13, d23 and fkv.
__global__ void __launch_bounds__(256) sgs_visc_kernel(DevGrid G, SgsDev S, const double *__restrict__ u,
                                                       const double *__restrict__ v, const double *__restrict__ w,
                                                       const double *__restrict__ es, const double *__restrict__ qt,
                                                       const double *__restrict__ dens, SgsDij D, SgsVisc O)
{
    const int i = 4 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 4 + blockIdx.y * blockDim.y + threadIdx.y;
    const int k = 1 + blockIdx.z;
    if (i > G.nx - 2 || j > G.ny - 2) return;
    const int nz = G.nz;
    const Grad g{G, S, 1. / G.dx, 1. / G.dy};
    const long long c = gidx(G, i, j, k);
    const double d11 = g.gx(u, i, j, k), d22 = g.gy(v, i, j, k), d33 = g.gz_w(w, i, j, k);
    double d12 = 0., d13 = 0., d23 = 0.;
    if (k >= 2 && k <= nz - 1) {
        d13 = 0.5 * (0.25 * (g.gz_uv(u, 0, i, j, k) + g.gz_uv(u, 0, i + 1, j, k) + g.gz_uv(u, 0, i, j, k - 1) +
                             g.gz_uv(u, 0, i + 1, j, k - 1)) +
                     0.25 * (g.gx(w, i - 1, j, k + 1) + g.gx(w, i, j, k + 1) + g.gx(w, i - 1, j, k) + g.gx(w, i, j, k)));
        d12 = 0.5 * (0.25 * (g.gy(u, i, j, k) + g.gy(u, i + 1, j, k) + g.gy(u, i, j - 1, k) + g.gy(u, i + 1, j - 1, k)) +
                     0.25 * (g.gx(v, i - 1, j + 1, k) + g.gx(v, i, j + 1, k) + g.gx(v, i - 1, j, k) + g.gx(v, i, j, k)));
        d23 = 0.5 * (0.25 * (g.gz_uv(v, 1, i, j, k) + g.gz_uv(v, 1, i, j + 1, k) + g.gz_uv(v, 1, i, j, k - 1) +
                             g.gz_uv(v, 1, i, j + 1, k - 1)) +
                     0.25 * (g.gy(w, i, j - 1, k + 1) + g.gy(w, i, j, k + 1) + g.gy(w, i, j - 1, k) + g.gy(w, i, j, k)));
    }
    D.d[0][c] = d11; D.d[1][c] = d22; D.d[2][c] = d33;
    D.d[3][c] = d12; D.d[4][c] = d13; D.d[5][c] = d23;
    if (!O.fkv && !O.fe) return;   // deformation only (unit entry of efud)
    if (S.diff_on) {               // fixed diffusion coefficient (subgrid.f90:131-133)
        sgs_store_visc(S, O, c, k, fabs(S.diff), dens);
        return;
    }
    // N2 (subgrid.f90:929-963): ptv at k-1, k, k+1 of the own column
    auto ptv = [&](int kk) {
        const long long q = gidx(G, i, j, kk);
        return ld(es, q) * (1. + SGS_EPSM * (qt ? ld(qt, q) : 0.));
    };
    double n2;
    if (k == 1) n2 = ld(S.n2c, 0) * (ptv(2) - ptv(1)) / ld(S.n2d, 0);
    else if (k == nz) n2 = ld(S.n2c, nz - 1) * (ptv(nz) - ptv(nz - 1)) / ld(S.n2d, nz - 1);
    else n2 = ld(S.n2c, k - 1) * (ptv(k + 1) - ptv(k - 1)) / ld(S.n2d, k - 1);
    // S2 = max(2 sum(dij*dij), 1e-12), the sum in array element order (l fastest)
    double sm = 0.;
    sm = sm + d11 * d11; sm = sm + d12 * d12; sm = sm + d13 * d13;
    sm = sm + d12 * d12; sm = sm + d22 * d22; sm = sm + d23 * d23;
    sm = sm + d13 * d13; sm = sm + d23 * d23; sm = sm + d33 * d33;
    const double s2 = fmax_ref(2. * sm, 1.e-12);
    const double ri = n2 / fmax_ref(s2, 1.e-12) / fabs(S.pran);
    const double fri = ri <= SGS_RIC ? sqrt(1. - fmax_ref(ri, -0.25) / SGS_RIC) : 0.;
    sgs_store_visc(S, O, c, k, ld(S.cs2d, k - 1) * sqrt(s2) * fmax_ref(fri, 0.), dens);
}

// density-weighted viscosity and diffusivity of every cell (the unit entries, whose
// turbu%fkv is an input): fe, nut as sgs_store_visc, over the whole allocation
__global__ void __launch_bounds__(256) sgs_prep_kernel(DevGrid G, SgsDev S, const double *__restrict__ dens,
                                                       const double *__restrict__ fkv, double *fe, double *nut)
{
    const long long n = G.ps * G.nz;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int k = 1 + (int)(q / G.ps);
        const double t0 = ld(dens, q) * ld(fkv, q);
        const double t = S.pran < 0. ? ld(S.func, k - 1) * t0 : t0;
        fe[q] = t;
        nut[q] = t / fabs(S.pran);
    }
}

// efud (subgrid.f90:187-456): out := (in + eh) + ev for u, v (levels 1..nz-1) and
// w (levels 2..nz-1), in = 0 when null.  fkv and the dij fields carry periodic ghosts.
__global__ void __launch_bounds__(256, 4) sgs_mom_kernel(DevGrid G, SgsDev S, const double *__restrict__ u,
                                                      const double *__restrict__ v, const double *__restrict__ fev,
                                                      SgsDij D, const double *mflux,
                                                      const double *in_u, const double *in_v, const double *in_w,
                                                      double *out_u, double *out_v, double *out_w)
{
    const int i = 4 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 4 + blockIdx.y * blockDim.y + threadIdx.y;
    const int k = 1 + blockIdx.z;   // 1 .. nz-1
    if (i > G.nx - 2 || j > G.ny - 2) return;
    const double dx1 = 1. / G.dx, dy1 = 1. / G.dy;
    // efud's fkv (dens*fkv, damped when pran < 0) and fkh = f_an(k)*fkv (anis_k)
    auto fe = [&](int ii, int jj, int kk) { return ld(fev, gidx(G, ii, jj, kk)); };
    auto fh = [&](int ii, int jj, int kk) {
        const double t = fe(ii, jj, kk);
        return S.anis_k ? ld(S.fan, kk - 1) * t : t;
    };
    // dij = 2*dij (:229)
    auto Dq = [&](int qd, int ii, int jj, int kk) { return 2. * ld(D.d[qd], gidx(G, ii, jj, kk)); };
    const long long c = gidx(G, i, j, k);
    const int nz = G.nz;

    // surface momentum flux (:318-333)
    double su1 = 0., sv1 = 0.;
    if (k == 1 && S.momsf > 0) {
        const long long q1 = gidx(G, i, j, 1);
        const double ua = 0.5 * (ld(u, q1 + 1) + ld(u, q1)), va = 0.5 * (ld(v, q1 + G.px) + ld(v, q1));
        double windm = ua * ua;
        windm = windm + va * va;
        windm = fmax_ref(S.min_w, sqrt(windm));
        const double mf = mflux ? ld(mflux, (long long)(j - 1) * G.nx + (i - 1)) : 0.;
        su1 = mf * 0.5 * (ld(u, q1 + 1) + ld(u, q1)) / windm;
        sv1 = mf * 0.5 * (ld(v, q1 + G.px) + ld(v, q1)) / windm;
    }

    // ---- u ----
    {
        const double f11p = fh(i, j, k) * Dq(0, i, j, k);
        const double f11m = fh(i - 1, j, k) * Dq(0, i - 1, j, k);
        const double f12p = 0.25 * (fh(i, j, k) * Dq(3, i, j, k) + fh(i, j + 1, k) * Dq(3, i, j + 1, k) +
                                    fh(i - 1, j, k) * Dq(3, i - 1, j, k) + fh(i - 1, j + 1, k) * Dq(3, i - 1, j + 1, k));
        const double f12m = 0.25 * (fh(i, j - 1, k) * Dq(3, i, j - 1, k) + fh(i, j, k) * Dq(3, i, j, k) +
                                    fh(i - 1, j - 1, k) * Dq(3, i - 1, j - 1, k) + fh(i - 1, j, k) * Dq(3, i - 1, j, k));
        const double f13p = 0.25 * (fe(i, j, k) * Dq(4, i, j, k) + fe(i - 1, j, k) * Dq(4, i - 1, j, k) +
                                    fe(i - 1, j, k + 1) * Dq(4, i - 1, j, k + 1) + fe(i, j, k + 1) * Dq(4, i, j, k + 1));
        const double f13m = k >= 2 ? 0.25 * (fe(i, j, k - 1) * Dq(4, i, j, k - 1) + fe(i - 1, j, k - 1) * Dq(4, i - 1, j, k - 1) +
                                             fe(i - 1, j, k) * Dq(4, i - 1, j, k) + fe(i, j, k) * Dq(4, i, j, k))
                                   : su1;
        double eh = (f11p - f11m) * dx1;
        eh = eh + (f12p - f12m) * dy1;
        const double ev = (f13p - f13m) * ld(G.dz1w, k - 1);
        out_u[c] = (in_u ? in_u[c] : 0.) + eh + ev;
    }
    // ---- v ----
    {
        const double f21p = 0.25 * (fh(i, j, k) * Dq(3, i, j, k) + fh(i, j - 1, k) * Dq(3, i, j - 1, k) +
                                    fh(i + 1, j - 1, k) * Dq(3, i + 1, j - 1, k) + fh(i + 1, j, k) * Dq(3, i + 1, j, k));
        const double f21m = 0.25 * (fh(i - 1, j, k) * Dq(3, i - 1, j, k) + fh(i - 1, j - 1, k) * Dq(3, i - 1, j - 1, k) +
                                    fh(i, j - 1, k) * Dq(3, i, j - 1, k) + fh(i, j, k) * Dq(3, i, j, k));
        const double f22p = fh(i, j, k) * Dq(1, i, j, k);
        const double f22m = fh(i, j - 1, k) * Dq(1, i, j - 1, k);
        const double f23p = 0.25 * (fe(i, j, k) * Dq(5, i, j, k) + fe(i, j - 1, k) * Dq(5, i, j - 1, k) +
                                    fe(i, j - 1, k + 1) * Dq(5, i, j - 1, k + 1) + fe(i, j, k + 1) * Dq(5, i, j, k + 1));
        const double f23m = k >= 2 ? 0.25 * (fe(i, j, k - 1) * Dq(5, i, j, k - 1) + fe(i, j - 1, k - 1) * Dq(5, i, j - 1, k - 1) +
                                             fe(i, j - 1, k) * Dq(5, i, j - 1, k) + fe(i, j, k) * Dq(5, i, j, k))
                                   : sv1;
        double eh = (f21p - f21m) * dx1;
        eh = eh + (f22p - f22m) * dy1;
        const double ev = (f23p - f23m) * ld(G.dz1w, k - 1);
        out_v[c] = (in_v ? in_v[c] : 0.) + eh + ev;
    }
    // ---- w (levels 2 .. nz-1) ----
    if (k >= 2 && k <= nz - 1) {
        const double f31p = 0.25 * (fh(i, j, k) * Dq(4, i, j, k) + fh(i, j, k - 1) * Dq(4, i, j, k - 1) +
                                    fh(i + 1, j, k - 1) * Dq(4, i + 1, j, k - 1) + fh(i + 1, j, k) * Dq(4, i + 1, j, k));
        const double f31m = 0.25 * (fh(i - 1, j, k) * Dq(4, i - 1, j, k) + fh(i - 1, j, k - 1) * Dq(4, i - 1, j, k - 1) +
                                    fh(i, j, k - 1) * Dq(4, i, j, k - 1) + fh(i, j, k) * Dq(4, i, j, k));
        const double f32p = 0.25 * (fh(i, j, k) * Dq(5, i, j, k) + fh(i, j, k - 1) * Dq(5, i, j, k - 1) +
                                    fh(i, j + 1, k - 1) * Dq(5, i, j + 1, k - 1) + fh(i, j + 1, k) * Dq(5, i, j + 1, k));
        const double f32m = 0.25 * (fh(i, j - 1, k) * Dq(5, i, j - 1, k) + fh(i, j - 1, k - 1) * Dq(5, i, j - 1, k - 1) +
                                    fh(i, j, k - 1) * Dq(5, i, j, k - 1) + fh(i, j, k) * Dq(5, i, j, k));
        const double f33p = fe(i, j, k) * Dq(2, i, j, k);
        const double f33m = fe(i, j, k - 1) * Dq(2, i, j, k - 1);
        double eh = (f31p - f31m) * dx1;
        eh = eh + (f32p - f32m) * dy1;
        const double ev = (f33p - f33m) * ld(G.dz1, k - 1);
        out_w[c] = (in_w ? in_w[c] : 0.) + eh + ev;
    }
}

// eff (subgrid.f90:604-789) with grad_quick (gradients.f90:62-187), CONSERVATIVE:
// out := SGS tendency of each density-weighted scalar on levels 1..nz-1.  One thread
// per cell serves every field: the diffusivities of the seven points are loaded once.
__global__ void __launch_bounds__(256, 5) sgs_scal_kernel(DevGrid G, SgsDev S, const double *__restrict__ nutv, SgsScal A)
{
    const int i = 4 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 4 + blockIdx.y * blockDim.y + threadIdx.y;
    const int k = 1 + blockIdx.z;   // 1 .. nz-1
    if (i > G.nx - 2 || j > G.ny - 2) return;
    const double dx1 = 1. / G.dx, dy1 = 1. / G.dy;
    const long long c = gidx(G, i, j, k), px = G.px, ps = G.ps;
    const double fan = S.anis_k ? ld(S.fan, k - 1) : 1.;
    auto nuh = [&](long long q) {
        const double t = ld(nutv, q);
        return S.anis_k ? fan * t : t;
    };
    const double h0 = nuh(c), hxp = nuh(c + 1), hxm = nuh(c - 1), hyp = nuh(c + px), hym = nuh(c - px);
    const double n0 = ld(nutv, c), nzp = ld(nutv, c + ps), nzm = k >= 2 ? ld(nutv, c - ps) : 0.;
    const double d1k = ld(G.dz1, k - 1), d1km = k >= 2 ? ld(G.dz1, k - 2) : 0., dzw = ld(G.dz1w, k - 1);
    for (int f = 0; f < A.nf; f++) {
        const double *x = A.x[f];
        const double *x0 = A.x0[f];
        const bool sub = S.diff_on && x0;
        const double x0k = sub ? ld(x0, k - 1) : 0., x0p = sub ? ld(x0, k) : 0., x0m = (sub && k >= 2) ? ld(x0, k - 2) : 0.;
        auto xs = [&](long long q, double xz) { return sub ? ld(x, q) - xz : ld(x, q); };
        const double xc = xs(c, x0k);
        const double fxp = 0.5 * (hxp + h0) * ((xs(c + 1, x0k) - xc) * dx1);
        const double fxm = 0.5 * (h0 + hxm) * ((xc - xs(c - 1, x0k)) * dx1);
        const double fyp = 0.5 * (hyp + h0) * ((xs(c + px, x0k) - xc) * dy1);
        const double fym = 0.5 * (h0 + hym) * ((xc - xs(c - px, x0k)) * dy1);
        const double fzp = 0.5 * (nzp + n0) * ((xs(c + ps, x0p) - xc) * d1k);
        double e = (fxp - fxm) * dx1;
        e = e + (fyp - fym) * dy1;
        double ez;
        if (k == 1) {
            double fsv = 0.;
            if (A.fs[f]) {
                fsv = ld(A.fs[f], (long long)(j - 1) * G.nx + (i - 1));
                if (A.fs_neg[f]) fsv = -fsv;
            }
            ez = (fzp - fsv) * dzw;
        } else {
            const double fzm = 0.5 * (n0 + nzm) * ((xc - xs(c - ps, x0m)) * d1km);
            ez = (fzp - fzm) * dzw;
        }
        A.out[f][c] = e + ez;
    }
}

inline dim3 sgs_grid(const DevGrid &g, int nzb) { return dim3((g.maxx + 31) / 32, (g.maxy + 7) / 8, nzb); }

}  // namespace

cudaError_t launch_sgs_visc(const DevGrid &g, const SgsDev &s, const double *u, const double *v, const double *w,
                            const double *es, const double *qt, const double *dens, const SgsDij &d,
                            const SgsVisc &o, cudaStream_t st)
{
    if (g.nz < 5) return cudaErrorInvalidValue;
    if (o.fe && (!o.nut || !dens)) return cudaErrorInvalidValue;
    if ((o.fkv || o.fe) && !s.diff_on && !es) return cudaErrorInvalidValue;
    sgs_visc_kernel<<<sgs_grid(g, g.nz), dim3(32, 8), 0, st>>>(g, s, u, v, w, es, qt, dens, d, o);
    return cudaGetLastError();
}

cudaError_t launch_sgs_prep(const DevGrid &g, const SgsDev &s, const double *dens, const double *fkv, double *fe,
                            double *nut, cudaStream_t st)
{
    sgs_prep_kernel<<<1184, 256, 0, st>>>(g, s, dens, fkv, fe, nut);
    return cudaGetLastError();
}

cudaError_t launch_sgs_mom(const DevGrid &g, const SgsDev &s, const double *u, const double *v, const double *fe,
                           const SgsDij &d, const double *mflux, const double *in_u, const double *in_v,
                           const double *in_w, double *out_u, double *out_v, double *out_w, cudaStream_t st)
{
    if (g.nz < 5) return cudaErrorInvalidValue;
    sgs_mom_kernel<<<sgs_grid(g, g.nz - 1), dim3(32, 8), 0, st>>>(g, s, u, v, fe, d, mflux, in_u, in_v, in_w, out_u,
                                                                   out_v, out_w);
    return cudaGetLastError();
}

cudaError_t launch_sgs_scal(const DevGrid &g, const SgsDev &s, const double *nut, const SgsScal &a, cudaStream_t st)
{
    if (g.nz < 5 || a.nf <= 0 || a.nf > MG_MAXF) return cudaErrorInvalidValue;
    sgs_scal_kernel<<<sgs_grid(g, g.nz - 1), dim3(32, 8), 0, st>>>(g, s, nut, a);
    return cudaGetLastError();
}

// Per-level factors (host): z0 (define_grid.f90:132-135), length_scale
// (subgrid.f90:1183-1232, l_d = 1e8 without TKE), the pran < 0 damping (:234-239),
// f_an (:244-249), the N2 coefficients (:929-963) and the d/dz denominators of
// grad_wind_3d (gradients.f90:884-905), and delta.  Layout prof[q*nz + k-1], q = 0..10.
void sgs_host_profiles(int nz, double dx, double dy, double dz, const double *f, const double *pt0, const double *qv0,
                       int anis, double zdec, double zrough, double *prof)
{
    double *z0 = prof, *cs2d = prof + nz, *func = prof + 2 * nz, *fan = prof + 3 * nz;
    double *n2c = prof + 4 * nz, *n2d = prof + 5 * nz;
    double *du = prof + 6 * nz, *dv = prof + 7 * nz, *dw = prof + 8 * nz, *dwt = prof + 9 * nz;
    double *dl = prof + 10 * nz;
    for (int q = 0; q < SGS_NPROF * nz; q++) prof[q] = 0.;
    z0[0] = 0.5 * dz * f[0];
    for (int k = 2; k <= nz; k++) z0[k - 1] = z0[k - 2] + 0.5 * dz * (f[k - 2] + f[k - 1]);
    const double l_d = 1e8;
    for (int k = 1; k <= nz; k++) {
        const double deltas = anis ? dz * f[k - 1] : std::pow(dx * dy * dz * f[k - 1], 1. / 3.);
        const double l_z = SGS_VK * (z0[k - 1] + zrough);
        const double delta = 1. / std::sqrt(1. / (deltas * deltas) + 1. / (l_d * l_d) + 1. / (l_z * l_z));
        const double cd = SGS_CS * delta;
        cs2d[k - 1] = cd * cd;
        dl[k - 1] = delta;
        const double fv = 1. - std::exp(6. * (z0[k - 1] - zdec) / zdec);
        func[k - 1] = fv > 0. ? fv : 0.;
        if (anis) {
            const double t = std::pow(dx * dy, 1. / 2.) / (dz * f[k - 1]);
            fan[k - 1] = t * t;
        } else {
            fan[k - 1] = 1.;
        }
        const double ref = pt0[k - 1] * (1. + SGS_EPSM * qv0[k - 1]);
        n2c[k - 1] = (k == 1 || k == nz) ? 0.5 * SGS_G / ref : SGS_G / ref;
    }
    for (int k = 2; k <= nz - 1; k++) n2d[k - 1] = dz * (0.5 * f[k] + f[k - 1] + 0.5 * f[k - 2]);
    n2d[0] = 0.5 * dz * (f[1] + f[0]);
    n2d[nz - 1] = 0.5 * dz * (f[nz - 1] + f[nz - 2]);
    for (int k = 2; k <= nz - 2; k++) {
        du[k - 1] = dz * (0.5 * f[k + 1] + f[k - 1] + f[k - 2] + 0.5 * f[k - 2]);
        dv[k - 1] = dz * (0.5 * f[k + 1] + f[k - 1] + f[k] + 0.5 * f[k - 2]);
        dw[k - 1] = dz * (f[k - 2] + f[k - 1] + f[k]);
    }
    dwt[nz - 2] = dz * (f[nz - 1] + f[nz - 2] + f[nz - 3]);
}
