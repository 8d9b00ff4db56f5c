// k_acoustic.cu -- the compressible model's acoustic sub-steps (prognostic_pressure),
// plain FP64, compiled with -fmad=false.
//
// Replaces src/INTEG/prognostic_pressure.f90:64-259 for the dry ISENTROPIC CONSERVATIVE
// build (div_pressure compiled out, nhydro = 0, sorder = 2, sponge off), with its
// callees: advect with limiter=.false., full=.false. (src/TOOLS/advection.f90:84-314,
// unsplit; the faces of src/TOOLS/advq_lw_nolim.f90, or of advq_quick_nolim.f90 for the
// quick scheme), integ_scal and integ_mom
// (src/INTEG/integpack.f90:54-260), equation_of_state (src/TOOLS/thermodynamics.f90:
// 74-294: potential temperature in, density in, conservative), buoyancy (:472-493,
// the non-ANELASTIC branch), caldiv and gradp (src/TOOLS/gradients.f90:986-1052,
// 1205-1292; gpz(1) = 0 without ANELASTIC) and horav.
//
// One sub-step is two kernels over the interior cells, each followed by the periodic
// ghost refresh of what it wrote:
//   ac_scal_kernel  advective tendencies of density and es (x, y, z faces of the cell,
//                   as the reference subtracts them direction by direction), the
//                   tendency accumulators and the integ_scal update of every scalar,
//                   then, on the cell's new values, the equation of state (pressure,
//                   sound speed, es and qt through the reference's divide-and-multiply
//                   round trip), and the divergence of the momentum (caldiv: the
//                   momentum is not changed before it in the sub-step);
//   (level means of the sound speed, horav)
//   ac_mom_kernel   pressure gradient, divergence-damping gradient, buoyancy, the
//                   tendency accumulators and the integ_mom update.
// The reference's whole-array passes are pointwise where they are fused here, so the
// fused order gives the same values.
// Everything matches the CPU restatement bit for bit except the power of the equation
// of state (CUDA's pow against the C library's) and the order of the level sums.
#include <math.h>

#include "mg_common.cuh"

namespace {

constexpr double AC_G = 9.81, AC_PREF = 100000., AC_CPA = 1004., AC_CVA = 716., AC_CPV = 1827., AC_CVV = 1388.5;
constexpr double AC_ADIV = 0.2;   // prognostic_pressure.f90:53

struct AcDev {
    int nscal, cst_cp;
    double a_lm, b_lm, dtau;
    const double *p0;                       // base-state pressure (nz)
    const double *su, *sv, *sw, *sdens, *ses, *sqt;
    const double *sscal[MG_MAXF];
    const double *uadv, *vadv, *wadv;
    const double *dens, *es;                // sub-step inputs (ping-pong with dens2, es2)
    double *dens2, *es2;
    double *p, *u, *v, *w, *qt;
    double *scal[MG_MAXF];
    double *tu, *tv, *tw, *tdens, *tes, *tqt;
    double *tscal[MG_MAXF];
    double *cs2, *div;
    const double *damp;                     // level means of cs2 (nz)
};

// interior cell of a linear thread index; false past the end
__device__ __forceinline__ bool ac_cell(const DevGrid &G, long long t, int &i, int &j, int &k)
{
    const int mx = G.maxx, my = G.maxy;
    if (t >= (long long)mx * my * G.nz) return false;
    i = (int)(t % mx) + 4;
    j = (int)((t / mx) % my) + 4;
    k = (int)(t / ((long long)mx * my)) + 1;
    return true;
}

// face flux of advsx_lw_nl / advsy_lw_nl (advq_lw_nolim.f90:80-88): between xl and xr,
// face velocity uu; the Courant number uses dt0
__device__ __forceinline__ double lwnl_face_h(double xl, double xr, double uu, double dt0, double d1)
{
    const double mu = fabs(uu) * dt0 * d1;
    const double ffip1 = xr - xl;
    const double fl = xl + 0.5 * ffip1 * (1. - mu);
    const double fr = xr - 0.5 * ffip1 * (1. - mu);
    return 0.5 * fl * (uu + fabs(uu)) + 0.5 * fr * (uu - fabs(uu));
}

// face flux k+1/2 of advsz_lw_nl (advq_lw_nolim.f90:218-227), 1 <= k <= nz-1
__device__ __forceinline__ double lwnl_face_z(const DevGrid &G, const double *x, const double *w, long long c, int k)
{
    const double ww = __ldg(w + c + G.ps);
    const double d1 = __ldg(G.dz1 + k - 1), d1w = __ldg(G.dz1w + k - 1);
    const double mu = fabs(ww) * G.dt0 * d1;
    const double xx = __ldg(x + c), xp = __ldg(x + c + G.ps);
    const double ffip1 = (xp - xx) * d1;
    const double fl = xx + 0.5 * ffip1 * (1. - mu) / d1w;
    const double fr = xp - 0.5 * ffip1 * (1. - mu) / d1w;
    return 0.5 * fl * (ww + fabs(ww)) + 0.5 * fr * (ww - fabs(ww));
}

// face flux of advsx_quick_nl / advsy_quick_nl (advq_quick_nolim.f90:80-94): between
// x0 and xp1, with xm1 and xp2 beside them
__device__ __forceinline__ double quicknl_face_h(double xm1, double x0, double xp1, double xp2, double uu)
{
    const double cc = 1. / 4.;
    const double ffip1 = (xp1 - x0), ffip2 = (xp2 - xp1), ffim1 = (x0 - xm1);
    const double phil = ffip1 - cc * (ffip1 - ffim1);
    const double phir = ffip1 + cc * (ffip2 - ffip1);
    const double fl = x0 + 0.5 * phil;
    const double fr = xp1 - 0.5 * phir;
    return 0.5 * fl * (uu + fabs(uu)) + 0.5 * fr * (uu - fabs(uu));
}

// face flux k+1/2 of advsz_quick_nl (advq_quick_nolim.f90:218-272), 1 <= k <= nz-1, 'nnf'
// (bc51 = bc61 = 0: the one-sided slopes of the end faces are the reference's
// 0*(...) + 1*ffip1); c is the cell (k) of the column whose base is c0 (level 1)
__device__ __forceinline__ double quicknl_face_z(const DevGrid &G, const double *x, const double *w, long long c0, int k)
{
    const int nz = G.nz;
    const double cc = 1. / 4., bc = 0.;
    auto X = [&](int l) { return __ldg(x + c0 + (long long)(l - 1) * G.ps); };
    auto D1 = [&](int l) { return __ldg(G.dz1 + l - 1); };
    const double xx = X(k), ww = __ldg(w + c0 + (long long)k * G.ps);
    const double ffip1 = (X(k + 1) - xx) * D1(k);
    double ffip2, ffim1;
    if (k == 1) {
        ffip2 = (X(3) - X(2)) * D1(2);
        ffim1 = bc * (X(nz - 4) - X(nz - 5)) * D1(nz - 5) + (1. - bc) * ffip1;
    } else if (k == nz - 1) {
        ffim1 = (xx - X(k - 1)) * D1(k - 1);
        ffip2 = bc * (X(6) - X(5)) * D1(5) + (1. - bc) * ffip1;
    } else {
        ffip2 = (X(k + 2) - X(k + 1)) * D1(k + 1);
        ffim1 = (xx - X(k - 1)) * D1(k - 1);
    }
    const double phil = ffip1 - cc * (ffip1 - ffim1);
    const double phir = ffip1 + cc * (ffip2 - ffip1);
    const double d1w = __ldg(G.dz1w + k - 1);
    const double fl = xx + 0.5 * phil / d1w;
    const double fr = X(k + 1) - 0.5 * phir / d1w;
    return 0.5 * fl * (ww + fabs(ww)) + 0.5 * fr * (ww - fabs(ww));
}

// advection_x/y/z (advection.f90:556-798, non-split: xs = xs - xx per direction) of one
// field at cell c, starting from the slow tendency s; QUICK selects advq_quick_nolim's
// faces, false advq_lw_nolim's
template <bool QUICK>
__device__ __forceinline__ double nl_tendency(const DevGrid &G, const AcDev &A, const double *x, double s, long long c,
                                              int k)
{
    const double dx1 = 1. / G.dx, dy1 = 1. / G.dy;
    auto L = [&](long long q) { return __ldg(x + q); };
    double fxm, fxp, fym, fyp;
    if constexpr (QUICK) {
        fxm = quicknl_face_h(L(c - 2), L(c - 1), L(c), L(c + 1), __ldg(A.uadv + c));
        fxp = quicknl_face_h(L(c - 1), L(c), L(c + 1), L(c + 2), __ldg(A.uadv + c + 1));
        fym = quicknl_face_h(L(c - 2 * G.px), L(c - G.px), L(c), L(c + G.px), __ldg(A.vadv + c));
        fyp = quicknl_face_h(L(c - G.px), L(c), L(c + G.px), L(c + 2 * G.px), __ldg(A.vadv + c + G.px));
    } else {
        fxm = lwnl_face_h(L(c - 1), L(c), __ldg(A.uadv + c), G.dt0, dx1);
        fxp = lwnl_face_h(L(c), L(c + 1), __ldg(A.uadv + c + 1), G.dt0, dx1);
        fym = lwnl_face_h(L(c - G.px), L(c), __ldg(A.vadv + c), G.dt0, dy1);
        fyp = lwnl_face_h(L(c), L(c + G.px), __ldg(A.vadv + c + G.px), G.dt0, dy1);
    }
    s = s - (0. + (fxp - fxm) * dx1);
    s = s - (0. + (fyp - fym) * dy1);
    const int nz = G.nz;
    const double d1w = __ldg(G.dz1w + k - 1);
    const long long c0 = c - (long long)(k - 1) * G.ps;
    auto FZ = [&](int kf) {   // face kf+1/2
        if constexpr (QUICK) return quicknl_face_z(G, x, A.wadv, c0, kf);
        else return lwnl_face_z(G, x, A.wadv, c0 + (long long)(kf - 1) * G.ps, kf);
    };
    double zz;
    if (k == 1)   // 'nnf' bottom: xa(1) = xa(1) + (Flux(1) - 0.)*dz1w(1)
        zz = 0. + ((nz >= 2 ? FZ(1) : 0.) - 0.) * d1w;
    else if (k == nz)   // 'nnf' top: xa(nz) = xa(nz) + (0. - Flux(nz-1))*dz1w(nz)
        zz = 0. + (0. - FZ(k - 1)) * d1w;
    else
        zz = 0. + (FZ(k) - FZ(k - 1)) * d1w;
    return s - zz;
}

// equation_of_state(state, density_in=dens, pressure_out=p, thermo_out, conservative=.true.)
// for potential temperature (thermodynamics.f90:126-134, 193-203, 208-211, 254-258,
// 266-288) on a cell's density d and density-weighted es, qt (updated in place)
__device__ __forceinline__ void ac_eos(const AcDev &A, int k, long long c, double d, double &es_w, double &qt_w)
{
    const double es = es_w / d, qt = qt_w / d;
    double cp = AC_CPA, cv = AC_CVA;
    if (!A.cst_cp) {   // get_cp_cv_3d (:331-343), lmicro = 0: qv = qt
        const double qv = qt;
        cp = (1. - qt) * AC_CPA + AC_CPV * qv;
        cv = (1. - qt) * AC_CVA + AC_CVV * qv;
    }
    const double exn = pow(d * (cp - cv) * es / AC_PREF, (AC_CPA - AC_CVA) / AC_CVA);
    const double tt = es * exn;
    const double pp = d * (cp - cv) * tt;
    A.cs2[c] = AC_CPA / AC_CVA * pp / d;
    A.p[c] = pp - __ldg(A.p0 + k - 1);
    es_w = es * d;
    qt_w = qt * d;
}

// six CTAs per SM (40 registers, a few spilled): the kernel waits on its stencil loads,
// and the extra warps hide them (+5 % against 54 registers and four CTAs)
template <bool QUICK>
__global__ void __launch_bounds__(256, 6) ac_scal_kernel(const __grid_constant__ DevGrid G, const __grid_constant__ AcDev A)
{
    int i, j, k;
    if (!ac_cell(G, (long long)blockIdx.x * blockDim.x + threadIdx.x, i, j, k)) return;
    const long long c = gidx(G, i, j, k);
    // advect (density with adv=.false., es in flux form), then integ_scal (integpack.f90:171-217)
    const double densa = nl_tendency<QUICK>(G, A, A.dens, __ldg(A.sdens + c), c, k);
    const double esa = nl_tendency<QUICK>(G, A, A.es, __ldg(A.ses + c), c, k);
    const double td = densa + A.b_lm * A.tdens[c];
    const double te = esa + A.b_lm * A.tes[c];
    const double tq = __ldg(A.sqt + c) + A.b_lm * A.tqt[c];
    A.tdens[c] = td;
    A.tes[c] = te;
    A.tqt[c] = tq;
    const double dn = __ldg(A.dens + c) + A.a_lm * A.dtau * td;
    double en = __ldg(A.es + c) + A.a_lm * A.dtau * te;
    double qn = A.qt[c] + A.a_lm * A.dtau * tq;
    for (int h = 0; h < A.nscal; h++) {
        const double ts = __ldg(A.sscal[h] + c) + A.b_lm * A.tscal[h][c];
        A.tscal[h][c] = ts;
        A.scal[h][c] = A.scal[h][c] + A.a_lm * A.dtau * ts;
    }
    ac_eos(A, k, c, dn, en, qn);
    A.dens2[c] = dn;
    A.es2[c] = en;
    A.qt[c] = qn;
    // caldiv (gradients.f90:1014-1039) of the momentum
    const double dx1 = 1. / G.dx, dy1 = 1. / G.dy;
    double dv = 0.;
    dv = dv + (A.u[c + 1] - A.u[c]) * dx1;
    dv = dv + (A.v[c + G.px] - A.v[c]) * dy1;
    if (k < G.nz) dv = dv + (A.w[c + G.ps] - A.w[c]) * __ldg(G.dz1w + k - 1);
    else dv = dv + (0. - A.w[c]) * __ldg(G.dz1w + k - 1);
    A.div[c] = dv;
}

// gradp of the pressure and of the divergence (gpz(1) = 0), buoyancy of the density,
// winda (prognostic_pressure.f90:186-202) and integ_mom (integpack.f90:100-119, tauw = 1)
__global__ void ac_mom_kernel(const __grid_constant__ DevGrid G, const __grid_constant__ AcDev A)
{
    int i, j, k;
    if (!ac_cell(G, (long long)blockIdx.x * blockDim.x + threadIdx.x, i, j, k)) return;
    const long long c = gidx(G, i, j, k);
    const double dx1 = 1. / G.dx, dy1 = 1. / G.dy;
    const double pc = __ldg(A.p + c), dc = __ldg(A.div + c);
    const double gpx = (pc - __ldg(A.p + c - 1)) * dx1, gpy = (pc - __ldg(A.p + c - G.px)) * dy1;
    const double gdx = (dc - __ldg(A.div + c - 1)) * dx1, gdy = (dc - __ldg(A.div + c - G.px)) * dy1;
    double gpz = 0., gdz = 0., buoy;
    const double rc = __ldg(A.dens + c);
    if (k >= 2) {
        const double dz1 = __ldg(G.dz1 + k - 2);
        gpz = (pc - __ldg(A.p + c - G.ps)) * dz1;
        gdz = (dc - __ldg(A.div + c - G.ps)) * dz1;
        buoy = -(0.5 * AC_G * (rc + __ldg(A.dens + c - G.ps) - __ldg(G.den0 + k - 1) - __ldg(G.den0 + k - 2)));
    } else {
        buoy = -(AC_G * (rc - __ldg(G.den0)));
    }
    const double damp = __ldg(A.damp + k - 1);
    const double wu = __ldg(A.su + c) - gpx + AC_ADIV * A.dtau * damp * gdx;
    const double wv = __ldg(A.sv + c) - gpy + AC_ADIV * A.dtau * damp * gdy;
    const double ww = k == 1 ? 0. : __ldg(A.sw + c) - gpz + AC_ADIV * A.dtau * damp * gdz + buoy;
    const double tu = wu + A.b_lm * A.tu[c];
    const double tv = wv + A.b_lm * A.tv[c];
    const double tw = ww + A.b_lm * A.tw[c];
    A.tu[c] = tu;
    A.tv[c] = tv;
    A.tw[c] = tw;
    A.u[c] = A.u[c] + A.a_lm * A.dtau * tu;
    A.v[c] = A.v[c] + A.a_lm * A.dtau * tv;
    A.w[c] = 1. * (A.w[c] + A.a_lm * A.dtau * tw);
}

}  // namespace

// ntau sub-steps on device fields (halo'd layout, periodic ghost cells refreshed after
// every kernel); f: the AcousticFields pointers, lvl: nz doubles of scratch
cudaError_t launch_acoustic(const DevGrid &g, const AcousticFields &f, int im, int ntau, int cst_cp, double *lvl,
                            cudaStream_t s)
{
    if (ntau < 1 || (im != 1 && im != 2) || f.nscal < 0 || f.nscal > MG_MAXF - 4) return cudaErrorInvalidValue;
    if (g.scal_adv == MG_QUICK && g.nz < 6) return cudaErrorInvalidValue;   // the bottom face reads x(nz-5)
    AcDev A{};
    A.nscal = f.nscal;
    A.cst_cp = cst_cp;
    A.a_lm = im == 1 ? 1. : 0.5;
    A.b_lm = im == 1 ? 0. : 1.;
    A.dtau = g.dt0 * (1. / (double)ntau);
    A.p0 = f.p0;
    A.su = f.su; A.sv = f.sv; A.sw = f.sw; A.sdens = f.sdens; A.ses = f.ses; A.sqt = f.sqt;
    A.uadv = f.uadv; A.vadv = f.vadv; A.wadv = f.wadv;
    A.p = f.p; A.u = f.u; A.v = f.v; A.w = f.w; A.qt = f.qt;
    A.tu = f.tu; A.tv = f.tv; A.tw = f.tw; A.tdens = f.tdens; A.tes = f.tes; A.tqt = f.tqt;
    A.cs2 = f.cs2; A.div = f.div; A.damp = lvl;
    for (int h = 0; h < f.nscal; h++) {
        A.sscal[h] = f.sscal[h];
        A.scal[h] = f.scal[h];
        A.tscal[h] = f.tscal[h];
    }
    const long long n = (long long)g.maxx * g.maxy * g.nz;
    const unsigned nb = (unsigned)((n + 255) / 256);
    cudaError_t e;
    double *dens = f.dens, *dens2 = f.dens2, *es = f.es, *es2 = f.es2;
    {   // caldiv's windbc (gradients.f90:1011): the momentum's ghost cells, once; every
        // sub-step leaves them periodic
        double *wf[3] = {f.u, f.v, f.w};
        if ((e = launch_halo_fill(g, wf, 3, s)) != cudaSuccess) return e;
    }
    for (int it = 0; it < ntau; it++) {
        A.dens = dens; A.dens2 = dens2; A.es = es; A.es2 = es2;
        if (g.scal_adv == MG_QUICK)
            ac_scal_kernel<true><<<nb, 256, 0, s>>>(g, A);
        else
            ac_scal_kernel<false><<<nb, 256, 0, s>>>(g, A);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        {
            double *hf[7 + MG_MAXF];
            int nf = 0;
            hf[nf++] = dens2; hf[nf++] = es2; hf[nf++] = f.qt; hf[nf++] = f.p; hf[nf++] = f.cs2; hf[nf++] = f.div;
            for (int h = 0; h < f.nscal; h++) hf[nf++] = f.scal[h];
            if ((e = launch_halo_fill(g, hf, nf, s)) != cudaSuccess) return e;
        }
        if ((e = launch_level_mean(g, f.cs2, lvl, s)) != cudaSuccess) return e;
        // the new density is this sub-step's state from here on
        A.dens = dens2;
        ac_mom_kernel<<<nb, 256, 0, s>>>(g, A);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        {
            double *wf[3] = {f.u, f.v, f.w};
            if ((e = launch_halo_fill(g, wf, 3, s)) != cudaSuccess) return e;
        }
        double *t = dens; dens = dens2; dens2 = t;
        t = es; es = es2; es2 = t;
    }
    // the final density and es live in the buffers the caller passed as dens / es
    if (dens != f.dens) {
        if ((e = cudaMemcpyAsync(f.dens, dens, (size_t)g.ps * g.nz * 8, cudaMemcpyDeviceToDevice, s)) != cudaSuccess) return e;
        if ((e = cudaMemcpyAsync(f.es, es, (size_t)g.ps * g.nz * 8, cudaMemcpyDeviceToDevice, s)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}
