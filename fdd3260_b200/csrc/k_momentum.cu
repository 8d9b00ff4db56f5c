// k_momentum.cu -- K2: momentum tendency and stage update, plain FP64 form.
//
// Replaces, per stage, src/INTEG/momentum.f90:64-228 (explicit -rho0 grad(p/rho0)
// :121-144, buoyancy with imp_buoy :150-181 and src/TOOLS/thermodynamics.f90:472-534,
// assembly :193-205), src/INTEG/windadv.f90 qnadv_uvw/uadv_fd/vadv_fd/wadv_fd and
// the adv{u,v,w}{x,y,z}_fd stencils (:494-1127), and integ_mom
// (src/INTEG/integpack.f90:54-135).
//
// One block per 32x8 column tile marching k = 1..nz.  A five-level ring (k-2..k+2)
// of haloed planes (2 ghost cells) of the momentum and of the advective velocity
// derived from it is kept in shared memory; every stencil of the reference reads
// inside that ring.  Per cell and component the reference's accumulation order is
// kept: directions x,y,z for even ntime and z,y,x for odd ntime, each adding its
// flux divergence and then subtracting its artificial viscosity.
//
// Compiled with -fmad=false: bit-identical to the CPU restatement.
#include "mg_common.cuh"
#include "mimica_gpu.h"

namespace {

constexpr int TX = 32, TY = 8, R = 2;
constexpr int PW = TX + 2 * R, PH = TY + 2 * R, PL = PW * PH;
constexpr int NSLOT = 5;
constexpr double AVISC = 1. / 16.;   // windadv.f90:39

__device__ __forceinline__ double ldg(const double *p, long long i) { return __ldg(p + i); }

__global__ void __launch_bounds__(TX *TY) k2_kernel(DevGrid G, K2Args A)
{
    extern __shared__ double sm[];
    double *ring_m = sm;                       // [slot][3][PL] momentum (stencil values)
    double *ring_a = sm + NSLOT * 3 * PL;      // [slot][3][PL] advective velocity

    const int ntx = (G.maxx + TX - 1) / TX;
    const int ti = blockIdx.x % ntx, tj = blockIdx.x / ntx;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const int i0 = 4 + ti * TX, j0 = 4 + tj * TY;
    const int i = i0 + tx, j = j0 + ty;
    const int nx = G.nx, ny = G.ny, nz = G.nz;
    const bool act = (i <= nx - 2) && (j <= ny - 2);
    const double dx1 = 1. / G.dx, dy1 = 1. / G.dy, dt0 = G.dt0;
    const double dx2 = 1. / (2. * G.dx), dy2 = 1. / (2. * G.dy);
    const double dx3 = 1. / (3. * G.dx), dy3 = 1. / (3. * G.dy);
    double c1a, c2a, c1b, c2b;   // a: 4/3,1/3 (self-advection); b: 9/8,1/8 (cross terms)
    if (G.mom_ord == 4) { c1a = 4. / 3.; c2a = 1. / 3.; c1b = 9. / 8.; c2b = 1. / 8.; }
    else { c1a = 1.; c2a = 0.; c1b = 1.; c2b = 0.; }
    const double *dzw = G.dzw, *dz1w = G.dz1w, *dz1 = G.dz1;

    auto load_level = [&](int l) {
        const int slot = l % NSLOT;
        const double d0 = ldg(G.den0, l - 1), a0 = ldg(G.avden0, l - 1);
        for (int q = tid; q < 3 * PL; q += TX * TY) {
            int arr = q / PL, o = q - arr * PL;
            int r = o / PW, c = o - r * PW;
            int ii = i0 - R + c, jj = j0 - R + r;
            double mv = 0., av = 0.;
            if (ii >= 1 && ii <= nx && jj >= 1 && jj <= ny) {
                long long idx = gidx(G, ii, jj, l);
                const double *src = arr == 0 ? A.mu : (arr == 1 ? A.mv : A.mw);
                double w = arr == 2 ? a0 : d0;
                double x = ldg(src, idx);
                mv = A.in_is_leveln ? rep_value(A.rep, x, w) : x;
                av = mv / w;
                if (arr == 0) av = av - G.u0shift;
                else if (arr == 1) av = av - G.v0shift;
            }
            ring_m[(slot * 3 + arr) * PL + o] = mv;
            ring_a[(slot * 3 + arr) * PL + o] = av;
        }
    };
    // Per level k: lb[d+2] = this thread's element of ring slot (k+d) mod 5, d = -2..2.
    // MM/AA(c, d, di, dj): momentum / advective velocity of component c (0 u, 1 v, 2 w)
    // at (i+di, j+dj, k+d); d, di, dj are compile-time constants at every use.
    const double *lb[5];
#define MM(c, d, di, dj) lb[(d) + 2][(c) * PL + (dj) * PW + (di)]
#define AA(c, d, di, dj) lb[(d) + 2][NSLOT * 3 * PL + (c) * PL + (dj) * PW + (di)]
#define ZW(l) ldg(dzw, (l) - 1)
#define ZW1(l) ldg(dz1w, (l) - 1)
#define Z1(l) ldg(dz1, (l) - 1)

    load_level(1);
    if (nz >= 2) load_level(2);

    double bb_prev = 0.;   // buoyancy at level k-1 (cell centre)
    // vertical fluxes carried up the column (each computed once):
    //   fzu/fzv[m] = Flux(k-2+m) of advuz/advvz, m = 0..3;  fzw[m] = Flux(k-1+m) and
    //   azw[m] = Adv(k-2+m) of advwz;  pp_below = p(k-1)/rho0(k-1)
    double fzu0 = 0., fzu1 = 0., fzu2 = 0., fzu3 = 0., fzv0 = 0., fzv1 = 0., fzv2 = 0., fzv3 = 0.;
    double fzw0 = 0., fzw1 = 0., azw0 = 0., azw1 = 0., azw2 = 0.;
    double pp_below = 0.;
    const bool even = (A.ntime % 2) == 0;
    const double grav = 9.81, epsm = 0.60243, cdiag = 0.5;
    const int own = (ty + R) * PW + (tx + R);

    for (int k = 1; k <= nz; k++) {
        __syncthreads();
        if (k + 2 <= nz) load_level(k + 2);
        __syncthreads();
        if (!act) continue;   // no further barriers in this iteration
#pragma unroll
        for (int d = -2; d <= 2; d++) lb[d + 2] = ring_m + (((k + d + NSLOT) % NSLOT) * 3) * PL + own;

        // ---- advance the carried vertical fluxes ----
        {
            // advuz_fd/advvz_fd Flux(k+1) (windadv.f90:656-663): levels k+1, k+2; Flux(nz) = 0
            double fu = 0., fv = 0.;
            if (k + 1 <= nz - 1) {
                const double zp = ZW(k + 2), zc = ZW(k + 1), zs = zp + zc;
                double ww = c1b * (AA(2, 2, -1, 0) + AA(2, 2, 0, 0)) * 0.5 - c2b * (AA(2, 2, -2, 0) + AA(2, 2, 1, 0)) * 0.5;
                double fr = (zp * MM(0, 2, 0, 0) + zc * MM(0, 1, 0, 0)) / zs;
                fu = ww * fr;
                ww = c1b * (AA(2, 2, 0, -1) + AA(2, 2, 0, 0)) * 0.5 - c2b * (AA(2, 2, 0, -2) + AA(2, 2, 0, 1)) * 0.5;
                fr = (zp * MM(1, 2, 0, 0) + zc * MM(1, 1, 0, 0)) / zs;
                fv = ww * fr;
            }
            if (k == 1) {   // Flux(1): levels 1, 2
                const double zp = ZW(2), zc = ZW(1), zs = zp + zc;
                double ww = c1b * (AA(2, 1, -1, 0) + AA(2, 1, 0, 0)) * 0.5 - c2b * (AA(2, 1, -2, 0) + AA(2, 1, 1, 0)) * 0.5;
                double fr = (zp * MM(0, 1, 0, 0) + zc * MM(0, 0, 0, 0)) / zs;
                fzu3 = ww * fr;
                ww = c1b * (AA(2, 1, 0, -1) + AA(2, 1, 0, 0)) * 0.5 - c2b * (AA(2, 1, 0, -2) + AA(2, 1, 0, 1)) * 0.5;
                fr = (zp * MM(1, 1, 0, 0) + zc * MM(1, 0, 0, 0)) / zs;
                fzv3 = ww * fr;
            }
            fzu0 = fzu1; fzu1 = fzu2; fzu2 = fzu3; fzu3 = fu;
            fzv0 = fzv1; fzv1 = fzv2; fzv2 = fzv3; fzv3 = fv;
            // advwz_fd Flux(k), Adv(k) (:1087-1098)
            double fw = 0., aw_ = 0.;
            if (k <= nz - 2) {
                double ww = (AA(2, 1, 0, 0) + AA(2, 0, 0, 0)) * 0.5;
                double fr = (MM(2, 1, 0, 0) + MM(2, 0, 0, 0)) * 0.5;
                fw = ww * fr;
                const double zp = ZW(k + 1), zc = ZW(k), zs = zp + zc;
                double ww2 = (zp * AA(2, 2, 0, 0) + zc * AA(2, 0, 0, 0)) / zs;
                double fr2 = (zp * MM(2, 2, 0, 0) + zc * MM(2, 0, 0, 0)) / zs;
                aw_ = ww2 * fr2;
            } else if (k == nz - 1) {
                fw = 0.25 * (AA(2, 1, 0, 0) + AA(2, 0, 0, 0)) * (MM(2, 1, 0, 0) + MM(2, 0, 0, 0));
                const double s2 = ZW(nz) + ZW(nz - 1);
                aw_ = (0. + ZW(nz - 1) * AA(2, 0, 0, 0)) * (0. + ZW(nz - 1) * MM(2, 0, 0, 0)) / (s2 * s2);
            }
            fzw0 = fzw1; fzw1 = fw;
            azw0 = azw1; azw1 = azw2; azw2 = aw_;
        }

        // ---------------- u component ----------------
        double au = 0.;
        for (int pass = 0; pass < 3; pass++) {
            int dir = even ? pass : 2 - pass;
            if (dir == 0) {   // advux_fd
#define FX(p) (((AA(0, 0, (p) + 1, 0) + AA(0, 0, (p), 0)) * 0.5) * ((MM(0, 0, (p) + 1, 0) + MM(0, 0, (p), 0)) * 0.5))
#define AX(p) (((AA(0, 0, (p) + 2, 0) + AA(0, 0, (p), 0)) * 0.5) * ((MM(0, 0, (p) + 2, 0) + MM(0, 0, (p), 0)) * 0.5))
                au = au + c1a * (FX(0) - FX(-1)) * dx1 - c2a * (AX(0) - AX(-2)) * dx2;
#undef FX
#undef AX
                if (G.lavisc) {
                    double mu = fabs(AA(0, 0, 0, 0)) * dx1;
                    au = au - AVISC * mu * (-MM(0, 0, 2, 0) + 4. * MM(0, 0, 1, 0) - 6. * MM(0, 0, 0, 0) + 4. * MM(0, 0, -1, 0) - MM(0, 0, -2, 0));
                }
            } else if (dir == 1) {   // advuy_fd: vt1=vt(i-1), vt2=vt(i), vt3=vt(i-2), vt4=vt(i+1)
#define FY(p) ((c1b * (AA(1, 0, -1, (p) + 1) + AA(1, 0, 0, (p) + 1)) * 0.5 - c2b * (AA(1, 0, -2, (p) + 1) + AA(1, 0, 1, (p) + 1)) * 0.5) * \
               ((MM(0, 0, 0, (p) + 1) + MM(0, 0, 0, (p))) * 0.5))
                au = au + c1b * (FY(0) - FY(-1)) * dy1 - c2b * (FY(1) - FY(-2)) * dy3;
#undef FY
                if (G.lavisc) {
                    double mu = 0.25 * fabs(AA(1, 0, -1, 0) + AA(1, 0, 0, 0) + AA(1, 0, -1, 1) + AA(1, 0, 0, 1)) * dy1;
                    au = au - AVISC * mu * (-MM(0, 0, 0, 2) + 4. * MM(0, 0, 0, 1) - 6. * MM(0, 0, 0, 0) + 4. * MM(0, 0, 0, -1) - MM(0, 0, 0, -2));
                }
            } else {   // advuz_fd, Flux(k-2..k+1) = fzu0..fzu3
                if (k >= 3 && k <= nz - 1)
                    au = au + c1b * (fzu2 - fzu1) * ZW1(k) - c2b * (fzu3 - fzu0) / (ZW(k - 1) + ZW(k) + ZW(k + 1));
                else if (k == 1)
                    au = au + (fzu2 - 0.) * ZW1(1);
                else if (k == 2)
                    au = au + c1b * (fzu2 - fzu1) * ZW1(1) - c2b * (fzu3 - 0.) / (ZW(1) + ZW(2) + ZW(3));
                else
                    au = au + (0. - fzu1) * ZW1(nz);
                if (G.lavisc && k >= 3 && k <= nz - 2) {
                    double mu = 0.25 * fabs(AA(2, 0, -1, 0) + AA(2, 0, 0, 0) + AA(2, 1, -1, 0) + AA(2, 1, 0, 0)) * ZW1(k);
                    au = au - AVISC * mu * (-MM(0, 2, 0, 0) + 4. * MM(0, 1, 0, 0) - 6. * MM(0, 0, 0, 0) + 4. * MM(0, -1, 0, 0) - MM(0, -2, 0, 0));
                }
            }
        }

        // ---------------- v component ----------------
        double av = 0.;
        for (int pass = 0; pass < 3; pass++) {
            int dir = even ? pass : 2 - pass;
            if (dir == 0) {   // advvx_fd: ut1=ut(j-1), ut2=ut(j), ut3=ut(j-2), ut4=ut(j+1)
#define FX(p) ((c1b * (AA(0, 0, (p) + 1, -1) + AA(0, 0, (p) + 1, 0)) * 0.5 - c2b * (AA(0, 0, (p) + 1, -2) + AA(0, 0, (p) + 1, 1)) * 0.5) * \
               ((MM(1, 0, (p) + 1, 0) + MM(1, 0, (p), 0)) * 0.5))
                av = av + c1b * (FX(0) - FX(-1)) * dx1 - c2b * (FX(1) - FX(-2)) * dx3;
#undef FX
                if (G.lavisc) {
                    double mu = 0.25 * fabs(AA(0, 0, 0, -1) + AA(0, 0, 0, 0) + AA(0, 0, 1, -1) + AA(0, 0, 1, 0)) * dx1;
                    av = av - AVISC * mu * (-MM(1, 0, 2, 0) + 4. * MM(1, 0, 1, 0) - 6. * MM(1, 0, 0, 0) + 4. * MM(1, 0, -1, 0) - MM(1, 0, -2, 0));
                }
            } else if (dir == 1) {   // advvy_fd
#define FY(p) (((AA(1, 0, 0, (p) + 1) + AA(1, 0, 0, (p))) * 0.5) * ((MM(1, 0, 0, (p) + 1) + MM(1, 0, 0, (p))) * 0.5))
#define AY(p) (((AA(1, 0, 0, (p) + 2) + AA(1, 0, 0, (p))) * 0.5) * ((MM(1, 0, 0, (p) + 2) + MM(1, 0, 0, (p))) * 0.5))
                av = av + c1a * (FY(0) - FY(-1)) * dy1 - c2a * (AY(0) - AY(-2)) * dy2;
#undef FY
#undef AY
                if (G.lavisc) {
                    double mu = fabs(AA(1, 0, 0, 0)) * dy1;
                    av = av - AVISC * mu * (-MM(1, 0, 0, 2) + 4. * MM(1, 0, 0, 1) - 6. * MM(1, 0, 0, 0) + 4. * MM(1, 0, 0, -1) - MM(1, 0, 0, -2));
                }
            } else {   // advvz_fd, Flux(k-2..k+1) = fzv0..fzv3
                if (k >= 3 && k <= nz - 1)
                    av = av + c1b * (fzv2 - fzv1) * ZW1(k) - c2b * (fzv3 - fzv0) / (ZW(k - 1) + ZW(k) + ZW(k + 1));
                else if (k == 1)
                    av = av + (fzv2 - 0.) * ZW1(1);
                else if (k == 2)
                    av = av + c1b * (fzv2 - fzv1) * ZW1(2) - c2b * (fzv3 - 0.) / (ZW(1) + ZW(2) + ZW(3));
                else
                    av = av + (0. - fzv1) * ZW1(nz);
                if (G.lavisc && k >= 3 && k <= nz - 2) {
                    double mu = 0.25 * fabs(AA(2, 0, 0, -1) + AA(2, 0, 0, 0) + AA(2, 1, 0, -1) + AA(2, 1, 0, 0)) * ZW1(k);
                    av = av - AVISC * mu * (-MM(1, 2, 0, 0) + 4. * MM(1, 1, 0, 0) - 6. * MM(1, 0, 0, 0) + 4. * MM(1, -1, 0, 0) - MM(1, -2, 0, 0));
                }
            }
        }

        // ---------------- w component (k >= 2) ----------------
        double aw = 0.;
        if (k >= 2) {
            for (int pass = 0; pass < 3; pass++) {
                int dir = even ? pass : 2 - pass;
                if (dir == 0) {   // advwx_fd
#define HV(p, d) AA(0, d, p, 0)
#define WV(p) MM(2, 0, p, 0)
#define FH(p) ((k == 2 ? (HV((p) + 1, 0) + HV((p) + 1, -1)) * 0.5                                            \
                       : (k == nz ? (HV((p) + 1, 0) + HV((p) + 1, -1)) * 0.5                                  \
                                  : c1b * (HV((p) + 1, 0) + HV((p) + 1, -1)) * 0.5 -                          \
                                        c2b * (HV((p) + 1, 1) + HV((p) + 1, -2)) * 0.5)) *                    \
                ((WV((p) + 1) + WV(p)) * 0.5))
                    aw = aw + c1b * (FH(0) - FH(-1)) * dx1 - c2b * (FH(1) - FH(-2)) * dx3;
                    if (G.lavisc) {
                        double mu = 0.25 * fabs(HV(0, 0) + HV(0, -1) + HV(1, 0) + HV(1, -1)) * dx1;
                        aw = aw - AVISC * mu * (-WV(2) + 4. * WV(1) - 6. * WV(0) + 4. * WV(-1) - WV(-2));
                    }
#undef HV
#undef WV
                } else if (dir == 1) {   // advwy_fd
#define HV(p, d) AA(1, d, 0, p)
#define WV(p) MM(2, 0, 0, p)
                    aw = aw + c1b * (FH(0) - FH(-1)) * dy1 - c2b * (FH(1) - FH(-2)) * dy3;
                    if (G.lavisc) {
                        double mu = 0.25 * fabs(HV(0, 0) + HV(0, -1) + HV(1, 0) + HV(1, -1)) * dy1;
                        aw = aw - AVISC * mu * (-WV(2) + 4. * WV(1) - 6. * WV(0) + 4. * WV(-1) - WV(-2));
                    }
#undef HV
#undef WV
#undef FH
                } else {   // advwz_fd, Flux(k-1..k) = fzw0..1, Adv(k-2..k) = azw0..2
                    if (k >= 3 && k <= nz - 1)
                        aw = aw + c1a * (fzw1 - fzw0) * Z1(k - 1) - c2a * (azw2 - azw0) / (ZW(k) + ZW(k - 1));
                    else if (k == 2)
                        aw = aw + c1a * (fzw1 - fzw0) * Z1(1) - c2a * (azw2 - 0.) / (ZW(2) + ZW(1));
                    else
                        aw = aw + (0. - fzw0) * Z1(nz - 1);
                    if (G.lavisc && k >= 3 && k <= nz - 2) {
                        double mu = fabs(AA(2, 0, 0, 0)) * Z1(k - 1);
                        aw = aw - AVISC * mu * (-MM(2, 2, 0, 0) + 4. * MM(2, 1, 0, 0) - 6. * MM(2, 0, 0, 0) + 4. * MM(2, -1, 0, 0) - MM(2, -2, 0, 0));
                    }
                }
            }
        }

        const long long idx = gidx(G, i, j, k);
        if (A.mode == 1) {
            A.ou[idx] = au;
            A.ov[idx] = av;
            A.ow[idx] = aw;
            continue;
        }

        // ---------------- explicit pressure gradient (gradp on p/rho0) ----------------
        const double d0 = ldg(G.den0, k - 1), a0 = ldg(G.avden0, k - 1);
        const double ppc = ldg(A.p, idx) / d0;
        const double gpx = (ppc - ldg(A.p, gidx(G, i - 1, j, k)) / d0) * dx1;
        const double gpy = (ppc - ldg(A.p, gidx(G, i, j - 1, k)) / d0) * dy1;
        double gpz;
        if (k >= 2) gpz = (ppc - pp_below) * Z1(k - 1);
        else gpz = MM(2, 0, 0, 0) / (dt0 * ldg(G.avden0, 0));
        pp_below = ppc;
        double wsu = 0. - d0 * gpx;
        double wsv = 0. - d0 * gpy;
        double wsw = 0. - a0 * gpz;

        // ---------------- buoyancy (imp_buoy: state + cdiag*dt0*states) ----------------
        double buoy = 0.;
        if (G.with_buoy) {
            double dn = ldg(A.dens, idx);
            double esv = ldg(A.es, idx), qtv = A.qt ? ldg(A.qt, idx) : 0.;
            if (A.dens_is_leveln) {
                esv = rep_value(A.rep, esv, dn);
                if (A.qt) qtv = rep_value(A.rep, qtv, dn);
            }
            double est = esv + cdiag * dt0 * ldg(A.fes, idx);
            double qtt = A.qt ? qtv + cdiag * dt0 * ldg(A.fqt, idx) : 0.;
            double den1 = 1. / dn;
            double pt = den1 * est;
            double sumh = 0.;
            double ref = ldg(G.pt0, k - 1) * (1. + epsm * ldg(G.qv0, k - 1));
            double bb = dn * grav * (pt * (1. + epsm * den1 * (qtt - sumh) - den1 * sumh) / ref - 1.);
            buoy = k >= 2 ? 0.5 * (bb_prev + bb) : bb;
            bb_prev = bb;
        }

        // ---------------- assembly and integ_mom ----------------
        wsu = -au + wsu;
        wsv = -av + wsv;
        wsw = -aw + wsw + buoy;
        double tu_o = A.stage == 1 ? 0. : A.tu[idx];
        double tv_o = A.stage == 1 ? 0. : A.tv[idx];
        double tw_o = A.stage == 1 ? 0. : A.tw[idx];
        double tu = wsu + A.b * tu_o, tv = wsv + A.b * tv_o, tw = wsw + A.b * tw_o;
        double un = rep_value(A.rep, ldg(A.mu_n, idx), d0);
        double vn = rep_value(A.rep, ldg(A.mv_n, idx), d0);
        double wn = rep_value(A.rep, ldg(A.mw_n, idx), a0);
        A.ou[idx] = un + A.a_dt * tu;
        A.ov[idx] = vn + A.a_dt * tv;
        A.ow[idx] = 1. * (wn + A.a_dt * tw);
        A.tu[idx] = tu;
        A.tv[idx] = tv;
        A.tw[idx] = tw;
    }
#undef MM
#undef AA
#undef ZW
#undef ZW1
#undef Z1
}

}  // namespace

cudaError_t launch_k2(const DevGrid &g, const K2Args &a, cudaStream_t s)
{
    int ntx = (g.maxx + TX - 1) / TX, nty = (g.maxy + TY - 1) / TY;
    size_t sm = (size_t)2 * NSLOT * 3 * PL * sizeof(double);
    cudaError_t e = cudaFuncSetAttribute(k2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    k2_kernel<<<ntx * nty, dim3(TX, TY), sm, s>>>(g, a);
    return cudaGetLastError();
}
