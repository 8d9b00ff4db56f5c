// weno_partials.cuh -- closed-form partial derivatives of the WENO3-switch face flux
// (src/TOOLS/advq_weno.f90, as weno_face_up in schemes.cuh evaluates it), for the
// tangent-linear and adjoint kernels of the scalar advection.  Host-callable, so that a
// host program can check it against the scheme evaluated on dual numbers.
#pragma once
#include <cmath>

#include "schemes.cuh"

// Closed-form partials of the interior WENO face flux weno_face_up(xm1, x0, xp1, xp2, u)
// with respect to its four stencil values (J) and its velocity (Ju), along the branch
// the FP64 form takes: the upwind side, the positivity limiter's phi (1, or |x0/den|
// with den = min(candidates) - x0 + eps), and linear or nonlinear weights, each decided
// by the forward's own expressions.  The same derivatives as the scheme evaluated on dual
// numbers (|u| with slope +1 at 0), without carrying partials through every operation:
// on the common branch (phi = 1, linear weights) J is a constant vector times the face's
// upwind factor.
__host__ __device__ __forceinline__ void weno_face_partials(double xm1, double x0, double xp1, double xp2,
                                                            double uu, bool full_weights, double J[4], double &Ju)
{
    const double eps = 1.e-15, g1 = 1. / 3., g2 = 2. / 3., thres = 20.;
    const double ffim1 = (-(0.5 * xm1) + 1.5 * x0);
    const double ffip1 = (0.5 * x0 + 0.5 * xp1);
    const double ffip2 = (1.5 * xp1 - 0.5 * xp2);
    const bool pos = !(uu < 0.);
    // d(candidate)/d(xm1, x0, xp1, xp2)
    const double dcf[4] = {pos ? -0.5 : 0., pos ? 1.5 : 0., pos ? 0. : 1.5, pos ? 0. : -0.5};
    const double dcc[4] = {0., 0.5, 0.5, 0.};
    // positivity limiter (:462-491): phi = min(|(0 - x0)/((minp - x0) + eps)|, 1)
    int im = 0;
    double minp = ffim1;
    if (!(minp < ffip1)) { minp = ffip1; im = 1; }
    if (!(minp < ffip1)) { minp = ffip1; im = 1; }
    if (!(minp < ffip2)) { minp = ffip2; im = 2; }
    const double num = 0. - x0, den = (minp - x0) + eps;
    double phi = 1., dphi[4] = {0., 0., 0., 0.};
    if (!(fabs(num) >= fabs(den))) {
        const double q = num / den;
        if (fabs(q) < 1.) {
            phi = fabs(q);
            const double sg = q < 0. ? -1. : 1.;
            // dq = (dnum * den - num * dden) / den^2, dnum = -dx0, dden = dminp - dx0
            const double dmin[4] = {im == 0 ? -0.5 : 0., im == 0 ? 1.5 : (im == 1 ? 0.5 : 0.),
                                    im == 1 ? 0.5 : (im == 2 ? 1.5 : 0.), im == 2 ? -0.5 : 0.};
            const double r2 = 1. / (den * den);
            for (int m = 0; m < 4; m++) {
                const double dx0 = m == 1 ? 1. : 0.;
                dphi[m] = sg * ((-dx0) * den - num * (dmin[m] - dx0)) * r2;
            }
        }
    }
    const double cf = pos ? ffim1 : ffip2;
    const double far = phi * (cf - x0) + x0, cen = phi * (ffip1 - x0) + x0;
    double wf = g1, wc = g2, dwf[4] = {0., 0., 0., 0.};
    if (full_weights) {
        const double dout = pos ? (x0 - xm1) : (xp2 - xp1);
        const double dmid = xp1 - x0;
        const double eo = dout * dout, em = dmid * dmid;
        if (ratio_gt(tmax(eo, em), tmin(eo, em) + eps, thres)) {
            const double yo = eps + eo, ym = eps + em;
            const double a = g1 / (yo * yo), b = g2 / (ym * ym);
            const double sa = a + b;
            wf = a / sa; wc = b / sa;
            // da = -4 a dout / yo d(dout), db = -4 b dmid / ym d(dmid); dwf = (da b - a db) / s^2
            const double ka = -4. * a * dout / yo, kb = -4. * b * dmid / ym, r2 = 1. / (sa * sa);
            const double ddo[4] = {pos ? -1. : 0., pos ? 1. : 0., pos ? 0. : -1., pos ? 0. : 1.};
            const double ddm[4] = {0., -1., 1., 0.};
            for (int m = 0; m < 4; m++) dwf[m] = (ka * ddo[m] * b - a * kb * ddm[m]) * r2;
        }
    }
    const double F = wf * far + wc * cen;
    const double up = 0.5 * (pos ? (uu + fabs(uu)) : (uu - fabs(uu)));   // u, or 0 at u = 0
    for (int m = 0; m < 4; m++) {
        const double dx0 = m == 1 ? 1. : 0.;
        const double dfar = dphi[m] * (cf - x0) + phi * (dcf[m] - dx0) + dx0;
        const double dcen = dphi[m] * (ffip1 - x0) + phi * (dcc[m] - dx0) + dx0;
        J[m] = up * (dwf[m] * (far - cen) + wf * dfar + wc * dcen);
    }
    Ju = F;
}

