// schemes.cuh -- per-face / per-cell arithmetic of the reference's scalar
// advection schemes, as device functions shared by the FP64 kernels (double)
// and the mixed-precision kernels (float).  Every expression keeps the reference's
// evaluation order; the FP64 translation unit is compiled without FMA contraction
// so that results match the CPU restatement bit for bit.
#pragma once
#include <cuda_runtime.h>

template <typename T> __host__ __device__ __forceinline__ T tmin(T a, T b) { return a < b ? a : b; }
template <typename T> __host__ __device__ __forceinline__ T tmax(T a, T b) { return a > b ? a : b; }
__host__ __device__ __forceinline__ double dabs(double a) { return fabs(a); }
__host__ __device__ __forceinline__ float dabs(float a) { return fabsf(a); }
__host__ __device__ __forceinline__ double sign1(double b) { return copysign(1.0, b); }
__host__ __device__ __forceinline__ float sign1(float b) { return copysignf(1.0f, b); }

// RN(a/b) > thr for b > 0, decided without the division when a lies clearly on one
// side of thr*b (a relative band of 1e-7 around thr); bit-identical to the division.
template <typename T> __host__ __device__ __forceinline__ bool ratio_gt(T a, T b, T thr);
template <> __host__ __device__ __forceinline__ bool ratio_gt<double>(double a, double b, double thr)
{
    if (a > b * (thr * 1.0000001)) return true;
    if (a < b * (thr * 0.9999999)) return false;
    return a / b > thr;
}
template <> __host__ __device__ __forceinline__ bool ratio_gt<float>(float a, float b, float thr) { return a > thr * b; }

// min(|num/den|, 1) of the positivity limiters: 1 exactly whenever |num| >= |den|
// (then |num/den| >= 1 and its rounding too, or the quotient is inf/NaN and min()
// returns 1), so the division is only evaluated when it can matter.
template <typename T> __host__ __device__ __forceinline__ T min_abs_ratio_1(T num, T den);
template <> __host__ __device__ __forceinline__ double min_abs_ratio_1<double>(double num, double den)
{
    if (fabs(num) >= fabs(den)) return 1.;
    const double q = fabs(num / den);
    return q < 1. ? q : 1.;
}
template <> __host__ __device__ __forceinline__ float min_abs_ratio_1<float>(float num, float den)
{
    if (fabsf(num) >= fabsf(den)) return 1.f;
    const float q = fabsf(num / den);
    return q < 1.f ? q : 1.f;
}

// ---------------- WENO3-switch: src/TOOLS/advq_weno.f90 ----------------
// Face flux at i+1/2 (:92-110; weights :304-353, limiter :462-491).  The reference
// evaluates both sides, Flux = 0.5*Fl*(u+|u|) + 0.5*Fr*(u-|u|), with Fl = w0*ffim1 +
// w1*ffip1p and Fr = w2*ffip1m + w3*ffip2 from the limited candidates, and weights that
// are linear (1/3, 2/3) unless the smoothness ratio max/min(eta) exceeds 20, then
// g/(eps+eta)^2 normalised; (eps+eta)**2 is the correctly rounded product.
// weno_face_up evaluates only the upwind side's weights and reconstruction.  For u > 0
// the reference's downwind term is 0.5*Fr*(u-|u|) = 0.5*Fr*0, a zero, and adding a zero
// to the upwind term leaves its value unchanged (u < 0 alike), so the result equals the
// reference's up to the sign of a zero flux.  The downwind side's
// weights (and their divisions) are not computed.  The right side is the left side's
// formula on the mirrored stencil (xp2, xp1, x0): eta1 <-> eta3, the candidates
// 1.5*xp1 - 0.5*xp2 and 0.5*xp1 + 0.5*x0, and the weight sum g1/y3^2 + g2/y2^2; every
// swapped operand pair is an IEEE addition or product, which commutes bit for bit.  The
// positivity limiter scales all four candidates about x0 with phi from their minimum,
// as :462-491 do, before one side is chosen.  u = 0 takes the left side: its value is a
// zero either way, and on dual numbers (whose |u| has slope +1 at 0) the left side's
// term 0.5*Fl*(u+|u|) is the one whose derivative, Fl*du, the two-sided form has.
template <typename T>
__host__ __device__ __forceinline__ T weno_face_up(T xm1, T x0, T xp1, T xp2, T uu, bool full_weights)
{
    const T eps = T(1.e-15), g1 = T(1.) / T(3.), g2 = T(2.) / T(3.), thres = T(20.);
    T ffim1 = (-(T(0.5) * xm1) + T(1.5) * x0);
    T ffip1 = (T(0.5) * x0 + T(0.5) * xp1);
    T ffip2 = (T(1.5) * xp1 - T(0.5) * xp2);
    T minp = tmin(tmin(tmin(ffim1, ffip1), ffip1), ffip2);
    T phi = min_abs_ratio_1(T(0.) - x0, (minp - x0) + eps);
    const bool pos = !(uu < T(0.));
    const T far = phi * ((pos ? ffim1 : ffip2) - x0) + x0;
    const T cen = phi * (ffip1 - x0) + x0;
    T wf = g1, wc = g2;
    if (full_weights) {
        const T dout = pos ? (x0 - xm1) : (xp2 - xp1);
        const T dmid = xp1 - x0;
        const T eo = dout * dout, em = dmid * dmid;
        if (ratio_gt(tmax(eo, em), tmin(eo, em) + eps, thres)) {
            const T yo = eps + eo, ym = eps + em;
            const T a = g1 / (yo * yo), b = g2 / (ym * ym);
            const T s = a + b;
            wf = a / s; wc = b / s;
        }
    }
    const T F = wf * far + wc * cen;
    return T(0.5) * F * (pos ? (uu + dabs(uu)) : (uu - dabs(uu)));
}
// vertical bottom face (k=1), :232-241
template <typename T>
__host__ __device__ __forceinline__ T weno_face_bottom(T x1, T x2, T x3, T ww)
{
    const T g1 = T(1.) / T(3.), g2 = T(2.) / T(3.);
    T ffip1p = (T(0.5) * x1 + T(0.5) * x2);
    T ffip1m = ffip1p;
    T ffip2 = (T(1.5) * x2 - T(0.5) * x3);
    T Fl = ffip1p;
    T Fr = g2 * ffip1m + g1 * ffip2;
    return T(0.5) * Fl * (ww + dabs(ww)) + T(0.5) * Fr * (ww - dabs(ww));
}
// vertical top face (k=nz-1), :262-271
template <typename T>
__host__ __device__ __forceinline__ T weno_face_top(T xm1, T x0, T xp1, T ww)
{
    const T g1 = T(1.) / T(3.), g2 = T(2.) / T(3.);
    T ffim1 = (-(T(0.5) * xm1) + T(1.5) * x0);
    T ffip1p = (T(0.5) * x0 + T(0.5) * xp1);
    T ffip1m = ffip1p;
    T Fl = g1 * ffim1 + g2 * ffip1p;
    T Fr = ffip1m;
    return T(0.5) * Fl * (ww + dabs(ww)) + T(0.5) * Fr * (ww - dabs(ww));
}

// ---------------- MUSCL: src/TOOLS/advq_muscl.f90 ----------------
// limiter_muscl (:335-383) for one side: phil is muscl_phi(.., ffip1, ffim1), phir is
// muscl_phi(.., ffip1, ffip2); the reference's two sides are the same expressions on
// their own slope.
template <typename T>
__host__ __device__ __forceinline__ T muscl_phi(int lim, T lim_tol, T xx, T ffip1, T ffo)
{
    T r = T(1.);
    if (dabs(ffo) > lim_tol * dabs(xx) && dabs(ffip1) < dabs(ffo) / lim_tol) r = ffip1 / ffo;
    if (lim == 1) return (r + dabs(r)) / (T(1.) + dabs(r));                               // VL
    if (lim == 2) return tmax(T(0.), tmin(tmin(T(2.) * r, T(0.5) * (r + T(1.))), T(2.)));   // MC
    if (lim == 0) return tmax(T(0.), tmin(T(1.), r));                                      // minmod
    return T(0.5) * (r + T(1.));
}

// The face fluxes below evaluate only the upwind side.  The reference's flux is
// 0.5*u*(Fl*(1+sign(1,u)) + Fr*(1-sign(1,u))) (:99): for sign(1,u) = 1 the second product
// is Fr*0, a zero, and Fl*2 + 0 = Fl*2, so the value is 0.5*u*(Fl*2) (sign(1,u) = -1
// alike with Fr); it differs from the two-sided expression at most in the sign of a zero.
// sign(1,u) has copysign semantics, so u = -0 takes the Fr side as the reference does.

// horizontal face between i and i+1 (advq_muscl.f90:81-100); d = dx, d1 = 1/dx
template <typename T>
__host__ __device__ __forceinline__ T muscl_face_h(int lim, T lim_tol, T d, T d1, T xm1, T x0, T xp1, T xp2, T uu)
{
    const T eps = T(1.e-18);
    T slope_p = (xp1 - x0) * d1;
    T slope_p2 = (xp2 - xp1) * d1;
    T slope_m = (x0 - xm1) * d1;
    const bool pos = sign1(uu) > T(0.);
    T F;
    if (d * dabs(slope_m) > lim_tol * dabs(x0) + eps || d * dabs(slope_p2) > lim_tol * dabs(x0) + eps) {
        const T phi = muscl_phi(lim, lim_tol, x0, slope_p, pos ? slope_m : slope_p2);
        F = pos ? x0 + T(0.5) * phi * slope_m * d : xp1 - T(0.5) * phi * slope_p2 * d;
    } else {
        F = pos ? x0 + T(0.5) * slope_p * d : xp1 - T(0.5) * slope_p * d;
    }
    return T(0.5) * uu * (F * T(2.));
}

// vertical face k+1/2 (advq_muscl.f90:245-302).  kind: 0 core, 1 bottom (k=1), 2 top (k=nz-1).
// xm1..xp2 = x(k-1..k+2); d1m = dz1(k-1), d10 = dz1(k), d1p = dz1(k+1); fm = fdz0(k-1),
// fp = fdz0(k+1); dzw1 = dz1w(k).
template <typename T>
__host__ __device__ __forceinline__ T muscl_face_z(int kind, int lim, T lim_tol, T dz, T xm1, T x0, T xp1, T xp2,
                                          T d1m, T d10, T d1p, T fm, T fp, T dzw1, T ww)
{
    const T eps = T(1.e-18);
    T slope_p, slope_p2, slope_m;
    bool lim_on;
    if (kind == 1) {
        slope_p = (xp1 - x0) * d10;
        slope_p2 = (xp2 - xp1) * d1p;
        slope_m = slope_p;
        lim_on = fp * dz * dabs(slope_p2) > lim_tol * dabs(x0) + eps;
    } else {
        slope_p = (xp1 - x0) * d10;
        slope_m = (x0 - xm1) * d1m;
        if (kind == 2) {
            slope_p2 = slope_p;
            lim_on = fm * dz * dabs(slope_m) > lim_tol * dabs(x0) + eps;
        } else {
            slope_p2 = (xp2 - xp1) * d1p;
            lim_on = fm * dz * dabs(slope_m) > lim_tol * dabs(x0) + eps ||
                     fp * dz * dabs(slope_p2) > lim_tol * dabs(x0) + eps;
        }
    }
    const bool pos = sign1(ww) > T(0.);
    T F;
    if (lim_on) {
        const T phi = muscl_phi(lim, lim_tol, x0, slope_p, pos ? slope_m : slope_p2);
        F = pos ? x0 + T(0.5) * phi * slope_m / dzw1 : xp1 - T(0.5) * phi * slope_p2 / dzw1;
    } else {
        F = pos ? x0 + T(0.5) * slope_p / dzw1 : xp1 - T(0.5) * slope_p / dzw1;
    }
    return T(0.5) * ww * (F * T(2.));
}

// ---------------- lw: src/TOOLS/advq_lw.f90 (limiter 'MC', the module constant) ----------------
template <typename T>
__host__ __device__ __forceinline__ void lw_limiter(T lim_tol, T xx, T ffip1, T ffip2, T ffim1, T &phir, T &phil)
{
    const T eps = T(1.e-18);
    T rp1 = T(1.), rp2 = T(1.);
    if (dabs(ffim1) > lim_tol * dabs(xx) + eps) rp1 = ffip1 / ffim1;
    if (dabs(ffip2) > lim_tol * dabs(xx) + eps) rp2 = ffip1 / ffip2;
    phil = tmax(tmin(tmin(T(2.) * rp1, T(0.5) * (rp1 + T(1.))), T(2.)), T(0.));
    phir = tmax(tmin(tmin(T(2.) * rp2, T(0.5) * (rp2 + T(1.))), T(2.)), T(0.));
}

// horizontal face between i and i+1 (advq_lw.f90:82-101); d1 = 1/dx
template <typename T>
__host__ __device__ __forceinline__ T lw_face_h(T lim_tol, T dt0, T d1, T xm1, T x0, T xp1, T xp2, T uu)
{
    const T eps = T(1.e-18);
    const T ffip1 = xp1 - x0, ffim1 = x0 - xm1, ffip2 = xp2 - xp1;
    const T mu = dabs(uu) * dt0 * d1;
    T fl, fr;
    if (dabs(ffim1) > lim_tol * dabs(x0) + eps || dabs(ffip2) > lim_tol * dabs(x0) + eps) {
        T phir, phil;
        lw_limiter(lim_tol, x0, ffip1, ffip2, ffim1, phir, phil);
        fl = x0 + T(0.5) * phil * ffim1 * (T(1.) - mu);
        fr = xp1 - T(0.5) * phir * ffip2 * (T(1.) - mu);
    } else {
        fl = x0 + T(0.5) * ffip1 * (T(1.) - mu);
        fr = xp1 - T(0.5) * ffip1 * (T(1.) - mu);
    }
    return T(0.5) * uu * (fl * (sign1(uu) + T(1.)) - fr * (sign1(uu) - T(1.)));
}

// vertical face k+1/2 (advq_lw.f90:246-311).  kind: 0 core, 1 bottom (k=1, ffim1 = ffip1),
// 2 top (k=nz-1, ffip2 = ffip1).  d1m, d10, d1p = dz1(k-1), dz1(k), dz1(k+1); dzw1 = dz1w(k).
template <typename T>
__host__ __device__ __forceinline__ T lw_face_z(int kind, T lim_tol, T dz, T dt0, T xm1, T x0, T xp1, T xp2,
                                       T d1m, T d10, T d1p, T dzw1, T ww)
{
    const T eps = T(1.e-18);
    const T ffip1 = (xp1 - x0) * d10;
    const T ffim1 = kind == 1 ? ffip1 : (x0 - xm1) * d1m;
    const T ffip2 = kind == 2 ? ffip1 : (xp2 - xp1) * d1p;
    const T mu = dabs(ww) * dt0 * d10;
    T fl, fr;
    if (dz * dabs(ffim1) > lim_tol * dabs(x0) + eps || dz * dabs(ffip2) > lim_tol * dabs(x0) + eps) {
        T phir, phil;
        lw_limiter(lim_tol, x0, ffip1, ffip2, ffim1, phir, phil);
        fl = x0 + T(0.5) * phil * ffim1 * (T(1.) - mu) / dzw1;
        fr = xp1 - T(0.5) * phir * ffip2 * (T(1.) - mu) / dzw1;
    } else {
        fl = x0 + T(0.5) * ffip1 * (T(1.) - mu) / dzw1;
        fr = xp1 - T(0.5) * ffip1 * (T(1.) - mu) / dzw1;
    }
    return T(0.5) * ww * (fl * (sign1(ww) + T(1.)) - fr * (sign1(ww) - T(1.)));
}

// ---------------- QUICK: src/TOOLS/advq_quick.f90 ----------------
template <typename T>
__host__ __device__ __forceinline__ void quick_limiter(T lim_tol, T phic, T ffip1, T ffip2, T ffim1, T &phil, T &phir)
{
    const T eps = T(1.e-18);
    const T c1 = T(1.) / T(3.);
    const T thr = lim_tol * dabs(phic) + eps;
    T rp1 = T(1.), rp2 = T(1.), rp11 = T(1.), rp21 = T(1.);
    if (dabs(ffim1) > thr) rp1 = ffip1 / ffim1;
    if (dabs(ffip2) > thr) rp2 = ffip1 / ffip2;
    if (dabs(ffip1) > thr) {
        rp11 = ffim1 / ffip1;
        rp21 = ffip2 / ffip1;
    }
    phil = rp1 * (T(1.) - c1 * (T(1.) - rp11));
    phir = rp2 * (T(1.) - c1 * (T(1.) - rp21));
    if (dabs(ffim1) > thr || dabs(ffip2) > thr) {
        phil = tmax(T(0.), tmin(T(2.) * rp1, tmin(phil, T(2.))));
        phir = tmax(T(0.), tmin(T(2.) * rp2, tmin(phir, T(2.))));
    }
}

// horizontal face between i and i+1 (advq_quick.f90:79-93)
template <typename T>
__host__ __device__ __forceinline__ T quick_face_h(T lim_tol, T xm1, T x0, T xp1, T xp2, T uu)
{
    const T ffip1 = xp1 - x0, ffip2 = xp2 - xp1, ffim1 = x0 - xm1;
    T phil, phir;
    quick_limiter(lim_tol, x0, ffip1, ffip2, ffim1, phil, phir);
    const T Fl = x0 + T(0.5) * phil * ffim1;
    const T Fr = xp1 - T(0.5) * phir * ffip2;
    return T(0.5) * Fl * (uu + dabs(uu)) + T(0.5) * Fr * (uu - dabs(uu));
}

// vertical face k+1/2 (advq_quick.f90:235-279), kinds and arguments as lw_face_z
template <typename T>
__host__ __device__ __forceinline__ T quick_face_z(int kind, T lim_tol, T dz, T xm1, T x0, T xp1, T xp2, T d1m, T d10,
                                          T d1p, T dzw1, T ww)
{
    const T ffip1 = (xp1 - x0) * d10;
    const T ffip2 = kind == 2 ? ffip1 : (xp2 - xp1) * d1p;
    const T ffim1 = kind == 1 ? ffip1 : (x0 - xm1) * d1m;
    T phil, phir;
    quick_limiter(lim_tol, x0 / dz, ffip1, ffip2, ffim1, phil, phir);
    const T Fl = x0 + T(0.5) * phil * ffim1 / dzw1;
    const T Fr = xp1 - T(0.5) * phir * ffip2 / dzw1;
    return T(0.5) * Fl * (ww + dabs(ww)) + T(0.5) * Fr * (ww - dabs(ww));
}

// ---------------- PPM: src/TOOLS/advq_ppm.f90 ----------------
// spacing() of Fortran (2**(exponent-digits)), tiny() for 0
__device__ __forceinline__ double fspacing(double x)
{
    if (x == 0.0) return 2.2250738585072014e-308;
    int e = ilogb(x) - 52;
    if (e < -1022) return 2.2250738585072014e-308;
    return ldexp(1.0, e);
}
__device__ __forceinline__ float fspacing(float x)
{
    if (x == 0.0f) return 1.17549435e-38f;
    int e = ilogbf(x) - 23;
    if (e < -126) return 1.17549435e-38f;
    return ldexpf(1.0f, e);
}
__device__ __forceinline__ double tsqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float tsqrt(float x) { return sqrtf(x); }

// limiter_ppm :449-530 with ppmlimiter='PPM'
template <typename T>
__host__ __device__ __forceinline__ void ppm_limiter(T xx, T xp, T xm, T xplus, T xmin, T ffip1, T ffip2, T ffim1,
                                            T ffim2, T &phir, T &phil, T &phi1, T &phi2)
{
    const T eps = T(1.e-15), thres = T(10.);
    T rp1 = T(1.);
    phir = xplus; phil = xmin;
    T a, b;
    a = ffip1 - ffim1; b = ffip1 + ffim1;
    T gamma1 = T(0.5) * (a * a + b * b);
    a = ffip2 - ffip1; b = ffip2 + ffip1;
    T gamma2 = T(0.5) * (a * a + b * b);
    a = ffim1 - ffim2; b = ffim1 + ffim2;
    T gamma3 = T(0.5) * (a * a + b * b);
    const bool sel = ratio_gt(tmax(tmax(gamma1, gamma2), gamma3), tmin(tmin(gamma1, gamma2), gamma3) + eps, thres);
    phi1 = phir - phil;
    phi2 = T(3.) * (phil - T(2.) * xx + phir);
    if (sel) {
        if (phir < T(0.) || ((phir - xx) * (xp - phir) < T(0.) &&
                             (ffim1 * ffip2 >= T(0.) || ffim1 * ffip1 <= T(0.) || ffip2 * ffip1 <= T(0.)))) {
            if (dabs(phir - xx) < dabs(phir - xp)) phir = xx;
            else phir = xp;
        }
        if (phil < T(0.) || ((xx - phil) * (phil - xm) < T(0.) &&
                             (ffim2 * ffip1 >= T(0.) || ffim2 * ffim1 <= T(0.) || ffip1 * ffim1 <= T(0.)))) {
            if (dabs(phil - xx) < dabs(phil - xm)) phil = xx;
            else phil = xm;
        }
        phi1 = phir - phil;
        phi2 = T(3.) * (phil - T(2.) * xx + phir);
        T slope = -(T(0.5) * phi1 / (sign1(phi2) * tmax(dabs(phi2), eps)));
        if (dabs(ffim1) > tsqrt(fspacing(ffim1))) rp1 = ffip1 / ffim1;
        if (dabs(phi2) > eps && (slope > T(-0.5) || slope < T(0.5))) {
            T lim = tmax(T(0.), tmin(tmin(T(2.), T(0.5) * (rp1 + T(1.))), T(2.) * rp1));
            phir = xx + T(0.5) * ffim1 * lim;
            phil = xx - T(0.5) * ffim1 * lim;
            if ((xx - phil) * (phir - xx) < T(0.)) {
                phil = xx;
                phir = xx;
            }
            phi1 = phir - phil;
            phi2 = T(0.);
        }
    }
}

// uniform-grid face value xplus of cell i (advq_ppm.f90:108-110)
template <typename T>
__host__ __device__ __forceinline__ T ppm_xplus_core(T xm1, T x0, T xp1, T xp2)
{
    T ffip1 = (xp1 - x0), ffip2 = (xp2 - xp1), ffim1 = (x0 - xm1);
    T sl = T(0.5) * (ffip1 + ffim1);
    T slp1 = T(0.5) * (ffip2 + ffip1);
    return x0 + T(0.5) * ffip1 - T(1.) / T(6.) * (slp1 - sl);
}

// Courant-number fluxes (advq_ppm.f90:93-94)
template <typename T> __host__ __device__ __forceinline__ T ppm_fr(T phir, T mup, T phi1, T phi2)
{ return phir - T(0.5) * mup * (phi1 + (T(1.) - T(2.) / T(3.) * mup) * phi2); }
template <typename T> __host__ __device__ __forceinline__ T ppm_fl(T phil, T muc, T phi1, T phi2)
{ return phil + T(0.5) * muc * (phi1 - (T(1.) - T(2.) / T(3.) * muc) * phi2); }

// Horizontal cell reconstruction of cell c, pencil of length n (1-based).
// xv[0..4] = x(c-2..c+2) (entries outside the pencil unused).  kind:
//  0 core (5 <= c <= n-2), 1 left ghost (c = 3, :79-94), 2 first interior (c = 4,
//  xmin from the left-ghost xplus), 3 right ghost (c = n-1, :120-134).
// xmin of a cell is the unlimited xplus of the cell before it (:98,117).
// Returns phir, phil, phi1, phi2 (the velocity-independent part).
template <typename T>
__host__ __device__ __forceinline__ void ppm_cell_h(int kind, const T *xv, T &phir, T &phil, T &phi1, T &phi2)
{
    T xm2 = xv[0], xm1 = xv[1], x0 = xv[2], xp1 = xv[3], xp2 = xv[4];
    T ffip1, ffip2, ffim1, ffim2, xplus, xmin;
    if (kind == 1) {
        ffip1 = (xp1 - x0);
        ffip2 = (xp2 - xp1);
        ffim1 = (x0 - xm1);
        ffim2 = (x0 - xm1);
        xmin = T(0.5) * (xp1 + x0);
        xplus = x0 + T(0.5) * ffip1;
    } else if (kind == 3) {
        ffip1 = (xp1 - x0);
        ffip2 = (xp1 - x0);
        ffim1 = (x0 - xm1);
        ffim2 = (xm1 - xm2);
        xplus = x0 + T(0.5) * ffip1;
        xmin = ppm_xplus_core(xm2, xm1, x0, xp1);
    } else {
        ffip1 = (xp1 - x0);
        ffip2 = (xp2 - xp1);
        ffim1 = (x0 - xm1);
        ffim2 = (xm1 - xm2);
        xplus = ppm_xplus_core(xm1, x0, xp1, xp2);
        if (kind == 2) xmin = xm1 + T(0.5) * (x0 - xm1);
        else xmin = ppm_xplus_core(xm2, xm1, x0, xp1);
    }
    ppm_limiter(x0, xp1, xm1, xplus, xmin, ffip1, ffip2, ffim1, ffim2, phir, phil, phi1, phi2);
}

// Stretched-grid face value of cell k (advq_ppm.f90:374-383); dm1..dp2 = dz1w(k-1..k+2)
template <typename T>
__host__ __device__ __forceinline__ T ppm_xplus_z(T x0, T ffip1, T ffip2, T ffim1, T deltam1, T delta, T deltap1, T deltap2)
{
    T sl = delta / (deltam1 + delta + deltap1) *
           ((T(2.) * deltam1 + delta) / (deltap1 + delta) * ffip1 + (delta + T(2.) * deltap1) / (deltam1 + delta) * ffim1);
    T slp1 = deltap1 / (delta + deltap1 + deltap2) *
             ((T(2.) * delta + deltap1) / (deltap2 + deltap1) * ffip2 + (deltap1 + T(2.) * deltap2) / (delta + deltap1) * ffip1);
    return x0 + delta / (delta + deltap1) * ffip1 +
           T(1.) / (deltam1 + delta + deltap1 + deltap2) *
               (T(2.) * deltap1 * delta / (delta + deltap1) *
                    ((deltam1 + delta) / (T(2.) * delta + deltap1) - (deltap2 + deltap1) / (T(2.) * deltap1 + delta)) * ffip1 -
                delta * (deltam1 + delta) / (T(2.) * delta + deltap1) * slp1 +
                deltap1 * (deltap1 + deltap2) / (T(2.) * deltap1 + delta) * sl);
}

// =====================================================================================
// Mixed form: the scheme logic in FP32 on differences relative to the upwind cell
// value, the face flux u*(x_upwind + delta) in FP64.  Same algorithm as above
// (identical in exact arithmetic); FP32 only ever holds perturbations, so the
// cancellation in the flux differences costs no digits of the FP64 state.
// =====================================================================================

// WENO3-switch face i+1/2, returning the flux in FP64: the scheme logic runs in FP32 on
// the differences from x0; only the upwind side's weights are evaluated (the mirrored
// stencil for u < 0, as weno_face_up explains); the limiter sees all four candidates.
__device__ __forceinline__ double weno_face_up_mixed(double xm1, double x0, double xp1, double xp2, double uu,
                                                     bool full_weights)
{
    const float eps = 1.e-15f, thres = 20.f, g1 = 1.f / 3.f, g2 = 2.f / 3.f;
    const float a = (float)(xm1 - x0), b = (float)(xp1 - x0), c = (float)(xp2 - x0);
    const bool pos = uu > 0.;
    float wf = g1, wc = g2;
    if (full_weights) {
        const float dout = pos ? a : c - b;
        const float eo = dout * dout, em = b * b;
        if (fmaxf(eo, em) > thres * (fminf(eo, em) + eps)) {
            const float yo = eps + eo, ym = eps + em;
            // wf = g1/yo^2 / (g1/yo^2 + g2/ym^2) = g1 ym^2 / (g1 ym^2 + g2 yo^2)
            const float p = g1 * (ym * ym), q = g2 * (yo * yo), r = __frcp_rn(p + q);
            wf = p * r; wc = q * r;
        }
    }
    const float d1 = -0.5f * a, d2 = 0.5f * b, d3 = 1.5f * b - 0.5f * c;   // reconstructions minus x0
    const float mind = fminf(fminf(d1, d2), d3);
    const float x0f = (float)x0;
    const float den = mind + eps;
    const float phi = fabsf(x0f) >= fabsf(den) ? 1.f : fabsf(x0f / den);
    const float dsel = phi * (wf * (pos ? d1 : d3) + wc * d2);
    return uu == 0. ? 0. : uu * (x0 + (double)dsel);
}
__device__ __forceinline__ double weno_face_bottom_mixed(double x1, double x2, double x3, double ww)
{
    // Fl = (x1+x2)/2; Fr = g2 (x1+x2)/2 + g1 (1.5 x2 - 0.5 x3), relative to x1
    const float b = (float)(x2 - x1), c = (float)(x3 - x1);
    const float dl = 0.5f * b, dr = (2.f / 3.f) * (0.5f * b) + (1.f / 3.f) * (1.5f * b - 0.5f * c);
    return ww > 0. ? ww * (x1 + (double)dl) : (ww < 0. ? ww * (x1 + (double)dr) : 0.);
}
__device__ __forceinline__ double weno_face_top_mixed(double xm1, double x0, double xp1, double ww)
{
    const float a = (float)(xm1 - x0), b = (float)(xp1 - x0);
    const float dl = (1.f / 3.f) * (-0.5f * a) + (2.f / 3.f) * (0.5f * b), dr = 0.5f * b;
    return ww > 0. ? ww * (x0 + (double)dl) : (ww < 0. ? ww * (x0 + (double)dr) : 0.);
}

// MUSCL horizontal face between i and i+1, relative to x0 (upwind for u > 0) and xp1
__device__ __forceinline__ double muscl_face_h_mixed(int lim, float lim_tol, float d, float d1, double xm1, double x0,
                                                     double xp1, double xp2, double uu)
{
    const float eps = 1.e-18f;
    const float sp = (float)(xp1 - x0) * d1, sp2 = (float)(xp2 - xp1) * d1, sm = (float)(x0 - xm1) * d1;
    const float ax = fabsf((float)x0);
    const bool pos = uu >= 0.;
    float dd;   // upwind face value minus its cell value
    if (d * fabsf(sm) > lim_tol * ax + eps || d * fabsf(sp2) > lim_tol * ax + eps) {
        const float phi = muscl_phi(lim, lim_tol, (float)x0, sp, pos ? sm : sp2);
        dd = pos ? 0.5f * phi * sm * d : -0.5f * phi * sp2 * d;
    } else {
        dd = pos ? 0.5f * sp * d : -0.5f * sp * d;
    }
    return uu * ((pos ? x0 : xp1) + (double)dd);
}
__device__ __forceinline__ double muscl_face_z_mixed(int kind, int lim, float lim_tol, float dz, double xm1, double x0,
                                                     double xp1, double xp2, float d1m, float d10, float d1p, float fm,
                                                     float fp, float dzw1, double ww)
{
    const float eps = 1.e-18f;
    const float ax = fabsf((float)x0);
    const float sp = (float)(xp1 - x0) * d10;
    float sp2, sm;
    bool lim_on;
    if (kind == 1) {
        sp2 = (float)(xp2 - xp1) * d1p;
        sm = sp;
        lim_on = fp * dz * fabsf(sp2) > lim_tol * ax + eps;
    } else {
        sm = (float)(x0 - xm1) * d1m;
        if (kind == 2) {
            sp2 = sp;
            lim_on = fm * dz * fabsf(sm) > lim_tol * ax + eps;
        } else {
            sp2 = (float)(xp2 - xp1) * d1p;
            lim_on = fm * dz * fabsf(sm) > lim_tol * ax + eps || fp * dz * fabsf(sp2) > lim_tol * ax + eps;
        }
    }
    const float h = 0.5f / dzw1;
    const bool pos = ww >= 0.;
    float dd;   // upwind face value minus its cell value
    if (lim_on) {
        const float phi = muscl_phi(lim, lim_tol, (float)x0, sp, pos ? sm : sp2);
        dd = pos ? phi * sm * h : -(phi * sp2 * h);
    } else {
        dd = pos ? sp * h : -(sp * h);
    }
    return ww * ((pos ? x0 : xp1) + (double)dd);
}

// lw faces in the mixed form: FP32 slopes of differences relative to the upwind cell,
// FP64 flux (same switch structure as lw_face_h / lw_face_z)
__device__ __forceinline__ double lw_face_h_mixed(float lim_tol, float dt0, float d1, double xm1, double x0,
                                                  double xp1, double xp2, double uu)
{
    const float eps = 1.e-18f;
    const float sp = (float)(xp1 - x0), sp2 = (float)(xp2 - xp1), sm = (float)(x0 - xm1);
    const float ax = fabsf((float)x0);
    const float om = 1.f - fabsf((float)uu) * dt0 * d1;
    float dr, dl;
    if (fabsf(sm) > lim_tol * ax + eps || fabsf(sp2) > lim_tol * ax + eps) {
        float phir, phil;
        lw_limiter(lim_tol, (float)x0, sp, sp2, sm, phir, phil);
        dl = 0.5f * phil * sm * om;
        dr = -(0.5f * phir * sp2 * om);
    } else {
        dl = 0.5f * sp * om;
        dr = -dl;
    }
    return uu >= 0. ? uu * (x0 + (double)dl) : uu * (xp1 + (double)dr);
}
__device__ __forceinline__ double lw_face_z_mixed(int kind, float lim_tol, float dz, float dt0, double xm1, double x0,
                                                  double xp1, double xp2, float d1m, float d10, float d1p, float dzw1,
                                                  double ww)
{
    const float eps = 1.e-18f;
    const float sp = (float)(xp1 - x0) * d10;
    const float sm = kind == 1 ? sp : (float)(x0 - xm1) * d1m;
    const float sp2 = kind == 2 ? sp : (float)(xp2 - xp1) * d1p;
    const float ax = fabsf((float)x0);
    const float h = 0.5f * (1.f - fabsf((float)ww) * dt0 * d10) / dzw1;
    float dr, dl;
    if (dz * fabsf(sm) > lim_tol * ax + eps || dz * fabsf(sp2) > lim_tol * ax + eps) {
        float phir, phil;
        lw_limiter(lim_tol, (float)x0, sp, sp2, sm, phir, phil);
        dl = phil * sm * h;
        dr = -(phir * sp2 * h);
    } else {
        dl = sp * h;
        dr = -dl;
    }
    return ww >= 0. ? ww * (x0 + (double)dl) : ww * (xp1 + (double)dr);
}
// QUICK faces in the mixed form
__device__ __forceinline__ double quick_face_h_mixed(float lim_tol, double xm1, double x0, double xp1, double xp2,
                                                     double uu)
{
    const float sp = (float)(xp1 - x0), sp2 = (float)(xp2 - xp1), sm = (float)(x0 - xm1);
    float phil, phir;
    quick_limiter(lim_tol, (float)x0, sp, sp2, sm, phil, phir);
    const float dl = 0.5f * phil * sm, dr = -(0.5f * phir * sp2);
    return uu > 0. ? uu * (x0 + (double)dl) : (uu < 0. ? uu * (xp1 + (double)dr) : 0.);
}
__device__ __forceinline__ double quick_face_z_mixed(int kind, float lim_tol, float dz, double xm1, double x0,
                                                     double xp1, double xp2, float d1m, float d10, float d1p,
                                                     float dzw1, double ww)
{
    const float sp = (float)(xp1 - x0) * d10;
    const float sp2 = kind == 2 ? sp : (float)(xp2 - xp1) * d1p;
    const float sm = kind == 1 ? sp : (float)(x0 - xm1) * d1m;
    float phil, phir;
    quick_limiter(lim_tol, (float)x0 / dz, sp, sp2, sm, phil, phir);
    const float h = 0.5f / dzw1;
    const float dl = phil * sm * h, dr = -(phir * sp2 * h);
    return ww > 0. ? ww * (x0 + (double)dl) : (ww < 0. ? ww * (xp1 + (double)dr) : 0.);
}

// PPM: reconstruction of a cell relative to its own value x0; xv[] holds
// differences x(c-2..c+2) - x0 in FP32 and x0f the value itself (positivity tests).
// Outputs dr = phir - x0, dl = phil - x0, phi1, phi2.
__device__ __forceinline__ void ppm_limiter_rel(float x0f, float dp, float dm, float dplus, float dmin, float ffip1,
                                                float ffip2, float ffim1, float ffim2, float &dr, float &dl, float &phi1,
                                                float &phi2)
{
    // same logic as ppm_limiter with xx -> 0 (values relative to x0) and the
    // positivity tests phir < 0  <=>  dr < -x0
    const float eps = 1.e-15f, thres = 10.f;
    float rp1 = 1.f;
    dr = dplus; dl = dmin;
    float a, b;
    a = ffip1 - ffim1; b = ffip1 + ffim1;
    const float gamma1 = 0.5f * (a * a + b * b);
    a = ffip2 - ffip1; b = ffip2 + ffip1;
    const float gamma2 = 0.5f * (a * a + b * b);
    a = ffim1 - ffim2; b = ffim1 + ffim2;
    const float gamma3 = 0.5f * (a * a + b * b);
    const bool sel = fmaxf(fmaxf(gamma1, gamma2), gamma3) > thres * (fminf(fminf(gamma1, gamma2), gamma3) + eps);
    phi1 = dr - dl;
    phi2 = 3.f * (dl + dr);
    if (sel) {
        if (dr < -x0f || ((dr) * (dp - dr) < 0.f && (ffim1 * ffip2 >= 0.f || ffim1 * ffip1 <= 0.f || ffip2 * ffip1 <= 0.f))) {
            if (fabsf(dr) < fabsf(dr - dp)) dr = 0.f;
            else dr = dp;
        }
        if (dl < -x0f || ((-dl) * (dl - dm) < 0.f && (ffim2 * ffip1 >= 0.f || ffim2 * ffim1 <= 0.f || ffip1 * ffim1 <= 0.f))) {
            if (fabsf(dl) < fabsf(dl - dm)) dl = 0.f;
            else dl = dm;
        }
        phi1 = dr - dl;
        phi2 = 3.f * (dl + dr);
        const float slope = -(0.5f * phi1 / (copysignf(1.f, phi2) * fmaxf(fabsf(phi2), eps)));
        if (fabsf(ffim1) > sqrtf(fspacing(ffim1))) rp1 = ffip1 / ffim1;
        if (fabsf(phi2) > eps && (slope > -0.5f || slope < 0.5f)) {
            const float lim = fmaxf(0.f, fminf(fminf(2.f, 0.5f * (rp1 + 1.f)), 2.f * rp1));
            dr = 0.5f * ffim1 * lim;
            dl = -(0.5f * ffim1 * lim);
            if ((-dl) * (dr) < 0.f) { dl = 0.f; dr = 0.f; }
            phi1 = dr - dl;
            phi2 = 0.f;
        }
    }
}

// horizontal cell recon, mixed: xv = x(c-2..c+2) in FP64; outputs relative to x(c)
__device__ __forceinline__ void ppm_cell_h_mixed(int kind, const double *xv, float &dr, float &dl, float &phi1, float &phi2)
{
    const double x0 = xv[2];
    const float m2 = (float)(xv[0] - x0), m1 = (float)(xv[1] - x0), p1 = (float)(xv[3] - x0), p2 = (float)(xv[4] - x0);
    float ffip1, ffip2, ffim1, ffim2, dplus, dmin;
    if (kind == 1) {
        ffip1 = p1; ffip2 = p2 - p1; ffim1 = -m1; ffim2 = -m1;
        dmin = 0.5f * p1;
        dplus = 0.5f * ffip1;
    } else if (kind == 3) {
        ffip1 = p1; ffip2 = p1; ffim1 = -m1; ffim2 = m1 - m2;
        dplus = 0.5f * ffip1;
        dmin = m1 + 0.5f * (-m1) - (1.f / 6.f) * (0.5f * ((p1 - 0.f) + (0.f - m1)) - 0.5f * ((0.f - m1) + (m1 - m2)));
    } else {
        ffip1 = p1; ffip2 = p2 - p1; ffim1 = -m1; ffim2 = m1 - m2;
        dplus = 0.5f * ffip1 - (1.f / 6.f) * (0.5f * (ffip2 + ffip1) - 0.5f * (ffip1 + ffim1));
        if (kind == 2) dmin = m1 + 0.5f * (-m1);
        else dmin = m1 + 0.5f * (-m1) - (1.f / 6.f) * (0.5f * (p1 + (-m1)) - 0.5f * ((-m1) + (m1 - m2)));
    }
    ppm_limiter_rel((float)x0, p1, m1, dplus, dmin, ffip1, ffip2, ffim1, ffim2, dr, dl, phi1, phi2);
}
