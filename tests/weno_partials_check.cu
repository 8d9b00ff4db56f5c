// Host check of the closed-form WENO face partials (fdd3260_b200/csrc/weno_partials.cuh)
// against the face flux evaluated on 5-partial dual numbers (dual.cuh), on seeded random
// stencils built to reach every branch: both upwind sides and u = 0, linear and nonlinear
// weights, the positivity limiter on (phi < 1) and off, and the reduced-weight faces.
// Prints the worst relative differences and the branch counts.  Exit status 1 when a
// partial differs by more than 1e-11 relative on well-conditioned stencils (differences of
// order 1 to 10 on a base of 300), or by more than 1e-6 on any stencil: where the
// differences are 1e-3 of the base, the nonlinear weights' derivatives are large and
// cancel, and the two evaluation orders round differently (the closed form subtracts the
// two candidates before scaling by the weight derivative, the dual numbers after).
#include <cmath>
#include <cstdio>
#include <random>

#include "dual.cuh"
#include "weno_partials.cuh"

int main()
{
    std::mt19937_64 rng(12345);
    std::uniform_real_distribution<double> U(-1., 1.);
    double worst = 0., worst_wc = 0.;
    long n_nl = 0, n_lim = 0, n_neg = 0, n_zero = 0, n = 0;
    for (int t = 0; t < 200000; t++) {
        const int kind = t % 5;
        double base = 300. + 5. * U(rng), sc = kind == 0 ? 1e-3 : (kind == 1 ? 1. : 10.);
        double x[4];
        for (int m = 0; m < 4; m++) x[m] = base + sc * U(rng);
        if (kind == 3) {   // near-zero positive field with a dip: the positivity limiter
            for (int m = 0; m < 4; m++) x[m] = 1e-3 * (1. + U(rng));
            x[t % 4] = 1e-6;
        }
        if (kind == 4) {   // one step: a smoothness ratio far above 20
            x[0] = x[1] = base;
            x[2] = x[3] = base + sc;
        }
        double u = U(rng);
        if (t % 97 == 0) u = 0.;
        const bool full = (t % 7) != 0;
        double J[4], Ju;
        weno_face_partials(x[0], x[1], x[2], x[3], u, full, J, Ju);
        using D5 = D<5>;
        const D5 F = weno_face_up<D5>(D5::var(x[0], 0), D5::var(x[1], 1), D5::var(x[2], 2), D5::var(x[3], 3),
                                      D5::var(u, 4), full);
        double scale = std::fabs(Ju) + std::fabs(F.d[4]);
        for (int m = 0; m < 4; m++) scale += std::fabs(J[m]) + std::fabs(F.d[m]);
        double diff = std::fabs(Ju - F.d[4]);
        for (int m = 0; m < 4; m++) diff = std::fmax(diff, std::fabs(J[m] - F.d[m]));
        const double rel = diff / (scale > 0. ? scale : 1.);
        if (rel > worst) worst = rel;
        if ((kind == 1 || kind == 2) && rel > worst_wc) worst_wc = rel;
        // branch bookkeeping (the same decisions the forward makes)
        const double f1 = -(0.5 * x[0]) + 1.5 * x[1], f2 = 0.5 * x[1] + 0.5 * x[2], f3 = 1.5 * x[2] - 0.5 * x[3];
        const double mn = std::fmin(std::fmin(f1, f2), f3);
        if (std::fabs(0. - x[1]) < std::fabs((mn - x[1]) + 1e-15)) n_lim++;
        const double dout = u < 0. ? x[3] - x[2] : x[1] - x[0], dmid = x[2] - x[1];
        const double eo = dout * dout, em = dmid * dmid;
        if (full && ratio_gt(std::fmax(eo, em), std::fmin(eo, em) + 1e-15, 20.)) n_nl++;
        n_neg += u < 0.;
        n_zero += u == 0.;
        n++;
    }
    printf("faces %ld nonlinear %ld limited %ld u<0 %ld u=0 %ld worst_rel %.3e well_conditioned_worst_rel %.3e\n", n,
           n_nl, n_lim, n_neg, n_zero, worst, worst_wc);
    return worst_wc <= 1e-11 && worst <= 1e-6 && n_nl > 1000 && n_lim > 1000 && n_zero > 100 ? 0 : 1;
}
