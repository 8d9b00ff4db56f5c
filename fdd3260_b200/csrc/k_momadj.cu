// k_momadj.cu -- tangent linear and adjoint of the momentum advection operator
// qnadv_uvw (src/INTEG/windadv.f90:46-79 with uadv_fd :82-220, vadv_fd :223-357,
// wadv_fd :360-492 and the stencils :494-1127), FD4/FD2 with the artificial viscosity.
//
// The operator is evaluated per cell in gather form: each output (au, av or aw at one
// cell) recomputes the face fluxes it differences, with the advective velocities
// m/rho0 - shift formed from the same momentum loads.  The code keeps the reference's
// expressions and the direction order of ntime's parity, so its FP64 instance equals
// the K2 momentum advection bit for bit (a test checks it).
//   TL: the per-cell form on dual numbers with one partial (tangent = dm).
//   AD: the transposed stencils, hand-written in gather form (one thread per input cell
//       sums what every face flux and viscosity term that reads the cell passes back);
//       no atomics.  What the forward reads through periodic ghost images lands on the
//       interior cells they copy, so the ghosts of the result stay 0.
#include "dual.cuh"
#include "mg_common.cuh"
#include "mimica_gpu.h"

namespace {

constexpr double AVISC = 1. / 16.;   // windadv.f90:39


// advective velocity of momentum component f at level k (funcpack.f90:65-94)
template <typename T>
__device__ __forceinline__ T adv_vel(const DevGrid &G, int f, int k, const T &m)
{
    if (f == 0) return m / T(__ldg(G.den0 + k - 1)) - T(G.u0shift);
    if (f == 1) return m / T(__ldg(G.den0 + k - 1)) - T(G.v0shift);
    return m / T(__ldg(G.avden0 + k - 1));
}

// ---------------- the nine direction terms (oracle and K2 order of operations) ----------------
template <typename T, class L>
__device__ __forceinline__ T u_x(const DevGrid &G, const L &ld, int i, int j, int k, T ua)
{
    const bool fd4 = G.mom_ord == 4;
    const double dx1 = 1. / G.dx, dx2 = 1. / (2. * G.dx);
    const double c1 = fd4 ? 4. / 3. : 1., c2 = fd4 ? 1. / 3. : 0.;
    auto U = [&](int p) { return ld.m(0, p, j, k); };
    auto UT = [&](int p) { return ld.t(0, p, j, k); };
    auto F = [&](int p) { return ((UT(p + 1) + UT(p)) * T(0.5)) * ((U(p + 1) + U(p)) * T(0.5)); };
    auto A = [&](int p) { return ((UT(p + 2) + UT(p)) * T(0.5)) * ((U(p + 2) + U(p)) * T(0.5)); };
    ua = ua + T(c1) * (F(i) - F(i - 1)) * T(dx1) - T(c2) * (A(i) - A(i - 2)) * T(dx2);
    if (G.lavisc) {
        const T mu = dabs(UT(i)) * T(dx1);
        ua = ua - T(AVISC) * mu * (-U(i + 2) + T(4.) * U(i + 1) - T(6.) * U(i) + T(4.) * U(i - 1) - U(i - 2));
    }
    return ua;
}

template <typename T, class L>
__device__ __forceinline__ T u_y(const DevGrid &G, const L &ld, int i, int j, int k, T ua)
{
    const bool fd4 = G.mom_ord == 4;
    const double dy1 = 1. / G.dy, dy3 = 1. / (3. * G.dy);
    const double c1 = fd4 ? 9. / 8. : 1., c2 = fd4 ? 1. / 8. : 0.;
    auto U = [&](int q) { return ld.m(0, i, q, k); };
    auto V = [&](int di, int q) { return ld.t(1, i + di, q, k); };
    auto F = [&](int q) {
        const T vv = T(c1) * (V(-1, q + 1) + V(0, q + 1)) * T(0.5) - T(c2) * (V(-2, q + 1) + V(1, q + 1)) * T(0.5);
        const T fr = (U(q + 1) + U(q)) * T(0.5);
        return vv * fr;
    };
    ua = ua + T(c1) * (F(j) - F(j - 1)) * T(dy1) - T(c2) * (F(j + 1) - F(j - 2)) * T(dy3);
    if (G.lavisc) {
        const T mu = T(0.25) * dabs(V(-1, j) + V(0, j) + V(-1, j + 1) + V(0, j + 1)) * T(dy1);
        ua = ua - T(AVISC) * mu * (-U(j + 2) + T(4.) * U(j + 1) - T(6.) * U(j) + T(4.) * U(j - 1) - U(j - 2));
    }
    return ua;
}

// advuz_fd / advvz_fd (advhz): f = 0 (u, w at i-1, i, i-2, i+1) or 1 (v, w at j-1, j, j-2, j+1)
template <typename T, class L>
__device__ __forceinline__ T h_z(const DevGrid &G, const L &ld, int f, int i, int j, int k, T ua)
{
    const int nz = G.nz;
    const bool fd4 = G.mom_ord == 4;
    const double c1 = fd4 ? 9. / 8. : 1., c2 = fd4 ? 1. / 8. : 0.;
    auto dzw = [&](int q) { return __ldg(G.dzw + q - 1); };
    auto dz1w = [&](int q) { return __ldg(G.dz1w + q - 1); };
    auto U = [&](int q) { return ld.m(f, i, j, q); };
    auto W = [&](int d, int q) { return f == 0 ? ld.t(2, i + d, j, q) : ld.t(2, i, j + d, q); };
    auto F = [&](int q) -> T {
        if (q >= nz) return T(0.);
        const T ww = T(c1) * (W(-1, q + 1) + W(0, q + 1)) * T(0.5) - T(c2) * (W(-2, q + 1) + W(1, q + 1)) * T(0.5);
        const T fr = (T(dzw(q + 1)) * U(q + 1) + T(dzw(q)) * U(q)) / T(dzw(q + 1) + dzw(q));
        return ww * fr;
    };
    if (k >= 3 && k <= nz - 1)
        ua = ua + T(c1) * (F(k) - F(k - 1)) * T(dz1w(k)) - T(c2) * (F(k + 1) - F(k - 2)) / T(dzw(k - 1) + dzw(k) + dzw(k + 1));
    else if (k == 1)
        ua = ua + (F(1) - T(0.)) * T(dz1w(1));
    else if (k == 2)
        ua = ua + T(c1) * (F(2) - F(1)) * T(dz1w(f == 1 ? 2 : 1)) - T(c2) * (F(3) - T(0.)) / T(dzw(1) + dzw(2) + dzw(3));
    else   // k == nz
        ua = ua + (T(0.) - F(nz - 1)) * T(dz1w(nz));
    if (G.lavisc && k >= 3 && k <= nz - 2) {
        const T mu = T(0.25) * dabs(W(-1, k) + W(0, k) + W(-1, k + 1) + W(0, k + 1)) * T(dz1w(k));
        ua = ua - T(AVISC) * mu * (-U(k + 2) + T(4.) * U(k + 1) - T(6.) * U(k) + T(4.) * U(k - 1) - U(k - 2));
    }
    return ua;
}

template <typename T, class L>
__device__ __forceinline__ T v_x(const DevGrid &G, const L &ld, int i, int j, int k, T va)
{
    const bool fd4 = G.mom_ord == 4;
    const double dx1 = 1. / G.dx, dx3 = 1. / (3. * G.dx);
    const double c1 = fd4 ? 9. / 8. : 1., c2 = fd4 ? 1. / 8. : 0.;
    auto V = [&](int p) { return ld.m(1, p, j, k); };
    auto UT = [&](int p, int dj) { return ld.t(0, p, j + dj, k); };
    auto F = [&](int p) {
        const T uu = T(c1) * (UT(p + 1, -1) + UT(p + 1, 0)) * T(0.5) - T(c2) * (UT(p + 1, -2) + UT(p + 1, 1)) * T(0.5);
        const T fr = (V(p + 1) + V(p)) * T(0.5);
        return uu * fr;
    };
    va = va + T(c1) * (F(i) - F(i - 1)) * T(dx1) - T(c2) * (F(i + 1) - F(i - 2)) * T(dx3);
    if (G.lavisc) {
        const T mu = T(0.25) * dabs(UT(i, -1) + UT(i, 0) + UT(i + 1, -1) + UT(i + 1, 0)) * T(dx1);
        va = va - T(AVISC) * mu * (-V(i + 2) + T(4.) * V(i + 1) - T(6.) * V(i) + T(4.) * V(i - 1) - V(i - 2));
    }
    return va;
}

template <typename T, class L>
__device__ __forceinline__ T v_y(const DevGrid &G, const L &ld, int i, int j, int k, T va)
{
    const bool fd4 = G.mom_ord == 4;
    const double dy1 = 1. / G.dy, dy2 = 1. / (2. * G.dy);
    const double c1 = fd4 ? 4. / 3. : 1., c2 = fd4 ? 1. / 3. : 0.;
    auto V = [&](int q) { return ld.m(1, i, q, k); };
    auto VT = [&](int q) { return ld.t(1, i, q, k); };
    auto F = [&](int q) { return ((VT(q + 1) + VT(q)) * T(0.5)) * ((V(q + 1) + V(q)) * T(0.5)); };
    auto A = [&](int q) { return ((VT(q + 2) + VT(q)) * T(0.5)) * ((V(q + 2) + V(q)) * T(0.5)); };
    va = va + T(c1) * (F(j) - F(j - 1)) * T(dy1) - T(c2) * (A(j) - A(j - 2)) * T(dy2);
    if (G.lavisc) {
        const T mu = dabs(VT(j)) * T(dy1);
        va = va - T(AVISC) * mu * (-V(j + 2) + T(4.) * V(j + 1) - T(6.) * V(j) + T(4.) * V(j - 1) - V(j - 2));
    }
    return va;
}

// advwx_fd / advwy_fd (advwh): dir 0 (x, velocity ua) or 1 (y, velocity va); levels 2..nz
template <typename T, class L>
__device__ __forceinline__ T w_h(const DevGrid &G, const L &ld, int dir, int i, int j, int k, T wa)
{
    const int nz = G.nz;
    const bool fd4 = G.mom_ord == 4;
    const double d = dir == 0 ? G.dx : G.dy;
    const double d1 = 1. / d, d3 = 1. / (3. * d);
    const double c1 = fd4 ? 9. / 8. : 1., c2 = fd4 ? 1. / 8. : 0.;
    auto HT = [&](int p, int q) { return dir == 0 ? ld.t(0, p, j, q) : ld.t(1, i, p, q); };
    auto Wm = [&](int p, int q) { return dir == 0 ? ld.m(2, p, j, q) : ld.m(2, i, p, q); };
    const int s = dir == 0 ? i : j;
    auto FF = [&](int p) -> T {
        T uu;
        if (k == 2) uu = (HT(p + 1, 2) + HT(p + 1, 1)) * T(0.5);
        else if (k == nz) uu = (HT(p + 1, nz) + HT(p + 1, nz - 1)) * T(0.5);
        else uu = T(c1) * (HT(p + 1, k) + HT(p + 1, k - 1)) * T(0.5) - T(c2) * (HT(p + 1, k + 1) + HT(p + 1, k - 2)) * T(0.5);
        const T fr = (Wm(p + 1, k) + Wm(p, k)) * T(0.5);
        return uu * fr;
    };
    wa = wa + T(c1) * (FF(s) - FF(s - 1)) * T(d1) - T(c2) * (FF(s + 1) - FF(s - 2)) * T(d3);
    if (G.lavisc) {
        const T mu = T(0.25) * dabs(HT(s, k) + HT(s, k - 1) + HT(s + 1, k) + HT(s + 1, k - 1)) * T(d1);
        wa = wa - T(AVISC) * mu * (-Wm(s + 2, k) + T(4.) * Wm(s + 1, k) - T(6.) * Wm(s, k) + T(4.) * Wm(s - 1, k) - Wm(s - 2, k));
    }
    return wa;
}

template <typename T, class L>
__device__ __forceinline__ T w_z(const DevGrid &G, const L &ld, int i, int j, int k, T wa)
{
    const int nz = G.nz;
    const bool fd4 = G.mom_ord == 4;
    const double c1 = fd4 ? 4. / 3. : 1., c2 = fd4 ? 1. / 3. : 0.;
    auto dzw = [&](int q) { return __ldg(G.dzw + q - 1); };
    auto dz1 = [&](int q) { return __ldg(G.dz1 + q - 1); };
    auto W = [&](int q) { return ld.m(2, i, j, q); };
    auto WT = [&](int q) { return ld.t(2, i, j, q); };
    auto F = [&](int q) -> T {
        if (q == nz - 1) return T(0.25) * (WT(nz) + WT(nz - 1)) * (W(nz) + W(nz - 1));
        return ((WT(q + 1) + WT(q)) * T(0.5)) * ((W(q + 1) + W(q)) * T(0.5));
    };
    auto A = [&](int q) -> T {
        if (q == nz - 1) {
            const double s = dzw(nz) + dzw(nz - 1);
            return (T(0.) + T(dzw(nz - 1)) * WT(nz - 1)) * (T(0.) + T(dzw(nz - 1)) * W(nz - 1)) / T(s * s);
        }
        const T ww2 = (T(dzw(q + 1)) * WT(q + 2) + T(dzw(q)) * WT(q)) / T(dzw(q + 1) + dzw(q));
        const T fr2 = (T(dzw(q + 1)) * W(q + 2) + T(dzw(q)) * W(q)) / T(dzw(q + 1) + dzw(q));
        return ww2 * fr2;
    };
    if (k >= 3 && k <= nz - 1)
        wa = wa + T(c1) * (F(k) - F(k - 1)) * T(dz1(k - 1)) - T(c2) * (A(k) - A(k - 2)) / T(dzw(k) + dzw(k - 1));
    else if (k == 2)
        wa = wa + T(c1) * (F(2) - F(1)) * T(dz1(1)) - T(c2) * (A(2) - T(0.)) / T(dzw(2) + dzw(1));
    else if (k == nz)
        wa = wa + (T(0.) - F(nz - 1)) * T(dz1(nz - 1));
    if (G.lavisc && k >= 3 && k <= nz - 2) {
        const T mu = dabs(WT(k)) * T(dz1(k - 1));
        wa = wa - T(AVISC) * mu * (-W(k + 2) + T(4.) * W(k + 1) - T(6.) * W(k) + T(4.) * W(k - 1) - W(k - 2));
    }
    return wa;
}

// component c (0 u, 1 v, 2 w) of qnadv_uvw at interior cell (i,j,k): even ntime x, y, z;
// odd ntime z, y, x (windadv.f90:58-76)
template <typename T, class L>
__device__ __forceinline__ T adv_comp(const DevGrid &G, const L &ld, int c, int ntime, int i, int j, int k)
{
    T a = T(0.);
    if (c == 2 && k == 1) return a;   // w(1): the surface, no advective tendency
    const bool even = (ntime % 2) == 0;
    for (int pass = 0; pass < 3; pass++) {
        const int dir = even ? pass : 2 - pass;
        if (c == 0) a = dir == 0 ? u_x(G, ld, i, j, k, a) : (dir == 1 ? u_y(G, ld, i, j, k, a) : h_z(G, ld, 0, i, j, k, a));
        else if (c == 1) a = dir == 0 ? v_x(G, ld, i, j, k, a) : (dir == 1 ? v_y(G, ld, i, j, k, a) : h_z(G, ld, 1, i, j, k, a));
        else a = dir == 0 ? w_h(G, ld, 0, i, j, k, a) : (dir == 1 ? w_h(G, ld, 1, i, j, k, a) : w_z(G, ld, i, j, k, a));
    }
    return a;
}

// ---------------- loaders ----------------
struct Mom3 {
    const double *m[3];
};

// values and one tangent
struct LoadTL {
    const DevGrid &G;
    Mom3 v, d;
    __device__ D<1> m(int f, int i, int j, int k) const
    {
        const long long q = gidx(G, i, j, k);
        D<1> r(__ldg(v.m[f] + q));
        r.d[0] = __ldg(d.m[f] + q);
        return r;
    }
    __device__ D<1> t(int f, int i, int j, int k) const { return adv_vel(G, f, k, m(f, i, j, k)); }
};

// ---------------- kernels ----------------
__global__ void __launch_bounds__(128) mom_tl_kernel(DevGrid G, int ntime, Mom3 v, Mom3 d, Mom3 val, Mom3 tan)
{
    const int i = 4 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 4 + blockIdx.y;
    const int k = 1 + blockIdx.z;
    if (i > G.nx - 2) return;
    const LoadTL ld{G, v, d};
    const long long q = gidx(G, i, j, k);
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const D<1> a = adv_comp<D<1>>(G, ld, c, ntime, i, j, k);
        if (val.m[c]) const_cast<double *>(val.m[c])[q] = a.v;
        const_cast<double *>(tan.m[c])[q] = a.d[0];
    }
}

// ---------------- adjoint: the transposed stencils in gather form ----------------
// Each direction term is a sum of face fluxes Phi = a * b with constant coefficients
// (a: an average of advective velocities, b: an average of the advected momentum; the
// coefficients of the vertical terms depend on the level, as the forward's branches at
// the surface and the lid), plus the artificial viscosity mu |velocity| D4(momentum).
// The adjoint at an input cell sums, over every face that reads the cell, Phi-bar (the
// coefficient-weighted adjoints of the outputs that difference the face) times the
// partial of Phi, and likewise over the viscosity terms.  Positions wrap periodically in
// x and y, so what the forward reads through a ghost image is gathered by the interior
// cell it copies; outputs outside 1..nz (and w at the surface) do not exist.

__device__ __forceinline__ double sgnd(double x) { return x < 0. ? -1. : 1.; }   // d|x|/dx as dabs takes it
__device__ __forceinline__ double w4(int d) { return d == 0 ? -6. : ((d == 1 || d == -1) ? 4. : -1.); }

struct Gath {
    const DevGrid &G;
    Mom3 m, ab;
    double c1s, c2s, c1c, c2c;
    int i0, j0, k0;   // the thread's cell: every position is addressed from its index
    long long q0;
    __device__ Gath(const DevGrid &g, Mom3 m_, Mom3 ab_, int i, int j, int k) : G(g), m(m_), ab(ab_), i0(i), j0(j), k0(k)
    {
        const bool fd4 = g.mom_ord == 4;
        c1s = fd4 ? 4. / 3. : 1.; c2s = fd4 ? 1. / 3. : 0.;
        c1c = fd4 ? 9. / 8. : 1.; c2c = fd4 ? 1. / 8. : 0.;
        q0 = gidx(g, i, j, k);
    }
    // (along, transverse) -> (i, j): direction 0 is x, 1 is y
    __device__ static int ci(int dir, int a, int t) { return dir == 0 ? a : t; }
    __device__ static int cj(int dir, int a, int t) { return dir == 0 ? t : a; }
    // the positions visited lie within 2 cells of the thread's (outputs) or 3 (momenta);
    // only a viscosity term three cells along reads past the last ghost, and is moved to
    // its periodic image
    __device__ int img_a(int dir, int a) const
    {
        return dir == 0 ? (a + 1 > G.nx ? a - G.maxx : a) : (a + 1 > G.ny ? a - G.maxy : a);
    }
    __device__ long long idx(int i, int j, int k) const
    {
        return q0 + (i - i0) + (long long)(j - j0) * G.px + (long long)(k - k0) * G.ps;
    }
    __device__ double M(int f, int i, int j, int k) const { return __ldg(m.m[f] + idx(i, j, k)); }
    // advective velocity with the reciprocal profiles (its partial is the same factor)
    __device__ double T(int f, int i, int j, int k) const
    {
        const double x = M(f, i, j, k) * rden(f, k);
        return f == 0 ? x - G.u0shift : (f == 1 ? x - G.v0shift : x);
    }
    // output adjoints, halo-filled: the ghost cells hold the periodic images
    __device__ double A(int c, int i, int j, int k) const
    {
        if (k < 1 || k > G.nz || (c == 2 && k == 1)) return 0.;
        return __ldg(ab.m[c] + idx(i, j, k));
    }
    __device__ double Ma(int f, int dir, int a, int t, int k) const { return M(f, ci(dir, a, t), cj(dir, a, t), k); }
    __device__ double Ta(int f, int dir, int a, int t, int k) const { return T(f, ci(dir, a, t), cj(dir, a, t), k); }
    __device__ double Aa(int c, int dir, int a, int t, int k) const { return A(c, ci(dir, a, t), cj(dir, a, t), k); }
    __device__ double rden(int f, int k) const { return __ldg((f == 2 ? G.ravden0 : G.rden0) + k - 1); }
    __device__ double dzw(int q) const { return __ldg(G.dzw + q - 1); }
    __device__ double dz1w(int q) const { return __ldg(G.dz1w + q - 1); }
    __device__ double dz1(int q) const { return __ldg(G.dz1 + q - 1); }
    __device__ double d1(int dir) const { return dir == 0 ? 1. / G.dx : 1. / G.dy; }

    // ---- u_x (f 0, dir x) and v_y (f 1, dir y): the advected field is its own velocity ----
    __device__ double self_h(int f, int i, int j, int k) const
    {
        const int dir = f, a0 = dir == 0 ? i : j, t = dir == 0 ? j : i;
        const double h1 = d1(dir), h2 = dir == 0 ? 1. / (2. * G.dx) : 1. / (2. * G.dy), rd = rden(f, k);
        double r = 0.;
        for (int p = a0 - 1; p <= a0; p++) {   // F(p) = avg T(p, p+1) * avg m(p, p+1)
            const double fb = c1s * h1 * (Aa(f, dir, p, t, k) - Aa(f, dir, p + 1, t, k));
            r += fb * 0.5 * (0.5 * (Ma(f, dir, p + 1, t, k) + Ma(f, dir, p, t, k)) * rd +
                             0.5 * (Ta(f, dir, p + 1, t, k) + Ta(f, dir, p, t, k)));
        }
        for (int p = a0 - 2; p <= a0; p += 2) {   // A(p) = avg T(p, p+2) * avg m(p, p+2)
            const double gb = c2s * h2 * (Aa(f, dir, p + 2, t, k) - Aa(f, dir, p, t, k));
            r += gb * 0.5 * (0.5 * (Ma(f, dir, p + 2, t, k) + Ma(f, dir, p, t, k)) * rd +
                             0.5 * (Ta(f, dir, p + 2, t, k) + Ta(f, dir, p, t, k)));
        }
        if (G.lavisc) {
            for (int o = a0 - 2; o <= a0 + 2; o++) r -= AVISC * h1 * Aa(f, dir, o, t, k) * fabs(Ta(f, dir, o, t, k)) * w4(a0 - o);
            const double d4 = -Ma(f, dir, a0 + 2, t, k) + 4. * Ma(f, dir, a0 + 1, t, k) - 6. * Ma(f, dir, a0, t, k) +
                              4. * Ma(f, dir, a0 - 1, t, k) - Ma(f, dir, a0 - 2, t, k);
            r -= AVISC * h1 * Aa(f, dir, a0, t, k) * sgnd(Ta(f, dir, a0, t, k)) * rd * d4;
        }
        return r;
    }

    // ---- u_y (c 0: dir y, velocity v) and v_x (c 1: dir x, velocity u) ----
    // face bar at along-position q of line t
    __device__ double cross_fbar(int c, int dir, int q, int t, int k) const
    {
        const double h1 = d1(dir), h3 = dir == 0 ? 1. / (3. * G.dx) : 1. / (3. * G.dy);
        return c1c * h1 * (Aa(c, dir, q, t, k) - Aa(c, dir, q + 1, t, k)) - c2c * h3 * Aa(c, dir, q - 1, t, k) +
               c2c * h3 * Aa(c, dir, q + 2, t, k);
    }
    // partial wrt the advected momentum c at its own cell
    __device__ double cross_adv(int c, int i, int j, int k) const
    {
        const int dir = 1 - c, g = 1 - c;
        const int a0 = dir == 0 ? i : j, t = dir == 0 ? j : i;
        double r = 0.;
        for (int q = a0 - 1; q <= a0; q++) {
            const double vel = c1c * (Ta(g, dir, q + 1, t - 1, k) + Ta(g, dir, q + 1, t, k)) * 0.5 -
                               c2c * (Ta(g, dir, q + 1, t - 2, k) + Ta(g, dir, q + 1, t + 1, k)) * 0.5;
            r += cross_fbar(c, dir, q, t, k) * 0.5 * vel;
        }
        if (G.lavisc)
            for (int o = a0 - 2; o <= a0 + 2; o++) {
                const int ob = img_a(dir, o);
                const double mu = 0.25 * fabs(Ta(g, dir, ob, t - 1, k) + Ta(g, dir, ob, t, k) + Ta(g, dir, ob + 1, t - 1, k) +
                                              Ta(g, dir, ob + 1, t, k)) * d1(dir);
                r -= AVISC * Aa(c, dir, ob, t, k) * mu * w4(a0 - o);
            }
        return r;
    }
    // partial wrt the advecting momentum g = 1 - c at its own cell
    __device__ double cross_vel(int c, int i, int j, int k) const
    {
        const int dir = 1 - c, g = 1 - c;
        const int a0 = dir == 0 ? i : j, t0 = dir == 0 ? j : i;
        const double rd = rden(g, k);
        double r = 0.;
        const int ds[4] = {-1, 0, -2, 1};
        for (int n = 0; n < 4; n++) {   // the velocity at transverse offset d of line t = t0 - d, face q = a0 - 1
            const int t = t0 - ds[n];
            const double gam = n < 2 ? 0.5 * c1c : -0.5 * c2c;
            const double fr = 0.5 * (Ma(c, dir, a0, t, k) + Ma(c, dir, a0 - 1, t, k));
            r += cross_fbar(c, dir, a0 - 1, t, k) * fr * gam * rd;
        }
        if (G.lavisc)
            for (int t = t0; t <= t0 + 1; t++)
                for (int o = a0 - 1; o <= a0; o++) {
                    const double s = Ta(g, dir, o, t - 1, k) + Ta(g, dir, o, t, k) + Ta(g, dir, o + 1, t - 1, k) +
                                     Ta(g, dir, o + 1, t, k);
                    const double d4 = -Ma(c, dir, o + 2, t, k) + 4. * Ma(c, dir, o + 1, t, k) - 6. * Ma(c, dir, o, t, k) +
                                      4. * Ma(c, dir, o - 1, t, k) - Ma(c, dir, o - 2, t, k);
                    r -= AVISC * Aa(c, dir, o, t, k) * d4 * 0.25 * d1(dir) * sgnd(s) * rd;
                }
        return r;
    }

    // ---- h_z (f 0: u with w at x offsets; f 1: v with w at y offsets) ----
    // coefficient of face flux F(q) in the output at level ko (advhz's branches)
    __device__ double hz_coef(int f, int ko, int q) const
    {
        const int nz = G.nz;
        if (ko >= 3 && ko <= nz - 1) {
            const double s3 = dzw(ko - 1) + dzw(ko) + dzw(ko + 1);
            if (q == ko) return c1c * dz1w(ko);
            if (q == ko - 1) return -c1c * dz1w(ko);
            if (q == ko + 1) return -c2c / s3;
            if (q == ko - 2) return c2c / s3;
            return 0.;
        }
        if (ko == 1) return q == 1 ? dz1w(1) : 0.;
        if (ko == 2) {
            const double mz = dz1w(f == 1 ? 2 : 1);
            if (q == 2) return c1c * mz;
            if (q == 1) return -c1c * mz;
            if (q == 3) return -c2c / (dzw(1) + dzw(2) + dzw(3));
            return 0.;
        }
        return q == nz - 1 ? -dz1w(nz) : 0.;   // ko == nz
    }
    __device__ double hz_fbar(int f, int i, int j, int q) const
    {
        double r = 0.;
        for (int ko = q - 1; ko <= q + 2; ko++)
            if (ko >= 1 && ko <= G.nz) r += A(f, i, j, ko) * hz_coef(f, ko, q);
        return r;
    }
    __device__ double WTo(int f, int i, int j, int d, int q) const { return f == 0 ? T(2, i + d, j, q) : T(2, i, j + d, q); }
    __device__ double hz_adv(int f, int i, int j, int k) const
    {
        const int nz = G.nz;
        double r = 0.;
        for (int q = k - 1; q <= k; q++) {
            if (q < 1 || q > nz - 1) continue;
            const double ww = c1c * (WTo(f, i, j, -1, q + 1) + WTo(f, i, j, 0, q + 1)) * 0.5 -
                              c2c * (WTo(f, i, j, -2, q + 1) + WTo(f, i, j, 1, q + 1)) * 0.5;
            const double wgt = (q == k ? dzw(q) : dzw(q + 1)) / (dzw(q + 1) + dzw(q));
            r += hz_fbar(f, i, j, q) * ww * wgt;
        }
        if (G.lavisc)
            for (int ko = k - 2; ko <= k + 2; ko++) {
                if (ko < 3 || ko > nz - 2) continue;
                const double mu = 0.25 * fabs(WTo(f, i, j, -1, ko) + WTo(f, i, j, 0, ko) + WTo(f, i, j, -1, ko + 1) +
                                              WTo(f, i, j, 0, ko + 1)) * dz1w(ko);
                r -= AVISC * A(f, i, j, ko) * mu * w4(k - ko);
            }
        return r;
    }
    __device__ double hz_w(int f, int i, int j, int k) const   // partial wrt w at (i, j, k)
    {
        const int nz = G.nz;
        const double ra = rden(2, k);
        double r = 0.;
        const int q = k - 1;
        if (q >= 1 && q <= nz - 1) {
            const int ds[4] = {-1, 0, -2, 1};
            for (int n = 0; n < 4; n++) {
                const int ii = f == 0 ? i - ds[n] : i, jj = f == 0 ? j : j - ds[n];
                const double gam = n < 2 ? 0.5 * c1c : -0.5 * c2c;
                const double fr = (dzw(q + 1) * M(f, ii, jj, q + 1) + dzw(q) * M(f, ii, jj, q)) / (dzw(q + 1) + dzw(q));
                r += hz_fbar(f, ii, jj, q) * fr * gam * ra;
            }
        }
        if (G.lavisc)
            for (int s = 0; s <= 1; s++) {   // outputs at the column itself and one further along
                const int ii = f == 0 ? i + s : i, jj = f == 0 ? j : j + s;
                for (int ko = k - 1; ko <= k; ko++) {
                    if (ko < 3 || ko > nz - 2) continue;
                    const double sw = WTo(f, ii, jj, -1, ko) + WTo(f, ii, jj, 0, ko) + WTo(f, ii, jj, -1, ko + 1) +
                                      WTo(f, ii, jj, 0, ko + 1);
                    const double d4 = -M(f, ii, jj, ko + 2) + 4. * M(f, ii, jj, ko + 1) - 6. * M(f, ii, jj, ko) +
                                      4. * M(f, ii, jj, ko - 1) - M(f, ii, jj, ko - 2);
                    r -= AVISC * A(f, ii, jj, ko) * d4 * 0.25 * dz1w(ko) * sgnd(sw) * ra;
                }
            }
        return r;
    }

    // ---- w_h (dir 0: velocity u along x; dir 1: v along y), outputs w at levels 2..nz ----
    // weight of the velocity at level q in uu of the output at level kw
    __device__ double wh_lam(int kw, int q) const
    {
        const int nz = G.nz;
        if (kw == 2) return (q == 2 || q == 1) ? 0.5 : 0.;
        if (kw == nz) return (q == nz || q == nz - 1) ? 0.5 : 0.;
        if (q == kw || q == kw - 1) return 0.5 * c1c;
        if (q == kw + 1 || q == kw - 2) return -0.5 * c2c;
        return 0.;
    }
    __device__ double wh_fbar(int dir, int p, int t, int kw) const { return cross_fbar(2, dir, p, t, kw); }
    __device__ double wh_w(int dir, int i, int j, int k) const   // partial wrt w (advected) at (i, j, k)
    {
        if (k < 2) return 0.;
        const int a0 = dir == 0 ? i : j, t = dir == 0 ? j : i;
        double r = 0.;
        for (int p = a0 - 1; p <= a0; p++) {
            double uu = 0.;
            for (int q = k - 2; q <= k + 1; q++) {
                const double l = wh_lam(k, q);
                if (l != 0.) uu += l * Ta(dir, dir, p + 1, t, q);
            }
            r += wh_fbar(dir, p, t, k) * 0.5 * uu;
        }
        if (G.lavisc)
            for (int o = a0 - 2; o <= a0 + 2; o++) {
                const int ob = img_a(dir, o);
                const double mu = 0.25 * fabs(Ta(dir, dir, ob, t, k) + Ta(dir, dir, ob, t, k - 1) + Ta(dir, dir, ob + 1, t, k) +
                                              Ta(dir, dir, ob + 1, t, k - 1)) * d1(dir);
                r -= AVISC * Aa(2, dir, ob, t, k) * mu * w4(a0 - o);
            }
        return r;
    }
    __device__ double wh_vel(int dir, int i, int j, int k) const   // partial wrt the velocity momentum (u or v)
    {
        const int nz = G.nz;
        const int a0 = dir == 0 ? i : j, t = dir == 0 ? j : i;
        const double rd = rden(dir, k);
        double r = 0.;
        for (int kw = k - 1; kw <= k + 2; kw++) {
            if (kw < 2 || kw > nz) continue;
            const double l = wh_lam(kw, k);
            if (l == 0.) continue;
            const double fr = 0.5 * (Ma(2, dir, a0, t, kw) + Ma(2, dir, a0 - 1, t, kw));
            r += wh_fbar(dir, a0 - 1, t, kw) * fr * l * rd;
        }
        if (G.lavisc)
            for (int kw = k; kw <= k + 1; kw++) {
                if (kw < 2 || kw > nz) continue;
                for (int o = a0 - 1; o <= a0; o++) {
                    const double s = Ta(dir, dir, o, t, kw) + Ta(dir, dir, o, t, kw - 1) + Ta(dir, dir, o + 1, t, kw) +
                                     Ta(dir, dir, o + 1, t, kw - 1);
                    const double d4 = -Ma(2, dir, o + 2, t, kw) + 4. * Ma(2, dir, o + 1, t, kw) - 6. * Ma(2, dir, o, t, kw) +
                                      4. * Ma(2, dir, o - 1, t, kw) - Ma(2, dir, o - 2, t, kw);
                    r -= AVISC * Aa(2, dir, o, t, kw) * d4 * 0.25 * d1(dir) * sgnd(s) * rd;
                }
            }
        return r;
    }

    // ---- w_z, outputs w at levels 2..nz ----
    __device__ double wz_fcoef(int ko, int q) const
    {
        const int nz = G.nz;
        if (ko >= 3 && ko <= nz - 1) return q == ko ? c1s * dz1(ko - 1) : (q == ko - 1 ? -c1s * dz1(ko - 1) : 0.);
        if (ko == 2) return q == 2 ? c1s * dz1(1) : (q == 1 ? -c1s * dz1(1) : 0.);
        if (ko == nz) return q == nz - 1 ? -dz1(nz - 1) : 0.;
        return 0.;
    }
    __device__ double wz_acoef(int ko, int q) const
    {
        const int nz = G.nz;
        if (ko >= 3 && ko <= nz - 1) {
            const double s = dzw(ko) + dzw(ko - 1);
            return q == ko ? -c2s / s : (q == ko - 2 ? c2s / s : 0.);
        }
        if (ko == 2) return q == 2 ? -c2s / (dzw(2) + dzw(1)) : 0.;
        return 0.;
    }
    __device__ double wz_w(int i, int j, int k) const
    {
        const int nz = G.nz;
        const double ra = rden(2, k);
        auto W = [&](int q) { return M(2, i, j, q); };
        auto WT = [&](int q) { return T(2, i, j, q); };
        double r = 0.;
        for (int q = k - 1; q <= k; q++) {   // F(q) = avg WT(q, q+1) * avg W(q, q+1)
            if (q < 1 || q > nz - 1) continue;
            const double fb = A(2, i, j, q) * wz_fcoef(q, q) + A(2, i, j, q + 1) * wz_fcoef(q + 1, q);
            r += fb * 0.25 * ((W(q + 1) + W(q)) * ra + (WT(q + 1) + WT(q)));
        }
        for (int q = k - 2; q <= k; q += 2) {   // A(q): W(q) and W(q+2), or W(nz-1) alone at q = nz-1
            if (q < 1 || q > nz - 1) continue;
            const double gb = A(2, i, j, q) * wz_acoef(q, q) + A(2, i, j, q + 2) * wz_acoef(q + 2, q);
            if (gb == 0.) continue;
            if (q == nz - 1) {
                if (k != q) continue;
                const double dl = dzw(nz - 1), sg = dzw(nz) + dzw(nz - 1);
                r += gb * dl * dl / (sg * sg) * (W(q) * ra + WT(q));
            } else {
                const double al = dzw(q + 1), be = dzw(q), sg = al + be;
                const double ww2 = (al * WT(q + 2) + be * WT(q)) / sg, fr2 = (al * W(q + 2) + be * W(q)) / sg;
                r += gb * (k == q + 2 ? al : be) / sg * (fr2 * ra + ww2);
            }
        }
        if (G.lavisc) {
            for (int ko = k - 2; ko <= k + 2; ko++) {
                if (ko < 3 || ko > nz - 2) continue;
                r -= AVISC * A(2, i, j, ko) * fabs(WT(ko)) * dz1(ko - 1) * w4(k - ko);
            }
            if (k >= 3 && k <= nz - 2) {
                const double d4 = -W(k + 2) + 4. * W(k + 1) - 6. * W(k) + 4. * W(k - 1) - W(k - 2);
                r -= AVISC * A(2, i, j, k) * dz1(k - 1) * sgnd(WT(k)) * ra * d4;
            }
        }
        return r;
    }
};

// one output component per launch (C: 0 u, 1 v, 2 w): a third of the code each
template <int C>
__global__ void __launch_bounds__(128) mom_ad_gather_kernel(DevGrid G, Mom3 v, Mom3 ab, Mom3 bar)
{
    const int i = 4 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 4 + blockIdx.y;
    const int k = 1 + blockIdx.z;
    if (i > G.nx - 2) return;
    const Gath g(G, v, ab, i, j, k);
    const long long q = g.q0;
    double *b = const_cast<double *>(bar.m[C]);
    if constexpr (C == 0)   // u: u_x, u_y (advected), h_z (f 0, advected), v_x (velocity), w_h x (velocity)
        b[q] += g.self_h(0, i, j, k) + g.cross_adv(0, i, j, k) + g.hz_adv(0, i, j, k) + g.cross_vel(1, i, j, k) +
                g.wh_vel(0, i, j, k);
    else if constexpr (C == 1)   // v: v_y, v_x (advected), h_z (f 1, advected), u_y (velocity), w_h y (velocity)
        b[q] += g.self_h(1, i, j, k) + g.cross_adv(1, i, j, k) + g.hz_adv(1, i, j, k) + g.cross_vel(0, i, j, k) +
                g.wh_vel(1, i, j, k);
    else   // w: w_z, w_h x and y (advected), h_z f 0 and f 1 (velocity)
        b[q] += g.wz_w(i, j, k) + g.wh_w(0, i, j, k) + g.wh_w(1, i, j, k) + g.hz_w(0, i, j, k) + g.hz_w(1, i, j, k);
}

}  // namespace

// val (optional) := qnadv_uvw(m) (positive convention), tan := its derivative along dm
cudaError_t launch_qnadv_tl(const DevGrid &g, int ntime, const double *mu, const double *mv, const double *mw,
                            const double *dmu, const double *dmv, const double *dmw, double *au, double *av, double *aw,
                            double *dau, double *dav, double *daw, cudaStream_t s)
{
    const dim3 grid((g.maxx + 127) / 128, g.maxy, g.nz);
    mom_tl_kernel<<<grid, 128, 0, s>>>(g, ntime, Mom3{{mu, mv, mw}}, Mom3{{dmu, dmv, dmw}}, Mom3{{au, av, aw}},
                                       Mom3{{dau, dav, daw}});
    return cudaGetLastError();
}

// bar += (d qnadv / d m)^T abar (bar arrays must be zeroed by the caller for a plain adjoint);
// abar is read on the interior (its ghost cells are overwritten with periodic images),
// the ghost entries of bar are left as they are
cudaError_t launch_qnadv_ad(const DevGrid &g, const double *mu, const double *mv, const double *mw, double *aubar,
                            double *avbar, double *awbar, double *mubar, double *mvbar, double *mwbar, cudaStream_t s)
{
    double *ab[3] = {aubar, avbar, awbar};
    cudaError_t e = launch_halo_fill(g, ab, 3, s);
    if (e != cudaSuccess) return e;
    const dim3 grid((g.maxx + 127) / 128, g.maxy, g.nz);
    const Mom3 v{{mu, mv, mw}}, ab3{{aubar, avbar, awbar}}, bar{{mubar, mvbar, mwbar}};
    mom_ad_gather_kernel<0><<<grid, 128, 0, s>>>(g, v, ab3, bar);
    mom_ad_gather_kernel<1><<<grid, 128, 0, s>>>(g, v, ab3, bar);
    mom_ad_gather_kernel<2><<<grid, 128, 0, s>>>(g, v, ab3, bar);
    return cudaGetLastError();
}
