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
//   AD: the per-cell form on dual numbers with 8 partials, seeded with 8 of the cell's
//       stencil inputs at a time (the input offsets of each component are found once by
//       a probe pass); the local Jacobian row times the output adjoint is scattered
//       onto the inputs with atomics.  Inputs in periodic ghost cells are scattered onto
//       the interior cells they are images of, so the ghosts of the result stay 0.
#include <vector>

#include "dual.cuh"
#include "mg_common.cuh"
#include "mimica_gpu.h"

namespace {

constexpr double AVISC = 1. / 16.;   // windadv.f90:39
constexpr int NCH = 8;                // partials per AD pass
constexpr int NOFF = 3 * 5 * 5 * 5;   // (field, di, dj, dk) offsets, |d| <= 2

__device__ __forceinline__ int wrap_x(const DevGrid &G, int i) { return i < 4 ? i + G.maxx : (i > G.nx - 2 ? i - G.maxx : i); }
__device__ __forceinline__ int wrap_y(const DevGrid &G, int j) { return j < 4 ? j + G.maxy : (j > G.ny - 2 ? j - G.maxy : j); }
__device__ __forceinline__ int off_code(int f, int di, int dj, int dk) { return ((f * 5 + di + 2) * 5 + dj + 2) * 5 + dk + 2; }

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
__device__ T u_x(const DevGrid &G, const L &ld, int i, int j, int k, T ua)
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
__device__ T u_y(const DevGrid &G, const L &ld, int i, int j, int k, T ua)
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
__device__ T h_z(const DevGrid &G, const L &ld, int f, int i, int j, int k, T ua)
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
__device__ T v_x(const DevGrid &G, const L &ld, int i, int j, int k, T va)
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
__device__ T v_y(const DevGrid &G, const L &ld, int i, int j, int k, T va)
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
__device__ T w_h(const DevGrid &G, const L &ld, int dir, int i, int j, int k, T wa)
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
__device__ T w_z(const DevGrid &G, const L &ld, int i, int j, int k, T wa)
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
__device__ T adv_comp(const DevGrid &G, const L &ld, int c, int ntime, int i, int j, int k)
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

// records the offsets an output reads (probe pass, plain values)
struct LoadProbe {
    const DevGrid &G;
    Mom3 v;
    int i0, j0, k0;
    int *mask;
    __device__ double m(int f, int i, int j, int k) const
    {
        mask[off_code(f, i - i0, j - j0, k - k0)] = 1;
        return __ldg(v.m[f] + gidx(G, i, j, k));
    }
    __device__ double t(int f, int i, int j, int k) const { return adv_vel(G, f, k, m(f, i, j, k)); }
};

// 8 partials, seeded on the inputs whose compact slot lies in [s0, s0 + 8)
struct LoadAD {
    const DevGrid &G;
    Mom3 v;
    int i0, j0, k0, s0;
    const short *slot;   // offset code -> compact slot of this component, or -1
    __device__ D<NCH> m(int f, int i, int j, int k) const
    {
        D<NCH> r(__ldg(v.m[f] + gidx(G, i, j, k)));
        const int s = slot[off_code(f, i - i0, j - j0, k - k0)] - s0;
        if (s >= 0 && s < NCH) r.d[s] = 1.;
        return r;
    }
    __device__ D<NCH> t(int f, int i, int j, int k) const { return adv_vel(G, f, k, m(f, i, j, k)); }
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
    for (int c = 0; c < 3; c++) {
        const D<1> a = adv_comp<D<1>>(G, ld, c, ntime, i, j, k);
        if (val.m[c]) const_cast<double *>(val.m[c])[q] = a.v;
        const_cast<double *>(tan.m[c])[q] = a.d[0];
    }
}

__global__ void mom_probe_kernel(DevGrid G, int ntime, Mom3 v, int i0, int j0, int *masks)
{
    const int c = blockIdx.x;
    for (int k = 1; k <= G.nz; k++) {
        const LoadProbe ld{G, v, i0, j0, k, masks + c * NOFF};
        (void)adv_comp<double>(G, ld, c, ntime, i0, j0, k);
    }
}

__global__ void __launch_bounds__(128) mom_ad_kernel(DevGrid G, int ntime, int c, int s0, int nslot, Mom3 v,
                                                     const double *abar, const short *slot, const int *offs,
                                                     Mom3 bar)
{
    const int i = 4 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 4 + blockIdx.y;
    const int k = 1 + blockIdx.z;
    if (i > G.nx - 2) return;
    const long long q = gidx(G, i, j, k);
    const double ab = abar[q];
    if (ab == 0.) return;
    const LoadAD ld{G, v, i, j, k, s0, slot};
    const D<NCH> a = adv_comp<D<NCH>>(G, ld, c, ntime, i, j, k);
    for (int t = 0; t < NCH && s0 + t < nslot; t++) {
        const int code = offs[s0 + t];
        const int dk = code % 5 - 2, dj = (code / 5) % 5 - 2, di = (code / 25) % 5 - 2, f = code / 125;
        // the offsets are the union over all levels; near the surface and the lid some of
        // them point outside 1..nz, where the stencils read nothing (the partial is 0)
        if (k + dk < 1 || k + dk > G.nz) continue;
        const long long tq = gidx(G, wrap_x(G, i + di), wrap_y(G, j + dj), k + dk);
        atomicAdd(const_cast<double *>(bar.m[f]) + tq, a.d[t] * ab);
    }
}

}  // namespace

// host: offsets (per component) that qnadv_uvw reads, from a probe of one column
struct MomAdjPlan {
    short *slot = nullptr;   // [3][NOFF]
    int *offs = nullptr;     // [3][NOFF] compact slot -> offset code
    int nslot[3] = {0, 0, 0};
};

cudaError_t mom_adj_plan(const DevGrid &g, int ntime, const double *mu, const double *mv, const double *mw, void **plan,
                         cudaStream_t s)
{
    MomAdjPlan *p = new MomAdjPlan();
    int *mask = nullptr;
    cudaError_t e = cudaMalloc(&mask, 3 * NOFF * sizeof(int));
    if (e == cudaSuccess) e = cudaMemsetAsync(mask, 0, 3 * NOFF * sizeof(int), s);
    if (e == cudaSuccess) {
        // the deep interior column reads no periodic image twice
        mom_probe_kernel<<<3, 1, 0, s>>>(g, ntime, Mom3{{mu, mv, mw}}, 4 + g.maxx / 2, 4 + g.maxy / 2, mask);
        e = cudaGetLastError();
    }
    std::vector<int> hm(3 * NOFF, 0);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hm.data(), mask, hm.size() * sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    std::vector<short> hs(3 * NOFF, -1);
    std::vector<int> ho(3 * NOFF, 0);
    for (int c = 0; c < 3 && e == cudaSuccess; c++)
        for (int o = 0; o < NOFF; o++)
            if (hm[c * NOFF + o]) {
                hs[c * NOFF + o] = (short)p->nslot[c];
                ho[c * NOFF + p->nslot[c]] = o;
                p->nslot[c]++;
            }
    if (e == cudaSuccess) e = cudaMalloc(&p->slot, hs.size() * sizeof(short));
    if (e == cudaSuccess) e = cudaMalloc(&p->offs, ho.size() * sizeof(int));
    if (e == cudaSuccess) e = cudaMemcpyAsync(p->slot, hs.data(), hs.size() * sizeof(short), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(p->offs, ho.data(), ho.size() * sizeof(int), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(mask);
    if (e != cudaSuccess) {
        cudaFree(p->slot); cudaFree(p->offs);
        delete p;
        return e;
    }
    *plan = p;
    return cudaSuccess;
}

void mom_adj_plan_destroy(void *plan)
{
    MomAdjPlan *p = (MomAdjPlan *)plan;
    if (!p) return;
    cudaFree(p->slot);
    cudaFree(p->offs);
    delete p;
}

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

// bar += (d qnadv / d m)^T abar (bar arrays must be zeroed by the caller for a plain adjoint)
cudaError_t launch_qnadv_ad(const DevGrid &g, void *plan, int ntime, const double *mu, const double *mv, const double *mw,
                            const double *aubar, const double *avbar, const double *awbar, double *mubar, double *mvbar,
                            double *mwbar, cudaStream_t s)
{
    MomAdjPlan *p = (MomAdjPlan *)plan;
    if (!p) return cudaErrorInvalidValue;
    const dim3 grid((g.maxx + 127) / 128, g.maxy, g.nz);
    const double *ab[3] = {aubar, avbar, awbar};
    for (int c = 0; c < 3; c++)
        for (int s0 = 0; s0 < p->nslot[c]; s0 += NCH) {
            mom_ad_kernel<<<grid, 128, 0, s>>>(g, ntime, c, s0, p->nslot[c], Mom3{{mu, mv, mw}}, ab[c], p->slot + c * NOFF,
                                               p->offs + c * NOFF, Mom3{{mubar, mvbar, mwbar}});
            cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) return e;
        }
    return cudaSuccess;
}
