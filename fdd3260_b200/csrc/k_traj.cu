// k_traj.cu -- the pointwise and short-stencil parts of one integrator stage, their
// tangent linear and their adjoint, for the trajectory adjoint of the FP64 path.
//
// A stage (src/INTEG/time_step.f90:256-281 with momentum.f90:64-228, scalars.f90,
// integpack.f90:54-284, integ.h) on top of the advection tendencies A (K1 unit mode)
// and qnadv (K2 unit mode):
//   gp   = backward differences of p/rho0; gpz(1) = mw(1)/(dt0 avden0(1))   (gradp)
//   bb   = rho g (theta (1 + eps qt/rho)/ref - 1), theta = (psi_es + cdiag dt0 A_es)/rho,
//          qt = psi_qt + cdiag dt0 A_qt; buoy = averages of bb to the w faces  (imp_buoy)
//   ws   = -qnadv + (0 - rho0 gp) [+ buoy for w]
//   t    = ws + b t_prev;  m_out = m_n + a dt0 t                            (integ_mom)
//   t_f  = A_f + b t_prev_f;  psi_out = s_n rho_n + a dt0 t_f  (rho: rho_n + ...)  (integ_scal)
// The forward and tangent-linear kernels are one template instantiated on double and
// on dual numbers with one partial; each expression keeps the reference's operation
// order, so the double instance reproduces the fused stage kernels.  The adjoint
// kernels are written in gather form (each thread sums what reads its own cell), so
// they need no atomics; the adjoints of periodic ghost reads land on the interior cells
// the ghosts copy.
#include "dual.cuh"
#include "mg_common.cuh"

namespace {

constexpr double GRAV = 9.81, EPSM = 0.60243, CDIAG = 0.5;

using D1 = D<1>;

template <typename T> struct Val;
template <> struct Val<double> {
    __device__ static double get(const double *v, const double *, long long q) { return __ldg(v + q); }
    __device__ static void put(double *v, double *, long long q, double x) { v[q] = x; }
};
template <> struct Val<D1> {
    __device__ static D1 get(const double *v, const double *d, long long q)
    {
        D1 r(__ldg(v + q));
        r.d[0] = __ldg(d + q);
        return r;
    }
    __device__ static void put(double *v, double *d, long long q, const D1 &x)
    {
        if (v) v[q] = x.v;
        d[q] = x.d[0];
    }
};

__device__ __forceinline__ int wrap_x(const DevGrid &G, int i) { return i < 4 ? i + G.maxx : (i > G.nx - 2 ? i - G.maxx : i); }
__device__ __forceinline__ int wrap_y(const DevGrid &G, int j) { return j < 4 ? j + G.maxy : (j > G.ny - 2 ? j - G.maxy : j); }

// rho g (theta (1 + eps qt / rho) / ref - 1) at one level (thermodynamics.f90:472-534)
template <typename T>
__device__ __forceinline__ T bb_level(const DevGrid &G, int k, const T &dn, const T &est, const T &qtt)
{
    const double ref = __ldg(G.pt0 + k - 1) * (1. + EPSM * __ldg(G.qv0 + k - 1));
    const T den1 = T(1.) / dn;
    const T pt = den1 * est;
    const T sumh = T(0.);
    return dn * T(GRAV) * (pt * (T(1.) + T(EPSM) * den1 * (qtt - sumh) - den1 * sumh) / T(ref) - T(1.));
}

// ---------------- momentum assembly and update ----------------
template <typename T>
__global__ void stage_mom_kernel(DevGrid G, TrajMomArgs A)
{
    const int i = 4 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 4 + blockIdx.y;
    const int k = 1 + blockIdx.z;
    if (i > G.nx - 2) return;
    const long long c = gidx(G, i, j, k), px = G.px, ps = G.ps;
    auto L = [&](int f, long long q) { return Val<T>::get(A.v[f], A.d[f], q); };
    const double d0 = __ldg(G.den0 + k - 1), a0 = __ldg(G.avden0 + k - 1);
    const double dx1 = 1. / G.dx, dy1 = 1. / G.dy;
    // explicit pressure gradient of p/rho0 (gradp)
    const T ppc = L(TM_P, c) / T(d0);
    const T gpx = (ppc - L(TM_P, c - 1) / T(d0)) * T(dx1);
    const T gpy = (ppc - L(TM_P, c - px) / T(d0)) * T(dy1);
    T gpz;
    if (k >= 2) gpz = (ppc - L(TM_P, c - ps) / T(__ldg(G.den0 + k - 2))) * T(__ldg(G.dz1 + k - 2));
    else gpz = L(TM_MW, c) / T(G.dt0 * __ldg(G.avden0));
    T wsu = T(0.) - T(d0) * gpx;
    T wsv = T(0.) - T(d0) * gpy;
    T wsw = T(0.) - T(a0) * gpz;
    // implicit buoyancy at the w face k
    T buoy = T(0.);
    if (G.with_buoy) {
        auto bb = [&](int kk) {
            const long long q = c + (long long)(kk - k) * ps;
            const T est = L(TM_ES, q) + T(CDIAG * G.dt0) * L(TM_AES, q);
            const T qtt = A.v[TM_QT] ? L(TM_QT, q) + T(CDIAG * G.dt0) * L(TM_AQT, q) : T(0.);
            return bb_level(G, kk, L(TM_RHO, q), est, qtt);
        };
        const T bk = bb(k);
        buoy = k >= 2 ? T(0.5) * (bb(k - 1) + bk) : bk;
    }
    wsu = -L(TM_AU, c) + wsu;
    wsv = -L(TM_AV, c) + wsv;
    wsw = -L(TM_AW, c) + wsw + buoy;
    // integ_mom: t = ws + b t_prev, m = m_n + a dt0 t
    const T tu = wsu + T(A.b) * (A.b != 0. ? L(TM_TU, c) : T(0.));
    const T tv = wsv + T(A.b) * (A.b != 0. ? L(TM_TV, c) : T(0.));
    const T tw = wsw + T(A.b) * (A.b != 0. ? L(TM_TW, c) : T(0.));
    Val<T>::put(A.out[0], A.dout[0], c, tu);
    Val<T>::put(A.out[1], A.dout[1], c, tv);
    Val<T>::put(A.out[2], A.dout[2], c, tw);
    Val<T>::put(A.out[3], A.dout[3], c, L(TM_UN, c) * T(d0) + T(A.a_dt) * tu);
    Val<T>::put(A.out[4], A.dout[4], c, L(TM_VN, c) * T(d0) + T(A.a_dt) * tv);
    Val<T>::put(A.out[5], A.dout[5], c, T(1.) * (L(TM_WN, c) * T(a0) + T(A.a_dt) * tw));
}

// ---------------- scalar update (integ_scal) ----------------
template <typename T>
__global__ void stage_scal_kernel(DevGrid G, TrajScalArgs A)
{
    const int i = 4 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 4 + blockIdx.y;
    const int k = 1 + blockIdx.z;
    if (i > G.nx - 2) return;
    const long long c = gidx(G, i, j, k);
    const T dens2 = Val<T>::get(A.rhon, A.drhon, c);
    for (int f = 0; f < A.nf; f++) {
        const T ts = Val<T>::get(A.adv[f], A.dadv[f], c) + T(A.b) * (A.b != 0. ? Val<T>::get(A.tprev[f], A.dtprev[f], c) : T(0.));
        Val<T>::put(A.tout[f], A.dtout[f], c, ts);
        const T old = f == 0 ? dens2 : Val<T>::get(A.sn[f], A.dsn[f], c) * dens2;
        Val<T>::put(A.out[f], A.dout[f], c, old + T(A.a_dt) * ts);
    }
}

// ---------------- conversions between natural and stage variables ----------------
// dir 0: m = u rho0 (w: avden0), psi_f = s_f rho (f >= 1); dir 1: the inverse
template <typename T>
__global__ void convert_kernel(DevGrid G, TrajConv A)
{
    const long long n = G.ps * G.nz;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int k = 1 + (int)(q / G.ps);
        const double d0 = __ldg(G.den0 + k - 1), a0 = __ldg(G.avden0 + k - 1);
        for (int f = 0; f < 3; f++) {
            const T x = Val<T>::get(A.in[f], A.din[f], q);
            const double w = f == 2 ? a0 : d0;
            Val<T>::put(A.out[f], A.dout[f], q, A.dir == 0 ? x * T(w) : x / T(w));
        }
        const T rho = Val<T>::get(A.rho, A.drho, q);
        for (int f = 0; f < A.ns; f++) {
            const T x = Val<T>::get(A.in[3 + f], A.din[3 + f], q);
            Val<T>::put(A.out[3 + f], A.dout[3 + f], q, A.dir == 0 ? x * rho : x / rho);
        }
    }
}

// ---------------- adjoints ----------------
// momentum assembly: from mbar (m_out), tcarry (b_next t_next-bar), produces
// tbar_prev (= b tbar, to the previous stage), mnbar += rho0 mbar (natural level n),
// abar (qnadv adjoint input, = -ws-bar), pbar += gradp^T, mwbar_in(1) += gpz(1) term,
// rho/es/qt/aes/aqt adjoints of the buoyancy (accumulated).
__global__ void stage_mom_ad_kernel(DevGrid G, TrajMomAd A)
{
    const int i = 4 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 4 + blockIdx.y;
    const int k = 1 + blockIdx.z;
    if (i > G.nx - 2) return;
    const int nz = G.nz;
    const long long c = gidx(G, i, j, k), ps = G.ps;
    const double dx1 = 1. / G.dx, dy1 = 1. / G.dy;
    // ws-bar of a cell: a dt0 mbar + carry
    auto wsb = [&](int f, long long q) {
        const double mb = __ldg(A.mbar[f] + q);
        return A.a_dt * mb + (A.tcarry[f] ? __ldg(A.tcarry[f] + q) : 0.);
    };
    const double wu = wsb(0, c), wv = wsb(1, c), ww = wsb(2, c);
    const double d0 = __ldg(G.den0 + k - 1), a0 = __ldg(G.avden0 + k - 1);
    for (int f = 0; f < 3; f++) {
        const double wsf = f == 0 ? wu : (f == 1 ? wv : ww);
        if (A.tprev_bar[f]) A.tprev_bar[f][c] = A.b * wsf;
        A.abar[f][c] = -wsf;
        A.mnbar[f][c] += (f == 2 ? a0 : d0) * __ldg(A.mbar[f] + c);
    }
    // gradp^T: pp-bar(c) = sum over the gradients that read pp(c)
    //   gpx(c) = (pp(c) - pp(i-1)) dx1 -> ws-bar_u(c) (-d0) dx1 at c, -(...) at the cell i+1
    auto gxb = [&](int ii, int jj) {   // gpx-bar of the interior cell (ii, jj, k)
        return -d0 * wsb(0, gidx(G, wrap_x(G, ii), wrap_y(G, jj), k));
    };
    auto gyb = [&](int ii, int jj) { return -d0 * wsb(1, gidx(G, wrap_x(G, ii), wrap_y(G, jj), k)); };
    double ppb = gxb(i, j) * dx1 - gxb(i + 1, j) * dx1;
    ppb += gyb(i, j) * dy1 - gyb(i, j + 1) * dy1;
    auto gzb = [&](int kk) { return -__ldg(G.avden0 + kk - 1) * wsb(2, gidx(G, i, j, kk)); };
    if (k >= 2) ppb += gzb(k) * __ldg(G.dz1 + k - 2);
    if (k + 1 <= nz) ppb -= gzb(k + 1) * __ldg(G.dz1 + k - 1);
    A.pbar[c] += ppb / d0;
    if (k == 1) A.mwin_bar[c] += gzb(1) / (G.dt0 * __ldg(G.avden0));
    // buoyancy: bb(k) feeds buoy(k) (weight 1 at k = 1, 1/2 above) and buoy(k+1) (1/2)
    if (G.with_buoy) {
        double bbb = (k == 1 ? 1. : 0.5) * ww;
        if (k + 1 <= nz) bbb += 0.5 * wsb(2, c + ps);
        const D<3> dn = D<3>::var(__ldg(A.rho + c), 0);
        const D<3> est = D<3>::var(__ldg(A.es + c) + CDIAG * G.dt0 * __ldg(A.aes + c), 1);
        const D<3> qtt = A.qt ? D<3>::var(__ldg(A.qt + c) + CDIAG * G.dt0 * __ldg(A.aqt + c), 2) : D<3>(0.);
        const D<3> b = bb_level(G, k, dn, est, qtt);
        A.rho_bar[c] += bbb * b.d[0];
        A.es_bar[c] += bbb * b.d[1];
        A.aes_bar[c] += CDIAG * G.dt0 * (bbb * b.d[1]);
        if (A.qt) {
            A.qt_bar[c] += bbb * b.d[2];
            A.aqt_bar[c] += CDIAG * G.dt0 * (bbb * b.d[2]);
        }
    }
}

// scalar update: tbar = a dt0 psi-bar + carry -> adv-bar (+=), tprev-bar = b tbar,
// s_n-bar += rho_n psi-bar, rho_n-bar += s_n psi-bar (f >= 1) or psi-bar (f = 0)
__global__ void stage_scal_ad_kernel(DevGrid G, TrajScalAd A)
{
    const int i = 4 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 4 + blockIdx.y;
    const int k = 1 + blockIdx.z;
    if (i > G.nx - 2) return;
    const long long c = gidx(G, i, j, k);
    const double rhon = __ldg(A.rhon + c);
    double rnb = 0.;
    for (int f = 0; f < A.nf; f++) {
        const double pb = __ldg(A.psibar[f] + c);
        const double tb = A.a_dt * pb + (A.tcarry[f] ? __ldg(A.tcarry[f] + c) : 0.);
        A.advbar[f][c] += tb;
        if (A.tprev_bar[f]) A.tprev_bar[f][c] = A.b * tb;
        if (f == 0) {
            rnb += pb;
        } else {
            A.snbar[f][c] += rhon * pb;
            rnb += __ldg(A.sn[f] + c) * pb;
        }
    }
    A.snbar[0][c] += rnb;   // the level-n density
}

// conversions: dir 0 (m = u w, psi = s rho; in = the natural s): u-bar += w m-bar,
// s-bar += rho psi-bar, rho-bar += s psi-bar; dir 1 (u = m / w, s = psi / rho; in = the
// natural s of the output): m-bar += u-bar / w, psi-bar += s-bar / rho,
// rho-bar -= s s-bar / rho (= psi s-bar / rho^2) (interior cells)
__global__ void convert_ad_kernel(DevGrid G, TrajConvAd A)
{
    const int i = 4 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 4 + blockIdx.y;
    const int k = 1 + blockIdx.z;
    if (i > G.nx - 2) return;
    const long long c = gidx(G, i, j, k);
    const double d0 = __ldg(G.den0 + k - 1), a0 = __ldg(G.avden0 + k - 1);
    for (int f = 0; f < 3; f++) {
        const double w = f == 2 ? a0 : d0;
        const double ob = __ldg(A.outbar[f] + c);
        A.inbar[f][c] += A.dir == 0 ? w * ob : ob / w;
    }
    const double rho = __ldg(A.rho + c);
    double rb = 0.;
    for (int f = 0; f < A.ns; f++) {
        const double ob = __ldg(A.outbar[3 + f] + c);
        const double x = __ldg(A.in[3 + f] + c);
        if (A.dir == 0) {
            A.inbar[3 + f][c] += rho * ob;
            rb += x * ob;
        } else {
            A.inbar[3 + f][c] += ob / rho;
            rb -= x * ob / rho;
        }
    }
    A.rhobar[c] += rb;
}

__global__ void axpy_kernel(long long n, double *y, const double *x, double alpha)
{
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        y[q] += alpha * x[q];
}

inline dim3 cell_grid(const DevGrid &g) { return dim3((g.maxx + 127) / 128, g.maxy, g.nz); }

}  // namespace

cudaError_t launch_stage_mom(const DevGrid &g, const TrajMomArgs &a, int tangent, cudaStream_t s)
{
    if (tangent) stage_mom_kernel<D1><<<cell_grid(g), 128, 0, s>>>(g, a);
    else stage_mom_kernel<double><<<cell_grid(g), 128, 0, s>>>(g, a);
    return cudaGetLastError();
}
cudaError_t launch_stage_scal(const DevGrid &g, const TrajScalArgs &a, int tangent, cudaStream_t s)
{
    if (a.nf > MG_MAXF) return cudaErrorInvalidValue;
    if (tangent) stage_scal_kernel<D1><<<cell_grid(g), 128, 0, s>>>(g, a);
    else stage_scal_kernel<double><<<cell_grid(g), 128, 0, s>>>(g, a);
    return cudaGetLastError();
}
cudaError_t launch_convert(const DevGrid &g, const TrajConv &a, int tangent, cudaStream_t s)
{
    if (tangent) convert_kernel<D1><<<1184, 256, 0, s>>>(g, a);
    else convert_kernel<double><<<1184, 256, 0, s>>>(g, a);
    return cudaGetLastError();
}
cudaError_t launch_stage_mom_ad(const DevGrid &g, const TrajMomAd &a, cudaStream_t s)
{
    stage_mom_ad_kernel<<<cell_grid(g), 128, 0, s>>>(g, a);
    return cudaGetLastError();
}
cudaError_t launch_stage_scal_ad(const DevGrid &g, const TrajScalAd &a, cudaStream_t s)
{
    stage_scal_ad_kernel<<<cell_grid(g), 128, 0, s>>>(g, a);
    return cudaGetLastError();
}
cudaError_t launch_convert_ad(const DevGrid &g, const TrajConvAd &a, cudaStream_t s)
{
    convert_ad_kernel<<<cell_grid(g), 128, 0, s>>>(g, a);
    return cudaGetLastError();
}

// y += alpha x over the whole allocation
cudaError_t launch_axpy(const DevGrid &g, double *y, const double *x, double alpha, cudaStream_t s)
{
    axpy_kernel<<<1184, 256, 0, s>>>(g.ps * g.nz, y, x, alpha);
    return cudaGetLastError();
}
