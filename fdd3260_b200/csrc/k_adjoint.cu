// k_adjoint.cu -- tangent-linear and adjoint of the scalar advection operator.
//
// The operator is the advective tendency of one density-weighted field x,
//     A(x, m) = -(Tx + Ty + Tz),  Tx = (F(i+1/2) - F(i-1/2)) * dx1, ...
// with the WENO3-switch face fluxes of src/TOOLS/advq_weno.f90 (x :61-131, y :134-199,
// z :202-301) and the advective velocity u = m/rho0 - shift of
// src/TOOLS/funcpack.f90:65-94 -- the tendency mg_advection_ac adds to xs.
//
// The Jacobian of every face flux with respect to its four stencil values and its
// velocity is obtained by evaluating the forward scheme templates on dual numbers
// (dual.cuh): the switch to nonlinear weights and the positivity limiter follow the
// branch the FP64 form takes, and the smoothness weights are differentiated.  The
// face template is the upwind-only one the forward kernel runs (weno_face_up): the
// downwind side's term is zero with a zero derivative, so only the upwind side's
// weights are carried on dual numbers.
//   TL: dA = J (dx, dm), per direction a face pass (each face's tangent flux once) and a
//       difference pass over the cells.
//   AD: (xbar, mbar) = J^T Abar, deterministic per direction: one kernel computes Fbar * J
//       of the faces around a tile into shared memory and sums, for each cell of the
//       tile, the four faces that read it; the adjoints of the periodic ghost cells are
//       then folded onto the cells they are images of.
#include "dual.cuh"
#include "mg_common.cuh"
#include "mimica_gpu.h"
#include "weno_partials.cuh"

namespace {

using D5 = D<5>;

struct AdvIn {
    const double *x, *mu, *mv, *mw;
};

// partials of the face flux of direction dir whose lower cell is (i,j,k):
// J[m] with respect to the stencil cell (lower - 1 + m) along dir, m = 0..3, and
// Jv with respect to the momentum that carries the face velocity; returns false when
// the face does not exist (z faces k+1/2 with k outside 1..nz-1)
__device__ bool face_jac(const DevGrid &G, int dir, const AdvIn &in, int i, int j, int k, double J[4], double &Jv)
{
    const int nz = G.nz;
    if (dir == 2 && (k < 1 || k > nz - 1)) return false;
    for (int m = 0; m < 4; m++) J[m] = 0.;
    Jv = 0.;
    if (dir == 0 || dir == 1) {
        const long long st = dir == 0 ? 1 : G.px;
        const long long c = gidx(G, i, j, k);
        const double d0 = __ldg(G.den0 + k - 1);
        const double mom = dir == 0 ? __ldg(in.mu + c + 1) : __ldg(in.mv + c + G.px);
        const double shift = dir == 0 ? G.u0shift : G.v0shift;
        double Ju;
        weno_face_partials(__ldg(in.x + c - st), __ldg(in.x + c), __ldg(in.x + c + st), __ldg(in.x + c + 2 * st),
                           mom / d0 - shift, true, J, Ju);
        Jv = Ju / d0;
        return true;
    }
    const long long c = gidx(G, i, j, k);
    const long long st = G.ps;
    const double a1 = __ldg(G.avden0 + k);   // w(k+1) carries face k+1/2
    const D5 w = D5::var(__ldg(in.mw + c + st) / a1, 4);
    D5 F;
    if (k == 1) {   // bottom face: x(1), x(2), x(3) at stencil positions 1..3
        const D5 x1 = D5::var(__ldg(in.x + c), 1), x2 = D5::var(__ldg(in.x + c + st), 2);
        const D5 x3 = D5::var(__ldg(in.x + c + 2 * st), 3);
        F = weno_face_bottom<D5>(x1, x2, x3, w);
    } else if (k == nz - 1) {   // top face: x(nz-2), x(nz-1), x(nz) at positions 0..2
        const D5 a = D5::var(__ldg(in.x + c - st), 0), b = D5::var(__ldg(in.x + c), 1);
        const D5 cc = D5::var(__ldg(in.x + c + st), 2);
        F = weno_face_top<D5>(a, b, cc, w);
    } else {
        double Ju;
        weno_face_partials(__ldg(in.x + c - st), __ldg(in.x + c), __ldg(in.x + c + st), __ldg(in.x + c + 2 * st), w.v,
                           k >= 3 && k <= nz - 3, J, Ju);
        Jv = Ju / a1;
        return true;
    }
    for (int m = 0; m < 4; m++) J[m] = F.d[m];
    Jv = F.d[4] / a1;
    return true;
}

__device__ __forceinline__ double face_metric(const DevGrid &G, int dir, int k)
{
    return dir == 0 ? 1. / G.dx : (dir == 1 ? 1. / G.dy : __ldg(G.dz1w + k - 1));
}

// ---- tangent linear, face pass of one direction: dF[face] = J (dx stencil, dm) ----
// faces indexed by their lower cell, as the adjoint's face pass
__global__ void __launch_bounds__(256, 3) adv_tl_face_kernel(DevGrid G, int dir, AdvIn in, AdvIn d, double *dF)
{
    const int maxx = G.maxx, maxy = G.maxy, nz = G.nz;
    const int ni = dir == 0 ? maxx + 1 : maxx, nj = dir == 1 ? maxy + 1 : maxy, nk = dir == 2 ? nz - 1 : nz;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)ni * nj * nk) return;
    const int i = (int)(t % ni) + (dir == 0 ? 3 : 4), j = (int)((t / ni) % nj) + (dir == 1 ? 3 : 4);
    const int k = (int)(t / ((long long)ni * nj)) + 1;
    const long long c = gidx(G, i, j, k);
    const long long st = dir == 0 ? 1 : (dir == 1 ? G.px : G.ps);
    const double *dm = dir == 0 ? d.mu : (dir == 1 ? d.mv : d.mw);
    double J[4], Jv;
    face_jac(G, dir, in, i, j, k, J, Jv);   // every face of the range exists
    double v = 0.;
    for (int m = 0; m < 4; m++)
        if (J[m] != 0.) v += J[m] * __ldg(d.x + c + (m - 1) * st);
    dF[c] = v + Jv * __ldg(dm + c + st);
}

// ---- tangent linear, difference pass: dA (-)= (dF(c+1/2) - dF(c-1/2)) * metric ----
__global__ void adv_tl_diff_kernel(DevGrid G, int dir, const double *dF, double *dA, int first)
{
    const int maxx = G.maxx, maxy = G.maxy, nz = G.nz;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)maxx * maxy * nz) return;
    const int i = (int)(t % maxx) + 4, j = (int)((t / maxx) % maxy) + 4, k = (int)(t / ((long long)maxx * maxy)) + 1;
    const long long c = gidx(G, i, j, k);
    const long long st = dir == 0 ? 1 : (dir == 1 ? G.px : G.ps);
    const double up = (dir == 2 && k == nz) ? 0. : __ldg(dF + c);
    const double lo = (dir == 2 && k == 1) ? 0. : __ldg(dF + c - st);
    const double v = (up - lo) * face_metric(G, dir, k);
    dA[c] = first ? -v : dA[c] - v;
}

// ---- adjoint of one direction in one pass: face partials and gather per tile ----
// A tile is LA cells along the direction times LB across it (x: 32 x 8 rows at one level;
// y: 16 rows x 32 columns at one level; z: 16 levels x 32 columns at one row), over every
// cell, ghosts included.  Its CTA computes Fbar * J of the LA + 3 faces along each line
// whose stencil or velocity touches the tile (lower cells a0-2 .. a0+LA; faces that do not
// exist are zeros) into shared memory, then each cell sums the four faces that read it and
// the face its velocity carries, as adv_ad_face_kernel + adv_ad_gather_kernel do with the
// face values in global memory.
template <int DIR>
struct AdTile {
    static constexpr int LA = DIR == 0 ? 32 : 16, LB = DIR == 0 ? 8 : 32, NF = (LA + 3) * LB;
};

template <int DIR>
__global__ void __launch_bounds__(256) adv_ad_fused_kernel(DevGrid G, AdvIn in, const double *Abar, double *xbar,
                                                          double *mbar)
{
    using T = AdTile<DIR>;
    __shared__ double gs[5][T::NF];
    const int nx = G.nx, ny = G.ny, nz = G.nz;
    const int na = DIR == 0 ? nx : (DIR == 1 ? ny : nz), nb = DIR == 0 ? ny : nx;
    const int ta = (na + T::LA - 1) / T::LA, tb = (nb + T::LB - 1) / T::LB;
    const int t = blockIdx.x % (ta * tb), fixed = blockIdx.x / (ta * tb) + 1;   // k (x, y) or j (z)
    const int a0 = 1 + (t % ta) * T::LA, b0 = 1 + (t / ta) * T::LB;
    const long long sa = DIR == 0 ? 1 : (DIR == 1 ? G.px : G.ps);
    auto cell = [&](int a, int b, int &i, int &j, int &k) {
        if (DIR == 0) { i = a; j = b; k = fixed; }
        else if (DIR == 1) { i = b; j = a; k = fixed; }
        else { i = b; j = fixed; k = a; }
    };
    auto interior = [&](int ii, int jj, int kk) { return ii >= 4 && ii <= nx - 2 && jj >= 4 && jj <= ny - 2 && kk >= 1 && kk <= nz; };
    for (int q = threadIdx.x; q < T::NF; q += blockDim.x) {
        // x: consecutive q run along a (x) for coalescing; y/z: along b (x)
        const int fa = DIR == 0 ? q % (T::LA + 3) : q / T::LB, fb = DIR == 0 ? q / (T::LA + 3) : q % T::LB;
        const int l = a0 - 2 + fa, bb = b0 + fb;
        int i, j, k;
        cell(l, bb, i, j, k);
        bool ok;
        if (DIR == 0) ok = l >= 3 && l <= nx - 2 && j >= 4 && j <= ny - 2 && k >= 1 && k <= nz;
        else if (DIR == 1) ok = l >= 3 && l <= ny - 2 && i >= 4 && i <= nx - 2 && k >= 1 && k <= nz;
        else ok = l >= 1 && l <= nz - 1 && i >= 4 && i <= nx - 2 && j >= 4 && j <= ny - 2;
        double g[5] = {0., 0., 0., 0., 0.};
        if (ok) {
            const long long c = gidx(G, i, j, k);
            const int ui = DIR == 0 ? i + 1 : i, uj = DIR == 1 ? j + 1 : j, uk = DIR == 2 ? k + 1 : k;
            double Fbar = 0.;
            if (interior(i, j, k)) Fbar -= Abar[c] * face_metric(G, DIR, k);
            if (interior(ui, uj, uk)) Fbar += Abar[c + sa] * face_metric(G, DIR, uk);
            double J[4], Jv;
            if (face_jac(G, DIR, in, i, j, k, J, Jv)) {
                for (int m = 0; m < 4; m++) g[m] = Fbar * J[m];
                g[4] = Fbar * Jv;
            }
        }
        for (int m = 0; m < 5; m++) gs[m][q] = g[m];
    }
    __syncthreads();
    // face (lower cell l, cross index fb) sits at smem index face_at(l - (a0 - 2), fb)
    auto face_at = [&](int fa, int fb) { return DIR == 0 ? fb * (T::LA + 3) + fa : fa * T::LB + fb; };
    for (int q = threadIdx.x; q < T::LA * T::LB; q += blockDim.x) {
        const int ca = DIR == 0 ? q % T::LA : q / T::LB, cb = DIR == 0 ? q / T::LA : q % T::LB;
        const int p = a0 + ca, bb = b0 + cb;
        if (p > na || bb > nb) continue;
        int i, j, k;
        cell(p, bb, i, j, k);
        const long long c = gidx(G, i, j, k);
        // cell p is stencil position m of the face with lower cell p + 1 - m
        const int f0 = p + 1 - (a0 - 2);
        const double s = ((gs[0][face_at(f0, cb)] + gs[1][face_at(f0 - 1, cb)]) + gs[2][face_at(f0 - 2, cb)]) +
                         gs[3][face_at(f0 - 3, cb)];
        xbar[c] += s;
        // the face with lower cell p-1 is carried by the velocity at index p
        mbar[c] += gs[4][face_at(f0 - 2, cb)];
    }
}

// adjoint of the periodic ghost images: ghost columns then ghost rows are added onto
// the cells they copy, then zeroed (each destination receives from one ghost per pass)
__global__ void fold_x_kernel(DevGrid G, double *f)
{
    const int ny = G.ny, nz = G.nz, maxx = G.maxx;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 5LL * ny * nz) return;
    const int q = (int)(t % 5), j = (int)((t / 5) % ny) + 1, k = (int)(t / (5LL * ny)) + 1;
    const int gi = q < 3 ? q + 1 : G.nx - 4 + q;   // 1,2,3, nx-1, nx
    const int si = gi <= 3 ? gi + maxx : gi - maxx;
    const long long gc = gidx(G, gi, j, k);
    f[gidx(G, si, j, k)] += f[gc];
    f[gc] = 0.;
}
__global__ void fold_y_kernel(DevGrid G, double *f)
{
    const int nx = G.nx, nz = G.nz, maxy = G.maxy;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 5LL * nx * nz) return;
    const int i = (int)(t % nx) + 1, q = (int)((t / nx) % 5), k = (int)(t / (5LL * nx)) + 1;
    const int gj = q < 3 ? q + 1 : G.ny - 4 + q;
    const int sj = gj <= 3 ? gj + maxy : gj - maxy;
    const long long gc = gidx(G, i, gj, k);
    f[gidx(G, i, sj, k)] += f[gc];
    f[gc] = 0.;
}

inline unsigned nblk(long long n) { return (unsigned)((n + 255) / 256); }

}  // namespace

// dA = J (dx, dm) over the interior; scratch: one field (the face tangents of a direction)
cudaError_t launch_advection_tl(const DevGrid &g, const double *x, const double *mu, const double *mv, const double *mw,
                                const double *dx, const double *dmu, const double *dmv, const double *dmw, double *dA,
                                double *scratch, cudaStream_t s)
{
    const AdvIn in{x, mu, mv, mw}, d{dx, dmu, dmv, dmw};
    const long long ncell = (long long)g.maxx * g.maxy * g.nz;
    for (int dir = 0; dir < 3; dir++) {
        const long long nf = (long long)(dir == 0 ? g.maxx + 1 : g.maxx) * (dir == 1 ? g.maxy + 1 : g.maxy) *
                             (dir == 2 ? g.nz - 1 : g.nz);
        adv_tl_face_kernel<<<nblk(nf), 256, 0, s>>>(g, dir, in, d, scratch);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        adv_tl_diff_kernel<<<nblk(ncell), 256, 0, s>>>(g, dir, scratch, dA, dir == 0);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// xbar, mubar, mvbar, mwbar are overwritten (accumulate = 0) or added to (1: their ghost
// cells are zero on entry; the ghost folds below move the kernels' ghost contributions
// onto the cells they image and leave the ghosts zero)
cudaError_t launch_advection_ad(const DevGrid &g, const double *x, const double *mu, const double *mv, const double *mw,
                                const double *Abar, double *xbar, double *mubar, double *mvbar, double *mwbar,
                                cudaStream_t s, int accumulate)
{
    const size_t fbytes = (size_t)g.ps * g.nz * 8;
    cudaError_t e;
    double *outs[4] = {xbar, mubar, mvbar, mwbar};
    for (int q = 0; q < 4 && !accumulate; q++)
        if ((e = cudaMemsetAsync(outs[q], 0, fbytes, s)) != cudaSuccess) return e;
    const AdvIn in{x, mu, mv, mw};
    auto tiles = [&](int na, int la, int nb, int lb, int nfix) {
        return (unsigned)(((na + la - 1) / la) * ((nb + lb - 1) / lb) * nfix);
    };
    adv_ad_fused_kernel<0><<<tiles(g.nx, AdTile<0>::LA, g.ny, AdTile<0>::LB, g.nz), 256, 0, s>>>(g, in, Abar, xbar, mubar);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    adv_ad_fused_kernel<1><<<tiles(g.ny, AdTile<1>::LA, g.nx, AdTile<1>::LB, g.nz), 256, 0, s>>>(g, in, Abar, xbar, mvbar);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    adv_ad_fused_kernel<2><<<tiles(g.nz, AdTile<2>::LA, g.nx, AdTile<2>::LB, g.ny), 256, 0, s>>>(g, in, Abar, xbar, mwbar);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    for (int q = 0; q < 4; q++) {
        fold_x_kernel<<<nblk(5LL * g.ny * g.nz), 256, 0, s>>>(g, outs[q]);
        fold_y_kernel<<<nblk(5LL * g.nx * g.nz), 256, 0, s>>>(g, outs[q]);
    }
    return cudaGetLastError();
}
