// k_scalar.cu -- K1: flux-form advection of all density-weighted scalars (and the
// density itself) fused with the Heun stage update, plain FP64 form.
//
// Replaces, per stage, src/TOOLS/advection.f90 advect/advection_ac ->
// advection_x/y/z (:556-798) -> advs{x,y,z}_{weno,ppm,muscl}
// (src/TOOLS/advq_weno.f90, advq_ppm.f90, advq_muscl.f90) and integ_scal
// (src/INTEG/integpack.f90:137-261).
//
// Grid: blockIdx.x = field, blockIdx.y = 32x8 column tile.  Blocks of one tile are
// consecutive in launch order, so the momentum and density tiles they all read are
// served from L2 after the first block touches them.  Each block marches k = 1..nz:
// the x/y stencils read plane k staged in shared memory (3 ghost cells each side),
// the z stencil reads a five-level register window of the thread's own column.
// Per cell the tendency is T = ((0 - Tx) - Ty) - Tz, the reference's accumulation
// order (advection_x/y/z subtract each direction's tendency in turn).
//
// Compiled with -fmad=false: bit-identical to the CPU restatement.
#include "mg_common.cuh"
#include "schemes.cuh"

namespace {

constexpr int TX = 32, TY = 8, H = 3;
constexpr int SW = TX + 2 * H, SH = TY + 2 * H;

__device__ __forceinline__ double ldg(const double *p, long long i) { return __ldg(p + i); }

// advective velocity from momentum (get_advective, src/TOOLS/funcpack.f90:65-94)
__device__ __forceinline__ double mom_val(const K1Args &A, const double *m, long long idx, double w)
{
    double x = ldg(m, idx);
    if (A.mom_rep < 0) return x;
    return rep_value(A.mom_rep, x, w);
}

template <int SCHEME>
__global__ void __launch_bounds__(TX *TY) k1_kernel(DevGrid G, K1Args A)
{
    extern __shared__ double sm[];
    double *sx = sm;                        // SH*SW   stencil values of plane k
    double *su = sx + SH * SW;              // TY*(TX+1)  u_adv at x-faces
    double *sv = su + TY * (TX + 1);        // (TY+1)*TX  v_adv at y-faces
    double *fx = sv + (TY + 1) * TX;        // TY*(TX+1)  x-face fluxes
    double *fy = fx + TY * (TX + 1);        // (TY+1)*TX  y-face fluxes
    double *crx = fy + (TY + 1) * TX;       // PPM: 4 * TY*(TX+2)
    double *cry = crx + 4 * TY * (TX + 2);  // PPM: 4 * (TY+2)*TX

    const int f = blockIdx.x;
    const int ntx = (G.maxx + TX - 1) / TX;
    const int ti = blockIdx.y % ntx, tj = blockIdx.y / ntx;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const int i0 = 4 + ti * TX, j0 = 4 + tj * TY;
    const int i = i0 + tx, j = j0 + ty;
    const int nx = G.nx, ny = G.ny, nz = G.nz;
    const bool act = (i <= nx - 2) && (j <= ny - 2);
    const int ic = min(i, nx - 2), jc = min(j, ny - 2);
    const bool weighted = !(A.dens_first && f == 0);
    const bool conv = (A.stage == 1) && weighted;
    const double *xin = A.xin[f];
    const double *dens_n = A.dens_n;
    const double dx1 = 1. / G.dx, dy1 = 1. / G.dy, dt0 = G.dt0;

    auto sval = [&](long long idx) -> double {
        double x = ldg(xin, idx);
        return conv ? rep_value(A.rep, x, ldg(dens_n, idx)) : x;
    };
    auto wadv = [&](int kk) -> double {  // w_adv at own column, level kk
        long long idx = gidx(G, ic, jc, kk);
        double a0 = ldg(G.avden0, kk - 1);
        return mom_val(A, A.mw, idx, a0) / a0;
    };

    // z window: zx[m] = x(k-1+m), m = 0..4 ; zw[m] = w_adv(k+m), m = 0..2
    double zx[5], zw[3];
    zx[0] = 0.;
    for (int m = 1; m < 5; m++) zx[m] = (m <= nz) ? sval(gidx(G, ic, jc, m)) : 0.;
    for (int m = 0; m < 3; m++) zw[m] = (1 + m <= nz) ? wadv(1 + m) : 0.;

    double Fzo = 0.;                 // z-face flux below the current level
    // PPM vertical chain: reconstruction of the cell below, carried upward
    double pr_fr = 0., pr_xplus = 0.;
    if (SCHEME == MG_PPM) {
        // cell 1 (:328-343): bottom special, bc51 = 0
        double x1 = zx[1], x2 = zx[2], x3 = zx[3];
        double d1 = ldg(G.dz1, 0);
        double mup = fabs(zw[1]) * dt0 * d1;
        double ffip1 = x2 - x1, ffip2 = x3 - x2, ffim1 = 0., ffim2 = 0.;
        double xmin = x1 - 0.5 * ffip1, xplus = x1 + 0.5 * ffip1;
        double phir, phil, phi1, phi2;
        ppm_limiter(x1, x2, x2, xplus, xmin, ffip1, ffip2, ffim1, ffim2, phir, phil, phi1, phi2);
        pr_fr = ppm_fr(phir, mup, phi1, phi2);
        pr_xplus = xplus;
    }

    for (int k = 1; k <= nz; k++) {
        __syncthreads();
        // ---- stage plane k into shared memory ----
        const double d0 = ldg(G.den0, k - 1);
        for (int q = tid; q < SH * SW; q += TX * TY) {
            int r = q / SW, c = q - r * SW;
            int ii = i0 - H + c, jj = j0 - H + r;
            bool corner = (r < H || r >= TY + H) && (c < H || c >= TX + H);
            double v = 0.;
            if (!corner && ii >= 1 && ii <= nx && jj >= 1 && jj <= ny) v = sval(gidx(G, ii, jj, k));
            sx[q] = v;
        }
        for (int q = tid; q < TY * (TX + 1); q += TX * TY) {
            int r = q / (TX + 1), c = q - r * (TX + 1);
            int ii = i0 + c, jj = min(j0 + r, ny);
            double v = 0.;
            if (ii <= nx) v = mom_val(A, A.mu, gidx(G, ii, jj, k), d0) / d0 - G.u0shift;
            su[q] = v;
        }
        for (int q = tid; q < (TY + 1) * TX; q += TX * TY) {
            int r = q / TX, c = q - r * TX;
            int ii = min(i0 + c, nx), jj = j0 + r;
            double v = 0.;
            if (jj <= ny) v = mom_val(A, A.mv, gidx(G, ii, jj, k), d0) / d0 - G.v0shift;
            sv[q] = v;
        }
        __syncthreads();

        // ---- horizontal fluxes ----
        if (SCHEME == MG_PPM) {
            // cell reconstructions: x cells c = i0-1+q, q in [0, TX+2); y cells likewise
            for (int q = tid; q < TY * (TX + 2); q += TX * TY) {
                int r = q / (TX + 2), c = q - r * (TX + 2);
                int cell = i0 - 1 + c;
                double xv[5];
                for (int m = 0; m < 5; m++) xv[m] = sx[(r + H) * SW + (c - 1 + H) - 2 + m];
                int kind = cell == 3 ? 1 : (cell == 4 ? 2 : (cell == nx - 1 ? 3 : 0));
                double pr = 0., pl = 0., p1 = 0., p2 = 0.;
                if (cell <= nx - 1) ppm_cell_h(kind, xv, pr, pl, p1, p2);
                int o = r * (TX + 2) + c;
                crx[o] = pr; crx[TY * (TX + 2) + o] = pl; crx[2 * TY * (TX + 2) + o] = p1; crx[3 * TY * (TX + 2) + o] = p2;
            }
            for (int q = tid; q < (TY + 2) * TX; q += TX * TY) {
                int r = q / TX, c = q - r * TX;
                int cell = j0 - 1 + r;
                double xv[5];
                for (int m = 0; m < 5; m++) xv[m] = sx[(r - 1 + H - 2 + m) * SW + (c + H)];
                int kind = cell == 3 ? 1 : (cell == 4 ? 2 : (cell == ny - 1 ? 3 : 0));
                double pr = 0., pl = 0., p1 = 0., p2 = 0.;
                if (cell <= ny - 1) ppm_cell_h(kind, xv, pr, pl, p1, p2);
                int o = r * TX + c;
                cry[o] = pr; cry[(TY + 2) * TX + o] = pl; cry[2 * (TY + 2) * TX + o] = p1; cry[3 * (TY + 2) * TX + o] = p2;
            }
            __syncthreads();
        }
        // x faces q = 0..TX: face between cells i0+q-1 and i0+q
        for (int q = tid; q < TY * (TX + 1); q += TX * TY) {
            int r = q / (TX + 1), c = q - r * (TX + 1);
            double uu = su[q];
            double F;
            const double *row = sx + (r + H) * SW + H;   // row[m] = x(i0+m)
            int il = c - 1;                               // left cell offset
            if (SCHEME == MG_WENO) {
                F = weno_face(row[il - 1], row[il], row[il + 1], row[il + 2], uu, true);
            } else if (SCHEME == MG_MUSCL) {
                F = muscl_face_h(G.muscl_lim, G.lim_tol, G.dx, dx1, row[il - 1], row[il], row[il + 1], row[il + 2], uu);
            } else {
                // Fr of cell i0+c-1 (slot c) and Fl of cell i0+c (slot c+1)
                double mu_ = fabs(uu) * dt0 * dx1;
                int o0 = r * (TX + 2) + c, o1 = o0 + 1, S = TY * (TX + 2);
                double fr = ppm_fr(crx[o0], mu_, crx[2 * S + o0], crx[3 * S + o0]);
                double fl = ppm_fl(crx[S + o1], mu_, crx[2 * S + o1], crx[3 * S + o1]);
                F = 0.5 * fr * (uu + fabs(uu)) + 0.5 * fl * (uu - fabs(uu));
            }
            fx[q] = F;
        }
        // y faces q = 0..TY: face between rows j0+q-1 and j0+q
        for (int q = tid; q < (TY + 1) * TX; q += TX * TY) {
            int r = q / TX, c = q - r * TX;
            double vv = sv[q];
            double F;
            const double *col = sx + H * SW + (c + H);    // col[m*SW] = x(j0+m)
            int jl = r - 1;
            if (SCHEME == MG_WENO) {
                F = weno_face(col[(jl - 1) * SW], col[jl * SW], col[(jl + 1) * SW], col[(jl + 2) * SW], vv, true);
            } else if (SCHEME == MG_MUSCL) {
                F = muscl_face_h(G.muscl_lim, G.lim_tol, G.dy, dy1, col[(jl - 1) * SW], col[jl * SW],
                                 col[(jl + 1) * SW], col[(jl + 2) * SW], vv);
            } else {
                double mu_ = fabs(vv) * dt0 * dy1;
                int o0 = r * TX + c, o1 = o0 + TX, S = (TY + 2) * TX;
                double fr = ppm_fr(cry[o0], mu_, cry[2 * S + o0], cry[3 * S + o0]);
                double fl = ppm_fl(cry[S + o1], mu_, cry[2 * S + o1], cry[3 * S + o1]);
                F = 0.5 * fr * (vv + fabs(vv)) + 0.5 * fl * (vv - fabs(vv));
            }
            fy[q] = F;
        }
        __syncthreads();
        const double Tx = (fx[ty * (TX + 1) + tx + 1] - fx[ty * (TX + 1) + tx]) * dx1;
        const double Ty = (fy[(ty + 1) * TX + tx] - fy[ty * TX + tx]) * dy1;

        // ---- vertical flux at face k+1/2 and tendency ----
        const double dzw1 = ldg(G.dz1w, k - 1);
        double Fzn = 0.;
        if (k <= nz - 1) {
            const double ww = zw[1];                      // w_adv(k+1)
            if (SCHEME == MG_WENO) {
                if (k == 1) Fzn = weno_face_bottom(zx[1], zx[2], zx[3], ww);
                else if (k == nz - 1) Fzn = weno_face_top(zx[0], zx[1], zx[2], ww);
                else Fzn = weno_face(zx[0], zx[1], zx[2], zx[3], ww, (k >= 3 && k <= nz - 3));
            } else if (SCHEME == MG_MUSCL) {
                int kind = k == 1 ? 1 : (k == nz - 1 ? 2 : 0);
                double d1m = k >= 2 ? ldg(G.dz1, k - 2) : 0., d10 = ldg(G.dz1, k - 1), d1p = ldg(G.dz1, k);
                double fm = k >= 2 ? ldg(G.fdz0, k - 2) : 0., fp = ldg(G.fdz0, k);
                Fzn = muscl_face_z(kind, G.muscl_lim, G.lim_tol, G.dz, zx[0], zx[1], zx[2], zx[3], d1m, d10, d1p, fm, fp,
                                   dzw1, ww);
            } else {
                // reconstruction of cell k+1 (advq_ppm.f90:345-414)
                const int c = k + 1;
                double xm1 = zx[1], x0 = zx[2], xp1 = zx[3], xp2 = zx[4], xm2 = zx[0];
                double d1c = ldg(G.dz1, c - 1);
                double muc = fabs(zw[1]) * dt0 * d1c;
                double fl;
                if (c == nz) {
                    double ffim1 = x0 - xm1;
                    fl = x0 + 0.5 * ffim1 * (1. - muc);
                } else {
                    double mup = fabs(zw[2]) * dt0 * d1c;
                    double ffip1, ffip2, ffim1, ffim2, xplus;
                    double xmin = pr_xplus;
                    if (c == 2) {
                        ffip1 = xp1 - x0; ffip2 = xp2 - xp1; ffim1 = (x0 - xm1); ffim2 = 0.;
                        xplus = x0 + 0.5 * ffip1;
                    } else if (c == nz - 1) {
                        ffip1 = xp1 - x0; ffim1 = x0 - xm1; ffim2 = xm1 - xm2; ffip2 = ffip1;
                        xplus = x0 + 0.5 * ffip1;
                    } else {
                        ffip1 = (xp1 - x0); ffip2 = (xp2 - xp1); ffim1 = (x0 - xm1); ffim2 = (xm1 - xm2);
                        xplus = ppm_xplus_z(x0, ffip1, ffip2, ffim1, ldg(G.dz1w, c - 2), ldg(G.dz1w, c - 1),
                                            ldg(G.dz1w, c), ldg(G.dz1w, c + 1));
                    }
                    double phir, phil, phi1, phi2;
                    ppm_limiter(x0, xp1, xm1, xplus, xmin, ffip1, ffip2, ffim1, ffim2, phir, phil, phi1, phi2);
                    fl = ppm_fl(phil, muc, phi1, phi2);
                    double frn = ppm_fr(phir, mup, phi1, phi2);
                    Fzn = 0.5 * pr_fr * (ww + fabs(ww)) + 0.5 * fl * (ww - fabs(ww));
                    pr_fr = frn;
                    pr_xplus = xplus;
                    fl = 0.;  // consumed
                }
                if (c == nz) Fzn = 0.5 * pr_fr * (ww + fabs(ww)) + 0.5 * fl * (ww - fabs(ww));
            }
        }
        double Tz;
        if (k == 1) Tz = (Fzn - 0.) * dzw1;
        else if (k == nz) Tz = (0. - Fzo) * dzw1;
        else Tz = (Fzn - Fzo) * dzw1;
        Fzo = Fzn;
        const double T = ((0. - Tx) - Ty) - Tz;

        // ---- epilogue ----
        if (act) {
            const long long idx = gidx(G, i, j, k);
            if (A.mode == 1) {
                double *xs = A.xout[f];
                xs[idx] = ((xs[idx] - Tx) - Ty) - Tz;
            } else {
                double told = A.stage == 1 ? 0. : A.tend[f][idx];
                double tn = T + A.b * told;
                double xo = ldg(A.xold[f], idx);
                double old = weighted ? rep_value(A.rep, xo, ldg(dens_n, idx)) : xo;
                A.xout[f][idx] = old + A.a_dt * tn;
                A.tend[f][idx] = tn;
                if (A.fst[f]) A.fst[f][idx] = T;
            }
        }

        // ---- advance the z window ----
        zx[0] = zx[1]; zx[1] = zx[2]; zx[2] = zx[3]; zx[3] = zx[4];
        zx[4] = (k + 4 <= nz) ? sval(gidx(G, ic, jc, k + 4)) : 0.;
        zw[0] = zw[1]; zw[1] = zw[2];
        zw[2] = (k + 3 <= nz) ? wadv(k + 3) : 0.;
    }
}

}  // namespace

static size_t k1_smem(int scheme)
{
    size_t n = SH * SW + TY * (TX + 1) + (TY + 1) * TX + TY * (TX + 1) + (TY + 1) * TX;
    if (scheme == MG_PPM) n += 4 * TY * (TX + 2) + 4 * (TY + 2) * TX;
    return n * sizeof(double);
}

cudaError_t launch_k1(const DevGrid &g, const K1Args &a, cudaStream_t s)
{
    if (a.nf <= 0 || a.nf > MG_MAXF) return cudaErrorInvalidValue;
    int ntx = (g.maxx + TX - 1) / TX, nty = (g.maxy + TY - 1) / TY;
    dim3 grid(a.nf, ntx * nty), block(TX, TY);
    size_t sm = k1_smem(g.scal_adv);
    cudaError_t e;
    switch (g.scal_adv) {
    case MG_WENO:
        e = cudaFuncSetAttribute(k1_kernel<MG_WENO>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
        k1_kernel<MG_WENO><<<grid, block, sm, s>>>(g, a);
        break;
    case MG_PPM:
        e = cudaFuncSetAttribute(k1_kernel<MG_PPM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
        k1_kernel<MG_PPM><<<grid, block, sm, s>>>(g, a);
        break;
    default:
        e = cudaFuncSetAttribute(k1_kernel<MG_MUSCL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
        k1_kernel<MG_MUSCL><<<grid, block, sm, s>>>(g, a);
        break;
    }
    return cudaGetLastError();
}
