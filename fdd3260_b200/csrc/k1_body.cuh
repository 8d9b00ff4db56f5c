// k1_body.cuh -- body of the K1 kernel (scalar advection + stage update), templated
// on the scheme, the arithmetic form and the stage; instantiated by k_scalar.cu (plain
// FP64, compiled without FMA contraction) and k_scalar_mixed.cu (FP32 scheme logic on
// differences, FP64 fluxes and state).
//
// One CTA (288 threads: 8 cell warps + 1 helper warp) owns a 32 x 8 column tile and
// marches up a segment [kb, ke] of its levels (A.nseg segments per tile, so that small
// grids fill the GPU and the last wave of CTAs is short).  A segment above the surface
// first runs level kb-1 as a prologue that computes only its vertical face kb-1/2, the
// flux the first level of the segment differences (the same arithmetic on the same
// values as the segment below, so the result does not depend on the split).  Per level, the fields are processed in groups of PF (2 for WENO and
// MUSCL, 1 for PPM, whose per-field reconstruction arrays are large): the haloed planes
// of a group arrive by TMA (NPS group slots in flight), their x/y faces are computed as
// independent chains, one barrier publishes them, then each cell thread finishes the
// vertical face and the stage update of every field of the group.
#pragma once
#include <algorithm>
#include "mg_common.cuh"
#include "schemes.cuh"
#include "tma.cuh"

namespace {

constexpr int TX = 32, TY = 8, H = 3;
constexpr int SW = TX + 2 * H, SH = TY + 2 * H;   // haloed plane box 38 x 14
constexpr int NT = TX * (TY + 1);                 // 288 threads: 8 cell warps + 1 helper warp
constexpr int PLANE_BYTES = SW * SH * 8;          // 4256
constexpr int PLANE_SLOT = 4352;                  // 128-byte multiple
constexpr int VW = 34, VH = 9;                    // momentum box (x from i0-1, y from j0)
constexpr int VBOX_BYTES = VW * VH * 8;           // 2448
constexpr int VBOX_SLOT = 2560;
constexpr int NCELL = TX * TY;
constexpr int FXN = TY * (TX + 1), FYN = (TY + 1) * TX;   // x faces, y faces of one field
constexpr int NHALO = SW * SH - TX * TY;          // 276 plane elements outside the cells
constexpr int K1_FC = 6;                          // field count with kernels of its own (density + 5 scalars)

// fields per group, group slots of planes in flight, face buffers: parity-double-buffered
// (a group's faces are written while the cells still read the previous group's) when a
// group is one field, and in stage 2 and unit mode, which have no density plane; single
// in stage 1 of two-field groups, whose density products need a barrier before the faces
// anyway (two face buffers and the density plane would leave one CTA per SM at 6 fields)
__host__ __device__ constexpr int k1_pf(int scheme) { return scheme == MG_PPM ? 1 : 2; }
__host__ __device__ constexpr int k1_nps(int scheme) { return scheme == MG_PPM ? 4 : 2; }
__host__ __device__ constexpr int k1_nfb(int scheme, int stage) { return (k1_pf(scheme) == 1 || stage != 1) ? 2 : 1; }

struct Layout {
    int zs;             // z-ring slots
    size_t planes, vbu, vbv, densp, su, sv, fx, fy, mbar, zring, wring, zf, chain, crx, cry, total;
};

// stage: 1, 2, or 0 (unit mode); only stage 1 keeps the density plane
__host__ __device__ inline Layout make_layout(int scheme, int nf, int stage)
{
    Layout L;
    const int PF = k1_pf(scheme), NPS = k1_nps(scheme), NFB = k1_nfb(scheme, stage);
    L.zs = scheme == MG_PPM ? 5 : 4;   // window x(k-1..k+L), L = 3 (PPM) or 2
    size_t o = 0;
    L.planes = o; o += (size_t)NPS * PF * PLANE_SLOT;
    L.vbu = o; o += VBOX_SLOT;
    L.vbv = o; o += VBOX_SLOT;
    L.densp = o;
    if (stage == 1) o += PLANE_SLOT;
    L.su = o; o += TY * (TX + 1) * 8;
    L.sv = o; o += (TY + 1) * TX * 8;
    L.fx = o; o += (size_t)NFB * PF * FXN * 8;
    L.fy = o; o += (size_t)NFB * PF * FYN * 8;
    o = (o + 127) / 128 * 128;
    L.mbar = o; o += 128;
    L.zring = o; o += (size_t)nf * L.zs * NCELL * 8;
    L.wring = o; o += (size_t)L.zs * NCELL * 8;
    L.zf = o; o += (size_t)nf * NCELL * 8;
    L.chain = o;
    L.crx = o;
    L.cry = o;
    if (scheme == MG_PPM) {
        o += (size_t)2 * nf * NCELL * 8;
        L.crx = o; o += (size_t)NFB * 4 * TY * (TX + 2) * 8;
        L.cry = o; o += (size_t)NFB * 4 * (TY + 2) * TX * 8;
    }
    L.total = o + 128;   // slack for 128-byte alignment of the base
    return L;
}

// the largest layout over the stages and unit mode (the launch checks)
inline size_t k1_smem_max(int scheme, int nf)
{
    return std::max(make_layout(scheme, nf, 0).total, std::max(make_layout(scheme, nf, 1).total, make_layout(scheme, nf, 2).total));
}

// k segments per column tile: the count that minimises (waves of CTAs) x (levels per
// segment + 3, the prologue and the pipeline fill), with segments of at least 8 levels.
// PPM keeps one: its vertical reconstruction chain carries more than one face.
inline int k1_segments(const DevGrid &g, int scheme, size_t smem)
{
    if (scheme == MG_PPM) return 1;
    int dev = 0, nsm = 148;
    if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        nsm = 148;
    const long long per_sm = std::max<long long>(1, std::min<long long>(2, (228LL * 1024) / ((long long)smem + 1024)));
    const long long slots = (long long)nsm * per_sm;
    const long long tiles = (long long)((g.maxx + TX - 1) / TX) * ((g.maxy + TY - 1) / TY);
    int best = 1;
    double bt = 1e300;
    for (int sgm = 1; sgm <= std::max(1, g.nz / 8); sgm++) {
        const double t = (double)((tiles * sgm + slots - 1) / slots) * ((double)g.nz / sgm + 3.);
        if (t < 0.999 * bt) { bt = t; best = sgm; }
    }
    return best;
}

__device__ __forceinline__ double ldg(const double *p, long long i) { return __ldg(p + i); }

// plane element of halo index h in [0, NHALO): rows 0..2 and 11..13, then the halo
// columns of the cell rows
__device__ __forceinline__ int halo_elem(int h)
{
    if (h < 2 * H * SW) {
        const int r = h / SW, c = h - r * SW;
        return (r < H ? r : r + TY) * SW + c;
    }
    const int h2 = h - 2 * H * SW, r = h2 / (2 * H), cc = h2 - r * (2 * H);
    return (r + H) * SW + (cc < H ? cc : cc + TX);
}

// STAGE 1, 2: Heun stage update of density + density-weighted scalars (field 0 is the
// density); STAGE 0: unit mode (advection_ac of one field, xout := ((xout-Tx)-Ty)-Tz)
// SGS: the stage adds stored SGS tendencies (A.sgs), loaded one group ahead; a variant of
// its own so that the kernels without SGS keep their register budget
// FC: the field count when it is known at compile time (0: A.nf at run time); with it the
// group loop unrolls and every shared-memory offset of the z-window is a constant
// bid: the block's index in the domain's own grid of tiles x segments
template <int SCHEME, bool MIXED, int STAGE, bool SGS, int FC>
__device__ __forceinline__ void k1_run(const DevGrid &G, const K1Args &A, const K1Maps &M, const int bid)
{
    constexpr int PF = k1_pf(SCHEME), NPS = k1_nps(SCHEME), NFB = k1_nfb(SCHEME, STAGE);
    constexpr bool CONV1 = STAGE == 1;   // stage-1 inputs are natural: psi = s * rho
    extern __shared__ unsigned char smraw[];
    // 128-byte alignment by an offset from the shared array itself, so that every pointer
    // derived from it stays a shared-memory pointer
    unsigned char *sm = smraw + ((128u - (smem_u32(smraw) & 127u)) & 127u);
    const int F = FC > 0 ? FC : A.nf;
    const Layout Ly = make_layout(SCHEME, F, STAGE);
    constexpr int ZS = SCHEME == MG_PPM ? 5 : 4;   // z-ring slots
    constexpr int L = SCHEME == MG_PPM ? 3 : 2;    // window x(k-1 .. k+L)
    double *planes = (double *)(sm + Ly.planes);
    double *vbu = (double *)(sm + Ly.vbu), *vbv = (double *)(sm + Ly.vbv);
    double *densp = (double *)(sm + Ly.densp);
    double *su = (double *)(sm + Ly.su), *sv = (double *)(sm + Ly.sv);
    double *fx = (double *)(sm + Ly.fx), *fy = (double *)(sm + Ly.fy);
    uint64_t *mb = (uint64_t *)(sm + Ly.mbar);    // [0, NPS) plane groups, [NPS] momentum boxes
    double *zring = (double *)(sm + Ly.zring), *wring = (double *)(sm + Ly.wring);
    double *zf = (double *)(sm + Ly.zf);
    double *chain = (double *)(sm + Ly.chain);   // PPM: [0][f] Fr of the cell below, [1][f] its xplus
    double *crx = (double *)(sm + Ly.crx), *cry = (double *)(sm + Ly.cry);

    const int ntx = (G.maxx + TX - 1) / TX, nty = (G.maxy + TY - 1) / TY;
    const int tile = bid % (ntx * nty), seg = bid / (ntx * nty);
    const int ti = tile % ntx, tj = tile / ntx;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const int i0 = 4 + ti * TX, j0 = 4 + tj * TY;
    const int nx = G.nx, ny = G.ny, nz = G.nz;
    const bool cellt = ty < TY;
    const int i = i0 + tx, j = j0 + ty;
    const bool act = cellt && (i <= nx - 2) && (j <= ny - 2);
    const int ic = min(i, nx - 2), jc = min(j, ny - 2);
    const int cid = ty * TX + tx;   // cell slot (valid for cell threads)
    const int own_e = (ty + H) * SW + tx + H;   // own cell in a plane (cell threads)
    const double dx1 = 1. / G.dx, dy1 = 1. / G.dy, dt0 = G.dt0;
    const bool conv1 = CONV1;
    const int NG = (F + PF - 1) / PF;      // field groups per level
    // this CTA's levels [kb, ke], the prologue level kp (= kb - 1 above the surface), and
    // its plane groups [qb, qe); slots and barrier phases count from qb
    const int kb = 1 + (int)(((long long)seg * nz) / A.nseg), ke = (int)(((long long)(seg + 1) * nz) / A.nseg);
    const int kp = kb > 1 ? kb - 1 : 1;
    const int qb = (kb - 1) * NG, qe = ke * NG;
    const int zmax = min(nz, ke + L);      // last level the z-window needs
    const int MB_VEL = NPS;

    if (tid == 0) {
        for (int b = 0; b <= NPS; b++) mbar_init(&mb[b], 1);
        fence_mbar_init();
    }
    __syncthreads();

    auto issue_group = [&](int qg) {   // group qg = (k-1)*NG + g: planes of fields g*PF ..
        const int k = qg / NG + 1, g = qg - (k - 1) * NG;
        const int slot = (qg - qb) % NPS;
        const int nfg = min(PF, F - g * PF);
        fence_proxy_async_shared();
        mbar_arrive_expect_tx(&mb[slot], nfg * PLANE_BYTES);
        for (int u = 0; u < nfg; u++)
            tma_load_3d(planes + (size_t)(slot * PF + u) * (PLANE_SLOT / 8), &M.x[g * PF + u], i0 - 4, j0 - 4, k - 1,
                        &mb[slot]);
    };
    auto issue_vel = [&](int k) {
        fence_proxy_async_shared();
        mbar_arrive_expect_tx(&mb[MB_VEL], 2 * VBOX_BYTES);
        tma_load_3d(vbu, &M.mu, i0 - 2, j0 - 1, k - 1, &mb[MB_VEL]);
        tma_load_3d(vbv, &M.mv, i0 - 2, j0 - 1, k - 1, &mb[MB_VEL]);
    };
    auto issue_z = [&](int l) {   // own-column values of every field and w at level l
        if (cellt && l <= zmax) {
            const long long idx = gidx(G, ic, jc, l);
            const int s = l % ZS;
            for (int f = 0; f < F; f++) cp_async_8(&zring[(f * ZS + s) * NCELL + cid], A.xin[f] + idx);
            cp_async_8(&wring[s * NCELL + cid], A.mw + idx);
        }
        cp_async_commit();
    };

    if (tid == 0) {
        for (int q0 = qb; q0 < qb + NPS - 1 && q0 < qe; q0++) issue_group(q0);
        issue_vel(kb);
    }
    for (int l = max(1, kp - 1); l <= kp + L; l++) issue_z(l);

    double dn_old = 0., dn_new = 0., rdn_new = 0.;   // density of the own cell: level n and new (stage 2)
    int k_cur = kp;
    // per-field vertical state
    if (cellt)
        for (int f = 0; f < F; f++) zf[f * NCELL + cid] = 0.;

    int zsl[L + 2];   // z-ring slot of level k-1+m, refreshed per level
    // stencil value of a field at level l = k-1+m of the own column (stage 1: the other
    // fields' entries are multiplied by the density entry of the same level once, when
    // the level arrives)
#define ZVAL(f, m) (zring[((f) * ZS + zsl[(m)]) * NCELL + cid])
    auto wval = [&](int m) -> double {   // w_adv at level k-1+m of the own column
        const double a0 = ldg(G.avden0, k_cur - 2 + m);
        double x = wring[((k_cur - 1 + m) % ZS) * NCELL + cid];
        if (conv1) x = x * a0;
        return x / a0;
    };

    double wz2 = 0., wz3 = 0.;   // w_adv of the own column at levels k+1 and k+2
    // stage 2: level-n value and tendency of the group's fields, loaded one group ahead
    const long long idx0 = gidx(G, ic, jc, 1);
    const long long idxb = idx0 + (long long)(kb - 1) * G.ps;
    double nx_xold[PF], nx_tend[PF];
    double nx_sgs[PF];   // SGS tendencies (both stages), loaded one group ahead as well
#pragma unroll
    for (int u = 0; u < PF; u++) {
        nx_xold[u] = 0.;
        nx_tend[u] = 0.;
        nx_sgs[u] = 0.;
        if (STAGE == 2 && act && u < F) {
            nx_xold[u] = ldg_stream(A.xold[u] + idxb);
            nx_tend[u] = ldg_stream(A.tend[u] + idxb);
        }
        if (SGS && act && u < F && A.sgs[u]) nx_sgs[u] = ldg_stream(A.sgs[u] + idxb);
    }
    // mixed form: per-level coefficients loaded one level ahead of their use (rho0(k), the
    // cell's 1/dz and avden0 at level k+1, the vertical face's w), off the critical path
    // of the level's first faces (the mixed step 1863 -> 1902 Mcell-updates/s); the FP64
    // form loads them where they are used, its registers having no room for three more
    // (with their reciprocals, the context's 1/rho0 profiles, for the two divisions per
    // level that the mixed form turns into products)
    double nd0 = 0., ndzw = 0., naw = 1., nrd0 = 0., nraw = 1.;
    if constexpr (MIXED) {
        nd0 = ldg(G.den0, kp - 1);
        nrd0 = ldg(G.rden0, kp - 1);
        ndzw = ldg(G.dz1w, kp - 1);
        naw = kp <= nz - 1 ? ldg(G.avden0, kp) : 1.;
        nraw = kp <= nz - 1 ? ldg(G.ravden0, kp) : 1.;
    }
    for (int k = kp; k <= ke; k++) {
        const bool pro = k < kb;   // prologue level: its vertical face only
        k_cur = k;
        const double lv_d0 = nd0, lv_dzw = ndzw, lv_aw = naw, lv_rd0 = nrd0, lv_raw = nraw;
        if (MIXED && k + 1 <= ke) {
            nd0 = ldg(G.den0, k);
            nrd0 = ldg(G.rden0, k);
            ndzw = ldg(G.dz1w, k);
            naw = k + 1 <= nz - 1 ? ldg(G.avden0, k + 1) : 1.;
            nraw = k + 1 <= nz - 1 ? ldg(G.ravden0, k + 1) : 1.;
        }
#pragma unroll
        for (int m = 0; m < L + 2; m++) zsl[m] = (k - 1 + m) % ZS;
        const double d0 = MIXED ? lv_d0 : ldg(G.den0, k - 1);
        const double rd0 = MIXED ? lv_rd0 : 0.;   // the mixed form multiplies by 1/rho0
        // momentum boxes of level k -> face velocities.  Each thread converts the two
        // velocities of its own faces (su[tid]: x face, sv[tid]: y face), so the faces need
        // no barrier after this; the boxes are refilled for level k+1 after this level's
        // first face barrier, which every thread passes after its conversion.
        if (!pro) {
            mbar_wait_bounded(&mb[MB_VEL], (uint32_t)((k - kb) & 1), A.err);
            if (tid < TY * (TX + 1)) {
                const int r = tid / (TX + 1), c = tid - r * (TX + 1);
                double m = vbu[r * VW + c + 1];
                if (conv1) m = m * d0;
                su[tid] = (MIXED ? m * rd0 : m / d0) - G.u0shift;
            }
            {
                const int r = tid / TX, c = tid - r * TX;
                double m = vbv[r * VW + c + 1];
                if (conv1) m = m * d0;
                sv[tid] = (MIXED ? m * rd0 : m / d0) - G.v0shift;
            }
        }
#pragma unroll 1
        for (int g = 0; g < NG; g++) {
            const int qg = (k - 1) * NG + g, qr = qg - qb, gb = g * PF;
            // this group's stage-2 operands, then the next group's loads (they complete
            // while this group's faces are computed)
            double cur_xold[PF], cur_tend[PF], cur_sgs[PF];
#pragma unroll
            for (int u = 0; u < PF; u++) {
                cur_xold[u] = nx_xold[u];
                cur_tend[u] = nx_tend[u];
                cur_sgs[u] = nx_sgs[u];
            }
            double *fxb = fx + (NFB == 2 ? (qr & 1) : 0) * PF * FXN;
            double *fyb = fy + (NFB == 2 ? (qr & 1) : 0) * PF * FYN;
            double plane_xo[PF];
            if (!pro) {
            if ((STAGE == 2 || SGS) && act && qg + 1 < qe) {
                const int gn = g + 1 < NG ? g + 1 : 0, kn = g + 1 < NG ? k : k + 1;
                const long long idn = idx0 + (long long)(kn - 1) * G.ps;
#pragma unroll
                for (int u = 0; u < PF; u++)
                    if (gn * PF + u < F) {
                        if (STAGE == 2) {
                            nx_xold[u] = ldg_stream(A.xold[gn * PF + u] + idn);
                            nx_tend[u] = ldg_stream(A.tend[gn * PF + u] + idn);
                        }
                        if (SGS) nx_sgs[u] = A.sgs[gn * PF + u] ? ldg_stream(A.sgs[gn * PF + u] + idn) : 0.;
                    }
            }
            // slot (qg+NPS-1)%NPS last held group qg-1, whose faces all threads finished
            // before the face barrier of group qg-1
            if (tid == 0 && qg + NPS - 1 < qe) issue_group(qg + NPS - 1);
            mbar_wait_bounded(&mb[qr % NPS], (uint32_t)((qr / NPS) & 1), A.err);
            double *plq = planes + (size_t)(qr % NPS) * PF * (PLANE_SLOT / 8);
            // level-n values of the own cell (stage 1: they are the planes' own elements,
            // read before the density products below)
#pragma unroll
            for (int u = 0; u < PF; u++) plane_xo[u] = (cellt && gb + u < F) ? plq[u * (PLANE_SLOT / 8) + own_e] : 0.;
            if constexpr (CONV1) {
                // psi = s * rho in place, once per element: each cell thread scales its own
                // element, the halo elements are shared out.  Group 0 holds the density
                // (field 0), which is kept in densp for the later groups of the level.
#pragma unroll
                for (int u = 0; u < PF; u++) {
                    const int f = gb + u;
                    if (f >= F) continue;
                    double *plw = plq + u * (PLANE_SLOT / 8);
                    if (f == 0) {
                        for (int e = tid; e < SW * SH; e += NT) densp[e] = plw[e];
                    } else {
                        const double *dsrc = g == 0 ? plq : densp;   // group 0: the density plane itself
                        if (cellt) plw[own_e] = plane_xo[u] * dsrc[own_e];
                        for (int h = tid; h < NHALO; h += NT) {
                            const int e = halo_elem(h);
                            plw[e] = plw[e] * dsrc[e];
                        }
                    }
                }
            }
            if ((CONV1 && (PF == 2 || g > 0)) || NFB == 1) __syncthreads();
            double *crxq = crx + (NFB == 2 ? (qr & 1) : 0) * 4 * TY * (TX + 2);
            double *cryq = cry + (NFB == 2 ? (qr & 1) : 0) * 4 * (TY + 2) * TX;
            if constexpr (SCHEME == MG_PPM) {
                const double *pl = plq;
                auto V = [&](int e) -> double { return pl[e]; };
                for (int qq = tid; qq < TY * (TX + 2) + (TY + 2) * TX; qq += NT) {
                    double xv[5], pr = 0., pL = 0., p1 = 0., p2 = 0.;
                    if (qq < TY * (TX + 2)) {
                        int r = qq / (TX + 2), c = qq - r * (TX + 2);
                        int cell = i0 - 1 + c;
                        for (int m = 0; m < 5; m++) xv[m] = V((r + H) * SW + c + m);
                        int kind = cell == 3 ? 1 : (cell == 4 ? 2 : (cell == nx - 1 ? 3 : 0));
                        if (cell <= nx - 1) {
                            if constexpr (MIXED) {
                                float a_, b_, c_, d_;
                                ppm_cell_h_mixed(kind, xv, a_, b_, c_, d_);
                                pr = a_; pL = b_; p1 = c_; p2 = d_;
                            } else {
                                ppm_cell_h(kind, xv, pr, pL, p1, p2);
                            }
                        }
                        const int o = r * (TX + 2) + c, S = TY * (TX + 2);
                        crxq[o] = pr; crxq[S + o] = pL; crxq[2 * S + o] = p1; crxq[3 * S + o] = p2;
                    } else {
                        int q2 = qq - TY * (TX + 2);
                        int r = q2 / TX, c = q2 - r * TX;
                        int cell = j0 - 1 + r;
                        for (int m = 0; m < 5; m++) xv[m] = V((r + m) * SW + c + H);
                        int kind = cell == 3 ? 1 : (cell == 4 ? 2 : (cell == ny - 1 ? 3 : 0));
                        if (cell <= ny - 1) {
                            if constexpr (MIXED) {
                                float a_, b_, c_, d_;
                                ppm_cell_h_mixed(kind, xv, a_, b_, c_, d_);
                                pr = a_; pL = b_; p1 = c_; p2 = d_;
                            } else {
                                ppm_cell_h(kind, xv, pr, pL, p1, p2);
                            }
                        }
                        const int o = r * TX + c, S = (TY + 2) * TX;
                        cryq[o] = pr; cryq[S + o] = pL; cryq[2 * S + o] = p1; cryq[3 * S + o] = p2;
                    }
                }
                __syncthreads();
            }
#pragma unroll
            for (int u = 0; u < PF; u++) {
                if (PF > 1 && gb + u >= F) continue;
                const double *pl = plq + u * (PLANE_SLOT / 8);
                auto V = [&](int e) -> double { return pl[e]; };
                double *fxq = fxb + u * FXN, *fyq = fyb + u * FYN;
                    // x face (threads 0..263: (TX+1)*TY faces) and y face (all 288 threads:
                    // TX*(TY+1) faces), written as two independent chains for instruction-level
                    // parallelism
                    {
                        const bool hasx = tid < TY * (TX + 1);
                        const int rx = hasx ? tid / (TX + 1) : 0, cx = hasx ? tid - rx * (TX + 1) : 0;
                        const int ry = tid / TX, cy = tid - ry * TX;
                        const double uu = hasx ? su[tid] : 0., vv = sv[tid];   // the thread's own entries
                        const int bx = (rx + H) * SW + H + cx - 1;   // x(i0 + cx - 1) in row rx
                        const int by = (ry - 1 + H) * SW + H + cy;   // x(j0 + ry - 1) in column cy
                        double Fx, Fy;
                        if (SCHEME == MG_WENO) {
                            if constexpr (MIXED) {
                                Fx = weno_face_up_mixed(V(bx - 1), V(bx), V(bx + 1), V(bx + 2), uu, true);
                                Fy = weno_face_up_mixed(V(by - SW), V(by), V(by + SW), V(by + 2 * SW), vv, true);
                            } else {
                                Fx = weno_face_up(V(bx - 1), V(bx), V(bx + 1), V(bx + 2), uu, true);
                                Fy = weno_face_up(V(by - SW), V(by), V(by + SW), V(by + 2 * SW), vv, true);
                            }
                        } else if (SCHEME == MG_MUSCL) {
                            if constexpr (MIXED) {
                                Fx = muscl_face_h_mixed(G.muscl_lim, (float)G.lim_tol, (float)G.dx, (float)dx1, V(bx - 1), V(bx),
                                                        V(bx + 1), V(bx + 2), uu);
                                Fy = muscl_face_h_mixed(G.muscl_lim, (float)G.lim_tol, (float)G.dy, (float)dy1, V(by - SW), V(by),
                                                        V(by + SW), V(by + 2 * SW), vv);
                            } else {
                                Fx = muscl_face_h(G.muscl_lim, G.lim_tol, G.dx, dx1, V(bx - 1), V(bx), V(bx + 1), V(bx + 2), uu);
                                Fy = muscl_face_h(G.muscl_lim, G.lim_tol, G.dy, dy1, V(by - SW), V(by), V(by + SW), V(by + 2 * SW), vv);
                            }
                        } else if (SCHEME == MG_LW) {
                            if constexpr (MIXED) {
                                Fx = lw_face_h_mixed((float)G.lim_tol, (float)dt0, (float)dx1, V(bx - 1), V(bx), V(bx + 1), V(bx + 2), uu);
                                Fy = lw_face_h_mixed((float)G.lim_tol, (float)dt0, (float)dy1, V(by - SW), V(by), V(by + SW),
                                                     V(by + 2 * SW), vv);
                            } else {
                                Fx = lw_face_h(G.lim_tol, dt0, dx1, V(bx - 1), V(bx), V(bx + 1), V(bx + 2), uu);
                                Fy = lw_face_h(G.lim_tol, dt0, dy1, V(by - SW), V(by), V(by + SW), V(by + 2 * SW), vv);
                            }
                        } else if (SCHEME == MG_QUICK) {
                            if constexpr (MIXED) {
                                Fx = quick_face_h_mixed((float)G.lim_tol, V(bx - 1), V(bx), V(bx + 1), V(bx + 2), uu);
                                Fy = quick_face_h_mixed((float)G.lim_tol, V(by - SW), V(by), V(by + SW), V(by + 2 * SW), vv);
                            } else {
                                Fx = quick_face_h(G.lim_tol, V(bx - 1), V(bx), V(bx + 1), V(bx + 2), uu);
                                Fy = quick_face_h(G.lim_tol, V(by - SW), V(by), V(by + SW), V(by + 2 * SW), vv);
                            }
                        } else if constexpr (MIXED) {
                            // relative reconstructions: cell base values from the plane
                            const double mux = fabs(uu) * dt0 * dx1;
                            const int o0 = rx * (TX + 2) + cx, o1 = o0 + 1, S = TY * (TX + 2);
                            const float frx = ppm_fr((float)crxq[o0], (float)mux, (float)crxq[2 * S + o0], (float)crxq[3 * S + o0]);
                            const float flx = ppm_fl((float)crxq[S + o1], (float)mux, (float)crxq[2 * S + o1], (float)crxq[3 * S + o1]);
                            Fx = uu > 0. ? uu * (V(bx) + (double)frx) : (uu < 0. ? uu * (V(bx + 1) + (double)flx) : 0.);
                            const double muy = fabs(vv) * dt0 * dy1;
                            const int p0 = ry * TX + cy, p1 = p0 + TX, Sy = (TY + 2) * TX;
                            const float fry = ppm_fr((float)cryq[p0], (float)muy, (float)cryq[2 * Sy + p0], (float)cryq[3 * Sy + p0]);
                            const float fly = ppm_fl((float)cryq[Sy + p1], (float)muy, (float)cryq[2 * Sy + p1], (float)cryq[3 * Sy + p1]);
                            Fy = vv > 0. ? vv * (V(by) + (double)fry) : (vv < 0. ? vv * (V(by + SW) + (double)fly) : 0.);
                        } else {
                            const double mux = fabs(uu) * dt0 * dx1;
                            const int o0 = rx * (TX + 2) + cx, o1 = o0 + 1, S = TY * (TX + 2);
                            const double frx = ppm_fr(crxq[o0], mux, crxq[2 * S + o0], crxq[3 * S + o0]);
                            const double flx = ppm_fl(crxq[S + o1], mux, crxq[2 * S + o1], crxq[3 * S + o1]);
                            Fx = 0.5 * frx * (uu + fabs(uu)) + 0.5 * flx * (uu - fabs(uu));
                            const double muy = fabs(vv) * dt0 * dy1;
                            const int p0 = ry * TX + cy, p1 = p0 + TX, Sy = (TY + 2) * TX;
                            const double fry = ppm_fr(cryq[p0], muy, cryq[2 * Sy + p0], cryq[3 * Sy + p0]);
                            const double fly = ppm_fl(cryq[Sy + p1], muy, cryq[2 * Sy + p1], cryq[3 * Sy + p1]);
                            Fy = 0.5 * fry * (vv + fabs(vv)) + 0.5 * fly * (vv - fabs(vv));
                        }
                        if (hasx) fxq[tid] = Fx;
                        fyq[tid] = Fy;
                    }
            }
            __syncthreads();   // faces of group qg complete
            // every thread has read the momentum boxes of level k
            if (g == 0 && tid == 0 && k + 1 <= ke) issue_vel(k + 1);
            }
            if (!cellt) continue;

            // ---- vertical faces k+1/2 of the own column ----
            if (g == 0) {
                cp_async_wait_all();
                if (conv1) {
                    // newly arrived levels: the whole window at the first level (without level
                    // 0 at the surface), else k+L
                    const int m_lo = k == kp ? (k == 1 ? 1 : 0) : L + 1;
                    for (int m = m_lo; m <= L + 1; m++) {
                        if (k - 1 + m > nz) break;
                        const int sl = (k - 1 + m) % ZS;
                        const double dn = zring[sl * NCELL + cid];
                        for (int gg = 1; gg < F; gg++) zring[(gg * ZS + sl) * NCELL + cid] *= dn;
                    }
                }
                if (k <= nz - 1) {   // wval(2)
                    const double a0 = MIXED ? lv_aw : ldg(G.avden0, k);
                    double x = wring[((k + 1) % ZS) * NCELL + cid];
                    if (conv1) x = x * a0;
                    wz2 = MIXED ? x * lv_raw : x / a0;
                } else {
                    wz2 = 0.;
                }
                if (SCHEME == MG_PPM) wz3 = k + 2 <= nz ? wval(3) : 0.;
            }
#pragma unroll
            for (int u = 0; u < PF; u++) {
                const int f = gb + u;
                if (PF > 1 && f >= F) continue;
                const double *fxq = fxb + u * FXN, *fyq = fyb + u * FYN;
                const double Tx = pro ? 0. : (fxq[ty * (TX + 1) + tx + 1] - fxq[ty * (TX + 1) + tx]) * dx1;
                const double Ty = pro ? 0. : (fyq[(ty + 1) * TX + tx] - fyq[ty * TX + tx]) * dy1;
                    const double dzw1 = MIXED ? lv_dzw : ldg(G.dz1w, k - 1);
                    double Fzn = 0.;
                    double *zfo = &zf[f * NCELL + cid];
                    if (k <= nz - 1) {
                        const double ww = wz2;
                        if (SCHEME == MG_WENO) {
                            if constexpr (MIXED) {
                                if (k == 1) Fzn = weno_face_bottom_mixed(ZVAL(f, 1), ZVAL(f, 2), ZVAL(f, 3), ww);
                                else if (k == nz - 1) Fzn = weno_face_top_mixed(ZVAL(f, 0), ZVAL(f, 1), ZVAL(f, 2), ww);
                                else Fzn = weno_face_up_mixed(ZVAL(f, 0), ZVAL(f, 1), ZVAL(f, 2), ZVAL(f, 3), ww, (k >= 3 && k <= nz - 3));
                            } else {
                                if (k == 1) Fzn = weno_face_bottom(ZVAL(f, 1), ZVAL(f, 2), ZVAL(f, 3), ww);
                                else if (k == nz - 1) Fzn = weno_face_top(ZVAL(f, 0), ZVAL(f, 1), ZVAL(f, 2), ww);
                                else Fzn = weno_face_up(ZVAL(f, 0), ZVAL(f, 1), ZVAL(f, 2), ZVAL(f, 3), ww, (k >= 3 && k <= nz - 3));
                            }
                        } else if (SCHEME == MG_MUSCL) {
                            const int kind = k == 1 ? 1 : (k == nz - 1 ? 2 : 0);
                            const double d1m = k >= 2 ? ldg(G.dz1, k - 2) : 0., d10 = ldg(G.dz1, k - 1), d1p = ldg(G.dz1, k);
                            const double fm = k >= 2 ? ldg(G.fdz0, k - 2) : 0., fp = ldg(G.fdz0, k);
                            const double xm1 = k >= 2 ? ZVAL(f, 0) : 0.;
                            const double xp2 = k + 2 <= nz ? ZVAL(f, 3) : 0.;
                            if constexpr (MIXED)
                                Fzn = muscl_face_z_mixed(kind, G.muscl_lim, (float)G.lim_tol, (float)G.dz, xm1, ZVAL(f, 1), ZVAL(f, 2), xp2,
                                                         (float)d1m, (float)d10, (float)d1p, (float)fm, (float)fp, (float)dzw1, ww);
                            else
                                Fzn = muscl_face_z(kind, G.muscl_lim, G.lim_tol, G.dz, xm1, ZVAL(f, 1), ZVAL(f, 2), xp2, d1m, d10,
                                                   d1p, fm, fp, dzw1, ww);
                        } else if (SCHEME == MG_LW || SCHEME == MG_QUICK) {
                            const int kind = k == 1 ? 1 : (k == nz - 1 ? 2 : 0);
                            const double d1m = k >= 2 ? ldg(G.dz1, k - 2) : 0., d10 = ldg(G.dz1, k - 1), d1p = ldg(G.dz1, k);
                            const double xm1 = k >= 2 ? ZVAL(f, 0) : 0.;
                            const double xp2 = k + 2 <= nz ? ZVAL(f, 3) : 0.;
                            if constexpr (MIXED) {
                                if constexpr (SCHEME == MG_LW)
                                    Fzn = lw_face_z_mixed(kind, (float)G.lim_tol, (float)G.dz, (float)dt0, xm1, ZVAL(f, 1), ZVAL(f, 2), xp2,
                                                          (float)d1m, (float)d10, (float)d1p, (float)dzw1, ww);
                                else
                                    Fzn = quick_face_z_mixed(kind, (float)G.lim_tol, (float)G.dz, xm1, ZVAL(f, 1), ZVAL(f, 2), xp2,
                                                             (float)d1m, (float)d10, (float)d1p, (float)dzw1, ww);
                            } else {
                                if constexpr (SCHEME == MG_LW)
                                    Fzn = lw_face_z(kind, G.lim_tol, G.dz, dt0, xm1, ZVAL(f, 1), ZVAL(f, 2), xp2, d1m, d10, d1p, dzw1, ww);
                                else
                                    Fzn = quick_face_z(kind, G.lim_tol, G.dz, xm1, ZVAL(f, 1), ZVAL(f, 2), xp2, d1m, d10, d1p, dzw1, ww);
                            }
                        } else if constexpr (MIXED) {
                            // chain values relative: prfr = Fr(k) - x(k), prxp = xplus(k) - x(k)
                            double *prfr = &chain[f * NCELL + cid], *prxp = &chain[(F + f) * NCELL + cid];
                            if (k == 1) {
                                const double x1 = ZVAL(f, 1);
                                const float b1 = (float)(ZVAL(f, 2) - x1), b2 = (float)(ZVAL(f, 3) - x1);
                                const float mup = (float)(fabs(wz2) * dt0 * ldg(G.dz1, 0));
                                const float ffip1 = b1, ffip2 = b2 - b1;
                                float dr, dl, phi1, phi2;
                                ppm_limiter_rel((float)x1, b1, b1, 0.5f * ffip1, -0.5f * ffip1, ffip1, ffip2, 0.f, 0.f, dr, dl, phi1, phi2);
                                *prfr = ppm_fr(dr, mup, phi1, phi2);
                                *prxp = 0.5f * ffip1;
                            }
                            const int c = k + 1;
                            const double x0 = ZVAL(f, 2), xkm = ZVAL(f, 1);
                            const float m1 = (float)(xkm - x0);
                            const float m2 = k >= 2 ? (float)(ZVAL(f, 0) - x0) : 0.f;
                            const float p1 = c + 1 <= nz ? (float)(ZVAL(f, 3) - x0) : 0.f;
                            const float p2 = c + 2 <= nz ? (float)(ZVAL(f, 4) - x0) : 0.f;
                            const double d1c = ldg(G.dz1, c - 1);
                            const float muc = (float)(fabs(ww) * dt0 * d1c);
                            float dfl;
                            if (c == nz) {
                                dfl = 0.5f * (-m1) * (1.f - muc);
                            } else {
                                const float mup = (float)(fabs(wz3) * dt0 * d1c);
                                float ffip1, ffip2, ffim1, ffim2, dplus;
                                const float dmin = (float)(*prxp) + m1;   // xplus(k) - x(k+1)
                                if (c == 2) {
                                    ffip1 = p1; ffip2 = p2 - p1; ffim1 = -m1; ffim2 = 0.f;
                                    dplus = 0.5f * ffip1;
                                } else if (c == nz - 1) {
                                    ffip1 = p1; ffim1 = -m1; ffim2 = m1 - m2; ffip2 = ffip1;
                                    dplus = 0.5f * ffip1;
                                } else {
                                    ffip1 = p1; ffip2 = p2 - p1; ffim1 = -m1; ffim2 = m1 - m2;
                                    dplus = ppm_xplus_z(0.f, ffip1, ffip2, ffim1, (float)ldg(G.dz1w, c - 2), (float)ldg(G.dz1w, c - 1),
                                                        (float)ldg(G.dz1w, c), (float)ldg(G.dz1w, c + 1));
                                }
                                float dr, dl, phi1, phi2;
                                ppm_limiter_rel((float)x0, p1, m1, dplus, dmin, ffip1, ffip2, ffim1, ffim2, dr, dl, phi1, phi2);
                                dfl = ppm_fl(dl, muc, phi1, phi2);
                                const double fzn_up = ww > 0. ? ww * (xkm + *prfr) : (ww < 0. ? ww * (x0 + (double)dfl) : 0.);
                                *prfr = ppm_fr(dr, mup, phi1, phi2);
                                *prxp = dplus;
                                Fzn = fzn_up;
                            }
                            if (c == nz) Fzn = ww > 0. ? ww * (xkm + *prfr) : (ww < 0. ? ww * (x0 + (double)dfl) : 0.);
                        } else {
                            double *prfr = &chain[f * NCELL + cid], *prxp = &chain[(F + f) * NCELL + cid];
                            if (k == 1) {
                                // cell 1 (advq_ppm.f90:328-343): bottom special, bc51 = 0
                                const double x1 = ZVAL(f, 1), x2 = ZVAL(f, 2), x3 = ZVAL(f, 3);
                                const double mup = fabs(wz2) * dt0 * ldg(G.dz1, 0);   // w(2) at k = 1
                                const double ffip1 = x2 - x1, ffip2 = x3 - x2;
                                const double xmin = x1 - 0.5 * ffip1, xplus = x1 + 0.5 * ffip1;
                                double phir, phil, phi1, phi2;
                                ppm_limiter(x1, x2, x2, xplus, xmin, ffip1, ffip2, 0., 0., phir, phil, phi1, phi2);
                                *prfr = ppm_fr(phir, mup, phi1, phi2);
                                *prxp = xplus;
                            }
                            // reconstruction of cell c = k+1 (:345-414)
                            const int c = k + 1;
                            const double xm2 = k >= 2 ? ZVAL(f, 0) : 0., xm1 = ZVAL(f, 1), x0 = ZVAL(f, 2);
                            const double xp1 = c + 1 <= nz ? ZVAL(f, 3) : 0., xp2 = c + 2 <= nz ? ZVAL(f, 4) : 0.;
                            const double d1c = ldg(G.dz1, c - 1);
                            const double muc = fabs(ww) * dt0 * d1c;
                            if (c == nz) {
                                const double fl = x0 + 0.5 * (x0 - xm1) * (1. - muc);
                                Fzn = 0.5 * (*prfr) * (ww + fabs(ww)) + 0.5 * fl * (ww - fabs(ww));
                            } else {
                                const double mup = fabs(wz3) * dt0 * d1c;
                                double ffip1, ffip2, ffim1, ffim2, xplus;
                                const double xmin = *prxp;
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
                                const double fl = ppm_fl(phil, muc, phi1, phi2);
                                Fzn = 0.5 * (*prfr) * (ww + fabs(ww)) + 0.5 * fl * (ww - fabs(ww));
                                *prfr = ppm_fr(phir, mup, phi1, phi2);
                                *prxp = xplus;
                            }
                        }
                    }
                    double Tz;
                    if (k == 1) Tz = (Fzn - 0.) * dzw1;
                    else if (k == nz) Tz = (0. - *zfo) * dzw1;
                    else Tz = (Fzn - *zfo) * dzw1;
                    *zfo = Fzn;

                // ---- epilogue ----
                if (act && !pro) {
                    const long long idx = idx0 + (long long)(k - 1) * G.ps;
                    if constexpr (STAGE == 0) {
                        double *xs = A.xout[f];
                        xs[idx] = ((xs[idx] - Tx) - Ty) - Tz;
                    } else {
                        double T;
                        if constexpr (SGS) {
                            const bool has = A.sgs[f] != nullptr, spost = (A.sgs_post >> f) & 1u;
                            const double sgv = cur_sgs[u];
                            T = (((has && !spost ? 0. + sgv : 0.) - Tx) - Ty) - Tz;
                            if (has && spost) T = T + sgv;
                        } else {
                            T = ((0. - Tx) - Ty) - Tz;
                        }
                        const double told = STAGE == 1 ? 0. : cur_tend[u];
                        const double tn = T + A.b * told;
                        const bool weighted = f > 0;
                        // level n (natural); stage 2 overwrites it in place
                        const double xo = STAGE == 1 ? plane_xo[u] : cur_xold[u];
                        if (f == 0) dn_old = xo;
                        const double old = weighted ? xo * dn_old : xo;
                        const double xnew = old + A.a_dt * tn;
                        if constexpr (STAGE == 2) {
                            // get_scalars (funcpack.f90:488-542): natural value with the new density
                            if constexpr (MIXED) {   // one reciprocal per cell
                                if (f == 0) { dn_new = xnew; rdn_new = rcp_nr(xnew); }
                                A.xout[f][idx] = weighted ? xnew * rdn_new : xnew;
                            } else {
                                if (f == 0) dn_new = xnew;
                                A.xout[f][idx] = weighted ? xnew / dn_new : xnew;
                            }
                        } else {
                            A.xout[f][idx] = xnew;
                            A.tend[f][idx] = tn;
                        }
                        if (A.fst[f]) A.fst[f][idx] = T;
                    }
                }
            }
        }
        if (cellt) issue_z(k + L + 1);
        else cp_async_commit();
    }
    cp_async_wait_all();
#undef ZVAL
}

template <int SCHEME, bool MIXED, int STAGE, bool SGS, int FC = 0>
__global__ void __launch_bounds__(NT, 2)
    k1_kernel(const __grid_constant__ DevGrid G, const __grid_constant__ K1Args A, const __grid_constant__ K1Maps M)
{
    k1_run<SCHEME, MIXED, STAGE, SGS, FC>(G, A, M, blockIdx.x);
}

// One launch over the blocks of several domains (an ensemble stage): block b of the
// launch runs block items[b].b of domain items[b].m, whose grid, arguments and tensor
// maps (in global memory, written before the launch and never changed while it runs)
// are mem[items[b].m].
template <int SCHEME, bool MIXED, int STAGE, int FC = 0>
__global__ void __launch_bounds__(NT, 2) k1_group_kernel(const K1Member *__restrict__ mem, const GItem *__restrict__ items)
{
    const GItem it = items[blockIdx.x];
    const K1Member &m = mem[it.m];
    if (threadIdx.x == 0 && threadIdx.y == 0) {   // the thread that issues the bulk copies
        const int F = FC > 0 ? FC : m.A.nf;
        for (int f = 0; f < F; f++) tensormap_acquire(&m.M.x[f]);
        tensormap_acquire(&m.M.mu);
        tensormap_acquire(&m.M.mv);
    }
    k1_run<SCHEME, MIXED, STAGE, false, FC>(m.G, m.A, m.M, it.b);
}

}  // namespace
