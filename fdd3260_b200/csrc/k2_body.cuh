// k2_body.cuh -- body of the K2 kernel (momentum tendency + stage update), templated
// on the arithmetic form; instantiated by k_momentum.cu (plain FP64, no FMA
// contraction: bit-identical to the CPU restatement) and k_momentum_mixed.cu (FP32
// stencils and fluxes, FP64 accumulation, pressure gradient, buoyancy and state).
#pragma once
#include <type_traits>
#include "mg_common.cuh"
#include "mimica_gpu.h"
#include "tma.cuh"

namespace {

constexpr int TX = 32, TY = 8, RH = 2;
constexpr int PW = TX + 2 * RH, PH = TY + 2 * RH, PL = PW * PH;
constexpr int NSLOT = 5;
// raw momentum of one level, three TMA boxes of 38 x 12 doubles: x from cell i0-3 (an
// even 0-based start, as TMA requires), y from j0-2; ring column c is box column c+1
constexpr int SBW = TX + 2 * RH + 2, SBH = TY + 2 * RH;
constexpr int STG_BYTES = SBW * SBH * 8;   // 3648
constexpr int STG_SLOT = 3712;              // 128-byte multiple

template <typename R> __host__ __device__ constexpr size_t k2_ring_bytes() { return ((size_t)2 * NSLOT * 3 * PL * sizeof(R) + 127) / 128 * 128; }
template <typename R> __host__ __device__ constexpr size_t k2_smem_bytes() { return k2_ring_bytes<R>() + 3 * STG_SLOT + 128 + 128; }
constexpr double AVISC = 1. / 16.;   // windadv.f90:39

// k segments per column tile, as K1's (k1_body.cuh): the count that minimises (waves of
// CTAs) x (levels per segment + 2, the prologue's flux levels and the ring fill), with
// segments of at least 8 levels; CTAs per SM from the shared memory (at most 2 by the
// registers of 256 threads)
inline int k2_segments(const DevGrid &g, size_t smem)
{
    int dev = 0, nsm = 148;
    if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        nsm = 148;
    long long per_sm = (228LL * 1024) / ((long long)smem + 1024);
    per_sm = per_sm < 1 ? 1 : (per_sm > 2 ? 2 : per_sm);
    const long long slots = (long long)nsm * per_sm;
    const long long tiles = (long long)((g.maxx + TX - 1) / TX) * ((g.maxy + TY - 1) / TY);
    int best = 1;
    double bt = 1e300;
    for (int sgm = 1; sgm <= (g.nz / 8 > 1 ? g.nz / 8 : 1); sgm++) {
        const double t = (double)((tiles * sgm + slots - 1) / slots) * ((double)g.nz / sgm + 2.);
        if (t < 0.999 * bt) { bt = t; best = sgm; }
    }
    return best;
}

__device__ __forceinline__ double ldg(const double *p, long long i) { return __ldg(p + i); }
__device__ __forceinline__ double abs_r(double x) { return fabs(x); }
__device__ __forceinline__ float abs_r(float x) { return fabsf(x); }

// EVEN: the parity of ntime (the direction order of windadv.f90:103,158), so that each
// instantiation evaluates the three directions as straight-line code
// bid: the block's index in the domain's own grid of tiles x segments
template <bool MIXED, bool EVEN>
__device__ __forceinline__ void k2_run(const DevGrid &G, const K2Args &A, const K2Maps &M, const int bid)
{
    // R: type of the stencil arithmetic (FP64 plain form, FP32 mixed form)
    using R = typename std::conditional<MIXED, float, double>::type;
    extern __shared__ unsigned char sm_raw[];
    // 128-byte alignment by an offset from the shared array itself, so that every pointer
    // derived from it stays a shared-memory pointer
    unsigned char *smb = sm_raw + ((128u - (smem_u32(sm_raw) & 127u)) & 127u);
    R *sm = reinterpret_cast<R *>(smb);
    R *ring_m = sm;                            // [slot][3][PL] momentum (stencil values)
    R *ring_a = sm + NSLOT * 3 * PL;           // [slot][3][PL] advective velocity
    double *stg = reinterpret_cast<double *>(smb + k2_ring_bytes<R>());   // [3][SBH][SBW] raw level
    uint64_t *mbar = reinterpret_cast<uint64_t *>(smb + k2_ring_bytes<R>() + 3 * STG_SLOT);

    const int ntx = (G.maxx + TX - 1) / TX, nty = (G.maxy + TY - 1) / TY;
    const int tile = bid % (ntx * nty), seg = bid / (ntx * nty);
    const int ti = tile % ntx, tj = tile / ntx;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const int i0 = 4 + ti * TX, j0 = 4 + tj * TY;
    const int i = i0 + tx, j = j0 + ty;
    const int nx = G.nx, ny = G.ny, nz = G.nz;
    const bool act = (i <= nx - 2) && (j <= ny - 2);
    const double dx1d = 1. / G.dx, dy1d = 1. / G.dy, dt0 = G.dt0;
    const R dx1 = (R)dx1d, dy1 = (R)dy1d;
    const R dx2 = (R)(1. / (2. * G.dx)), dy2 = (R)(1. / (2. * G.dy));
    const R dx3 = (R)(1. / (3. * G.dx)), dy3 = (R)(1. / (3. * G.dy));
    R c1a, c2a, c1b, c2b;   // a: 4/3,1/3 (self-advection); b: 9/8,1/8 (cross terms)
    if (G.mom_ord == 4) { c1a = (R)(4. / 3.); c2a = (R)(1. / 3.); c1b = (R)(9. / 8.); c2b = (R)(1. / 8.); }
    else { c1a = 1; c2a = 0; c1b = 1; c2b = 0; }
    const R AVR = (R)AVISC, HALF = (R)0.5, QUART = (R)0.25, FOUR = (R)4., SIX = (R)6.;
    const double *dzw = G.dzw, *dz1w = G.dz1w, *dz1 = G.dz1;

    if (tid == 0) {
        mbar_init(mbar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    // raw level l -> staging (single slot; the l-th copy completes phase (l-1)&1)
    // this CTA's levels [kb, ke]; a segment above the surface starts at kp = kb - 3 with
    // prologue levels that only advance the carried vertical fluxes
    const int kb = 1 + (int)(((long long)seg * nz) / A.nseg), ke = (int)(((long long)(seg + 1) * nz) / A.nseg);
    const int kp = kb > 3 ? kb - 3 : 1;
    const int lmax = min(nz, ke + 2);   // last level the ring needs
    auto issue_raw = [&](int l) {
        fence_proxy_async_shared();
        mbar_arrive_expect_tx(mbar, 3 * STG_BYTES);
        for (int c = 0; c < 3; c++)
            tma_load_3d(stg + c * (STG_SLOT / 8), &M.m[c], i0 - 4, j0 - 3, l - 1, mbar);
    };
    // staging -> ring slot of level l: stencil momentum and advective velocity (zero
    // outside the domain, as the reference's arrays are read there)
    // This thread's ring elements of a level: o = tid and o = tid + 256 of each component's
    // PW x PH plane (PL = 432 < 512), with their staging offsets and whether they lie in
    // the domain; the same for every level, so they are found once.
    static_assert(PL > TX * TY && PL <= 2 * TX * TY, "two ring elements per thread and component");
    const int ro1 = tid + TX * TY;
    const bool has1 = ro1 < PL;
    auto stg_of = [&](int o, bool &in) {
        const int r = o / PW, c = o - r * PW;
        const int ii = i0 - RH + c, jj = j0 - RH + r;
        in = ii >= 1 && ii <= nx && jj >= 1 && jj <= ny;
        return r * SBW + c + 1;
    };
    bool in0, in1 = false;
    const int so0 = stg_of(tid, in0);
    const int so1 = has1 ? stg_of(ro1, in1) : 0;
    auto convert_level = [&](int l) {
        mbar_wait_bounded(mbar, (uint32_t)((l - kp) & 1), A.err);
        const int slot = l % NSLOT;
        const double d0 = ldg(G.den0, l - 1), a0 = ldg(G.avden0, l - 1);
        // the mixed form multiplies by the level's reciprocal densities instead of dividing
        const double rd0 = MIXED ? ldg(G.rden0, l - 1) : 0., ra0 = MIXED ? ldg(G.ravden0, l - 1) : 0.;
#pragma unroll
        for (int arr = 0; arr < 3; arr++) {
            const double w = arr == 2 ? a0 : d0;
            const double shift = arr == 0 ? G.u0shift : (arr == 1 ? G.v0shift : 0.);
            auto one = [&](int o, int so, bool in) {
                double mv = 0., av = 0.;
                if (in) {
                    const double x = stg[arr * (STG_SLOT / 8) + so];
                    mv = A.in_is_leveln ? rep_value(A.rep, x, w) : x;
                    av = MIXED ? mv * (arr == 2 ? ra0 : rd0) : mv / w;
                    if (arr < 2) av = av - shift;
                }
                ring_m[(slot * 3 + arr) * PL + o] = (R)mv;
                ring_a[(slot * 3 + arr) * PL + o] = (R)av;
            };
            one(tid, so0, in0);
            if (has1) one(ro1, so1, in1);
        }
    };
    // Per level k: lb[d+2] = this thread's element of ring slot (k+d) mod 5, d = -2..2.
    // MM/AA(c, d, di, dj): momentum / advective velocity of component c (0 u, 1 v, 2 w)
    // at (i+di, j+dj, k+d); d, di, dj are compile-time constants at every use.
    const R *lb[5];
#define MM(c, d, di, dj) lb[(d) + 2][(c) * PL + (dj) * PW + (di)]
#define AA(c, d, di, dj) lb[(d) + 2][NSLOT * 3 * PL + (c) * PL + (dj) * PW + (di)]
#define ZW(l) ((R)ldg(dzw, (l) - 1))
#define ZW1(l) ((R)ldg(dz1w, (l) - 1))
#define Z1(l) ((R)ldg(dz1, (l) - 1))
// accumulation of one direction's contribution: (acc + a) - b in the plain form (the
// reference's order), acc + (a - b) evaluated in R and added in FP64 in the mixed form
#define ACC2(acc, a, b) do { if constexpr (MIXED) acc = acc + (double)((a) - (b)); else acc = acc + (a) - (b); } while (0)
#define ACC1(acc, a) do { acc = acc + (a); } while (0)
#define SUB1(acc, a) do { acc = acc - (a); } while (0)

    if (tid == 0) issue_raw(kp);
    convert_level(kp);
    __syncthreads();
    if (kp + 1 <= lmax) {
        if (tid == 0) issue_raw(kp + 1);
        convert_level(kp + 1);
        __syncthreads();
    }
    if (tid == 0 && kp + 2 <= lmax) issue_raw(kp + 2);

    double bb_prev = 0.;   // buoyancy at level k-1 (cell centre)
    // vertical fluxes carried up the column (each computed once):
    //   fzu/fzv[m] = Flux(k-2+m) of advuz/advvz, m = 0..3;  fzw[m] = Flux(k-1+m) and
    //   azw[m] = Adv(k-2+m) of advwz;  pp_below = p(k-1)/rho0(k-1)
    R fzu0 = 0, fzu1 = 0, fzu2 = 0, fzu3 = 0, fzv0 = 0, fzv1 = 0, fzv2 = 0, fzv3 = 0;
    R fzw0 = 0, fzw1 = 0, azw0 = 0, azw1 = 0, azw2 = 0;
    double pp_below = 0.;
    const double grav = 9.81, epsm = 0.60243, cdiag = 0.5;
    const int own = (ty + RH) * PW + (tx + RH);

    // buoyancy bb of a cell (imp_buoy: state + cdiag*dt0*states)
    auto buoy_bb = [&](int k, double dn, double esv, double qtv, double fesv, double fqtv) {
        if (A.dens_is_leveln) {
            esv = rep_value(A.rep, esv, dn);
            if (A.qt) qtv = rep_value(A.rep, qtv, dn);
        }
        double est = esv + cdiag * dt0 * fesv;
        double qtt = A.qt ? qtv + cdiag * dt0 * fqtv : 0.;
        double sumh = 0.;
        double ref = ldg(G.pt0, k - 1) * (1. + epsm * ldg(G.qv0, k - 1));
        if constexpr (MIXED) {   // reciprocals instead of the two divisions
            const double den1 = rcp_nr(dn), pt = den1 * est;
            return dn * grav * (pt * (1. + epsm * den1 * (qtt - sumh) - den1 * sumh) * rcp_nr(ref) - 1.);
        } else {
            double den1 = 1. / dn;
            double pt = den1 * est;
            return dn * grav * (pt * (1. + epsm * den1 * (qtt - sumh) - den1 * sumh) / ref - 1.);
        }
    };
    // a segment above the surface: p/rho0 and the buoyancy of level kb-1, as the
    // segment below computes them
    if (kb > 1 && act && A.mode != 1) {
        const long long idm = gidx(G, i, j, kb - 1);
        pp_below = MIXED ? ldg(A.p, idm) * ldg(G.rden0, kb - 2) : ldg(A.p, idm) / ldg(G.den0, kb - 2);
        if (G.with_buoy)
            bb_prev = buoy_bb(kb - 1, ldg(A.dens, idm), ldg(A.es, idm), A.qt ? ldg(A.qt, idm) : 0., ldg(A.fes, idm),
                              A.qt ? ldg(A.fqt, idm) : 0.);
    }

    for (int k = kp; k <= ke; k++) {
        const bool pro = k < kb;   // prologue level: the carried vertical fluxes only
        __syncthreads();   // ring slot (k+2)%5 (level k-3) no longer read
        if (k + 2 <= lmax) convert_level(k + 2);
        __syncthreads();   // ring complete for level k; the staging slot is free
        if (tid == 0 && k + 3 <= lmax) issue_raw(k + 3);
        if (!act) continue;   // no further barriers in this iteration
        // epilogue operands of this level, issued before the stencil arithmetic
        const long long idx = gidx(G, i, j, k);
        double e_p = 0., e_pw = 0., e_ps = 0., e_dn = 0., e_es = 0., e_qt = 0., e_fes = 0., e_fqt = 0.;
        double e_tu = 0., e_tv = 0., e_tw = 0., e_un = 0., e_vn = 0., e_wn = 0.;
        if (A.mode != 1 && !pro) {
            e_p = ldg(A.p, idx);
            e_pw = ldg(A.p, idx - 1);
            e_ps = ldg(A.p, idx - G.px);
            if (G.with_buoy) {
                e_dn = ldg_stream(A.dens + idx);
                e_es = ldg_stream(A.es + idx);
                e_fes = ldg_stream(A.fes + idx);
                if (A.qt) { e_qt = ldg_stream(A.qt + idx); e_fqt = ldg_stream(A.fqt + idx); }
            }
            // single-use operands are read without allocating L1 lines, which the level
            // coefficients and the pressure's neighbours keep
            if (A.stage != 1) { e_tu = ld_stream(A.tu + idx); e_tv = ld_stream(A.tv + idx); e_tw = ld_stream(A.tw + idx); }
            e_un = ldg_stream(A.mu_n + idx);
            e_vn = ldg_stream(A.mv_n + idx);
            e_wn = ldg_stream(A.mw_n + idx);
        }
#pragma unroll
        for (int d = -2; d <= 2; d++) lb[d + 2] = ring_m + (((k + d + NSLOT) % NSLOT) * 3) * PL + own;

        // ---- advance the carried vertical fluxes ----
        {
            // advuz_fd/advvz_fd Flux(k+1) (windadv.f90:656-663): levels k+1, k+2; Flux(nz) = 0
            R fu = 0, fv = 0;
            if (k + 1 <= nz - 1) {
                const R zp = ZW(k + 2), zc = ZW(k + 1), zs = zp + zc;
                R ww = c1b * (AA(2, 2, -1, 0) + AA(2, 2, 0, 0)) * HALF - c2b * (AA(2, 2, -2, 0) + AA(2, 2, 1, 0)) * HALF;
                R fr = (zp * MM(0, 2, 0, 0) + zc * MM(0, 1, 0, 0)) / zs;
                fu = ww * fr;
                ww = c1b * (AA(2, 2, 0, -1) + AA(2, 2, 0, 0)) * HALF - c2b * (AA(2, 2, 0, -2) + AA(2, 2, 0, 1)) * HALF;
                fr = (zp * MM(1, 2, 0, 0) + zc * MM(1, 1, 0, 0)) / zs;
                fv = ww * fr;
            }
            if (k == 1) {   // Flux(1): levels 1, 2
                const R zp = ZW(2), zc = ZW(1), zs = zp + zc;
                R ww = c1b * (AA(2, 1, -1, 0) + AA(2, 1, 0, 0)) * HALF - c2b * (AA(2, 1, -2, 0) + AA(2, 1, 1, 0)) * HALF;
                R fr = (zp * MM(0, 1, 0, 0) + zc * MM(0, 0, 0, 0)) / zs;
                fzu3 = ww * fr;
                ww = c1b * (AA(2, 1, 0, -1) + AA(2, 1, 0, 0)) * HALF - c2b * (AA(2, 1, 0, -2) + AA(2, 1, 0, 1)) * HALF;
                fr = (zp * MM(1, 1, 0, 0) + zc * MM(1, 0, 0, 0)) / zs;
                fzv3 = ww * fr;
            }
            fzu0 = fzu1; fzu1 = fzu2; fzu2 = fzu3; fzu3 = fu;
            fzv0 = fzv1; fzv1 = fzv2; fzv2 = fzv3; fzv3 = fv;
            // advwz_fd Flux(k), Adv(k) (:1087-1098)
            R fw = 0, aw_ = 0;
            if (k <= nz - 2) {
                R ww = (AA(2, 1, 0, 0) + AA(2, 0, 0, 0)) * HALF;
                R fr = (MM(2, 1, 0, 0) + MM(2, 0, 0, 0)) * HALF;
                fw = ww * fr;
                const R zp = ZW(k + 1), zc = ZW(k), zs = zp + zc;
                R ww2 = (zp * AA(2, 2, 0, 0) + zc * AA(2, 0, 0, 0)) / zs;
                R fr2 = (zp * MM(2, 2, 0, 0) + zc * MM(2, 0, 0, 0)) / zs;
                aw_ = ww2 * fr2;
            } else if (k == nz - 1) {
                fw = QUART * (AA(2, 1, 0, 0) + AA(2, 0, 0, 0)) * (MM(2, 1, 0, 0) + MM(2, 0, 0, 0));
                const R s2 = ZW(nz) + ZW(nz - 1);
                aw_ = ((R)0 + ZW(nz - 1) * AA(2, 0, 0, 0)) * ((R)0 + ZW(nz - 1) * MM(2, 0, 0, 0)) / (s2 * s2);
            }
            fzw0 = fzw1; fzw1 = fw;
            azw0 = azw1; azw1 = azw2; azw2 = aw_;
        }
        if (pro) continue;

        // ---------------- u component ----------------
        double au = 0.;
        {
            auto dx_ = [&]() {   // advux_fd
#define FX(p) (((AA(0, 0, (p) + 1, 0) + AA(0, 0, (p), 0)) * HALF) * ((MM(0, 0, (p) + 1, 0) + MM(0, 0, (p), 0)) * HALF))
#define AX(p) (((AA(0, 0, (p) + 2, 0) + AA(0, 0, (p), 0)) * HALF) * ((MM(0, 0, (p) + 2, 0) + MM(0, 0, (p), 0)) * HALF))
                ACC2(au, c1a * (FX(0) - FX(-1)) * dx1, c2a * (AX(0) - AX(-2)) * dx2);
#undef FX
#undef AX
                if (G.lavisc) {
                    const R mu = abs_r(AA(0, 0, 0, 0)) * dx1;
                    SUB1(au, AVR * mu * (-MM(0, 0, 2, 0) + FOUR * MM(0, 0, 1, 0) - SIX * MM(0, 0, 0, 0) + FOUR * MM(0, 0, -1, 0) - MM(0, 0, -2, 0)));
                }
            };
            auto dy_ = [&]() {   // advuy_fd: vt1=vt(i-1), vt2=vt(i), vt3=vt(i-2), vt4=vt(i+1)
#define FY(p) ((c1b * (AA(1, 0, -1, (p) + 1) + AA(1, 0, 0, (p) + 1)) * HALF - c2b * (AA(1, 0, -2, (p) + 1) + AA(1, 0, 1, (p) + 1)) * HALF) * \
               ((MM(0, 0, 0, (p) + 1) + MM(0, 0, 0, (p))) * HALF))
                ACC2(au, c1b * (FY(0) - FY(-1)) * dy1, c2b * (FY(1) - FY(-2)) * dy3);
#undef FY
                if (G.lavisc) {
                    const R mu = QUART * abs_r(AA(1, 0, -1, 0) + AA(1, 0, 0, 0) + AA(1, 0, -1, 1) + AA(1, 0, 0, 1)) * dy1;
                    SUB1(au, AVR * mu * (-MM(0, 0, 0, 2) + FOUR * MM(0, 0, 0, 1) - SIX * MM(0, 0, 0, 0) + FOUR * MM(0, 0, 0, -1) - MM(0, 0, 0, -2)));
                }
            };
            auto dz_ = [&]() {   // advuz_fd, Flux(k-2..k+1) = fzu0..fzu3
                if (k >= 3 && k <= nz - 1)
                    ACC2(au, c1b * (fzu2 - fzu1) * ZW1(k), c2b * (fzu3 - fzu0) / (ZW(k - 1) + ZW(k) + ZW(k + 1)));
                else if (k == 1)
                    ACC1(au, (fzu2 - (R)0) * ZW1(1));
                else if (k == 2)
                    ACC2(au, c1b * (fzu2 - fzu1) * ZW1(1), c2b * (fzu3 - (R)0) / (ZW(1) + ZW(2) + ZW(3)));
                else
                    ACC1(au, ((R)0 - fzu1) * ZW1(nz));
                if (G.lavisc && k >= 3 && k <= nz - 2) {
                    const R mu = QUART * abs_r(AA(2, 0, -1, 0) + AA(2, 0, 0, 0) + AA(2, 1, -1, 0) + AA(2, 1, 0, 0)) * ZW1(k);
                    SUB1(au, AVR * mu * (-MM(0, 2, 0, 0) + FOUR * MM(0, 1, 0, 0) - SIX * MM(0, 0, 0, 0) + FOUR * MM(0, -1, 0, 0) - MM(0, -2, 0, 0)));
                }
            };
            // the reference's direction order, which alternates with ntime's parity
            if constexpr (EVEN) { dx_(); dy_(); dz_(); } else { dz_(); dy_(); dx_(); }
        }
        // ---------------- v component ----------------
        double av = 0.;
        {
            auto dx_ = [&]() {   // advvx_fd: ut1=ut(j-1), ut2=ut(j), ut3=ut(j-2), ut4=ut(j+1)
#define FX(p) ((c1b * (AA(0, 0, (p) + 1, -1) + AA(0, 0, (p) + 1, 0)) * HALF - c2b * (AA(0, 0, (p) + 1, -2) + AA(0, 0, (p) + 1, 1)) * HALF) * \
               ((MM(1, 0, (p) + 1, 0) + MM(1, 0, (p), 0)) * HALF))
                ACC2(av, c1b * (FX(0) - FX(-1)) * dx1, c2b * (FX(1) - FX(-2)) * dx3);
#undef FX
                if (G.lavisc) {
                    const R mu = QUART * abs_r(AA(0, 0, 0, -1) + AA(0, 0, 0, 0) + AA(0, 0, 1, -1) + AA(0, 0, 1, 0)) * dx1;
                    SUB1(av, AVR * mu * (-MM(1, 0, 2, 0) + FOUR * MM(1, 0, 1, 0) - SIX * MM(1, 0, 0, 0) + FOUR * MM(1, 0, -1, 0) - MM(1, 0, -2, 0)));
                }
            };
            auto dy_ = [&]() {   // advvy_fd
#define FY(p) (((AA(1, 0, 0, (p) + 1) + AA(1, 0, 0, (p))) * HALF) * ((MM(1, 0, 0, (p) + 1) + MM(1, 0, 0, (p))) * HALF))
#define AY(p) (((AA(1, 0, 0, (p) + 2) + AA(1, 0, 0, (p))) * HALF) * ((MM(1, 0, 0, (p) + 2) + MM(1, 0, 0, (p))) * HALF))
                ACC2(av, c1a * (FY(0) - FY(-1)) * dy1, c2a * (AY(0) - AY(-2)) * dy2);
#undef FY
#undef AY
                if (G.lavisc) {
                    const R mu = abs_r(AA(1, 0, 0, 0)) * dy1;
                    SUB1(av, AVR * mu * (-MM(1, 0, 0, 2) + FOUR * MM(1, 0, 0, 1) - SIX * MM(1, 0, 0, 0) + FOUR * MM(1, 0, 0, -1) - MM(1, 0, 0, -2)));
                }
            };
            auto dz_ = [&]() {   // advvz_fd, Flux(k-2..k+1) = fzv0..fzv3
                if (k >= 3 && k <= nz - 1)
                    ACC2(av, c1b * (fzv2 - fzv1) * ZW1(k), c2b * (fzv3 - fzv0) / (ZW(k - 1) + ZW(k) + ZW(k + 1)));
                else if (k == 1)
                    ACC1(av, (fzv2 - (R)0) * ZW1(1));
                else if (k == 2)
                    ACC2(av, c1b * (fzv2 - fzv1) * ZW1(2), c2b * (fzv3 - (R)0) / (ZW(1) + ZW(2) + ZW(3)));
                else
                    ACC1(av, ((R)0 - fzv1) * ZW1(nz));
                if (G.lavisc && k >= 3 && k <= nz - 2) {
                    const R mu = QUART * abs_r(AA(2, 0, 0, -1) + AA(2, 0, 0, 0) + AA(2, 1, 0, -1) + AA(2, 1, 0, 0)) * ZW1(k);
                    SUB1(av, AVR * mu * (-MM(1, 2, 0, 0) + FOUR * MM(1, 1, 0, 0) - SIX * MM(1, 0, 0, 0) + FOUR * MM(1, -1, 0, 0) - MM(1, -2, 0, 0)));
                }
            };
            // the reference's direction order, which alternates with ntime's parity
            if constexpr (EVEN) { dx_(); dy_(); dz_(); } else { dz_(); dy_(); dx_(); }
        }
        // ---------------- w component (k >= 2) ----------------
        double aw = 0.;
        if (k >= 2) {
            {
                auto dx_ = [&]() {   // advwx_fd
#define HV(p, d) AA(0, d, p, 0)
#define WV(p) MM(2, 0, p, 0)
#define FH(p) ((k == 2 ? (HV((p) + 1, 0) + HV((p) + 1, -1)) * HALF                                            \
                       : (k == nz ? (HV((p) + 1, 0) + HV((p) + 1, -1)) * HALF                                  \
                                  : c1b * (HV((p) + 1, 0) + HV((p) + 1, -1)) * HALF -                          \
                                        c2b * (HV((p) + 1, 1) + HV((p) + 1, -2)) * HALF)) *                    \
                ((WV((p) + 1) + WV(p)) * HALF))
                    ACC2(aw, c1b * (FH(0) - FH(-1)) * dx1, c2b * (FH(1) - FH(-2)) * dx3);
                    if (G.lavisc) {
                        const R mu = QUART * abs_r(HV(0, 0) + HV(0, -1) + HV(1, 0) + HV(1, -1)) * dx1;
                        SUB1(aw, AVR * mu * (-WV(2) + FOUR * WV(1) - SIX * WV(0) + FOUR * WV(-1) - WV(-2)));
                    }
#undef HV
#undef WV
                };
                auto dy_ = [&]() {   // advwy_fd
#define HV(p, d) AA(1, d, 0, p)
#define WV(p) MM(2, 0, 0, p)
                    ACC2(aw, c1b * (FH(0) - FH(-1)) * dy1, c2b * (FH(1) - FH(-2)) * dy3);
                    if (G.lavisc) {
                        const R mu = QUART * abs_r(HV(0, 0) + HV(0, -1) + HV(1, 0) + HV(1, -1)) * dy1;
                        SUB1(aw, AVR * mu * (-WV(2) + FOUR * WV(1) - SIX * WV(0) + FOUR * WV(-1) - WV(-2)));
                    }
#undef HV
#undef WV
#undef FH
                };
                auto dz_ = [&]() {   // advwz_fd, Flux(k-1..k) = fzw0..1, Adv(k-2..k) = azw0..2
                    if (k >= 3 && k <= nz - 1)
                        ACC2(aw, c1a * (fzw1 - fzw0) * Z1(k - 1), c2a * (azw2 - azw0) / (ZW(k) + ZW(k - 1)));
                    else if (k == 2)
                        ACC2(aw, c1a * (fzw1 - fzw0) * Z1(1), c2a * (azw2 - (R)0) / (ZW(2) + ZW(1)));
                    else
                        ACC1(aw, ((R)0 - fzw0) * Z1(nz - 1));
                    if (G.lavisc && k >= 3 && k <= nz - 2) {
                        const R mu = abs_r(AA(2, 0, 0, 0)) * Z1(k - 1);
                        SUB1(aw, AVR * mu * (-MM(2, 2, 0, 0) + FOUR * MM(2, 1, 0, 0) - SIX * MM(2, 0, 0, 0) + FOUR * MM(2, -1, 0, 0) - MM(2, -2, 0, 0)));
                    }
                };
                // the reference's direction order, which alternates with ntime's parity
                if constexpr (EVEN) { dx_(); dy_(); dz_(); } else { dz_(); dy_(); dx_(); }
            }
        }

        if (A.mode == 1) {
            A.ou[idx] = au;
            A.ov[idx] = av;
            A.ow[idx] = aw;
            continue;
        }

        // ---------------- explicit pressure gradient (gradp on p/rho0) ----------------
        const double d0 = ldg(G.den0, k - 1), a0 = ldg(G.avden0, k - 1);
        // p/rho0: the mixed form multiplies by the context's 1/rho0 profile (the same
        // product at a segment's first level, above), the FP64 form divides
        double ppc, gpx, gpy;
        if constexpr (MIXED) {
            const double rd0 = ldg(G.rden0, k - 1);
            ppc = e_p * rd0;
            gpx = (ppc - e_pw * rd0) * dx1d;
            gpy = (ppc - e_ps * rd0) * dy1d;
        } else {
            ppc = e_p / d0;
            gpx = (ppc - e_pw / d0) * dx1d;
            gpy = (ppc - e_ps / d0) * dy1d;
        }
        double gpz;
        if (k >= 2) gpz = (ppc - pp_below) * ldg(dz1, k - 2);
        else gpz = (double)MM(2, 0, 0, 0) / (dt0 * ldg(G.avden0, 0));
        pp_below = ppc;
        double wsu = (A.su ? A.su[idx] : 0.) - d0 * gpx;
        double wsv = (A.sv ? A.sv[idx] : 0.) - d0 * gpy;
        double wsw = (A.sw ? A.sw[idx] : 0.) - a0 * gpz;

        // ---------------- buoyancy (imp_buoy: state + cdiag*dt0*states) ----------------
        double buoy = 0.;
        if (G.with_buoy) {
            const double bb = buoy_bb(k, e_dn, e_es, A.qt ? e_qt : 0., e_fes, e_fqt);
            buoy = k >= 2 ? 0.5 * (bb_prev + bb) : bb;
            bb_prev = bb;
        }

        // ---------------- assembly and integ_mom ----------------
        wsu = -au + wsu;
        wsv = -av + wsv;
        wsw = -aw + wsw + buoy;
        double tu_o = A.stage == 1 ? 0. : e_tu;
        double tv_o = A.stage == 1 ? 0. : e_tv;
        double tw_o = A.stage == 1 ? 0. : e_tw;
        double tu = wsu + A.b * tu_o, tv = wsv + A.b * tv_o, tw = wsw + A.b * tw_o;
        double un = rep_value(A.rep, e_un, d0);
        double vn = rep_value(A.rep, e_vn, d0);
        double wn = rep_value(A.rep, e_wn, a0);
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

template <bool MIXED, bool EVEN>
__global__ void __launch_bounds__(TX *TY)
    k2_kernel(const __grid_constant__ DevGrid G, const __grid_constant__ K2Args A, const __grid_constant__ K2Maps M)
{
    k2_run<MIXED, EVEN>(G, A, M, blockIdx.x);
}

// One launch over the blocks of up to K2G_MAX domains: block b runs block items[b].b of
// domain items[b].m.  The domains' grids and arguments are a kernel parameter (constant
// bank: read-only, so the compiler reloads them where the single-domain kernel does
// instead of holding them in registers); their tensor maps are in global memory, written
// before the launch and unchanged while it runs.
template <bool MIXED, bool EVEN>
__global__ void __launch_bounds__(TX * TY, 2)
    k2_group_kernel(const __grid_constant__ K2GroupParams P, const K2Maps *__restrict__ maps, const GItem *__restrict__ items)
{
    const GItem it = items[blockIdx.x];
    const K2Maps &M = maps[it.m];
    if (threadIdx.x == 0 && threadIdx.y == 0)   // the thread that issues the bulk copies
        for (int c = 0; c < 3; c++) tensormap_acquire(&M.m[c]);
    k2_run<MIXED, EVEN>(P.a[it.m].G, P.a[it.m].A, M, it.b);
}

// K2 over the blocks of several members, all at one ntime parity
template <bool MIXED>
cudaError_t launch_k2_group_t(int even, const K2GroupParams &P, const K2Maps *maps, const GItem *items, int nitems,
                              cudaStream_t s)
{
    const size_t sm = k2_smem_bytes<typename std::conditional<MIXED, float, double>::type>();
    cudaError_t e = even ? cudaFuncSetAttribute(k2_group_kernel<MIXED, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm)
                         : cudaFuncSetAttribute(k2_group_kernel<MIXED, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    if (nitems < 1) return cudaErrorInvalidValue;
    if (even)
        k2_group_kernel<MIXED, true><<<nitems, dim3(TX, TY), sm, s>>>(P, maps, items);
    else
        k2_group_kernel<MIXED, false><<<nitems, dim3(TX, TY), sm, s>>>(P, maps, items);
    return cudaGetLastError();
}

}  // namespace
