// k_pressure.cu -- anelastic pressure projection on the GPU, plain FP64 form.
//
// Replaces src/PRESSURE/pressure_solver.f90 (solve_pressure :143-189, correction
// :342-412, rescale_pressure :415-459), fft_solve_serial
// (src/PRESSURE/fft_interface.f90:543-666: FFTW c2c 2-D transform per level,
// tridiag per wavenumber, inverse transform), tridiag/TRIDAG2
// (src/PRESSURE/fft_tools.f90:115-237), caldiv and gradp
// (src/TOOLS/gradients.f90:986-1052,1205-1292), cal_p1 (src/TOOLS/funcpack.f90:750-793)
// and horav (src/TOOLS/averages.f90:78-209).
//
// Pipeline of one pass (all on the context's stream):
//   1. fft_x_fwd: rhs = div(m)/(dt0*rho0) computed on the fly for 8 rows of one
//      level, two real rows packed in one complex row, shared-memory Stockham FFT
//      (radix 4/2/3/5), split into the two half spectra, stored transposed as
//      S[k][kx][ky] so that y transforms and the vertical solve are contiguous.
//   2. fft_y (forward): complex Stockham FFT of every (k,kx) row along ky.
//   3. tridiag: one (kx,ky) column per thread, Thomas elimination along k with the
//      time-invariant elimination factors GAM precomputed at plan creation.
//   4. fft_y (inverse).
//   5. fft_x_inv: Hermitian rebuild of two rows, inverse FFT, scale 1/N_h -> dp.
//   6. correction: p += rho0*dp, m -= dt0*rho0*grad(dp), ghost cells refreshed.
// The real-to-complex transform is the same DFT as the reference's c2c of real data
// (the spectrum is Hermitian); the reference keeps mode (0,0) and then removes the
// horizontal mean of dp, which is that mode -- here the mode is set to zero.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "mg_common.cuh"
#include "mimica_gpu.h"

namespace {

constexpr int MAXSTAGES = 16;
struct FftPlan1 {
    int n;                 // length
    int nst;               // stages
    unsigned long long rpack;   // radix of stage s in bits [4s, 4s+4)
    const double2 *tw;     // device twiddles exp(-2 pi i t/n), t in [0,n)
    const float2 *twf;     // the same twiddles rounded to FP32 (mixed form)
};

// complex arithmetic on double2 (plain form) and float2 (mixed form: FP32 spectra)
template <typename C> struct CT;
template <> struct CT<double2> { using R = double; };
template <> struct CT<float2> { using R = float; };
template <typename C> __device__ __forceinline__ C mkc(typename CT<C>::R x, typename CT<C>::R y) { C c; c.x = x; c.y = y; return c; }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) { return mkc<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { return mkc<C>(a.x + b.x, a.y + b.y); }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { return mkc<C>(a.x - b.x, a.y - b.y); }

// twiddle exp(sign * 2 pi i t / n), sign = -1 forward, +1 inverse
template <typename C> __device__ __forceinline__ C twid(const FftPlan1 &P, int t, int inv);
template <> __device__ __forceinline__ double2 twid<double2>(const FftPlan1 &P, int t, int inv)
{
    double2 w = __ldg(P.tw + t);
    return inv ? make_double2(w.x, -w.y) : w;
}
template <> __device__ __forceinline__ float2 twid<float2>(const FftPlan1 &P, int t, int inv)
{
    float2 w = __ldg(P.twf + t);
    return inv ? make_float2(w.x, -w.y) : w;
}

// multiply by -i (forward, sign = -1) or +i (inverse): the exact quarter-turn
template <typename C> __device__ __forceinline__ C rot(C v, int inv) { return inv ? mkc<C>(-v.y, v.x) : mkc<C>(v.y, -v.x); }

// DFT of R values in registers, o[q] = sum_r v[r] w^{rq}, w = exp(-+2 pi i / R); R = 2, 3, 4, 5, 8
template <typename C, int R> __device__ __forceinline__ void dft_small(C *v, int inv);
template <typename C> __device__ __forceinline__ void dft_small2(C &a, C &b)
{
    const C t = a;
    a = cadd(t, b);
    b = csub(t, b);
}
template <> __device__ __forceinline__ void dft_small<double2, 2>(double2 *v, int) { dft_small2(v[0], v[1]); }
template <> __device__ __forceinline__ void dft_small<float2, 2>(float2 *v, int) { dft_small2(v[0], v[1]); }
template <typename C> __device__ __forceinline__ void dft4(C *v, int inv)
{
    const C t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
    const C t2 = cadd(v[1], v[3]), t3 = rot(csub(v[1], v[3]), inv);
    v[0] = cadd(t0, t2);
    v[2] = csub(t0, t2);
    v[1] = cadd(t1, t3);
    v[3] = csub(t1, t3);
}
template <> __device__ __forceinline__ void dft_small<double2, 4>(double2 *v, int inv) { dft4(v, inv); }
template <> __device__ __forceinline__ void dft_small<float2, 4>(float2 *v, int inv) { dft4(v, inv); }
template <typename C> __device__ __forceinline__ void dft8(C *v, int inv)
{
    using R = typename CT<C>::R;
    const R h = (R)0.70710678118654752440084436210485;   // sqrt(1/2)
    // radix-2 over (r, r+4), then twiddles w8^{r}, then two radix-4 transforms
    C a[4], b[4];
#pragma unroll
    for (int r = 0; r < 4; r++) {
        a[r] = cadd(v[r], v[r + 4]);
        b[r] = csub(v[r], v[r + 4]);
    }
    // b[r] *= w8^r:  w8 = (h, -+h)
    const R sg = inv ? (R)1 : (R)-1;
    b[1] = mkc<C>(h * (b[1].x - sg * b[1].y), h * (b[1].y + sg * b[1].x));
    b[2] = rot(b[2], inv);
    b[3] = mkc<C>(-h * (b[3].x + sg * b[3].y), h * (sg * b[3].x - b[3].y));
    dft4(a, inv);
    dft4(b, inv);
#pragma unroll
    for (int q = 0; q < 4; q++) {
        v[2 * q] = a[q];
        v[2 * q + 1] = b[q];
    }
}
template <> __device__ __forceinline__ void dft_small<double2, 8>(double2 *v, int inv) { dft8(v, inv); }
template <> __device__ __forceinline__ void dft_small<float2, 8>(float2 *v, int inv) { dft8(v, inv); }
template <typename C> __device__ __forceinline__ void dft3(C *v, int inv)
{
    using R = typename CT<C>::R;
    const R s3 = (R)0.86602540378443864676372317075294;   // sin(2 pi/3)
    const C t1 = cadd(v[1], v[2]), t2 = csub(v[1], v[2]);
    const C m = mkc<C>(v[0].x - (R)0.5 * t1.x, v[0].y - (R)0.5 * t1.y);
    const C r = rot(mkc<C>(s3 * t2.x, s3 * t2.y), inv);
    v[0] = cadd(v[0], t1);
    v[1] = cadd(m, r);
    v[2] = csub(m, r);
}
template <> __device__ __forceinline__ void dft_small<double2, 3>(double2 *v, int inv) { dft3(v, inv); }
template <> __device__ __forceinline__ void dft_small<float2, 3>(float2 *v, int inv) { dft3(v, inv); }
template <typename C> __device__ __forceinline__ void dft5(C *v, int inv)
{
    using R = typename CT<C>::R;
    const R c1 = (R)0.30901699437494742410229341718282, c2 = (R)-0.80901699437494742410229341718282;
    const R s1 = (R)0.95105651629515357211643933337938, s2 = (R)0.58778525229247312916870595463907;
    const C t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]), t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
    const C a1 = mkc<C>(v[0].x + c1 * t1.x + c2 * t2.x, v[0].y + c1 * t1.y + c2 * t2.y);
    const C a2 = mkc<C>(v[0].x + c2 * t1.x + c1 * t2.x, v[0].y + c2 * t1.y + c1 * t2.y);
    const C b1 = rot(mkc<C>(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y), inv);
    const C b2 = rot(mkc<C>(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y), inv);
    v[0] = cadd(v[0], cadd(t1, t2));
    v[1] = cadd(a1, b1);
    v[4] = csub(a1, b1);
    v[2] = cadd(a2, b2);
    v[3] = csub(a2, b2);
}
template <> __device__ __forceinline__ void dft_small<double2, 5>(double2 *v, int inv) { dft5(v, inv); }
template <> __device__ __forceinline__ void dft_small<float2, 5>(float2 *v, int inv) { dft5(v, inv); }

// one Stockham stage of radix R: butterflies j = lt, lt+nt, ... < n/R; Ns = product of
// Row buffers of the shared-memory transforms keep one padding element after every 8
// (element i at i + i/8): the stride-R writes of a radix-8 stage (the first stage writes
// every 8th element) then fall in distinct banks.
__host__ __device__ constexpr int padded_len(int n) { return n + (n + 7) / 8; }
__device__ __forceinline__ int pidx(int i) { return i + (i >> 3); }

// the earlier radices (ns_shift = log2 Ns when Ns is a power of two, else -1)
template <typename C, int R>
__device__ __forceinline__ void stockham_stage(const FftPlan1 &P, const C *a, C *b, int lt, int nt, int inv,
                                               int Ns, int ns_shift)
{
    const int n = P.n, nb = n / R;
    const int tmul = n / (Ns * R);
    for (int j = lt; j < nb; j += nt) {
        const int jq = ns_shift >= 0 ? (j >> ns_shift) : j / Ns;
        const int kk = j - jq * Ns;
        const int tstep = kk * tmul;
        C v[R];
#pragma unroll
        for (int r = 0; r < R; r++) v[r] = a[pidx(j + r * nb)];
        if (tstep != 0) {
#pragma unroll
            for (int r = 1; r < R; r++) v[r] = cmul(v[r], twid<C>(P, tstep * r, inv));
        }
        dft_small<C, R>(v, inv);
        const int idxD = jq * Ns * R + kk;
#pragma unroll
        for (int r = 0; r < R; r++) b[pidx(idxD + r * Ns)] = v[r];
    }
}

// In-shared-memory Stockham FFT of one row: buffers a (input) and b (scratch), threads
// [0, nt) of a row group cooperate (lt = thread within the group).  Every stage ends in a
// block barrier.  Returns the buffer holding the result.
template <typename C>
__device__ C *stockham(const FftPlan1 &P, C *a, C *b, int lt, int nt, int inv)
{
    int Ns = 1;
    for (int s = 0; s < P.nst; s++) {
        const int Rr = (int)((P.rpack >> (4 * s)) & 15ull);
        const int sh = (Ns & (Ns - 1)) == 0 ? __ffs(Ns) - 1 : -1;
        switch (Rr) {
        case 8: stockham_stage<C, 8>(P, a, b, lt, nt, inv, Ns, sh); break;
        case 4: stockham_stage<C, 4>(P, a, b, lt, nt, inv, Ns, sh); break;
        case 2: stockham_stage<C, 2>(P, a, b, lt, nt, inv, Ns, sh); break;
        case 3: stockham_stage<C, 3>(P, a, b, lt, nt, inv, Ns, sh); break;
        default: stockham_stage<C, 5>(P, a, b, lt, nt, inv, Ns, sh); break;
        }
        __syncthreads();
        C *t = a; a = b; b = t;
        Ns *= Rr;
    }
    return a;
}

// -------------------- refinement control --------------------
struct Skip {
    const unsigned long long *flag;   // residual slot checked, or null (never skip)
    double tol;
};
__device__ __forceinline__ bool converged(const Skip &k)
{
    if (!k.flag) return false;
    const unsigned long long v = *(volatile const unsigned long long *)k.flag;
    return __longlong_as_double((long long)v) < k.tol;
}

// -------------------- step 1: rhs + x transform --------------------
constexpr int ROWS = 8;   // rows per x-transform block (4 packed pairs)
// element (kx, c) of a [kx][ROWS] staging tile of the x transforms, c = 0..7 in a row of
// its own: rows written at stride 8 by consecutive kx and read along c stay in distinct
// banks with c permuted by kx (by kx/2 for 8-byte elements, two rows per 128 bytes)
template <typename C>
__device__ __forceinline__ int stg(int kx, int c)
{
    return kx * ROWS + (c ^ ((sizeof(C) == 16 ? kx : kx >> 1) & 7));
}

struct XArgs {
    int mode;                     // 0: rhs = div(m)/(dt0*rho0) from momentum; 1: external rhs in rbuf;
                                  // 2: refinement residual r = (b - <b>_k) - A dp
    const double *mu, *mv, *mw;   // mode 0: momentum (halo'd layout)
    double *rbuf;                 // [nz][maxy][maxx]: mode 1/2 read; mode 0 writes b when store_b
    double *bsum;                 // [nz][groups] row-group sums of b (mode 0 writes when store_b, mode 2 reads)
    int store_b;
    const double *dp;             // mode 2: current solution [nz][maxy][maxx]
    const double *ak, *ck, *dka, *dkb;   // mode 2: vertical coefficients of the Poisson system
    void *spec;                   // S[k][kx][ky], complex of the form's precision
    double dt1;                   // 1/dt0
    unsigned long long *resid;    // this pass's residual slot (max |rhs|*dt0), or null
    Skip prev;                    // skip the pass when the previous pass's residual converged
};

// (A x) at one cell of the Poisson system solved by the transforms and the tridiagonal:
// the periodic 5-point horizontal Laplacian (whose DFT eigenvalues are wv, get_wv
// fft_tools.f90:82-107) plus the vertical rows of tridiag (fft_tools.f90:142-173).
__device__ __forceinline__ double poisson_apply(const DevGrid &G, const XArgs &A, int k, int jr, int t)
{
    const int maxx = G.maxx, maxy = G.maxy, nz = G.nz;
    const long long lev = (long long)maxx * maxy;
    const double *pl = A.dp + (long long)(k - 1) * lev;
    const long long o = (long long)jr * maxx + t;
    const double x = __ldg(pl + o);
    const double xw = __ldg(pl + (long long)jr * maxx + (t == 0 ? maxx - 1 : t - 1));
    const double xe = __ldg(pl + (long long)jr * maxx + (t == maxx - 1 ? 0 : t + 1));
    const double xs = __ldg(pl + (long long)(jr == 0 ? maxy - 1 : jr - 1) * maxx + t);
    const double xn = __ldg(pl + (long long)(jr == maxy - 1 ? 0 : jr + 1) * maxx + t);
    const double idx2 = 1. / (G.dx * G.dx), idy2 = 1. / (G.dy * G.dy);
    double v = (xe - 2. * x + xw) * idx2 + (xn - 2. * x + xs) * idy2;
    double dv;
    if (k == 1) dv = -__ldg(A.dka) - __ldg(A.dkb);
    else if (k == nz) dv = -__ldg(A.dka + nz - 1) + __ldg(A.dkb + nz - 1);
    else dv = -__ldg(A.dka + k - 1);
    v += dv * x;
    if (k > 1) v += __ldg(A.ak + k - 1) * __ldg(pl + o - lev);
    if (k < nz) v += __ldg(A.ck + k - 1) * __ldg(pl + o + lev);
    return v;
}

// The x-transform kernels keep the rows' buffers as two halves, [a_0..a_3 | b_0..b_3],
// so that one half is free when the other holds data: the half spectra move between
// shared memory and S[k][kx][ky] through a [kx][8 rows] staging tile in the free half,
// 8 consecutive ky (one 64/128-byte segment) per kx instead of 2 scattered values.
constexpr int XT_THREADS = 256;
// bid: the block's index in the domain's own grid (nz x row groups)
template <typename C>
__device__ __forceinline__ void fft_x_fwd_run(const DevGrid &G, const FftPlan1 &P, const XArgs &A, const int bid)
{
    using R = typename CT<C>::R;
    extern __shared__ double2 smraw_x[];
    C *smc = reinterpret_cast<C *>(smraw_x);
    C *spec = reinterpret_cast<C *>(A.spec);
    const int n = P.n, nh = n / 2 + 1, maxy = G.maxy;
    const int groups = (maxy + ROWS - 1) / ROWS;
    const int k = bid / groups + 1, jg = bid % groups;
    const int jb = jg * ROWS;                       // first interior row (0-based)
    const int nt_pair = blockDim.x / (ROWS / 2);
    const int pair = threadIdx.x / nt_pair, lt = threadIdx.x % nt_pair;
    const int np = padded_len(n);
    C *ahalf = smc, *bhalf = smc + (ROWS / 2) * np;
    C *a = ahalf + pair * np, *b = bhalf + pair * np;
    __shared__ unsigned long long bmax;
    __shared__ double wsum[32];
    if (converged(A.prev)) {   // uniform over the grid: nothing left to refine
        if (bid == 0 && threadIdx.x == 0 && A.resid) *A.resid = *A.prev.flag;
        return;
    }
    if (threadIdx.x == 0) bmax = 0ull;
    const double dx1 = 1. / G.dx, dy1 = 1. / G.dy;
    const double dzw1 = __ldg(G.dz1w + k - 1), d0 = __ldg(G.den0 + k - 1);
    const double rfac = A.dt1 / d0;   // rhs = div(m) * dt1 / rho0
    double bmean = 0.;
    if (A.mode == 2) {   // level mean of b from the row-group sums, fixed order
        for (int g = 0; g < groups; g++) bmean += A.bsum[(k - 1) * groups + g];
        bmean /= (double)G.maxx * (double)maxy;
    }
    auto rhs = [&](int jr, int t) -> double {   // jr: interior row 0-based, t: interior column 0-based
        if (jr >= maxy) return 0.;
        const long long o = ((long long)(k - 1) * maxy + jr) * G.maxx + t;
        if (A.mode == 1) return __ldg(A.rbuf + o);
        if (A.mode == 2) return (A.rbuf[o] - bmean) - poisson_apply(G, A, k, jr, t);
        const int i = t + 4, j = jr + 4;
        long long c = gidx(G, i, j, k);
        double d = 0.;
        d = d + (__ldg(A.mu + c + 1) - __ldg(A.mu + c)) * dx1;
        d = d + (__ldg(A.mv + c + G.px) - __ldg(A.mv + c)) * dy1;
        if (k < G.nz) d = d + (__ldg(A.mw + c + G.ps) - __ldg(A.mw + c)) * dzw1;
        else d = d + (0. - __ldg(A.mw + c)) * dzw1;
        const double bv = d * rfac;
        if (A.store_b) A.rbuf[o] = bv;
        return bv;
    };
    const int r0 = jb + 2 * pair, r1 = r0 + 1;
    double mx = 0., sm = 0.;
    if (A.mode == 0) {
        // rhs from the momentum, XU columns of both rows at a time: all their loads are
        // issued before the arithmetic (the momentum and b's buffer do not overlap)
        const double *__restrict__ mu = A.mu, *__restrict__ mv = A.mv, *__restrict__ mw = A.mw;
        double *__restrict__ rb = A.rbuf;
        const bool has0 = r0 < maxy, has1 = r1 < maxy, top = k >= G.nz;
        const long long cr0 = gidx(G, 4, (has0 ? r0 : 0) + 4, k), cr1 = gidx(G, 4, (has1 ? r1 : 0) + 4, k);
        const long long px = G.px, ps = G.ps;
        const long long o0 = ((long long)(k - 1) * maxy + r0) * G.maxx, o1 = o0 + G.maxx;
        constexpr int XU = 2;
        for (int tb = lt; tb < n; tb += XU * nt_pair) {
            double m0[XU][6], m1[XU][6];   // u(c), u(c+1), v(c), v(c+px), w(c), w(c+ps)
#pragma unroll
            for (int q = 0; q < XU; q++) {
                const int t = tb + q * nt_pair;
                if (t < n) {
                    if (has0) {
                        const long long c = cr0 + t;
                        m0[q][0] = __ldg(mu + c); m0[q][1] = __ldg(mu + c + 1);
                        m0[q][2] = __ldg(mv + c); m0[q][3] = __ldg(mv + c + px);
                        m0[q][4] = __ldg(mw + c); m0[q][5] = top ? 0. : __ldg(mw + c + ps);
                    }
                    if (has1) {
                        const long long c = cr1 + t;
                        m1[q][0] = __ldg(mu + c); m1[q][1] = __ldg(mu + c + 1);
                        m1[q][2] = __ldg(mv + c); m1[q][3] = __ldg(mv + c + px);
                        m1[q][4] = __ldg(mw + c); m1[q][5] = top ? 0. : __ldg(mw + c + ps);
                    }
                }
            }
            // the divergence of caldiv in its order of terms; at the top w(nz+1) = 0
            auto div = [&](const double *m) {
                double d = 0.;
                d = d + (m[1] - m[0]) * dx1;
                d = d + (m[3] - m[2]) * dy1;
                if (!top) d = d + (m[5] - m[4]) * dzw1;
                else d = d + (0. - m[4]) * dzw1;
                return d * rfac;
            };
#pragma unroll
            for (int q = 0; q < XU; q++) {
                const int t = tb + q * nt_pair;
                if (t < n) {
                    double v0 = 0., v1 = 0.;
                    if (has0) {
                        v0 = div(m0[q]);
                        if (A.store_b) rb[o0 + t] = v0;
                    }
                    if (has1) {
                        v1 = div(m1[q]);
                        if (A.store_b) rb[o1 + t] = v1;
                    }
                    mx = fmax(mx, fmax(fabs(v0), fabs(v1)));
                    sm += v0 + v1;
                    a[pidx(t)] = mkc<C>((R)v0, (R)v1);
                }
            }
        }
    } else if (A.mode == 2) {
        // refinement residual r = (b - <b>_k) - A dp, both rows of a column at a time with
        // their loads issued ahead of the arithmetic (poisson_apply's operands and order)
        const double *__restrict__ dp = A.dp, *__restrict__ rb = A.rbuf;
        const int maxx = G.maxx, nz = G.nz;
        const long long lev = (long long)maxx * maxy;
        const double idx2 = 1. / (G.dx * G.dx), idy2 = 1. / (G.dy * G.dy);
        double dv;
        if (k == 1) dv = -__ldg(A.dka) - __ldg(A.dkb);
        else if (k == nz) dv = -__ldg(A.dka + nz - 1) + __ldg(A.dkb + nz - 1);
        else dv = -__ldg(A.dka + k - 1);
        const double akk = k > 1 ? __ldg(A.ak + k - 1) : 0., ckk = k < nz ? __ldg(A.ck + k - 1) : 0.;
        const bool has[2] = {r0 < maxy, r1 < maxy};
        constexpr int XU = 1;
        for (int tb = lt; tb < n; tb += XU * nt_pair) {
            double m[XU][2][8];   // b, x, xw, xe, xs, xn, x below, x above
#pragma unroll
            for (int q = 0; q < XU; q++) {
                const int t = tb + q * nt_pair;
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int jr = h == 0 ? r0 : r1;
                    if (t < n && has[h]) {
                        const double *pl = dp + (long long)(k - 1) * lev;
                        const long long o = (long long)jr * maxx + t;
                        m[q][h][0] = rb[(long long)(k - 1) * lev + o];
                        m[q][h][1] = __ldg(pl + o);
                        m[q][h][2] = __ldg(pl + (long long)jr * maxx + (t == 0 ? maxx - 1 : t - 1));
                        m[q][h][3] = __ldg(pl + (long long)jr * maxx + (t == maxx - 1 ? 0 : t + 1));
                        m[q][h][4] = __ldg(pl + (long long)(jr == 0 ? maxy - 1 : jr - 1) * maxx + t);
                        m[q][h][5] = __ldg(pl + (long long)(jr == maxy - 1 ? 0 : jr + 1) * maxx + t);
                        m[q][h][6] = k > 1 ? __ldg(pl + o - lev) : 0.;
                        m[q][h][7] = k < nz ? __ldg(pl + o + lev) : 0.;
                    }
                }
            }
#pragma unroll
            for (int q = 0; q < XU; q++) {
                const int t = tb + q * nt_pair;
                if (t < n) {
                    double vv[2] = {0., 0.};
#pragma unroll
                    for (int h = 0; h < 2; h++) {
                        if (!has[h]) continue;
                        const double *e = m[q][h];
                        const double x = e[1];
                        double v = (e[3] - 2. * x + e[2]) * idx2 + (e[5] - 2. * x + e[4]) * idy2;
                        v += dv * x;
                        if (k > 1) v += akk * e[6];
                        if (k < nz) v += ckk * e[7];
                        vv[h] = (e[0] - bmean) - v;
                    }
                    mx = fmax(mx, fmax(fabs(vv[0]), fabs(vv[1])));
                    sm += vv[0] + vv[1];
                    a[pidx(t)] = mkc<C>((R)vv[0], (R)vv[1]);
                }
            }
        }
    } else {
        for (int t = lt; t < n; t += nt_pair) {
            const double v0 = rhs(r0, t), v1 = rhs(r1, t);
            mx = fmax(mx, fmax(fabs(v0), fabs(v1)));
            sm += v0 + v1;
            a[pidx(t)] = mkc<C>((R)v0, (R)v1);
        }
    }
    if (A.store_b) {   // deterministic block sum of b: fixed shuffle tree, warps in order
        for (int o = 16; o > 0; o >>= 1) sm += __shfl_xor_sync(0xffffffffu, sm, o);
        if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = sm;
    }
    __syncthreads();   // a[] complete, bmax initialised, warp sums written
    if (A.store_b && threadIdx.x == 0) {
        double t = 0.;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += wsum[w];
        A.bsum[(k - 1) * groups + jg] = t;
    }
    if (A.resid) {
        for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        if ((threadIdx.x & 31) == 0) atomicMax(&bmax, (unsigned long long)__double_as_longlong(mx * G.dt0));
    }
    C *res = stockham<C>(P, a, b, lt, nt_pair, 0);   // ends with a barrier
    if (A.resid && threadIdx.x == 0) atomicMax(A.resid, bmax);
    // split: A_k = (Z_k + conj Z_{n-k})/2, B_k = (Z_k - conj Z_{n-k})/(2i), rows r0 and r1;
    // kx < n/2 through the staging tile T[kx][8] in the free half, the Nyquist kx = n/2
    // directly
    const int hn = n / 2;
    C *T = (res == a) ? bhalf : ahalf;
    for (int kx = lt; kx < nh; kx += nt_pair) {
        C z = res[pidx(kx)], w = res[pidx((n - kx) % n)];
        C Av = mkc<C>((z.x + w.x) * (R)0.5, (z.y - w.y) * (R)0.5);
        C Bv = mkc<C>((z.y + w.y) * (R)0.5, (w.x - z.x) * (R)0.5);
        if (kx < hn) {
            T[stg<C>(kx, 2 * pair)] = Av;
            T[stg<C>(kx, 2 * pair + 1)] = Bv;
        } else {
            const long long base = ((long long)(k - 1) * nh + kx) * maxy;
            if (r0 < maxy) spec[base + r0] = Av;
            if (r1 < maxy) spec[base + r1] = Bv;
        }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < hn * ROWS; e += blockDim.x) {
        const int kx = e / ROWS, c = e - kx * ROWS, jr = jb + c;
        if (jr < maxy) spec[((long long)(k - 1) * nh + kx) * maxy + jr] = T[stg<C>(kx, c)];
    }
}

template <typename C>
__global__ void __launch_bounds__(XT_THREADS, 3)
    fft_x_fwd(const __grid_constant__ DevGrid G, const __grid_constant__ FftPlan1 P, const __grid_constant__ XArgs A)
{
    fft_x_fwd_run<C>(G, P, A, blockIdx.x);
}

// -------------------- steps 2/4: y transform --------------------
constexpr int YROWS = 4;   // (k,kx) rows per block

template <typename C>
__device__ __forceinline__ void fft_y_run(const FftPlan1 &P, void *spec_v, int nrows, int inv, const Skip &sk, const int bid)
{
    if (converged(sk)) return;
    extern __shared__ double2 smraw_y[];
    C *smc = reinterpret_cast<C *>(smraw_y);
    C *spec = reinterpret_cast<C *>(spec_v);
    const int n = P.n;
    const int nt_row = blockDim.x / YROWS;
    const int rr = threadIdx.x / nt_row, lt = threadIdx.x % nt_row;
    const long long row = (long long)bid * YROWS + rr;
    const int np = padded_len(n);
    C *a = smc + rr * 2 * np, *b = a + np;
    const bool ok = row < nrows;
    if (ok) {   // YI elements per thread at a time, their loads issued before the shared stores
        constexpr int YI = 8;
        for (int t0 = lt; t0 < n; t0 += YI * nt_row) {
            C v[YI];
#pragma unroll
            for (int q = 0; q < YI; q++) {
                const int t = t0 + q * nt_row;
                if (t < n) v[q] = spec[row * n + t];
            }
#pragma unroll
            for (int q = 0; q < YI; q++) {
                const int t = t0 + q * nt_row;
                if (t < n) a[pidx(t)] = v[q];
            }
        }
    }
    __syncthreads();
    C *res = stockham<C>(P, a, b, lt, nt_row, inv);
    if (ok)
        for (int t = lt; t < n; t += nt_row) spec[row * n + t] = res[pidx(t)];
}
template <typename C>
__global__ void fft_y(DevGrid G, const __grid_constant__ FftPlan1 P, void *spec_v, int nrows, int inv, Skip sk)
{
    (void)G;
    fft_y_run<C>(P, spec_v, nrows, inv, sk, blockIdx.x);
}

// FP32 spectra with n = 32*M, M a power of two from 2 to 16: one warp per row, no shared
// memory.  The row is a 32 x M matrix, element j1 + 32 j2 in lane j1 (a coalesced load):
// each lane transforms its M values in registers (radix 2), multiplies by the twiddles
// W_n^(j1 k2), and the 32-point transforms across the lanes run as five radix-2
// butterfly stages over __shfl_xor_sync; lane l then holds the outputs k2 + M*brev5(l),
// k2 = 0..M-1, which it stores as M/2 16-byte vectors.  Measured at 512 (65,792 rows):
// 167 us per launch against 213 us for the shared-memory Stockham transform.
constexpr int YW_WARPS = 8;   // rows (warps) per block of the shuffle transform
__host__ __device__ constexpr bool yshfl_ok(int n)
{
    return n == 64 || n == 128 || n == 256 || n == 512;
}
// the bit reversal of a within log2(m) bits (m a power of two)
__host__ __device__ constexpr int brev_bits(int a, int m)
{
    int r = 0;
    for (int b = 1; b < m; b <<= 1) r = (r << 1) | ((a & b) ? 1 : 0);
    return r;
}
template <int M>
__device__ __forceinline__ void yshfl_row(float2 *x, const float2 *__restrict__ tw, int inv)
{
    constexpr int n = 32 * M;
    const int lane = threadIdx.x & 31;
    float2 v[M];
#pragma unroll
    for (int j2 = 0; j2 < M; j2++) v[j2] = x[lane + 32 * j2];
    auto twiddle = [&](int t) {   // W_n^t, conjugated for the inverse
        float2 w = __ldg(tw + t);
        if (inv) w.y = -w.y;
        return w;
    };
    // M-point transforms over j2: bit reversal, then radix-2 stages (W_len^q = W_n^(q n/len))
#pragma unroll
    for (int a = 1; a < M; a++) {
        const int b = brev_bits(a, M);
        if (a < b) { const float2 t = v[a]; v[a] = v[b]; v[b] = t; }
    }
#pragma unroll
    for (int len = 2; len <= M; len <<= 1) {
        const int half = len >> 1;
#pragma unroll
        for (int st = 0; st < M; st += len)
#pragma unroll
            for (int q = 0; q < half; q++) {
                const float2 w = twiddle(q * (n / len));
                const float2 a = v[st + q], b = v[st + q + half];
                const float2 bw = make_float2(b.x * w.x - b.y * w.y, b.x * w.y + b.y * w.x);
                v[st + q] = make_float2(a.x + bw.x, a.y + bw.y);
                v[st + q + half] = make_float2(a.x - bw.x, a.y - bw.y);
            }
    }
#pragma unroll
    for (int k2 = 1; k2 < M; k2++) {
        const float2 w = twiddle((lane * k2) % n), a = v[k2];
        v[k2] = make_float2(a.x * w.x - a.y * w.y, a.x * w.y + a.y * w.x);
    }
    // 32-point transforms across the lanes: decimation in frequency, partner lane ^ s; the
    // upper lane's difference takes W_(2s)^(lane mod s) = W_n^((lane mod s) n/(2s))
#pragma unroll
    for (int s = 16; s >= 1; s >>= 1) {
        const bool upper = (lane & s) != 0;
        const float2 w = twiddle((lane & (s - 1)) * (n / (2 * s)));
#pragma unroll
        for (int k2 = 0; k2 < M; k2++) {
            const float ox = __shfl_xor_sync(0xffffffffu, v[k2].x, s);
            const float oy = __shfl_xor_sync(0xffffffffu, v[k2].y, s);
            if (!upper) {
                v[k2] = make_float2(v[k2].x + ox, v[k2].y + oy);
            } else {
                const float dx = ox - v[k2].x, dy = oy - v[k2].y;
                v[k2] = make_float2(dx * w.x - dy * w.y, dx * w.y + dy * w.x);
            }
        }
    }
    const int k1 = (int)(__brev((unsigned)lane) >> 27);
    float4 *o = reinterpret_cast<float4 *>(x + M * k1);
#pragma unroll
    for (int q = 0; q < M / 2; q++) o[q] = make_float4(v[2 * q].x, v[2 * q].y, v[2 * q + 1].x, v[2 * q + 1].y);
}
// bid: the block's index in the domain's own grid of (nrows / YW_WARPS) blocks
template <int M>
__device__ __forceinline__ void fft_y_shfl_run(const FftPlan1 &P, void *spec_v, int nrows, int inv, const Skip &sk,
                                               const int bid)
{
    if (converged(sk)) return;
    const long long row = (long long)bid * YW_WARPS + (threadIdx.x >> 5);
    if (row >= nrows) return;   // whole warps leave together
    yshfl_row<M>(reinterpret_cast<float2 *>(spec_v) + row * P.n, P.twf, inv);
}
template <int M>
__global__ void __launch_bounds__(32 * YW_WARPS) fft_y_shfl(const __grid_constant__ FftPlan1 P, void *spec_v, int nrows,
                                                            int inv, Skip sk)
{
    fft_y_shfl_run<M>(P, spec_v, nrows, inv, sk, blockIdx.x);
}
inline cudaError_t launch_y_shfl(const FftPlan1 &P, void *spec, int nrows, int inv, Skip sk, cudaStream_t s)
{
    const unsigned nb = (unsigned)((nrows + YW_WARPS - 1) / YW_WARPS);
    switch (P.n) {
    case 64: fft_y_shfl<2><<<nb, 32 * YW_WARPS, 0, s>>>(P, spec, nrows, inv, sk); break;
    case 128: fft_y_shfl<4><<<nb, 32 * YW_WARPS, 0, s>>>(P, spec, nrows, inv, sk); break;
    case 256: fft_y_shfl<8><<<nb, 32 * YW_WARPS, 0, s>>>(P, spec, nrows, inv, sk); break;
    default: fft_y_shfl<16><<<nb, 32 * YW_WARPS, 0, s>>>(P, spec, nrows, inv, sk); break;
    }
    return cudaGetLastError();
}

// -------------------- step 3: vertical tridiagonal --------------------
struct TriArgs {
    void *spec;
    double2 *scratch;        // mixed form: FP64 forward values [k][kx][ky]; null in the plain form
    const double *gam;       // [k][kx][ky], k = 2..nz (index k-1); k=1 unused
    const double *wv;        // wv(l,m), l fastest over maxx
    const double *ak, *ck, *dka, *dkb;   // per level coefficients (host-computed)
    int keep00;
    Skip sk;
};

__device__ __forceinline__ double dk_of(const TriArgs &T, int k, int nz, double wl)
{
    if (k == 1) return wl - __ldg(T.dka) - __ldg(T.dkb);
    if (k == nz) return wl - __ldg(T.dka + nz - 1) + __ldg(T.dkb + nz - 1);
    return wl - __ldg(T.dka + k - 1);
}

// The elimination runs in FP64 in both forms, including the values carried between the
// sweeps: the near-singular low-wavenumber columns amplify any rounding of them, and the
// divergence residual barely sees errors in those modes, so refinement could not repair
// them.  The mixed form reads its FP32 right-hand side, keeps the forward values in an
// FP64 scratch spectrum and writes the FP32 solution.
__device__ __forceinline__ double2 ld_spec(const double2 *s) { return *s; }
__device__ __forceinline__ double2 ld_spec(const float2 *s) { float2 v = *s; return make_double2(v.x, v.y); }
__device__ __forceinline__ void st_spec(double2 *s, double2 v) { *s = v; }
__device__ __forceinline__ void st_spec(float2 *s, double2 v) { *s = make_float2((float)v.x, (float)v.y); }

template <typename C>
__device__ __forceinline__ void tridiag_run(const DevGrid &G, const TriArgs &T, const int bid)
{
    if (converged(T.sk)) return;
    const int nh = G.maxx / 2 + 1, maxy = G.maxy, nz = G.nz;
    const long long col = (long long)bid * blockDim.x + threadIdx.x;
    if (col >= (long long)nh * maxy) return;
    const int kx = (int)(col / maxy), ky = (int)(col % maxy);
    const long long lstride = (long long)nh * maxy;
    C *s = reinterpret_cast<C *>(T.spec) + (long long)kx * maxy + ky;
    // forward values: in place (plain form) or in the FP64 scratch (mixed form)
    double2 *u64 = T.scratch ? T.scratch + (long long)kx * maxy + ky : reinterpret_cast<double2 *>(s);
    if (kx == 0 && ky == 0) {
        if (!T.keep00)
            for (int k = 0; k < nz; k++) st_spec(s + k * lstride, make_double2(0., 0.));
        return;
    }
    const double wl = __ldg(T.wv + (long long)ky * G.maxx + kx);
    const double *gam = T.gam + (long long)kx * maxy + ky;
    // forward elimination (TRIDAG2 :219-229), complex rhs solved as its two real parts;
    // the loads of TB levels are issued together ahead of their dependent chain
    constexpr int TB = 8;
    double2 uprev = make_double2(0., 0.);
    for (int k0 = 1; k0 <= nz; k0 += TB) {
        double2 rr[TB];
        double gg[TB];
#pragma unroll
        for (int u = 0; u < TB; u++) {
            const int k = k0 + u;
            if (k <= nz) {
                rr[u] = ld_spec(s + (k - 1) * lstride);
                gg[u] = k >= 2 ? __ldg(gam + (k - 1) * lstride) : 0.;
            }
        }
#pragma unroll
        for (int u = 0; u < TB; u++) {
            const int k = k0 + u;
            if (k <= nz) {
                const double a = k >= 2 ? __ldg(T.ak + k - 1) : 0.;
                const double bet = k >= 2 ? dk_of(T, k, nz, wl) - a * gg[u] : dk_of(T, 1, nz, wl);
                const double2 uk = make_double2((rr[u].x - a * uprev.x) / bet, (rr[u].y - a * uprev.y) / bet);
                u64[(k - 1) * lstride] = uk;
                uprev = uk;
            }
        }
    }
    // back substitution (:231-233), TB levels of loads at a time
    st_spec(s + (nz - 1) * lstride, uprev);
    for (int k0 = nz - 1; k0 >= 1; k0 -= TB) {
        double2 uu[TB];
        double gg[TB];
#pragma unroll
        for (int u = 0; u < TB; u++) {
            const int k = k0 - u;
            if (k >= 1) {
                uu[u] = u64[(k - 1) * lstride];
                gg[u] = __ldg(gam + k * lstride);   // GAM(k+1)
            }
        }
#pragma unroll
        for (int u = 0; u < TB; u++) {
            const int k = k0 - u;
            if (k >= 1) {
                const double2 uk = make_double2(uu[u].x - gg[u] * uprev.x, uu[u].y - gg[u] * uprev.y);
                st_spec(s + (k - 1) * lstride, uk);
                uprev = uk;
            }
        }
    }
}

template <typename C>
__global__ void tridiag_kernel(const __grid_constant__ DevGrid G, const __grid_constant__ TriArgs T)
{
    tridiag_run<C>(G, T, blockIdx.x);
}

// GAM(k) = C(k-1)/BET(k-1), BET(k) = B(k) - A(k)*GAM(k); zero pivots flagged
__global__ void gam_kernel(DevGrid G, TriArgs T, double *gam, int *err)
{
    const int nh = G.maxx / 2 + 1, maxy = G.maxy, nz = G.nz;
    const long long col = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= (long long)nh * maxy) return;
    const int kx = (int)(col / maxy), ky = (int)(col % maxy);
    const long long lstride = (long long)nh * maxy;
    const double wl = __ldg(T.wv + (long long)ky * G.maxx + kx);
    const bool skip = (kx == 0 && ky == 0);
    double bet = dk_of(T, 1, nz, wl);
    if (bet == 0. && !skip) atomicOr(err, 1);
    gam[col] = 0.;
    for (int k = 2; k <= nz; k++) {
        double g = __ldg(T.ck + k - 2) / bet;
        gam[(k - 1) * lstride + col] = g;
        bet = dk_of(T, k, nz, wl) - __ldg(T.ak + k - 1) * g;
        if (bet == 0. && !skip) atomicOr(err, 2);
    }
}

// -------------------- step 5: inverse x transform --------------------
__device__ __forceinline__ void prefetch_l2(const void *p)
{
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}
struct XInvArgs {
    const void *spec;
    double *dp;          // [nz][maxy][maxx] real
    double scale_div;    // divide by this (N_h), or 1
    int accumulate;      // refinement pass: dp += solution
    Skip sk;
};

template <typename C>
__device__ __forceinline__ void fft_x_inv_run(const DevGrid &G, const FftPlan1 &P, const XInvArgs &A, const int bid)
{
    if (converged(A.sk)) return;
    using R = typename CT<C>::R;
    extern __shared__ double2 smraw_xi[];
    C *smc = reinterpret_cast<C *>(smraw_xi);
    const C *spec = reinterpret_cast<const C *>(A.spec);
    const int n = P.n, nh = n / 2 + 1, maxy = G.maxy;
    const int groups = (maxy + ROWS - 1) / ROWS;
    const int k = bid / groups + 1, jg = bid % groups;
    const int jb = jg * ROWS;
    const int nt_pair = blockDim.x / (ROWS / 2);
    const int pair = threadIdx.x / nt_pair, lt = threadIdx.x % nt_pair;
    const int np = padded_len(n);
    C *ahalf = smc, *bhalf = smc + (ROWS / 2) * np;
    C *a = ahalf + pair * np, *b = bhalf + pair * np;
    const int r0 = jb + 2 * pair, r1 = r0 + 1;
    // the block's half spectra for kx < n/2, 8 consecutive ky per kx, staged in the b half
    const int hn = n / 2;
    // XI elements per thread at a time, all their loads issued before the shared stores
    constexpr int XI = 8;
    for (int e0 = threadIdx.x; e0 < hn * ROWS; e0 += XI * blockDim.x) {
        C v[XI];
#pragma unroll
        for (int q = 0; q < XI; q++) {
            const int e = e0 + q * blockDim.x;
            const int kx = e / ROWS, jr = jb + (e - kx * ROWS);
            v[q] = (e < hn * ROWS && jr < maxy) ? spec[((long long)(k - 1) * nh + kx) * maxy + jr] : mkc<C>(0, 0);
        }
#pragma unroll
        for (int q = 0; q < XI; q++) {
            const int e = e0 + q * blockDim.x;
            const int kx = e / ROWS, c = e - kx * ROWS;
            if (e < hn * ROWS) bhalf[stg<C>(kx, c)] = v[q];
        }
    }
    __syncthreads();
    // rebuild Z_k = A_k + i B_k over the full circle from the half spectra
    for (int kx = lt; kx < nh; kx += nt_pair) {
        C Av, Bv;
        if (kx < hn) {
            Av = bhalf[stg<C>(kx, 2 * pair)];
            Bv = bhalf[stg<C>(kx, 2 * pair + 1)];
        } else {
            const long long base = ((long long)(k - 1) * nh + kx) * maxy;
            Av = r0 < maxy ? spec[base + r0] : mkc<C>(0, 0);
            Bv = r1 < maxy ? spec[base + r1] : mkc<C>(0, 0);
        }
        a[pidx(kx)] = mkc<C>(Av.x - Bv.y, Av.y + Bv.x);
        if (kx > 0 && kx < n - kx) a[pidx(n - kx)] = mkc<C>(Av.x + Bv.y, Bv.x - Av.y);
    }
    __syncthreads();   // the b half is scratch for the transform from here on
    if (A.accumulate) {   // the rows dp is added to, brought into L2 while the transform runs
        for (int t = lt; t < n; t += nt_pair) {
            const long long o0 = ((long long)(k - 1) * maxy + r0) * G.maxx + t;
            if (r0 < maxy) prefetch_l2(A.dp + o0);
            if (r1 < maxy) prefetch_l2(A.dp + o0 + G.maxx);
        }
    }
    C *res = stockham<C>(P, a, b, lt, nt_pair, 1);
    for (int t = lt; t < n; t += nt_pair) {
        C z = res[pidx(t)];
        const long long o0 = ((long long)(k - 1) * maxy + r0) * G.maxx + t, o1 = o0 + G.maxx;
        if (A.accumulate) {
            if (r0 < maxy) A.dp[o0] = A.dp[o0] + (double)z.x / A.scale_div;
            if (r1 < maxy) A.dp[o1] = A.dp[o1] + (double)z.y / A.scale_div;
        } else {
            if (r0 < maxy) A.dp[o0] = (double)z.x / A.scale_div;
            if (r1 < maxy) A.dp[o1] = (double)z.y / A.scale_div;
        }
    }
    (void)sizeof(R);
}
template <typename C>
__global__ void __launch_bounds__(XT_THREADS, 3)
    fft_x_inv(const __grid_constant__ DevGrid G, const __grid_constant__ FftPlan1 P, const __grid_constant__ XInvArgs A)
{
    fft_x_inv_run<C>(G, P, A, blockIdx.x);
}

// -------------------- step 6: correction --------------------
// The blocks of a level are consecutive (corr_blocks_per_level of them), so a thread finds
// its level and cell with 32-bit arithmetic; 1/dx and 1/dy come from the host.
__host__ __device__ inline unsigned corr_blocks_per_level(const DevGrid &G, unsigned threads)
{
    return ((unsigned)G.maxx * (unsigned)G.maxy + threads - 1) / threads;
}
__device__ __forceinline__ void correction_run(const DevGrid &G, const double *dp, double *mu, double *mv, double *mw,
                                               double *p, int natural_uv, double dx1, double dy1, const int bid)
{
    const int maxx = G.maxx, maxy = G.maxy;
    const unsigned plane = (unsigned)maxx * (unsigned)maxy, bpl = corr_blocks_per_level(G, blockDim.x);
    const unsigned kl = (unsigned)bid / bpl;
    const unsigned rem = ((unsigned)bid - kl * bpl) * blockDim.x + threadIdx.x;
    if (rem >= plane || (int)kl >= G.nz) return;
    const int k = (int)kl + 1, jy = (int)(rem / (unsigned)maxx), ix = (int)(rem - (unsigned)jy * (unsigned)maxx);
    const int i = ix + 4, j = jy + 4;
    auto DP = [&](int a, int b, int kk) { return __ldg(dp + ((long long)(kk - 1) * maxy + b) * maxx + a); };
    const double d0 = __ldg(G.den0 + k - 1), a0 = __ldg(G.avden0 + k - 1);
    const double dpc = DP(ix, jy, k);
    const long long c = gidx(G, i, j, k);
    p[c] = p[c] + d0 * dpc;
    const double gpx = (dpc - DP(ix == 0 ? maxx - 1 : ix - 1, jy, k)) * dx1;
    const double gpy = (dpc - DP(ix, jy == 0 ? maxy - 1 : jy - 1, k)) * dy1;
    double gpz;
    if (k >= 2) gpz = (dpc - DP(ix, jy, k - 1)) * __ldg(G.dz1 + k - 2);
    else gpz = mw[c] / (G.dt0 * __ldg(G.avden0));
    const double mun = mu[c] - G.dt0 * d0 * gpx;
    const double mvn = mv[c] - G.dt0 * d0 * gpy;
    mw[c] = mw[c] - G.dt0 * a0 * gpz;
    // last correction of a step: get_velocities (funcpack.f90:328-334) fused for u, v
    mu[c] = natural_uv ? mun / d0 : mun;
    mv[c] = natural_uv ? mvn / d0 : mvn;
}
__global__ void correction_kernel(const __grid_constant__ DevGrid G, const double *dp, double *mu, double *mv, double *mw,
                                  double *p, int natural_uv, double dx1, double dy1)
{
    correction_run(G, dp, mu, mv, mw, p, natural_uv, dx1, dy1, blockIdx.x);
}

// -------------------- reductions --------------------
// per-level sums over the interior, fixed-order tree (deterministic)
// one block of LSUM_THREADS threads per level (a fixed-order tree: the sums do not depend
// on the launch); 1024 threads so that a few hundred levels fill the GPU
constexpr int LSUM_THREADS = 1024;
__device__ __forceinline__ void level_sums_run(const DevGrid &G, const double *x, const double *xold, int old_rep,
                                               double dt0, double *out_mean, double *out_mean_d, const int bid)
{
    __shared__ double s1[LSUM_THREADS], s2[LSUM_THREADS];
    const int k = bid + 1;
    const int maxx = G.maxx, maxy = G.maxy;
    const double a0 = __ldg(G.avden0 + k - 1);
    double acc = 0., accd = 0.;
    // q = jy * maxx + ix runs from threadIdx.x in steps of blockDim.x; (ix, jy) advance
    // incrementally instead of by a division per element
    // LI elements at a time: all their loads first, then the sums in element order
    constexpr int LI = 8;
    int ix = (int)threadIdx.x % maxx, jy = (int)threadIdx.x / maxx;
    while (jy < maxy) {
        double v[LI], wo[LI];
        bool in[LI];
#pragma unroll
        for (int q = 0; q < LI; q++) {
            in[q] = jy < maxy;
            v[q] = 0.;
            wo[q] = 0.;
            if (in[q]) {
                const long long c = gidx(G, ix + 4, jy + 4, k);
                v[q] = x[c];
                if (out_mean_d) wo[q] = __ldg(xold + c);
            }
            ix += blockDim.x;
            while (ix >= maxx) { ix -= maxx; ++jy; }
        }
#pragma unroll
        for (int q = 0; q < LI; q++) {
            if (!in[q]) continue;
            acc += v[q];
            if (out_mean_d) {
                double w = wo[q];
                if (old_rep >= 0) w = rep_value(old_rep, w, a0);
                accd += (v[q] - w) / dt0;
            }
        }
    }
    s1[threadIdx.x] = acc;
    s2[threadIdx.x] = accd;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            s1[threadIdx.x] += s1[threadIdx.x + w];
            s2[threadIdx.x] += s2[threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double nn = (double)maxx * (double)maxy;
        out_mean[k - 1] = s1[0] / nn;
        if (out_mean_d) out_mean_d[k - 1] = s2[0] / nn;
    }
}
__global__ void __launch_bounds__(LSUM_THREADS) level_sums(const __grid_constant__ DevGrid G, const double *x, const double *xold, int old_rep, double dt0,
                           double *out_mean, double *out_mean_d)
{
    level_sums_run(G, x, xold, old_rep, dt0, out_mean, out_mean_d, blockIdx.x);
}

// w -= <w>_k over all cells (cal_p1 :786-790); natural_w: then w/avden0 (get_velocities)
__device__ __forceinline__ void subtract_level_mean_run(const DevGrid &G, double *x, const double *mean, int natural_w,
                                                        const int bid, const int nblk)
{
    const long long n = G.ps * G.nz, ps = G.ps, stride = (long long)nblk * blockDim.x;
    // the level of element t advances with t (one 64-bit division per thread, not per
    // element), and SI elements per thread are loaded before any is written back
    long long t = (long long)bid * blockDim.x + threadIdx.x;
    long long k0 = t / ps, rem = t - k0 * ps;
    constexpr int SI = 4;
    while (t < n) {
        double v[SI];
        long long tt[SI];
        int kk[SI];
#pragma unroll
        for (int q = 0; q < SI; q++) {
            tt[q] = t;
            kk[q] = (int)k0;
            v[q] = t < n ? x[t] : 0.;
            t += stride;
            rem += stride;
            while (rem >= ps) { rem -= ps; ++k0; }
        }
#pragma unroll
        for (int q = 0; q < SI; q++) {
            if (tt[q] >= n) break;
            const double w = v[q] - __ldg(mean + kk[q]);
            x[tt[q]] = natural_w ? w / __ldg(G.avden0 + kk[q]) : w;
        }
    }
}
__global__ void subtract_level_mean(const __grid_constant__ DevGrid G, double *x, const double *mean, int natural_w)
{
    subtract_level_mean_run(G, x, mean, natural_w, blockIdx.x, gridDim.x);
}

__global__ void to_velocity_kernel(DevGrid G, double *mu, double *mv, double *mw)
{
    const long long n = G.ps * G.nz;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        int k = (int)(t / G.ps) + 1;
        const double d0 = __ldg(G.den0 + k - 1), a0 = __ldg(G.avden0 + k - 1);
        mu[t] = mu[t] / d0;
        mv[t] = mv[t] / d0;
        mw[t] = mw[t] / a0;
    }
}

__global__ void p1_kernel(DevGrid G, const double *wavd, double *p1)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int nz = G.nz;
    p1[nz - 1] = 0.;
    for (int k = nz - 1; k >= 1; k--)
        p1[k - 1] = p1[k] + wavd[k] * 0.5 * G.dz * (G.fdz0[k - 1] + G.fdz0[k]);
}

// caldiv over the interior, k = 2..nz-1, signed max (pressure_solver.f90:121-130), of the
// momentum; natural = 1: the inputs are velocities, and the momentum is formed on the fly as
// get_momentum does (rho0(k) u, rho0(k) v, avden0(k) w)
__global__ void maxdiv_kernel(DevGrid G, const double *mu, const double *mv, const double *mw, int natural,
                              double *partial)
{
    __shared__ double sm[256];
    const int maxx = G.maxx, maxy = G.maxy;
    const double dx1 = 1. / G.dx, dy1 = 1. / G.dy;
    double m = -INFINITY;
    const long long tot = (long long)maxx * maxy * (G.nz - 2);
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += (long long)gridDim.x * blockDim.x) {
        int ix = (int)(t % maxx), jy = (int)((t / maxx) % maxy), k = (int)(t / ((long long)maxx * maxy)) + 2;
        long long c = gidx(G, ix + 4, jy + 4, k);
        double d = 0.;
        if (natural) {
            const double r = __ldg(G.den0 + k - 1), a0 = __ldg(G.avden0 + k - 1), a1 = __ldg(G.avden0 + k);
            d = d + (r * mu[c + 1] - r * mu[c]) * dx1;
            d = d + (r * mv[c + G.px] - r * mv[c]) * dy1;
            d = d + (a1 * mw[c + G.ps] - a0 * mw[c]) * __ldg(G.dz1w + k - 1);
        } else {
            d = d + (mu[c + 1] - mu[c]) * dx1;
            d = d + (mv[c + G.px] - mv[c]) * dy1;
            d = d + (mw[c + G.ps] - mw[c]) * __ldg(G.dz1w + k - 1);
        }
        m = fmax(m, d);
    }
    sm[threadIdx.x] = m;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) sm[threadIdx.x] = fmax(sm[threadIdx.x], sm[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = sm[0];
}

__global__ void max_final(const double *partial, int n, double *out)
{
    __shared__ double sm[256];
    double m = -INFINITY;
    for (int t = threadIdx.x; t < n; t += blockDim.x) m = fmax(m, partial[t]);
    sm[threadIdx.x] = m;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) sm[threadIdx.x] = fmax(sm[threadIdx.x], sm[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = sm[0];
}

// copy a halo'd field's interior into a dense [nz][maxy][maxx] buffer and back
__global__ void interior_gather(DevGrid G, const double *src, double *dst)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)G.maxx * G.maxy * G.nz) return;
    int ix = (int)(t % G.maxx), jy = (int)((t / G.maxx) % G.maxy), k = (int)(t / ((long long)G.maxx * G.maxy)) + 1;
    dst[t] = src[gidx(G, ix + 4, jy + 4, k)];
}
__global__ void interior_scatter(DevGrid G, const double *src, double *dst)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)G.maxx * G.maxy * G.nz) return;
    int ix = (int)(t % G.maxx), jy = (int)((t / G.maxx) % G.maxy), k = (int)(t / ((long long)G.maxx * G.maxy)) + 1;
    dst[gidx(G, ix + 4, jy + 4, k)] = src[t];
}

// ghost cells := periodic images (statebc/windbc serial periodic branches)
struct HaloArgs { double *f[MG_MAXF]; int nf; };
__device__ __forceinline__ void halo_fill_run(const DevGrid &G, const HaloArgs &H, const int bid, const int nblk)
{
    // 32-bit index arithmetic: at most 5 (nx + maxy) < 41,100 ghost cells per level and
    // 4096 levels, below 2^31
    const int nx = G.nx, ny = G.ny, maxx = G.maxx, maxy = G.maxy;
    const unsigned per_plane = 5u * (unsigned)nx + 5u * (unsigned)maxy;
    const unsigned tot = per_plane * (unsigned)G.nz;
    for (unsigned t = (unsigned)bid * blockDim.x + threadIdx.x; t < tot; t += (unsigned)nblk * blockDim.x) {
        const unsigned kq = t / per_plane;
        const int k = (int)kq + 1;
        const unsigned g = t - kq * per_plane;
        int i, j;
        if (g < 5u * (unsigned)nx) {
            const int r = (int)(g / (unsigned)nx);
            i = (int)(g - (unsigned)r * (unsigned)nx) + 1;
            j = r < 3 ? r + 1 : ny - 4 + r;   // 1,2,3, ny-1, ny
        } else {
            const unsigned g2 = g - 5u * (unsigned)nx;
            j = (int)(g2 / 5u) + 4;
            const int c = (int)(g2 - (g2 / 5u) * 5u);
            i = c < 3 ? c + 1 : nx - 4 + c;
        }
        int si = i <= 3 ? i + maxx : (i >= nx - 1 ? i - maxx : i);
        int sj = j <= 3 ? j + maxy : (j >= ny - 1 ? j - maxy : j);
        long long dsti = gidx(G, i, j, k), srci = gidx(G, si, sj, k);
        for (int f = 0; f < H.nf; f++) H.f[f][dsti] = H.f[f][srci];
    }
}
__global__ void halo_fill_kernel(const __grid_constant__ DevGrid G, const __grid_constant__ HaloArgs H)
{
    halo_fill_run(G, H, blockIdx.x, gridDim.x);
}

// download conversion (get_velocities / get_scalars, funcpack.f90:65-178,429-485): the
// natural value of a resident field (REP_CONS: divided by its weight) written into a
// packed nx*ny*nz array (the reference layout without the row padding of the device
// layout), so that the host copy is one linear transfer
__global__ void to_natural_packed_kernel(DevGrid G, const double *src, const double *w, int kind, int rep, double *dst)
{
    const long long n = (long long)G.nx * G.ny * G.nz, plane = (long long)G.nx * G.ny;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(t / plane) + 1;
        const long long r = t - (k - 1) * plane;
        const int j = (int)(r / G.nx) + 1, i = (int)(r - (long long)(j - 1) * G.nx) + 1;
        const long long q = gidx(G, i, j, k);
        double x = src[q];
        if (rep == REP_CONS) {
            if (kind == 1) x = x / __ldg(G.den0 + k - 1);
            else if (kind == 2) x = x / __ldg(G.avden0 + k - 1);
            else if (kind == 3) x = x / w[q];
        }
        dst[t] = x;
    }
}

// packed nx*ny*nz -> device layout (the padding columns are left as they are)
__global__ void unpack_kernel(DevGrid G, const double *src, double *dst)
{
    const long long n = (long long)G.nx * G.ny * G.nz;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const long long row = t / G.nx;
        dst[row * G.px + (t - row * G.nx)] = src[t];
    }
}

// -------------------- grouped launches over several domains --------------------
// Each grouped kernel runs, in block b of its launch, block items[b].b of member
// items[b].m's own grid with that member's arguments (global memory, written before
// the launch and unchanged while it runs).  The bodies are the single-domain ones.
struct XFwdMember { DevGrid G; FftPlan1 P; XArgs A; };
struct YMember { FftPlan1 P; void *spec; int nrows, inv; Skip sk; };
struct TriMember { DevGrid G; TriArgs T; };
struct XInvMember { DevGrid G; FftPlan1 P; XInvArgs A; };
struct CorrMember { DevGrid G; const double *dp; double *mu, *mv, *mw, *p; int natural_uv; double dx1, dy1; };
struct LevelMember { DevGrid G; double *w; const double *wold; int wold_rep; double *mean; int natural_w, nb; };
struct HaloMember { DevGrid G; HaloArgs H; int nb; };

template <typename C>
__global__ void __launch_bounds__(XT_THREADS, 3) fft_x_fwd_grp(const XFwdMember *__restrict__ mem, const GItem *__restrict__ it)
{
    const GItem g = it[blockIdx.x];
    fft_x_fwd_run<C>(mem[g.m].G, mem[g.m].P, mem[g.m].A, g.b);
}
template <int M>
__global__ void __launch_bounds__(32 * YW_WARPS) fft_y_shfl_grp(const YMember *__restrict__ mem,
                                                                 const GItem *__restrict__ it)
{
    const GItem g = it[blockIdx.x];
    const YMember m = mem[g.m];   // a register copy: the row transform keeps its values in registers
    fft_y_shfl_run<M>(m.P, m.spec, m.nrows, m.inv, m.sk, g.b);
}
template <typename C>
__global__ void fft_y_grp(const YMember *__restrict__ mem, const GItem *__restrict__ it)
{
    const GItem g = it[blockIdx.x];
    const YMember &m = mem[g.m];
    fft_y_run<C>(m.P, m.spec, m.nrows, m.inv, m.sk, g.b);
}
template <typename C>
__global__ void tridiag_grp(const TriMember *__restrict__ mem, const GItem *__restrict__ it)
{
    const GItem g = it[blockIdx.x];
    tridiag_run<C>(mem[g.m].G, mem[g.m].T, g.b);
}
template <typename C>
__global__ void __launch_bounds__(XT_THREADS, 3) fft_x_inv_grp(const XInvMember *__restrict__ mem, const GItem *__restrict__ it)
{
    const GItem g = it[blockIdx.x];
    fft_x_inv_run<C>(mem[g.m].G, mem[g.m].P, mem[g.m].A, g.b);
}
__global__ void correction_grp(const CorrMember *__restrict__ mem, const GItem *__restrict__ it)
{
    const GItem g = it[blockIdx.x];
    const CorrMember &m = mem[g.m];
    correction_run(m.G, m.dp, m.mu, m.mv, m.mw, m.p, m.natural_uv, m.dx1, m.dy1, g.b);
}
__global__ void __launch_bounds__(LSUM_THREADS) level_sums_grp(const LevelMember *__restrict__ mem,
                                                               const GItem *__restrict__ it)
{
    const GItem g = it[blockIdx.x];
    const LevelMember &m = mem[g.m];
    level_sums_run(m.G, m.w, m.wold, m.wold_rep, m.G.dt0, m.mean, nullptr, g.b);
}
__global__ void subtract_level_mean_grp(const LevelMember *__restrict__ mem, const GItem *__restrict__ it)
{
    const GItem g = it[blockIdx.x];
    const LevelMember &m = mem[g.m];
    subtract_level_mean_run(m.G, m.w, m.mean, m.natural_w, g.b, m.nb);
}
__global__ void halo_fill_grp(const HaloMember *__restrict__ mem, const GItem *__restrict__ it)
{
    const GItem g = it[blockIdx.x];
    halo_fill_run(mem[g.m].G, mem[g.m].H, g.b, mem[g.m].nb);
}
// block m zeroes member m's residual slots
__global__ void resid_reset_grp(unsigned long long *const *__restrict__ resid)
{
    unsigned long long *r = resid[blockIdx.x];
    for (int q = threadIdx.x; q < MG_MAXPASS; q += blockDim.x) r[q] = 0ull;
}

// -------------------- host side: plan --------------------
bool factorize(int n, FftPlan1 *P)
{
    int m = n, s = 0;
    unsigned long long pk = 0;
    auto put = [&](int r) { pk |= (unsigned long long)r << (4 * s); s++; m /= r; };
    while (m % 8 == 0 && s < MAXSTAGES) put(8);
    while (m % 4 == 0 && s < MAXSTAGES) put(4);
    while (m % 2 == 0 && s < MAXSTAGES) put(2);
    while (m % 3 == 0 && s < MAXSTAGES) put(3);
    while (m % 5 == 0 && s < MAXSTAGES) put(5);
    P->nst = s;
    P->rpack = pk;
    return m == 1;
}

}  // namespace

struct PressurePlan {
    FftPlan1 px, py;
    double2 *twx = nullptr, *twy = nullptr;
    float2 *twxf = nullptr, *twyf = nullptr;
    int mixed = 0;                 // FP32 spectra and transforms
    double2 *tri = nullptr;        // mixed form: FP64 values between the tridiagonal sweeps
    double2 *spec = nullptr;       // [nz][nh][maxy]
    double *dp = nullptr;          // [nz][maxy][maxx]
    double *rbuf = nullptr;        // [nz][maxy][maxx] external rhs
    double *gam = nullptr;         // [nz][nh][maxy]
    double *wv = nullptr;          // [maxy][maxx]
    double *ak = nullptr, *ck = nullptr, *dka = nullptr, *dkb = nullptr;
    double *mean = nullptr, *mean_d = nullptr, *p1 = nullptr;
    double *partial = nullptr, *maxdiv = nullptr;
    unsigned long long *resid = nullptr;   // [MG_MAXPASS] residual per pass of the current projection
    double *bsum = nullptr;                // [nz][row groups] sums of b (refined projection)
    double *gamT = nullptr, *akT = nullptr, *ckT = nullptr;   // transposed system (adjoint), built on first use
    int npartial = 0;
    size_t bytes = 0;
    int xt = 32, yt = 32, tb = 128;   // launch shapes (threads per x row pair, per y row, per tridiagonal block)
};

static cudaError_t make_twiddles(int n, double2 **out)
{
    std::vector<double2> h(n);
    const long double PI = 3.141592653589793238462643383279502884L;
    for (int t = 0; t < n; t++) {
        long double ang = -2.0L * PI * (long double)t / (long double)n;
        h[t] = make_double2((double)cosl(ang), (double)sinl(ang));
    }
    cudaError_t e = cudaMalloc(out, n * sizeof(double2));
    if (e != cudaSuccess) return e;
    return cudaMemcpy(*out, h.data(), n * sizeof(double2), cudaMemcpyHostToDevice);
}

static cudaError_t make_twiddles_f(int n, float2 **out)
{
    std::vector<float2> h(n);
    const long double PI = 3.141592653589793238462643383279502884L;
    for (int t = 0; t < n; t++) {
        long double ang = -2.0L * PI * (long double)t / (long double)n;
        h[t] = make_float2((float)cosl(ang), (float)sinl(ang));
    }
    cudaError_t e = cudaMalloc(out, n * sizeof(float2));
    if (e != cudaSuccess) return e;
    return cudaMemcpy(*out, h.data(), n * sizeof(float2), cudaMemcpyHostToDevice);
}

cudaError_t pressure_plan_create(const DevGrid &g, const double *wv_host, int mixed, PressurePlan **out, int *pivot_error)
{
    *out = nullptr;
    *pivot_error = 0;
    PressurePlan *pp = new PressurePlan();
    cudaError_t e;
    int nh = g.maxx / 2 + 1;
    size_t nspec = (size_t)g.nz * nh * g.maxy, nreal = (size_t)g.nz * g.maxy * g.maxx;
#define CK(x) do { e = (x); if (e != cudaSuccess) { pressure_plan_destroy(pp); return e; } } while (0)
    pp->px.n = g.maxx;
    pp->py.n = g.maxy;
    if (!factorize(g.maxx, &pp->px) || !factorize(g.maxy, &pp->py)) {
        pressure_plan_destroy(pp);
        return cudaErrorInvalidValue;
    }
    pp->mixed = mixed ? 1 : 0;
    pp->xt = g.maxx / 8 < 32 ? 32 : (g.maxx / 8 > XT_THREADS / (ROWS / 2) ? XT_THREADS / (ROWS / 2) : g.maxx / 8);
    // fft_y<double2> holds 74 registers per thread: at most 512 threads per block (YROWS rows)
    pp->yt = g.maxy / 8 < 32 ? 32 : (g.maxy / 8 > 128 ? 128 : g.maxy / 8);
    pp->tb = 128;
    CK(make_twiddles(g.maxx, &pp->twx));
    CK(make_twiddles(g.maxy, &pp->twy));
    CK(make_twiddles_f(g.maxx, &pp->twxf));
    CK(make_twiddles_f(g.maxy, &pp->twyf));
    pp->px.tw = pp->twx;
    pp->py.tw = pp->twy;
    pp->px.twf = pp->twxf;
    pp->py.twf = pp->twyf;
    const size_t cbytes = pp->mixed ? sizeof(float2) : sizeof(double2);
    CK(cudaMalloc(&pp->spec, nspec * cbytes));
    if (pp->mixed) CK(cudaMalloc(&pp->tri, nspec * sizeof(double2)));
    CK(cudaMalloc(&pp->dp, nreal * sizeof(double)));
    CK(cudaMalloc(&pp->rbuf, nreal * sizeof(double)));
    CK(cudaMalloc(&pp->gam, nspec * sizeof(double)));
    CK(cudaMalloc(&pp->wv, (size_t)g.maxx * g.maxy * sizeof(double)));
    CK(cudaMemcpy(pp->wv, wv_host, (size_t)g.maxx * g.maxy * sizeof(double), cudaMemcpyHostToDevice));
    // per-level coefficients, fft_tools.f90:142-173 (host, same arithmetic as the reference)
    {
        const int nz = g.nz;
        std::vector<double> fdz(nz), dz1(nz), dz1w(nz), stab(nz);
        cudaMemcpy(fdz.data(), g.fdz0, nz * 8, cudaMemcpyDeviceToHost);
        cudaMemcpy(dz1.data(), g.dz1, nz * 8, cudaMemcpyDeviceToHost);
        cudaMemcpy(dz1w.data(), g.dz1w, nz * 8, cudaMemcpyDeviceToHost);
        cudaMemcpy(stab.data(), g.stab0, nz * 8, cudaMemcpyDeviceToHost);
        std::vector<double> ak(nz, 0.), ck(nz, 0.), dka(nz, 0.), dkb(nz, 0.);
        for (int k = 2; k <= nz - 1; k++) {
            double h = g.dz * (0.5 * fdz[k] + fdz[k - 1] + 0.5 * fdz[k - 2]);
            ak[k - 1] = dz1[k - 2] * dz1w[k - 1] - stab[k - 1] / h;
            ck[k - 1] = dz1[k - 1] * dz1w[k - 1] + stab[k - 1] / h;
            dka[k - 1] = dz1w[k - 1] * (dz1[k - 1] + dz1[k - 2]);
        }
        ak[0] = 0.;
        ck[0] = dz1[0] * dz1w[0] + stab[0] * dz1[0];
        dka[0] = dz1[0] * dz1w[0];
        dkb[0] = stab[0] * dz1[0];
        ak[nz - 1] = dz1w[nz - 1] * dz1[nz - 2] - stab[nz - 1] * dz1[nz - 2];
        ck[nz - 1] = 0.;
        dka[nz - 1] = dz1w[nz - 1] * dz1[nz - 2];
        dkb[nz - 1] = stab[nz - 1] * dz1[nz - 2];
        CK(cudaMalloc(&pp->ak, nz * 8)); CK(cudaMalloc(&pp->ck, nz * 8));
        CK(cudaMalloc(&pp->dka, nz * 8)); CK(cudaMalloc(&pp->dkb, nz * 8));
        CK(cudaMemcpy(pp->ak, ak.data(), nz * 8, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(pp->ck, ck.data(), nz * 8, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(pp->dka, dka.data(), nz * 8, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(pp->dkb, dkb.data(), nz * 8, cudaMemcpyHostToDevice));
    }
    CK(cudaMalloc(&pp->mean, g.nz * 8));
    CK(cudaMalloc(&pp->mean_d, g.nz * 8));
    CK(cudaMalloc(&pp->p1, g.nz * 8));
    pp->npartial = 1024;
    CK(cudaMalloc(&pp->partial, pp->npartial * 8));
    CK(cudaMalloc(&pp->maxdiv, 8));
    CK(cudaMalloc(&pp->resid, MG_MAXPASS * sizeof(unsigned long long)));
    CK(cudaMalloc(&pp->bsum, (size_t)g.nz * ((g.maxy + ROWS - 1) / ROWS) * sizeof(double)));
    CK(cudaMemset(pp->resid, 0, MG_MAXPASS * sizeof(unsigned long long)));
    // elimination factors and pivot check
    {
        int *derr;
        CK(cudaMalloc(&derr, sizeof(int)));
        CK(cudaMemset(derr, 0, sizeof(int)));
        TriArgs T{};
        T.wv = pp->wv; T.ak = pp->ak; T.ck = pp->ck; T.dka = pp->dka; T.dkb = pp->dkb;
        long long ncol = (long long)nh * g.maxy;
        gam_kernel<<<(unsigned)((ncol + 255) / 256), 256>>>(g, T, pp->gam, derr);
        e = cudaGetLastError();
        int herr = 0;
        if (e == cudaSuccess) e = cudaMemcpy(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost);
        cudaFree(derr);
        if (e != cudaSuccess) { pressure_plan_destroy(pp); return e; }
        *pivot_error = herr;
    }
    pp->bytes = nspec * (cbytes + 8 + (pp->mixed ? 16 : 0)) + nreal * 16 + (size_t)g.maxx * g.maxy * 8 + (size_t)(g.maxx + g.maxy) * 16;
#undef CK
    *out = pp;
    return cudaSuccess;
}

void pressure_plan_destroy(PressurePlan *pp)
{
    if (!pp) return;
    cudaFree(pp->twx); cudaFree(pp->twy); cudaFree(pp->twxf); cudaFree(pp->twyf); cudaFree(pp->spec); cudaFree(pp->tri); cudaFree(pp->dp); cudaFree(pp->rbuf);
    cudaFree(pp->gam); cudaFree(pp->wv); cudaFree(pp->ak); cudaFree(pp->ck); cudaFree(pp->dka); cudaFree(pp->dkb);
    cudaFree(pp->mean); cudaFree(pp->mean_d); cudaFree(pp->p1); cudaFree(pp->partial); cudaFree(pp->maxdiv);
    cudaFree(pp->resid); cudaFree(pp->bsum);
    cudaFree(pp->gamT); cudaFree(pp->akT); cudaFree(pp->ckT);
    delete pp;
}

size_t pressure_plan_bytes(const PressurePlan *pp) { return pp ? pp->bytes : 0; }

// ---- the autotuner's search space: radix sequences and launch shapes ----
static bool radices_ok(int n, unsigned long long pk, int nst)
{
    if (nst < 1 || nst > MAXSTAGES) return false;
    long long prod = 1;
    for (int q = 0; q < nst; q++) {
        const int r = (int)((pk >> (4 * q)) & 15ull);
        if (r != 2 && r != 3 && r != 4 && r != 5 && r != 8) return false;
        prod *= r;
    }
    return prod == n && (pk >> (4 * nst)) == 0ull;
}

void pressure_get_knobs(const PressurePlan *pp, PressureKnobs *k)
{
    k->xr = pp->px.rpack; k->xst = pp->px.nst;
    k->yr = pp->py.rpack; k->yst = pp->py.nst;
    k->xt = pp->xt; k->yt = pp->yt; k->tb = pp->tb;
}

bool pressure_knobs_valid(const DevGrid &g, const PressureKnobs &k)
{
    // thread counts: multiples of 8 (whole warps per block) within the launch limits, which
    // covers the defaults (maxx/8 and maxy/8, clamped) as well as the tuner's powers of two
    auto mult8_in = [](int v, int lo, int hi) { return v >= lo && v <= hi && v % 8 == 0; };
    auto pow2_in = [](int v, int lo, int hi) { return v >= lo && v <= hi && (v & (v - 1)) == 0; };
    return radices_ok(g.maxx, k.xr, k.xst) && radices_ok(g.maxy, k.yr, k.yst) && mult8_in(k.xt, 8, XT_THREADS / (ROWS / 2)) &&
           mult8_in(k.yt, 16, 128) && pow2_in(k.tb, 64, 256);
}

bool pressure_set_knobs(PressurePlan *pp, const DevGrid &g, const PressureKnobs &k)
{
    if (!pressure_knobs_valid(g, k)) return false;
    pp->px.rpack = k.xr; pp->px.nst = k.xst;
    pp->py.rpack = k.yr; pp->py.nst = k.yst;
    pp->xt = k.xt; pp->yt = k.yt; pp->tb = k.tb;
    return true;
}

// distinct radix sequences for n = 2^a 3^b 5^c: the power-of-two part as radix 8 (then 4
// or 2) or as radix 4 (then 2), the odd radices after or before it, each also reversed
int pressure_radix_candidates(int n, unsigned long long *pk, int *nst, int maxc)
{
    int a = 0, b = 0, c = 0, m = n;
    while (m % 2 == 0) { m /= 2; a++; }
    while (m % 3 == 0) { m /= 3; b++; }
    while (m % 5 == 0) { m /= 5; c++; }
    if (m != 1) return 0;
    std::vector<std::vector<int>> two(2), cand;
    for (int q = 0; q < a / 3; q++) two[0].push_back(8);
    if (a % 3 == 2) two[0].push_back(4);
    if (a % 3 == 1) two[0].push_back(2);
    for (int q = 0; q < a / 2; q++) two[1].push_back(4);
    if (a % 2) two[1].push_back(2);
    std::vector<int> odd;
    for (int q = 0; q < b; q++) odd.push_back(3);
    for (int q = 0; q < c; q++) odd.push_back(5);
    for (auto &t : two)
        for (int oddfirst = 0; oddfirst < 2; oddfirst++) {
            std::vector<int> v = oddfirst ? odd : t;
            const std::vector<int> &w = oddfirst ? t : odd;
            v.insert(v.end(), w.begin(), w.end());
            cand.push_back(v);
            cand.push_back(std::vector<int>(v.rbegin(), v.rend()));
        }
    int nc = 0;
    for (auto &v : cand) {
        if (v.empty() || (int)v.size() > MAXSTAGES) continue;
        unsigned long long p = 0;
        for (size_t q = 0; q < v.size(); q++) p |= (unsigned long long)v[q] << (4 * q);
        bool dup = false;
        for (int q = 0; q < nc; q++) dup = dup || (pk[q] == p && nst[q] == (int)v.size());
        if (dup || nc >= maxc) continue;
        pk[nc] = p;
        nst[nc] = (int)v.size();
        nc++;
    }
    return nc;
}
const double *pressure_p1_dev(const PressurePlan *pp) { return pp->p1; }
const double *pressure_maxdiv_dev(const PressurePlan *pp) { return pp->maxdiv; }
const unsigned long long *pressure_resid_dev(const PressurePlan *pp) { return pp->resid; }
cudaError_t pressure_resid_reset(PressurePlan *pp, cudaStream_t s)
{
    return cudaMemsetAsync(pp->resid, 0, MG_MAXPASS * sizeof(unsigned long long), s);
}
static Skip skip_self(const PressurePlan *pp, const PassCtl &pc)
{
    Skip k{nullptr, pc.tol};
    if (pc.slot >= 0 && pc.refine) k.flag = pp->resid + pc.slot;
    return k;
}

template <typename C>
static cudaError_t launch_x_fwd_t(const DevGrid &g, PressurePlan *pp, const XArgs &a, cudaStream_t s)
{
    int groups = (g.maxy + ROWS - 1) / ROWS;
    const int nt_pair = pp->xt;
    size_t sm = (size_t)(ROWS / 2) * 2 * padded_len(g.maxx) * sizeof(C);
    cudaError_t e = cudaFuncSetAttribute(fft_x_fwd<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    fft_x_fwd<C><<<g.nz * groups, nt_pair * (ROWS / 2), sm, s>>>(g, pp->px, a);
    return cudaGetLastError();
}
static cudaError_t launch_x_fwd(const DevGrid &g, PressurePlan *pp, const XArgs &a, cudaStream_t s)
{
    return pp->mixed ? launch_x_fwd_t<float2>(g, pp, a, s) : launch_x_fwd_t<double2>(g, pp, a, s);
}

static void set_resid(const PressurePlan *pp, const PassCtl &pc, XArgs &a)
{
    if (pc.slot >= 0 && pc.slot < MG_MAXPASS) {
        a.resid = pp->resid + pc.slot;
        if (pc.skip_prev && pc.slot > 0) a.prev = Skip{pp->resid + pc.slot - 1, pc.tol};
    }
}

cudaError_t launch_div_rhs(const DevGrid &g, PressurePlan *pp, const double *mu, const double *mv, const double *mw,
                           const PassCtl &pc, cudaStream_t s)
{
    XArgs a{};
    a.mode = 0;
    a.mu = mu; a.mv = mv; a.mw = mw; a.spec = pp->spec; a.dt1 = 1. / g.dt0;
    if (pc.store_b) { a.store_b = 1; a.rbuf = pp->rbuf; a.bsum = pp->bsum; }
    set_resid(pp, pc, a);
    return launch_x_fwd(g, pp, a, s);
}

cudaError_t launch_resid_rhs(const DevGrid &g, PressurePlan *pp, const PassCtl &pc, cudaStream_t s)
{
    XArgs a{};
    a.mode = 2;
    a.rbuf = pp->rbuf; a.bsum = pp->bsum; a.dp = pp->dp;
    a.ak = pp->ak; a.ck = pp->ck; a.dka = pp->dka; a.dkb = pp->dkb;
    a.spec = pp->spec; a.dt1 = 1. / g.dt0;
    set_resid(pp, pc, a);
    return launch_x_fwd(g, pp, a, s);
}

cudaError_t launch_load_rhs(const DevGrid &g, PressurePlan *pp, const double *tend, cudaStream_t s)
{
    long long n = (long long)g.maxx * g.maxy * g.nz;
    interior_gather<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(g, tend, pp->rbuf);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    XArgs a{};
    a.mode = 1;
    a.rbuf = pp->rbuf; a.spec = pp->spec;
    return launch_x_fwd(g, pp, a, s);
}

template <typename C>
static cudaError_t pressure_solve_t(const DevGrid &g, PressurePlan *pp, int keep00, Skip sk, int accumulate,
                                    cudaStream_t s, int transposed = 0)
{
    cudaError_t e;
    const int nh = g.maxx / 2 + 1;
    const int nrows = g.nz * nh;
    const int nt_row = pp->yt;
    size_t smy = (size_t)YROWS * 2 * padded_len(g.maxy) * sizeof(C);
    e = cudaFuncSetAttribute(fft_y<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smy);
    if (e != cudaSuccess) return e;
    // FP32 spectra of a length the warp-shuffle transform covers take it
    const bool shfl = sizeof(C) == sizeof(float2) && yshfl_ok(g.maxy);
    if (shfl)
        e = launch_y_shfl(pp->py, pp->spec, nrows, 0, sk, s);
    else {
        fft_y<C><<<(nrows + YROWS - 1) / YROWS, nt_row * YROWS, smy, s>>>(g, pp->py, pp->spec, nrows, 0, sk);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) return e;
    TriArgs T{};
    T.spec = pp->spec; T.gam = pp->gam; T.wv = pp->wv; T.ak = pp->ak; T.ck = pp->ck; T.dka = pp->dka; T.dkb = pp->dkb;
    if (transposed) { T.gam = pp->gamT; T.ak = pp->akT; T.ck = pp->ckT; }
    T.keep00 = keep00;
    T.sk = sk;
    T.scratch = pp->tri;
    long long ncol = (long long)nh * g.maxy;
    tridiag_kernel<C><<<(unsigned)((ncol + pp->tb - 1) / pp->tb), pp->tb, 0, s>>>(g, T);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (shfl)
        e = launch_y_shfl(pp->py, pp->spec, nrows, 1, sk, s);
    else {
        fft_y<C><<<(nrows + YROWS - 1) / YROWS, nt_row * YROWS, smy, s>>>(g, pp->py, pp->spec, nrows, 1, sk);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) return e;
    int groups = (g.maxy + ROWS - 1) / ROWS;
    const int nt_pair = pp->xt;
    size_t smx = (size_t)(ROWS / 2) * 2 * padded_len(g.maxx) * sizeof(C);
    e = cudaFuncSetAttribute(fft_x_inv<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smx);
    if (e != cudaSuccess) return e;
    XInvArgs xa{};
    xa.spec = pp->spec; xa.dp = pp->dp;
    xa.scale_div = keep00 ? 1.0 : (double)g.maxx * (double)g.maxy;
    xa.sk = sk;
    xa.accumulate = accumulate;
    fft_x_inv<C><<<g.nz * groups, nt_pair * (ROWS / 2), smx, s>>>(g, pp->px, xa);
    return cudaGetLastError();
}

cudaError_t pressure_solve(const DevGrid &g, PressurePlan *pp, double scale, int keep00, const PassCtl &pc,
                           cudaStream_t s)
{
    (void)scale;
    const Skip sk = skip_self(pp, pc);
    return pp->mixed ? pressure_solve_t<float2>(g, pp, keep00, sk, pc.refine, s)
                     : pressure_solve_t<double2>(g, pp, keep00, sk, pc.refine, s);
}

cudaError_t launch_store_solution(const DevGrid &g, PressurePlan *pp, double *out, cudaStream_t s)
{
    long long n = (long long)g.maxx * g.maxy * g.nz;
    interior_scatter<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(g, pp->dp, out);
    return cudaGetLastError();
}

cudaError_t launch_correction(const DevGrid &g, PressurePlan *pp, double *mu, double *mv, double *mw, double *p,
                              int natural_uv, cudaStream_t s)
{
    const unsigned nb = corr_blocks_per_level(g, 256) * (unsigned)g.nz;
    correction_kernel<<<nb, 256, 0, s>>>(g, pp->dp, mu, mv, mw, p, natural_uv, 1. / g.dx, 1. / g.dy);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    double *f[4] = {mu, mv, mw, p};
    return launch_halo_fill(g, f, 4, s);
}

cudaError_t launch_cal_p1(const DevGrid &g, PressurePlan *pp, double *mw, const double *wold, int wold_rep,
                          int want_p1, int natural_w, cudaStream_t s)
{
    level_sums<<<g.nz, LSUM_THREADS, 0, s>>>(g, mw, wold, wold_rep, g.dt0, pp->mean, want_p1 ? pp->mean_d : nullptr);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (want_p1) {
        p1_kernel<<<1, 32, 0, s>>>(g, pp->mean_d, pp->p1);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    subtract_level_mean<<<1184, 256, 0, s>>>(g, mw, pp->mean, natural_w);
    return cudaGetLastError();
}

cudaError_t launch_level_mean(const DevGrid &g, const double *x, double *mean, cudaStream_t s)
{
    level_sums<<<g.nz, LSUM_THREADS, 0, s>>>(g, x, nullptr, -1, g.dt0, mean, nullptr);
    return cudaGetLastError();
}

cudaError_t launch_to_velocity(const DevGrid &g, double *mu, double *mv, double *mw, cudaStream_t s)
{
    to_velocity_kernel<<<1184, 256, 0, s>>>(g, mu, mv, mw);
    return cudaGetLastError();
}

cudaError_t launch_maxdiv(const DevGrid &g, PressurePlan *pp, const double *mu, const double *mv, const double *mw,
                          cudaStream_t s, int natural)
{
    int nb = pp->npartial;
    maxdiv_kernel<<<nb, 256, 0, s>>>(g, mu, mv, mw, natural, pp->partial);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    max_final<<<1, 256, 0, s>>>(pp->partial, nb, pp->maxdiv);
    return cudaGetLastError();
}

cudaError_t launch_halo_fill(const DevGrid &g, double *const *fields, int nf, cudaStream_t s)
{
    HaloArgs H{};
    for (int b = 0; b < nf; b += MG_MAXF) {
        H.nf = nf - b < MG_MAXF ? nf - b : MG_MAXF;
        for (int f = 0; f < H.nf; f++) H.f[f] = fields[b + f];
        long long tot = (5LL * g.nx + 5LL * g.maxy) * g.nz;
        int blocks = (int)((tot + 255) / 256);
        if (blocks > 4096) blocks = 4096;
        halo_fill_kernel<<<blocks, 256, 0, s>>>(g, H);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t launch_to_natural_packed(const DevGrid &g, const double *src, const double *w, int weight_kind, int rep,
                                     double *dst, cudaStream_t s)
{
    to_natural_packed_kernel<<<1184, 256, 0, s>>>(g, src, w, weight_kind, rep, dst);
    return cudaGetLastError();
}
cudaError_t launch_unpack(const DevGrid &g, const double *src, double *dst, cudaStream_t s)
{
    unpack_kernel<<<1184, 256, 0, s>>>(g, src, dst);
    return cudaGetLastError();
}

// ======================== adjoint of the projection ========================
// One projection pass maps (m, p) to
//   m' = m - dt0 * R * G(dp),  p' = p + rho0 * dp,  dp = S(b),  b = D(m) * dt1 / rho0,
// with G the backward-difference gradient of correction_kernel (the bottom w row is set
// to zero from m_w(1) itself), S the transforms + tridiagonal solve (mode (0,0) zero,
// 1/N_h), D the divergence of fft_x_fwd, R = rho0 (u, v) or avden0 (w); cal_p1 then
// removes the level mean of w.  Its adjoint, pass by pass in reverse:
//   dpbar = rho0 * pbar - dt0 * G^T(R mbar),  bbar = S^T(dpbar),  mbar <- Z mbar + D^T(bbar dt1/rho0)
// where S^T has the same transforms around the transposed tridiagonal and Z zeroes the
// bottom w row.  Arrays: halo'd layout, interior adjoints, ghosts zero.
namespace {

__global__ void adj_sub_level_mean_kernel(DevGrid G, double *x, const double *mean)
{
    const int maxx = G.maxx, maxy = G.maxy;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)maxx * maxy * G.nz) return;
    const int ix = (int)(t % maxx), jy = (int)((t / maxx) % maxy), k = (int)(t / ((long long)maxx * maxy)) + 1;
    const long long c = gidx(G, ix + 4, jy + 4, k);
    x[c] = x[c] - mean[k - 1];
}

// dpbar (dense interior [nz][maxy][maxx]) = rho0 pbar - dt0 G^T(R mbar)
__global__ void adj_rhs_kernel(DevGrid G, const double *mub, const double *mvb, const double *mwb, const double *pb,
                               double *out)
{
    const int maxx = G.maxx, maxy = G.maxy, nz = G.nz;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)maxx * maxy * nz) return;
    const int ix = (int)(t % maxx), jy = (int)((t / maxx) % maxy), k = (int)(t / ((long long)maxx * maxy)) + 1;
    const int i = ix + 4, j = jy + 4;
    const long long c = gidx(G, i, j, k);
    const double d0 = __ldg(G.den0 + k - 1);
    const double dx1 = 1. / G.dx, dy1 = 1. / G.dy;
    // G_x dp(i) = (dp(i) - dp(i-1)) dx1 (periodic): G_x^T q(i) = (q(i) - q(i+1)) dx1
    const long long ce = gidx(G, ix == maxx - 1 ? 4 : i + 1, j, k);
    const long long cn = gidx(G, i, jy == maxy - 1 ? 4 : j + 1, k);
    double gt = (d0 * mub[c] - d0 * mub[ce]) * dx1 + (d0 * mvb[c] - d0 * mvb[cn]) * dy1;
    // G_z dp(k) = (dp(k) - dp(k-1)) dz1(k-1), k >= 2
    if (k >= 2) gt += __ldg(G.avden0 + k - 1) * mwb[c] * __ldg(G.dz1 + k - 2);
    if (k + 1 <= nz) gt -= __ldg(G.avden0 + k) * mwb[c + G.ps] * __ldg(G.dz1 + k - 1);
    out[t] = d0 * pb[c] - G.dt0 * gt;
}

// mbar <- Z mbar + D^T(q), q = bbar * dt1 / rho0 (dense interior bbar = dp)
__global__ void adj_div_kernel(DevGrid G, const double *bbar, double *mub, double *mvb, double *mwb)
{
    const int maxx = G.maxx, maxy = G.maxy, nz = G.nz;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)maxx * maxy * nz) return;
    const int ix = (int)(t % maxx), jy = (int)((t / maxx) % maxy), k = (int)(t / ((long long)maxx * maxy)) + 1;
    const int i = ix + 4, j = jy + 4;
    const long long c = gidx(G, i, j, k);
    const double dt1 = 1. / G.dt0, dx1 = 1. / G.dx, dy1 = 1. / G.dy;
    auto Q = [&](int a, int b, int kk) {
        return bbar[((long long)(kk - 1) * maxy + b) * maxx + a] * (dt1 / __ldg(G.den0 + kk - 1));
    };
    const double q = Q(ix, jy, k);
    // D: (mu(i+1) - mu(i)) dx1 + (mv(j+1) - mv(j)) dy1 + (mw(k+1) - mw(k)) dzw1(k), mw(nz+1) = 0
    mub[c] += (Q(ix == 0 ? maxx - 1 : ix - 1, jy, k) - q) * dx1;
    mvb[c] += (Q(ix, jy == 0 ? maxy - 1 : jy - 1, k) - q) * dy1;
    double wz = -q * __ldg(G.dz1w + k - 1);
    if (k >= 2) wz += Q(ix, jy, k - 1) * __ldg(G.dz1w + k - 2);
    mwb[c] = (k == 1 ? 0. : mwb[c]) + wz;
}

}  // namespace

cudaError_t pressure_adjoint(const DevGrid &g, PressurePlan *pp, int nsubp, double *mub, double *mvb, double *mwb,
                             double *pb, cudaStream_t s)
{
    if (pp->mixed) return cudaErrorInvalidValue;   // the adjoint runs in FP64
    cudaError_t e;
    const int nz = g.nz, nh = g.maxx / 2 + 1;
    const long long ncol = (long long)nh * g.maxy;
    if (!pp->gamT) {   // transposed system: sub-diagonal c(k-1), super-diagonal a(k+1)
        std::vector<double> ak(nz), ck(nz), akT(nz, 0.), ckT(nz, 0.);
        if ((e = cudaMemcpy(ak.data(), pp->ak, nz * 8, cudaMemcpyDeviceToHost)) != cudaSuccess) return e;
        if ((e = cudaMemcpy(ck.data(), pp->ck, nz * 8, cudaMemcpyDeviceToHost)) != cudaSuccess) return e;
        for (int k = 2; k <= nz; k++) akT[k - 1] = ck[k - 2];
        for (int k = 1; k <= nz - 1; k++) ckT[k - 1] = ak[k];
        if ((e = cudaMalloc(&pp->akT, nz * 8)) != cudaSuccess) return e;
        if ((e = cudaMalloc(&pp->ckT, nz * 8)) != cudaSuccess) return e;
        if ((e = cudaMalloc(&pp->gamT, (size_t)nz * ncol * 8)) != cudaSuccess) return e;
        if ((e = cudaMemcpy(pp->akT, akT.data(), nz * 8, cudaMemcpyHostToDevice)) != cudaSuccess) return e;
        if ((e = cudaMemcpy(pp->ckT, ckT.data(), nz * 8, cudaMemcpyHostToDevice)) != cudaSuccess) return e;
        int *derr;
        if ((e = cudaMalloc(&derr, sizeof(int))) != cudaSuccess) return e;
        cudaMemset(derr, 0, sizeof(int));
        TriArgs T{};
        T.wv = pp->wv; T.ak = pp->akT; T.ck = pp->ckT; T.dka = pp->dka; T.dkb = pp->dkb;
        gam_kernel<<<(unsigned)((ncol + 255) / 256), 256>>>(g, T, pp->gamT, derr);
        e = cudaGetLastError();
        int herr = 0;
        if (e == cudaSuccess) e = cudaMemcpy(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost);
        cudaFree(derr);
        if (e != cudaSuccess) return e;
        if (herr) return cudaErrorInvalidValue;
    }
    const long long n = (long long)g.maxx * g.maxy * nz;
    const unsigned nb = (unsigned)((n + 255) / 256);
    // cal_p1^T: remove the level mean of wbar (interior)
    level_sums<<<nz, LSUM_THREADS, 0, s>>>(g, mwb, mwb, -1, g.dt0, pp->mean, nullptr);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    adj_sub_level_mean_kernel<<<nb, 256, 0, s>>>(g, mwb, pp->mean);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    for (int ip = 0; ip < nsubp; ip++) {
        adj_rhs_kernel<<<nb, 256, 0, s>>>(g, mub, mvb, mwb, pb, pp->rbuf);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        XArgs a{};
        a.mode = 1;
        a.rbuf = pp->rbuf; a.spec = pp->spec;
        if ((e = launch_x_fwd(g, pp, a, s)) != cudaSuccess) return e;
        if ((e = pressure_solve_t<double2>(g, pp, 0, Skip{nullptr, 0.}, 0, s, 1)) != cudaSuccess) return e;
        adj_div_kernel<<<nb, 256, 0, s>>>(g, pp->dp, mub, mvb, mwb);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// ======================== grouped launches over several members ========================
void group_halo(GroupProgram &P, const std::vector<GroupHaloIn> &in)
{
    const int n = (int)in.size();
    std::vector<HaloMember> mem(n);
    std::vector<int> nb(n);
    std::vector<double> cost(n, 1.);
    for (int q = 0; q < n; q++) {
        const DevGrid &g = *in[q].G;
        mem[q].G = g;
        mem[q].H.nf = in[q].nf;
        for (int f = 0; f < in[q].nf; f++) mem[q].H.f[f] = in[q].f[f];
        const long long tot = (5LL * g.nx + 5LL * g.maxy) * g.nz;
        nb[q] = (int)std::min<long long>(4096, (tot + 255) / 256);
        mem[q].nb = nb[q];
    }
    const std::vector<GItem> it = group_items(nb, cost);
    const size_t mo = P.put(mem), io = P.put(it);
    const int ni = (int)it.size();
    P.ops.push_back([=](const unsigned char *d, cudaStream_t s) {
        halo_fill_grp<<<ni, 256, 0, s>>>((const HaloMember *)(d + mo), (const GItem *)(d + io));
        return cudaGetLastError();
    });
    P.launches++;
}

namespace {
// the members' indices grouped by the x transforms' threads per row pair
std::vector<std::vector<int>> by_xt(const std::vector<GroupProjIn> &in)
{
    std::vector<std::vector<int>> out;
    std::vector<int> keys;
    for (int q = 0; q < (int)in.size(); q++) {
        const int xt = in[q].pp->xt;
        size_t c = std::find(keys.begin(), keys.end(), xt) - keys.begin();
        if (c == keys.size()) { keys.push_back(xt); out.emplace_back(); }
        out[c].push_back(q);
    }
    return out;
}

// one grouped x transform (forward with the given per-member arguments, or inverse)
template <typename C>
void group_x(GroupProgram &P, const std::vector<GroupProjIn> &in, const std::vector<XArgs> *fwd,
             const std::vector<XInvArgs> *inv)
{
    for (const std::vector<int> &sub : by_xt(in)) {
        const int n = (int)sub.size();
        std::vector<int> nb(n);
        std::vector<double> cost(n);
        size_t sm = 0;
        for (int q = 0; q < n; q++) {
            const DevGrid &g = *in[sub[q]].G;
            nb[q] = g.nz * ((g.maxy + ROWS - 1) / ROWS);
            cost[q] = (double)g.maxx;
            sm = std::max(sm, (size_t)(ROWS / 2) * 2 * padded_len(g.maxx) * sizeof(C));
        }
        const std::vector<GItem> it = group_items(nb, cost);
        const int ni = (int)it.size(), threads = in[sub[0]].pp->xt * (ROWS / 2);
        size_t mo;
        if (fwd) {
            std::vector<XFwdMember> mem(n);
            for (int q = 0; q < n; q++) mem[q] = XFwdMember{*in[sub[q]].G, in[sub[q]].pp->px, (*fwd)[sub[q]]};
            mo = P.put(mem);
        } else {
            std::vector<XInvMember> mem(n);
            for (int q = 0; q < n; q++) mem[q] = XInvMember{*in[sub[q]].G, in[sub[q]].pp->px, (*inv)[sub[q]]};
            mo = P.put(mem);
        }
        const size_t io = P.put(it);
        const bool is_fwd = fwd != nullptr;
        P.ops.push_back([=](const unsigned char *d, cudaStream_t s) {
            cudaError_t e;
            if (is_fwd) {
                e = cudaFuncSetAttribute(fft_x_fwd_grp<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
                if (e != cudaSuccess) return e;
                fft_x_fwd_grp<C><<<ni, threads, sm, s>>>((const XFwdMember *)(d + mo), (const GItem *)(d + io));
            } else {
                e = cudaFuncSetAttribute(fft_x_inv_grp<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
                if (e != cudaSuccess) return e;
                fft_x_inv_grp<C><<<ni, threads, sm, s>>>((const XInvMember *)(d + mo), (const GItem *)(d + io));
            }
            return cudaGetLastError();
        });
        P.launches++;
    }
}

// y transform, tridiagonal, y transform, inverse x transform of every member (pressure_solve_t)
template <typename C>
void group_solve(GroupProgram &P, const std::vector<GroupProjIn> &in, const PassCtl &pc)
{
    const int n = (int)in.size();
    std::vector<Skip> sk(n);
    for (int q = 0; q < n; q++) sk[q] = skip_self(in[q].pp, pc);
    // y transforms: threads per row = the largest member's knob (the rows' arithmetic does
    // not depend on it)
    int yt = 16, tb = 64;
    size_t smy = 0;
    std::vector<int> nby(n), nbt(n);
    std::vector<double> cy(n), ct(n);
    for (int q = 0; q < n; q++) {
        const DevGrid &g = *in[q].G;
        const int nh = g.maxx / 2 + 1;
        yt = std::max(yt, in[q].pp->yt);
        tb = std::max(tb, in[q].pp->tb);
        smy = std::max(smy, (size_t)YROWS * 2 * padded_len(g.maxy) * sizeof(C));
        nby[q] = (g.nz * nh + YROWS - 1) / YROWS;
        cy[q] = (double)g.maxy;
        ct[q] = (double)g.nz;
    }
    for (int q = 0; q < n; q++) {
        const DevGrid &g = *in[q].G;
        nbt[q] = (int)(((long long)(g.maxx / 2 + 1) * g.maxy + tb - 1) / tb);
    }
    // members whose y transform is the warp-shuffle one (FP32 spectra of a covered length,
    // as pressure_solve_t chooses) take a launch per row length (variant log2(M)), the
    // others the Stockham launch (variant 0)
    std::vector<std::vector<int>> yv(5);
    for (int q = 0; q < n; q++) {
        const int my = in[q].G->maxy;
        yv[sizeof(C) == sizeof(float2) && yshfl_ok(my) ? (my == 64 ? 1 : my == 128 ? 2 : my == 256 ? 3 : 4) : 0]
            .push_back(q);
    }
    for (int dir = 0; dir < 2; dir++) {
        auto push_y = [&]() {
            for (int variant = 0; variant < 5; variant++) {
                const std::vector<int> &sub = yv[variant];
                if (sub.empty()) continue;
                std::vector<YMember> ym;
                std::vector<int> nb;
                std::vector<double> cost;
                for (int q : sub) {
                    const DevGrid &g = *in[q].G;
                    const int nrows = g.nz * (g.maxx / 2 + 1);
                    ym.push_back(YMember{in[q].pp->py, in[q].pp->spec, nrows, dir, sk[q]});
                    nb.push_back(variant == 0 ? nby[q] : (nrows + YW_WARPS - 1) / YW_WARPS);
                    cost.push_back(cy[q]);
                }
                const std::vector<GItem> it = group_items(nb, cost);
                const size_t mo = P.put(ym), io = P.put(it);
                const int ni = (int)it.size();
                if (variant == 0)
                    P.ops.push_back([=](const unsigned char *d, cudaStream_t s) {
                        cudaError_t e = cudaFuncSetAttribute(fft_y_grp<C>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                             (int)smy);
                        if (e != cudaSuccess) return e;
                        fft_y_grp<C><<<ni, yt * YROWS, smy, s>>>((const YMember *)(d + mo), (const GItem *)(d + io));
                        return cudaGetLastError();
                    });
                else
                    P.ops.push_back([=](const unsigned char *d, cudaStream_t s) {
                        const YMember *mm = (const YMember *)(d + mo);
                        const GItem *ii = (const GItem *)(d + io);
                        switch (variant) {
                        case 1: fft_y_shfl_grp<2><<<ni, 32 * YW_WARPS, 0, s>>>(mm, ii); break;
                        case 2: fft_y_shfl_grp<4><<<ni, 32 * YW_WARPS, 0, s>>>(mm, ii); break;
                        case 3: fft_y_shfl_grp<8><<<ni, 32 * YW_WARPS, 0, s>>>(mm, ii); break;
                        default: fft_y_shfl_grp<16><<<ni, 32 * YW_WARPS, 0, s>>>(mm, ii); break;
                        }
                        return cudaGetLastError();
                    });
                P.launches++;
            }
        };
        if (dir == 1) {   // the tridiagonal solve sits between the two y transforms
            std::vector<TriMember> tm(n);
            for (int q = 0; q < n; q++) {
                PressurePlan *pp = in[q].pp;
                TriArgs T{};
                T.spec = pp->spec; T.gam = pp->gam; T.wv = pp->wv; T.ak = pp->ak; T.ck = pp->ck; T.dka = pp->dka;
                T.dkb = pp->dkb; T.keep00 = 0; T.sk = sk[q]; T.scratch = pp->tri;
                tm[q] = TriMember{*in[q].G, T};
            }
            const std::vector<GItem> it2 = group_items(nbt, ct);
            const size_t mo2 = P.put(tm), io2 = P.put(it2);
            const int ni2 = (int)it2.size();
            P.ops.push_back([=](const unsigned char *d, cudaStream_t s) {
                tridiag_grp<C><<<ni2, tb, 0, s>>>((const TriMember *)(d + mo2), (const GItem *)(d + io2));
                return cudaGetLastError();
            });
            P.launches++;
        }
        push_y();
    }
    std::vector<XInvArgs> xa(n);
    for (int q = 0; q < n; q++) {
        const DevGrid &g = *in[q].G;
        xa[q] = XInvArgs{};
        xa[q].spec = in[q].pp->spec; xa[q].dp = in[q].pp->dp;
        xa[q].scale_div = (double)g.maxx * (double)g.maxy;
        xa[q].sk = sk[q];
        xa[q].accumulate = pc.refine;
    }
    group_x<C>(P, in, nullptr, &xa);
}

template <typename C>
void group_projection_t(GroupProgram &P, const std::vector<GroupProjIn> &in, int finalize, int nsub, int nref,
                        double tol)
{
    const int n = (int)in.size();
    {   // residual slots of every member
        std::vector<unsigned long long *> r(n);
        for (int q = 0; q < n; q++) r[q] = in[q].pp->resid;
        const size_t ro = P.put(r);
        P.ops.push_back([=](const unsigned char *d, cudaStream_t s) {
            resid_reset_grp<<<n, 64, 0, s>>>((unsigned long long *const *)(d + ro));
            return cudaGetLastError();
        });
        P.launches++;
    }
    for (int ip = 0; ip < nsub; ip++) {
        const int last = ip == nsub - 1;
        const int slot0 = ip * (1 + nref);
        const PassCtl p0 = {slot0, 0, 0, nref > 0, tol};
        std::vector<XArgs> xf(n);
        for (int q = 0; q < n; q++) {   // launch_div_rhs
            PressurePlan *pp = in[q].pp;
            XArgs a{};
            a.mode = 0;
            a.mu = in[q].mu; a.mv = in[q].mv; a.mw = in[q].mw; a.spec = pp->spec; a.dt1 = 1. / in[q].G->dt0;
            if (p0.store_b) { a.store_b = 1; a.rbuf = pp->rbuf; a.bsum = pp->bsum; }
            set_resid(pp, p0, a);
            xf[q] = a;
        }
        group_x<C>(P, in, &xf, nullptr);
        group_solve<C>(P, in, p0);
        for (int r = 0; r < nref; r++) {
            const PassCtl pr = {slot0 + 1 + r, 1, r > 0, 0, tol};
            for (int q = 0; q < n; q++) {   // launch_resid_rhs
                PressurePlan *pp = in[q].pp;
                XArgs a{};
                a.mode = 2;
                a.rbuf = pp->rbuf; a.bsum = pp->bsum; a.dp = pp->dp;
                a.ak = pp->ak; a.ck = pp->ck; a.dka = pp->dka; a.dkb = pp->dkb;
                a.spec = pp->spec; a.dt1 = 1. / in[q].G->dt0;
                set_resid(pp, pr, a);
                xf[q] = a;
            }
            group_x<C>(P, in, &xf, nullptr);
            group_solve<C>(P, in, pr);
        }
        {   // correction, then the ghost refresh of m and p
            std::vector<CorrMember> cm(n);
            std::vector<int> nb(n);
            std::vector<double> cost(n, 1.);
            std::vector<GroupHaloIn> h(n);
            for (int q = 0; q < n; q++) {
                const DevGrid &g = *in[q].G;
                cm[q] = CorrMember{g, in[q].pp->dp, in[q].mu, in[q].mv, in[q].mw, in[q].p, finalize && last, 1. / g.dx, 1. / g.dy};
                nb[q] = (int)(corr_blocks_per_level(g, 256) * (unsigned)g.nz);
                h[q].G = in[q].G;
                h[q].nf = 4;
                h[q].f[0] = in[q].mu; h[q].f[1] = in[q].mv; h[q].f[2] = in[q].mw; h[q].f[3] = in[q].p;
            }
            const std::vector<GItem> it = group_items(nb, cost);
            const size_t mo = P.put(cm), io = P.put(it);
            const int ni = (int)it.size();
            P.ops.push_back([=](const unsigned char *d, cudaStream_t s) {
                correction_grp<<<ni, 256, 0, s>>>((const CorrMember *)(d + mo), (const GItem *)(d + io));
                return cudaGetLastError();
            });
            P.launches++;
            group_halo(P, h);
        }
    }
    {   // cal_p1 without p1: level means of w, then w -= mean (natural w when finalizing)
        std::vector<LevelMember> lm(n);
        std::vector<int> nbs(n), nbm(n);
        std::vector<double> cs(n), cm(n, 1.);
        for (int q = 0; q < n; q++) {
            const DevGrid &g = *in[q].G;
            nbs[q] = g.nz;
            cs[q] = (double)g.maxx * g.maxy;
            nbm[q] = (int)std::min<long long>(1184, (g.ps * g.nz + 2047) / 2048);
            lm[q] = LevelMember{g, in[q].mw, in[q].wold, in[q].wold_rep, in[q].pp->mean, finalize, nbm[q]};
        }
        const std::vector<GItem> its = group_items(nbs, cs), itm = group_items(nbm, cm);
        const size_t mo = P.put(lm), io1 = P.put(its), io2 = P.put(itm);
        const int n1 = (int)its.size(), n2 = (int)itm.size();
        P.ops.push_back([=](const unsigned char *d, cudaStream_t s) {
            level_sums_grp<<<n1, LSUM_THREADS, 0, s>>>((const LevelMember *)(d + mo), (const GItem *)(d + io1));
            return cudaGetLastError();
        });
        P.ops.push_back([=](const unsigned char *d, cudaStream_t s) {
            subtract_level_mean_grp<<<n2, 256, 0, s>>>((const LevelMember *)(d + mo), (const GItem *)(d + io2));
            return cudaGetLastError();
        });
        P.launches += 2;
    }
}
}  // namespace

void group_projection(GroupProgram &P, const std::vector<GroupProjIn> &in, int finalize, int nsub, int nref, double tol)
{
    if (in.empty()) return;
    if (in[0].pp->mixed) group_projection_t<float2>(P, in, finalize, nsub, nref, tol);
    else group_projection_t<double2>(P, in, finalize, nsub, nref, tol);
}
