// k_check.cu -- the per-step checks of checkall (src/IO/check.f90:59-95): the maximum
// advective CFL number of checkwind (:102-337) and the bounds of checkx (:341-417)
// for es and qt, each with the location of its first occurrence, and the first
// non-finite value of u, v, w, es or qt (the library's MG_ERR_NAN; the reference has no
// such check: a NaN passes checkx's comparisons and ends its run later, if at all).
//
// One pass over the interior of the resident level-n state: every thread keeps its
// extremes with their linear indices L = ((k-1)*maxy + (j-4))*maxx + (i-4), which
// order cells as the reference's loops and maxloc/minloc do (k outermost, i fastest);
// ties go to the smaller L, so the result is the reference's first occurrence and
// independent of the launch shape.  Block partials are reduced by a second kernel.
#include <climits>

#include "mg_common.cuh"
#include "tma.cuh"

namespace {

constexpr long long NONE = LLONG_MAX;
constexpr int CHECK_BLOCKS = 592;   // 4 x 148 SMs
constexpr int NX = 6;               // cfl max, es max, es min, qt max, qt min, first non-finite

struct Ext {
    double v;
    long long L;
};

__device__ __forceinline__ void take_max(Ext &a, const Ext &b)
{
    if (b.L != NONE && (a.L == NONE || b.v > a.v || (b.v == a.v && b.L < a.L))) a = b;
}
__device__ __forceinline__ void take_min(Ext &a, const Ext &b)
{
    if (b.L != NONE && (a.L == NONE || b.v < a.v || (b.v == a.v && b.L < a.L))) a = b;
}

__device__ __forceinline__ void combine(Ext *a, const Ext *b)
{
    take_max(a[0], b[0]);
    take_max(a[1], b[1]);
    take_min(a[2], b[2]);
    take_max(a[3], b[3]);
    take_min(a[4], b[4]);
    if (b[5].L != NONE && (a[5].L == NONE || b[5].L < a[5].L)) a[5] = b[5];
}

__device__ void block_reduce(Ext *mine, Ext *out)
{
    __shared__ Ext sh[256][NX];
    for (int q = 0; q < NX; q++) sh[threadIdx.x][q] = mine[q];
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) combine(sh[threadIdx.x], sh[threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int q = 0; q < NX; q++) out[q] = sh[0][q];
}

__global__ void __launch_bounds__(256) check_partial_kernel(DevGrid G, const double *__restrict__ u,
                                                            const double *__restrict__ v,
                                                            const double *__restrict__ w,
                                                            const double *__restrict__ es,
                                                            const double *__restrict__ qt, Ext *part)
{
    Ext m[NX];
    for (int q = 0; q < NX; q++) m[q] = Ext{0., NONE};
    const long long n = (long long)G.maxx * G.maxy * G.nz;
    const double dx1 = 1. / G.dx, dy1 = 1. / G.dy, dt0 = G.dt0;
    for (long long L = blockIdx.x * (long long)blockDim.x + threadIdx.x; L < n; L += (long long)gridDim.x * blockDim.x) {
        const int i = 4 + (int)(L % G.maxx);
        const long long r = L / G.maxx;
        const int j = 4 + (int)(r % G.maxy);
        const int k = 1 + (int)(r / G.maxy);
        const long long c = gidx(G, i, j, k);
        // checkwind (:143-159): cfl = max(cflx, cfly, cflz), candidates > the running max 0
        const double cflx = dt0 * fabs(__ldg(u + c)) * dx1;
        const double cfly = dt0 * fabs(__ldg(v + c)) * dy1;
        const double cflz = dt0 * fabs(__ldg(w + c)) * __ldg(G.dz1w + k - 1);
        const double cfl = fmax_ref(fmax_ref(cflx, cfly), cflz);
        if (cfl > 0.) take_max(m[0], Ext{cfl, L});
        const double e = __ldg(es + c);
        take_max(m[1], Ext{e, L});
        take_min(m[2], Ext{e, L});
        bool finite = isfinite(cflx) && isfinite(cfly) && isfinite(cflz) && isfinite(e);
        if (qt) {
            const double q = __ldg(qt + c);
            take_max(m[3], Ext{q, L});
            take_min(m[4], Ext{q, L});
            finite = finite && isfinite(q);
        }
        if (!finite && m[5].L == NONE) m[5] = Ext{0., L};   // L grows along the loop: the first is the smallest
    }
    block_reduce(m, part + (size_t)blockIdx.x * NX);
}

__global__ void __launch_bounds__(256) check_final_kernel(const Ext *part, int nparts, Ext *out)
{
    Ext m[NX];
    for (int q = 0; q < NX; q++) m[q] = Ext{0., NONE};
    for (int b = threadIdx.x; b < nparts; b += blockDim.x) combine(m, part + (size_t)b * NX);
    block_reduce(m, out);
}

// The failure path of the bounded waits, exercised on purpose: one thread arms an
// mbarrier for 16 transaction bytes, issues no copy (nothing is in flight), and waits
// for it with the production wait and a cycle limit of the caller's choosing.  The wait
// runs out and raises the context's error flag, which the host reads as MG_ERR_TIMEOUT;
// the CTA then exits with nothing outstanding.
__global__ void selftest_wait_kernel(long long limit, int *err)
{
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
        mbar_arrive_expect_tx(&bar, 16);
        mbar_wait_bounded_n(&bar, 0, err, limit);
    }
}

}  // namespace

cudaError_t launch_selftest_wait(long long limit, int *err, cudaStream_t s)
{
    selftest_wait_kernel<<<1, 32, 0, s>>>(limit, err);
    return cudaGetLastError();
}

size_t check_scratch_bytes() { return (size_t)(CHECK_BLOCKS + 1) * NX * sizeof(Ext); }

// out (device): 6 x {double value, long long L} (L = LLONG_MAX when no candidate); the
// sixth is the first non-finite cell
cudaError_t launch_check(const DevGrid &g, const double *u, const double *v, const double *w, const double *es,
                         const double *qt, void *scratch, cudaStream_t s)
{
    Ext *part = (Ext *)scratch;
    const long long n = (long long)g.maxx * g.maxy * g.nz;
    int blocks = (int)((n + 255) / 256);
    if (blocks > CHECK_BLOCKS) blocks = CHECK_BLOCKS;
    check_partial_kernel<<<blocks, 256, 0, s>>>(g, u, v, w, es, qt, part);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    check_final_kernel<<<1, 256, 0, s>>>(part, blocks, part + (size_t)CHECK_BLOCKS * NX);
    return cudaGetLastError();
}
