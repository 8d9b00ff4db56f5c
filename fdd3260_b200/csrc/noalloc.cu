// noalloc.cu -- allocation-free variant of the projection residual.
//
// mg_maxdiv_noalloc computes the same quantity as the residual step of
// anelastic_pressure (src/PRESSURE/pressure_solver.f90:121-130: the signed maximum of
// caldiv, src/TOOLS/gradients.f90:986-1052, over the interior and k = 2..nz-1) with
// the same per-cell arithmetic as the context's maxdiv kernels, but it needs no
// context and allocates nothing: the per-block partial maxima live in the file-scope
// device array below, whose address is resolved once per device with
// cudaGetSymbolAddress.
//
// Limits and rules:
//  * scratch: NA_MAX_PARTIALS = 1024 block partials (8 KiB); the grid is capped at
//    that many blocks, each folding any number of cells with a grid-stride loop;
//  * domain: 1 <= maxx, maxy <= 4096 and 3 <= nz <= 4096 (larger sizes are rejected
//    with MG_ERR_PARAM before anything is launched);
//  * nothing in the scratch has to start at zero: every launched block writes its own
//    partial and the final reduction reads exactly those;
//  * the first call on a device resolves the scratch address; make it before any
//    stream capture that is to contain the call.  The address is kept for the life of
//    the process: after cudaDeviceReset (or any teardown of the device's primary
//    context) the module is loaded again and the array may move, so the entry must not
//    be used across a device reset;
//  * the scratch is one array per device: two calls in flight at the same time on one
//    device (other streams or host threads) race on it, so callers serialise them.
#include <mutex>

#include <cuda_runtime.h>

#include "mimica_gpu.h"

namespace {

constexpr int NA_MAX_PARTIALS = 1024;
constexpr int NA_THREADS = 256;
constexpr int NA_MAX_DEVICES = 64;

__device__ __align__(256) double g_maxdiv_partials[NA_MAX_PARTIALS];

double *g_scratch[NA_MAX_DEVICES] = {};
std::mutex g_scratch_mu;

// arrays in the reference layout: x(1:nx,1:ny,1:nz), C index ((k-1)*ny + (j-1))*nx + (i-1)
__global__ void na_maxdiv_partial(int maxx, int maxy, int nz, double dx, double dy, const double *dz1w,
                                  const double *mu, const double *mv, const double *mw, double *partial)
{
    __shared__ double sm[NA_THREADS];
    const int nx = maxx + 5, ny = maxy + 5;
    const long long plane = (long long)nx * ny;
    const double dx1 = 1. / dx, dy1 = 1. / dy;
    double m = -INFINITY;
    const long long tot = (long long)maxx * maxy * (nz - 2);
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += (long long)gridDim.x * blockDim.x) {
        const int ix = (int)(t % maxx), jy = (int)((t / maxx) % maxy), k = (int)(t / ((long long)maxx * maxy)) + 2;
        const long long c = (long long)(k - 1) * plane + (long long)(jy + 3) * nx + (ix + 3);
        double d = 0.;
        d = d + (mu[c + 1] - mu[c]) * dx1;
        d = d + (mv[c + nx] - mv[c]) * dy1;
        d = d + (mw[c + plane] - mw[c]) * dz1w[k - 1];
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

__global__ void na_max_final(const double *partial, int n, double *out)
{
    __shared__ double sm[NA_THREADS];
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

// scratch address of the current device.  Resolved again on every call outside a stream
// capture (a device reset reloads the module, and the symbol can move); a capture uses
// the address of the last call outside one, so that it issues no symbol lookup.
int scratch_of_current_device(cudaStream_t s, double **out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return MG_ERR_CUDA;
    if (dev < 0 || dev >= NA_MAX_DEVICES) return MG_ERR_PARAM;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess) return MG_ERR_CUDA;
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (!g_scratch[dev] || cs == cudaStreamCaptureStatusNone) {
        double *p = nullptr;
        cudaError_t rc = cudaGetSymbolAddress((void **)&p, g_maxdiv_partials);
        if (rc != cudaSuccess || !p) return MG_ERR_CUDA;
        g_scratch[dev] = p;
    }
    *out = g_scratch[dev];
    return MG_OK;
}

}  // namespace

extern "C" int mg_maxdiv_noalloc(int maxx, int maxy, int nz, double dx, double dy, const double *dz1w,
                                 const double *mu, const double *mv, const double *mw, double *maxdiv,
                                 void *stream)
{
    if (maxx < 1 || maxy < 1 || maxx > 4096 || maxy > 4096 || nz < 3 || nz > 4096) return MG_ERR_PARAM;
    if (!dz1w || !mu || !mv || !mw || !maxdiv || !(dx > 0.) || !(dy > 0.)) return MG_ERR_PARAM;
    cudaStream_t s = (cudaStream_t)stream;
    double *partial = nullptr;
    int st = scratch_of_current_device(s, &partial);
    if (st != MG_OK) return st;
    const long long tot = (long long)maxx * maxy * (nz - 2);
    long long nb = (tot + NA_THREADS - 1) / NA_THREADS;
    if (nb > NA_MAX_PARTIALS) nb = NA_MAX_PARTIALS;
    na_maxdiv_partial<<<(unsigned)nb, NA_THREADS, 0, s>>>(maxx, maxy, nz, dx, dy, dz1w, mu, mv, mw, partial);
    if (cudaGetLastError() != cudaSuccess) return MG_ERR_CUDA;
    na_max_final<<<1, NA_THREADS, 0, s>>>(partial, (int)nb, maxdiv);
    if (cudaGetLastError() != cudaSuccess) return MG_ERR_CUDA;
    return MG_OK;
}
