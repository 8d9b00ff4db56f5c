// tma.cuh -- Tensor Memory Accelerator (cp.async.bulk.tensor) and mbarrier helpers
// for sm_100a, written with inline PTX; plus cp.async (LDGSTS) helpers.
//
// Rules kept everywhere (see the CUDA/PTX documentation of the tiled bulk copy):
//  * tensor maps cover one device array; the innermost box start coordinate times
//    the element size is a multiple of 16 bytes (x even for doubles);
//  * shared-memory destinations are 128-byte aligned;
//  * loads only (no TMA store or reduce), no cluster multicast;
//  * every wait on an mbarrier is bounded by a clock64 deadline; on expiry the
//    waiting thread raises the kernel's error flag and carries on, so a kernel
//    always terminates (the host reports MG_ERR_TIMEOUT).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#ifndef MG_WAIT_CYCLES
#define MG_WAIT_CYCLES (4000000000LL)   // ~2 s at 2 GHz
#endif

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_shared()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// bounded wait of at most `limit` SM clock cycles; returns false (and raises *err) on timeout
__device__ __forceinline__ bool mbar_wait_bounded_n(uint64_t *bar, uint32_t parity, int *err, long long limit)
{
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (clock64() - t0 > limit) {
            if (err) atomicOr(err, 1);
            return false;
        }
    }
    return true;
}
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, int *err)
{
    return mbar_wait_bounded_n(bar, parity, err, MG_WAIT_CYCLES);
}

// A tensor map that the host wrote to global memory (cudaMemcpy) before the launch:
// acquire it for the tensor-map proxy before this thread's first bulk copy through it
// (system scope: the write came from the host).
__device__ __forceinline__ void tensormap_acquire(const CUtensorMap *map)
{
    asm volatile("fence.proxy.tensormap::generic.acquire.sys [%0], 128;" ::"l"((uint64_t)map) : "memory");
}

// 3-D tiled bulk copy global -> shared, completion signalled on bar
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int y, int z, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"(smem_u32(dst)), "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

// 8-byte asynchronous copy global -> shared (LDGSTS); visible to the issuing thread
// after cp_async_wait_all()
__device__ __forceinline__ void cp_async_8(void *dst, const void *src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
// read-only load of a streamed value that is used once: no L1 line is allocated for it,
// so the small per-level coefficient arrays stay in L1
__device__ __forceinline__ double ldg_stream(const double *p)
{
    double v;
    asm volatile("ld.global.nc.L1::no_allocate.f64 %0, [%1];" : "=d"(v) : "l"(p));
    return v;
}
// the same for a value this kernel later overwrites (not read through the non-coherent path)
__device__ __forceinline__ double ld_stream(const double *p)
{
    double v;
    asm volatile("ld.global.L1::no_allocate.f64 %0, [%1];" : "=d"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_group_1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

// ---- host: tensor map of a halo'd field (dims nx, ny, nz; row pitch px doubles) ----
#ifndef __CUDACC_RTC__
#include <cudaTypedefs.h>
static inline CUresult mg_encode_field_map(CUtensorMap *map, const double *base, int nx, int ny, int nz, int px,
                                           int boxx, int boxy)
{
    static PFN_cuTensorMapEncodeTiled_v12000 enc = nullptr;
    if (!enc) {
        cudaDriverEntryPointQueryResult q;
        void *fn = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn)
            return CUDA_ERROR_NOT_FOUND;
        enc = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    }
    cuuint64_t dims[3] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz};
    cuuint64_t strides[2] = {(cuuint64_t)px * 8, (cuuint64_t)px * 8 * (cuuint64_t)ny};
    cuuint32_t box[3] = {(cuuint32_t)boxx, (cuuint32_t)boxy, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    return enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, (void *)base, dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
}
#endif
