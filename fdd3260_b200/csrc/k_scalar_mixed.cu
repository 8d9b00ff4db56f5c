// k_scalar_mixed.cu -- K1, mixed form: the scheme logic (smoothness ratios,
// weights, limiters) in FP32 on differences relative to the upwind cell value, the
// face fluxes, tendencies and state in FP64.  Kernel body in k1_body.cuh.
#include "k1_body.cuh"


cudaError_t launch_k1_mixed(const DevGrid &g, const K1Args &a, const K1Maps &maps, cudaStream_t s)
{
    if (a.nf <= 0 || a.nf > MG_MAXF) return cudaErrorInvalidValue;
    const int ntx = (g.maxx + TX - 1) / TX, nty = (g.maxy + TY - 1) / TY;
    const dim3 grid(ntx * nty), block(TX, TY + 1);
    const size_t sm = make_layout(g.scal_adv, a.nf).total;
    if (sm > 232448) return cudaErrorInvalidValue;
    switch (g.scal_adv) {
    case MG_WENO: k1_kernel<MG_WENO, true><<<grid, block, sm, s>>>(g, a, maps); break;
    case MG_PPM: k1_kernel<MG_PPM, true><<<grid, block, sm, s>>>(g, a, maps); break;
    default: k1_kernel<MG_MUSCL, true><<<grid, block, sm, s>>>(g, a, maps); break;
    }
    return cudaGetLastError();
}

cudaError_t k1_mixed_init()
{
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(k1_kernel<MG_WENO, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 232448)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k1_kernel<MG_PPM, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 232448)) != cudaSuccess) return e;
    return cudaFuncSetAttribute(k1_kernel<MG_MUSCL, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 232448);
}
