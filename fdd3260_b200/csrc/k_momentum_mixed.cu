// k_momentum_mixed.cu -- K2, mixed form: FP32 stencil ring and flux arithmetic, FP64
// tendency accumulation, pressure gradient, buoyancy and stage update.  Body in
// k2_body.cuh.
#include "k2_body.cuh"

cudaError_t launch_k2_mixed(const DevGrid &g, const K2Args &a, const K2Maps &maps, cudaStream_t s)
{
    int ntx = (g.maxx + TX - 1) / TX, nty = (g.maxy + TY - 1) / TY;
    const size_t sm = k2_smem_bytes<float>();
    const bool even = (a.ntime % 2) == 0;   // direction order of the step (windadv.f90:103,158)
    cudaError_t e = even ? cudaFuncSetAttribute(k2_kernel<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm)
                         : cudaFuncSetAttribute(k2_kernel<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    K2Args as = a;
    if (as.nseg < 1 || as.nseg > g.nz) as.nseg = k2_segments(g, sm);
    if (even)
        k2_kernel<true, true><<<ntx * nty * as.nseg, dim3(TX, TY), sm, s>>>(g, as, maps);
    else
        k2_kernel<true, false><<<ntx * nty * as.nseg, dim3(TX, TY), sm, s>>>(g, as, maps);
    return cudaGetLastError();
}

cudaError_t launch_k2_group_mixed(int even, const K2GroupParams &P, const K2Maps *maps, const GItem *items, int nitems,
                            cudaStream_t s)
{
    return launch_k2_group_t<true>(even, P, maps, items, nitems, s);
}
