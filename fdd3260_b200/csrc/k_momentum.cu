// k_momentum.cu -- K2 (momentum tendency and stage update), plain FP64 form; body in
// k2_body.cuh.  Compiled with -fmad=false: bit-identical to the CPU restatement.
#include "k2_body.cuh"

cudaError_t launch_k2(const DevGrid &g, const K2Args &a, const K2Maps &maps, cudaStream_t s)
{
    int ntx = (g.maxx + TX - 1) / TX, nty = (g.maxy + TY - 1) / TY;
    const size_t sm = k2_smem_bytes<double>();
    const bool even = (a.ntime % 2) == 0;   // direction order of the step (windadv.f90:103,158)
    cudaError_t e = even ? cudaFuncSetAttribute(k2_kernel<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm)
                         : cudaFuncSetAttribute(k2_kernel<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    K2Args as = a;
    if (as.nseg < 1 || as.nseg > g.nz) as.nseg = k2_segments(g, sm);
    if (even)
        k2_kernel<false, true><<<ntx * nty * as.nseg, dim3(TX, TY), sm, s>>>(g, as, maps);
    else
        k2_kernel<false, false><<<ntx * nty * as.nseg, dim3(TX, TY), sm, s>>>(g, as, maps);
    return cudaGetLastError();
}

cudaError_t launch_k2_group(int even, const K2GroupParams &P, const K2Maps *maps, const GItem *items, int nitems,
                            cudaStream_t s)
{
    return launch_k2_group_t<false>(even, P, maps, items, nitems, s);
}
