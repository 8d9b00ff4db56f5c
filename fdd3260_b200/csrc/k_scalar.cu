// k_scalar.cu -- K1 (scalar advection fused with the Heun stage update), plain FP64
// form.  The kernel body is in k1_body.cuh.  This translation unit is compiled
// with -fmad=false: bit-identical to the CPU restatement.
#include "k1_body.cuh"

size_t k1_smem_bytes(int scheme, int nf) { return make_layout(scheme, nf).total; }

cudaError_t launch_k1(const DevGrid &g, const K1Args &a, const K1Maps &maps, cudaStream_t s)
{
    if (a.nf <= 0 || a.nf > MG_MAXF) return cudaErrorInvalidValue;
    const int ntx = (g.maxx + TX - 1) / TX, nty = (g.maxy + TY - 1) / TY;
    const dim3 grid(ntx * nty), block(TX, TY + 1);
    const size_t sm = make_layout(g.scal_adv, a.nf).total;
    if (sm > 232448) return cudaErrorInvalidValue;
    switch (g.scal_adv) {
    case MG_WENO: k1_kernel<MG_WENO, false><<<grid, block, sm, s>>>(g, a, maps); break;
    case MG_PPM: k1_kernel<MG_PPM, false><<<grid, block, sm, s>>>(g, a, maps); break;
    default: k1_kernel<MG_MUSCL, false><<<grid, block, sm, s>>>(g, a, maps); break;
    }
    return cudaGetLastError();
}

cudaError_t k1_init()
{
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(k1_kernel<MG_WENO, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 232448)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k1_kernel<MG_PPM, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 232448)) != cudaSuccess) return e;
    return cudaFuncSetAttribute(k1_kernel<MG_MUSCL, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 232448);
}
