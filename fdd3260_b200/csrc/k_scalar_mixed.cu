// k_scalar_mixed.cu -- K1, mixed form: the scheme logic (smoothness ratios,
// weights, limiters) in FP32 on differences relative to the upwind cell value, the
// face fluxes, tendencies and state in FP64.  Kernel body in k1_body.cuh.
#include "k1_body.cuh"

namespace {
template <int SCHEME, int STAGE>
cudaError_t launch_one(const DevGrid &g, const K1Args &a, const K1Maps &maps, cudaStream_t s)
{
    const size_t sm = make_layout(SCHEME, a.nf, STAGE).total;
    const int ntx = (g.maxx + TX - 1) / TX, nty = (g.maxy + TY - 1) / TY;
    K1Args as = a;
    if (as.nseg < 1 || as.nseg > g.nz) as.nseg = k1_segments(g, SCHEME, sm);
    if (SCHEME == MG_PPM) as.nseg = 1;
    bool sgs = false;
    for (int f = 0; f < a.nf; f++) sgs = sgs || a.sgs[f] != nullptr;
    if (STAGE != 0 && sgs)
        k1_kernel<SCHEME, true, STAGE, true><<<dim3(ntx * nty * as.nseg), dim3(TX, TY + 1), sm, s>>>(g, as, maps);
    else if (STAGE != 0 && a.nf == K1_FC)   // density + 5 scalars: the field count compiled in
        k1_kernel<SCHEME, true, STAGE, false, K1_FC><<<dim3(ntx * nty * as.nseg), dim3(TX, TY + 1), sm, s>>>(g, as, maps);
    else
        k1_kernel<SCHEME, true, STAGE, false><<<dim3(ntx * nty * as.nseg), dim3(TX, TY + 1), sm, s>>>(g, as, maps);
    return cudaGetLastError();
}
template <int SCHEME>
cudaError_t launch_scheme(const DevGrid &g, const K1Args &a, const K1Maps &maps, cudaStream_t s)
{
    if (a.mode == 1) return launch_one<SCHEME, 0>(g, a, maps, s);
    if (a.stage == 1) return launch_one<SCHEME, 1>(g, a, maps, s);
    return launch_one<SCHEME, 2>(g, a, maps, s);
}
template <int SCHEME>
cudaError_t init_scheme()
{
    cudaError_t e;
    const int mx = 232448;
    if ((e = cudaFuncSetAttribute(k1_kernel<SCHEME, true, 0, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k1_kernel<SCHEME, true, 1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k1_kernel<SCHEME, true, 2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k1_kernel<SCHEME, true, 1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k1_kernel<SCHEME, true, 1, false, K1_FC>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k1_kernel<SCHEME, true, 2, false, K1_FC>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx)) != cudaSuccess) return e;
    return cudaFuncSetAttribute(k1_kernel<SCHEME, true, 2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
}
template <int SCHEME, int STAGE>
cudaError_t group_one(int nf, const K1Member *mem, const GItem *items, int nitems, cudaStream_t s)
{
    const size_t sm = make_layout(SCHEME, nf, STAGE).total;
    if (nf == K1_FC) {
        cudaError_t e = cudaFuncSetAttribute(k1_group_kernel<SCHEME, true, STAGE, K1_FC>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
        k1_group_kernel<SCHEME, true, STAGE, K1_FC><<<nitems, dim3(TX, TY + 1), sm, s>>>(mem, items);
    } else {
        cudaError_t e = cudaFuncSetAttribute(k1_group_kernel<SCHEME, true, STAGE>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
        k1_group_kernel<SCHEME, true, STAGE><<<nitems, dim3(TX, TY + 1), sm, s>>>(mem, items);
    }
    return cudaGetLastError();
}
template <int SCHEME>
cudaError_t group_scheme(int stage, int nf, const K1Member *mem, const GItem *items, int nitems, cudaStream_t s)
{
    return stage == 1 ? group_one<SCHEME, 1>(nf, mem, items, nitems, s) : group_one<SCHEME, 2>(nf, mem, items, nitems, s);
}
}  // namespace

cudaError_t launch_k1_mixed(const DevGrid &g, const K1Args &a, const K1Maps &maps, cudaStream_t s)
{
    if (a.nf <= 0 || a.nf > MG_MAXF) return cudaErrorInvalidValue;
    if (a.mode != 1 && a.stage != 1 && a.stage != 2) return cudaErrorInvalidValue;
    if (k1_smem_max(g.scal_adv, a.nf) > 232448) return cudaErrorInvalidValue;
    switch (g.scal_adv) {
    case MG_WENO: return launch_scheme<MG_WENO>(g, a, maps, s);
    case MG_PPM: return launch_scheme<MG_PPM>(g, a, maps, s);
    case MG_LW: return launch_scheme<MG_LW>(g, a, maps, s);
    case MG_QUICK: return launch_scheme<MG_QUICK>(g, a, maps, s);
    default: return launch_scheme<MG_MUSCL>(g, a, maps, s);
    }
}

cudaError_t k1_mixed_init()
{
    cudaError_t e;
    if ((e = init_scheme<MG_WENO>()) != cudaSuccess) return e;
    if ((e = init_scheme<MG_PPM>()) != cudaSuccess) return e;
    if ((e = init_scheme<MG_LW>()) != cudaSuccess) return e;
    if ((e = init_scheme<MG_QUICK>()) != cudaSuccess) return e;
    return init_scheme<MG_MUSCL>();
}

// K1 over the blocks of several members (same scheme, stage and field count; no SGS)
cudaError_t launch_k1_group_mixed(int scheme, int stage, int nf, const K1Member *mem, const GItem *items, int nitems, cudaStream_t s)
{
    if (nf <= 0 || nf > MG_MAXF || (stage != 1 && stage != 2) || nitems < 1) return cudaErrorInvalidValue;
    if (k1_smem_max(scheme, nf) > 232448) return cudaErrorInvalidValue;
    switch (scheme) {
    case MG_WENO: return group_scheme<MG_WENO>(stage, nf, mem, items, nitems, s);
    case MG_PPM: return group_scheme<MG_PPM>(stage, nf, mem, items, nitems, s);
    case MG_LW: return group_scheme<MG_LW>(stage, nf, mem, items, nitems, s);
    case MG_QUICK: return group_scheme<MG_QUICK>(stage, nf, mem, items, nitems, s);
    default: return group_scheme<MG_MUSCL>(stage, nf, mem, items, nitems, s);
    }
}
