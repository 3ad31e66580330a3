// ensemble.cu -- launchers of the persistent ensemble kernel (FP32-mixed,
// same flags as fused_mixed.cu): occupancy query and cooperative launch.
#include <cuda_runtime.h>

#include "ensemble.cuh"
#include "stages.hpp"

namespace hcl::ensemble {

namespace {

using KernelFn = void (*)(const Prob*, const int*, Params, unsigned int*, int*);

template <int LIM, int NW>
KernelFn pick_rs(int rs)
{
    if (rs == RS_HLL) {
        return k_ensemble<LIM, RS_HLL, NW>;
    }
    if (rs == RS_HLLC) {
        return k_ensemble<LIM, RS_HLLC, NW>;
    }
    return k_ensemble<LIM, RS_SPLITTING, NW>;
}

template <int NW>
KernelFn pick_nw(int lim, int rs)
{
    switch (lim) {
    case LIM_CONSTANT:
        return pick_rs<LIM_CONSTANT, NW>(rs);
    case LIM_VANLEER:
        return pick_rs<LIM_VANLEER, NW>(rs);
    case LIM_MINMOD:
        return pick_rs<LIM_MINMOD, NW>(rs);
    default:
        return pick_rs<LIM_VANALBADA, NW>(rs);
    }
}

// nw: warps per CTA, 4 or 16
KernelFn pick(int lim, int rs, int nw)
{
    return nw == 16 ? pick_nw<16>(lim, rs) : pick_nw<4>(lim, rs);
}

size_t ring_bytes(int nw)
{
    return sizeof(double) * (size_t)nw * fused::kStripRingDoubles;
}

} // namespace

int max_blocks_per_sm(int lim, int rs, int nw)
{
    KernelFn fn = pick(lim, rs, nw);
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ring_bytes(nw));
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, 32 * nw, ring_bytes(nw));
    return n;
}

cudaError_t launch(int lim, int rs, int nw, int grid, const Prob* probs, const int* item_prob, const Params& ep,
                   unsigned int* barrier, int* status, cudaStream_t s)
{
    KernelFn fn = pick(lim, rs, nw);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(32 * nw);
    cfg.dynamicSmemBytes = ring_bytes(nw);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    ++g_launches;
    return cudaLaunchKernelEx(&cfg, fn, probs, item_prob, ep, barrier, status);
}

} // namespace hcl::ensemble
