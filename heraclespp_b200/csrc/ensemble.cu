// ensemble.cu -- launchers of the persistent ensemble kernel (FP32-mixed,
// same flags as fused_mixed.cu): occupancy query and cooperative launch.
#include <cuda_runtime.h>

#include "ensemble.cuh"
#include "stages.hpp"

namespace hcl::ensemble {

namespace {

using KernelFn = void (*)(const Prob*, const int*, Params, unsigned int*, int*);

template <int LIM>
KernelFn pick_rs(int rs)
{
    if (rs == RS_HLL) {
        return k_ensemble<LIM, RS_HLL>;
    }
    if (rs == RS_HLLC) {
        return k_ensemble<LIM, RS_HLLC>;
    }
    return k_ensemble<LIM, RS_SPLITTING>;
}

KernelFn pick(int lim, int rs)
{
    switch (lim) {
    case LIM_CONSTANT:
        return pick_rs<LIM_CONSTANT>(rs);
    case LIM_VANLEER:
        return pick_rs<LIM_VANLEER>(rs);
    case LIM_MINMOD:
        return pick_rs<LIM_MINMOD>(rs);
    default:
        return pick_rs<LIM_VANALBADA>(rs);
    }
}

} // namespace

int max_blocks_per_sm(int lim, int rs)
{
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, pick(lim, rs), 128, 0);
    return n;
}

cudaError_t launch(int lim, int rs, int grid, const Prob* probs, const int* item_prob, const Params& ep,
                   unsigned int* barrier, int* status, cudaStream_t s)
{
    KernelFn fn = pick(lim, rs);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(128);
    cfg.dynamicSmemBytes = 0;
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
