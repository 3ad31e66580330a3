// ensemble_adjoint.cu -- reverse pass of a batched ensemble in persistent
// launches: per checkpoint segment one launch of the ensemble's own forward
// kernel recomputes every problem's segment states (segment mode, recorded
// dts), then one cooperative launch sweeps every problem's segment back, step
// by step, with one grid barrier per step.  Three adjoint buffers rotate: step
// j reads lam[a] (the adjoint of its output), adds into lam[b] (its input),
// with each ghost's contribution sent to the interior cell the ghost is
// filled from, and clears the interior of lam[c], which step j-1 adds into.
// Same per-tile code and flags as the single-problem adjoint (adjoint.cu).
#include <cuda_runtime.h>

#include "adjoint_step.cuh"
#include "ensemble.cuh"
#include "per_device.hpp"
#include "stages.hpp"

namespace hcl::ensemble {

namespace {

using adjoint::AdjShape;

template <class R>
constexpr size_t rev_smem()
{
    return AdjShape<2, R, kRevTile, kRevTile, 1>::smem();
}

__global__ void k_seg_init(const AdjProb* __restrict__ probs, int nprob, int sg, int first)
{
    const int64_t gtid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t gsize = (int64_t)gridDim.x * blockDim.x;
    for (int p = 0; p < nprob; ++p) {
        const AdjProb& P = probs[p];
        const double* src = P.ckpt + P.sz * sg;
        double* dst = P.seg0.q;
        for (int64_t i = gtid; i < P.sz; i += gsize) {
            dst[i] = src[i];
        }
    }
    if (gtid < nprob) {
        StepCtl* c = probs[gtid].ctl;
        c->inv_dt_bits[0] = c->inv_dt_bits[1] = c->inv_dt_bits[2] = 0ull;
        c->t[0] = c->t[1] = 0.0;
        c->iter[0] = c->iter[1] = first;
        c->time_output_id[0] = c->time_output_id[1] = -1;
        c->iter_output_id[0] = c->iter_output_id[1] = -1;
        c->stop[0] = c->stop[1] = 0;
        c->errflag[0] = c->errflag[1] = 0;
        c->final_buf = 0;
        c->err = 0;
        c->bad_cell = ~0ull;
        c->last_dt = 0.0;
    }
}

template <class R>
__global__ void __launch_bounds__(kRevTile * kRevTile, sizeof(R) == 8 ? 2 : 3)
k_ens_reverse(const AdjProb* __restrict__ probs, const int* __restrict__ tile_prob, AdjParams ap,
              unsigned int* barrier, int* status)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ GridDev sg; // the tile's grid, read from shared memory by the tile code
    // lam[cur] holds the adjoint of the segment's last output state and the
    // interior of lam[cur + 1] is zero: the host clears all three buffers
    // before the first segment, and the last step of a segment clears the
    // buffer the next segment's first step adds into
    int cur = ap.cur;
    unsigned int phase = 0;
    for (int j = ap.len - 1; j >= 0; --j) {
        const int n = ap.first + j;
        const int nxt = cur == 2 ? 0 : cur + 1;
        const int clr = nxt == 2 ? 0 : nxt + 1;
        int loaded = -1;
        for (int item = blockIdx.x; item < ap.ntiles; item += gridDim.x) {
            const int p = tile_prob[item];
            const AdjProb& P = probs[p];
            if (p != loaded) {
                __syncthreads(); // the previous tile is done with sg
                const int nw = (int)(sizeof(GridDev) / sizeof(int));
                for (int i = threadIdx.x; i < nw; i += blockDim.x) {
                    reinterpret_cast<int*>(&sg)[i] = reinterpret_cast<const int*>(&P.g)[i];
                }
                loaded = p;
            }
            fused::StateDev U = P.seg0;
            U.q += P.sz * j;
            // the forward is the ensemble's FP32-mixed kernel: no FP64 forward rounding to reproduce
            adjoint::adjoint_tile<2, R, kRevTile, kRevTile, 1, kRevTile * kRevTile, false, false>(
                sg, U, P.lam[cur], P.lam[nxt], P.dts[n], item - P.tile0, smem_raw, &P.lam[clr], true);
        }
        if (!grid_barrier(barrier, (++phase) * gridDim.x, status)) {
            return;
        }
        cur = nxt;
    }
}

// shared-memory opt-in and resident CTAs per SM, once per device
template <class R>
int blocks_per_sm()
{
    static PerDevice cache;
    int dev = 0;
    cudaGetDevice(&dev);
    return cache.get(dev, [] {
        cudaFuncSetAttribute(k_ens_reverse<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rev_smem<R>());
        int n = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_ens_reverse<R>, kRevTile * kRevTile, rev_smem<R>());
        return n;
    });
}

template <class R>
cudaError_t launch_rev(int grid, const AdjProb* probs, const int* tile_prob, const AdjParams& ap,
                       unsigned int* barrier, int* status, cudaStream_t s)
{
    blocks_per_sm<R>();
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(kRevTile * kRevTile);
    cfg.dynamicSmemBytes = rev_smem<R>();
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    ++g_launches;
    return cudaLaunchKernelEx(&cfg, k_ens_reverse<R>, probs, tile_prob, ap, barrier, status);
}

} // namespace

int reverse_blocks_per_sm(bool fp64)
{
    return fp64 ? blocks_per_sm<double>() : blocks_per_sm<float>();
}

void seg_init(const AdjProb* probs, int nprob, int sg, int first, cudaStream_t s)
{
    k_seg_init<<<148 * 4, 256, 0, s>>>(probs, nprob, sg, first);
    ++g_launches;
}

cudaError_t reverse(bool fp64, int grid, const AdjProb* probs, const int* tile_prob, const AdjParams& ap,
                    unsigned int* barrier, int* status, cudaStream_t s)
{
    return fp64 ? launch_rev<double>(grid, probs, tile_prob, ap, barrier, status, s)
                : launch_rev<float>(grid, probs, tile_prob, ap, barrier, status, s);
}

} // namespace hcl::ensemble
