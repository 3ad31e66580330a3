// fused_strip3.cu -- instantiations and launcher of the 3-D column-march
// mixed step for every limiter x Riemann solver pair (same flags as
// fused_mixed.cu).
#include <cuda_runtime.h>

#include <algorithm>

#include "fused_strip3d.cuh"
#include "per_device.hpp"
#include "stages.hpp"

namespace hcl::fused {

bool strip3d_fx_eligible(const GridDev& g)
{
    return g.ndim == 3 && g.uniform_cart && g.geom == GEOM_CARTESIAN && g.gravity == GRAV_UNIFORM && g.ng >= 2 &&
           (g.nfx == 1 || g.nfx == 2);
}

bool strip3d_eligible(const GridDev& g)
{
    return g.ndim == 3 && g.uniform_cart && g.geom == GEOM_CARTESIAN && g.gravity == GRAV_UNIFORM && g.ng >= 2 &&
           g.nfx == 0;
}

namespace {

template <int LIM, int RS, int NFX>
void launch_lrf(const GridDev& g, const StateDev& in, const StateDev& out, StepCtl* ctl, const RunParamsDev& rp,
                int slot, int out_buf, int L, cudaStream_t s)
{
    constexpr int kSmem = (int)sizeof(S3SharedT<NFX>);
    // shared-memory opt-in and resident CTAs, once per device
    static PerDevice cache;
    int dev = 0;
    cudaGetDevice(&dev);
    const int resident = cache.get(dev, [&] {
        cudaFuncSetAttribute(k_strip3d<LIM, RS, NFX>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmem);
        int per_sm = 0, nsm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_strip3d<LIM, RS, NFX>, kS3Threads, kSmem);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        return std::max(1, per_sm) * (nsm > 0 ? nsm : 148);
    });
    const int ncol = ((g.nx[0] + 27) / 28) * ((g.nx[1] + 11) / 12);
    if (L <= 0) {
        // plane count per CTA that minimises (waves + 1/2) x (planes + 3): the
        // start-up planes of each CTA, and half a CTA of imbalance in the last
        // wave.  Chunks of at least 80 planes (RT 256^2 x 512: 2, 4, 6 and 8
        // chunks of the z column took 1.992, 1.963, 1.961 and 1.972 ms per
        // step; waves x (planes + 2) had picked 2)
        double best = -1;
        const int Lmin = std::min(80, g.nx[2]);
        for (int nzc = 1; nzc <= std::max(1, g.nx[2] / 4); ++nzc) {
            const int Lc = (g.nx[2] + nzc - 1) / nzc;
            if (Lc < Lmin) {
                break;
            }
            const long waves = ((long)ncol * nzc + resident - 1) / resident;
            const double cost = (waves + 0.5) * (Lc + 3);
            if (best < 0 || cost < best) {
                best = cost;
                L = Lc;
            }
        }
    }
    const int nzc = (g.nx[2] + L - 1) / L;
    k_strip3d<LIM, RS, NFX><<<ncol * nzc, kS3Threads, kSmem, s>>>(g, in, out, ctl, rp, slot, out_buf, L);
}

template <int LIM, int RS>
void launch_lr(const GridDev& g, const StateDev& in, const StateDev& out, StepCtl* ctl, const RunParamsDev& rp, int slot,
               int out_buf, int L, cudaStream_t s)
{
    if (g.nfx == 2) {
        launch_lrf<LIM, RS, 2>(g, in, out, ctl, rp, slot, out_buf, L, s);
    } else if (g.nfx == 1) {
        launch_lrf<LIM, RS, 1>(g, in, out, ctl, rp, slot, out_buf, L, s);
    } else {
        launch_lrf<LIM, RS, 0>(g, in, out, ctl, rp, slot, out_buf, L, s);
    }
}

template <int LIM>
void launch_l(const GridDev& g, const StateDev& in, const StateDev& out, StepCtl* ctl, const RunParamsDev& rp, int slot,
              int out_buf, int L, cudaStream_t s)
{
    if (g.riemann == RS_HLL) {
        launch_lr<LIM, RS_HLL>(g, in, out, ctl, rp, slot, out_buf, L, s);
    } else if (g.riemann == RS_HLLC) {
        launch_lr<LIM, RS_HLLC>(g, in, out, ctl, rp, slot, out_buf, L, s);
    } else {
        launch_lr<LIM, RS_SPLITTING>(g, in, out, ctl, rp, slot, out_buf, L, s);
    }
}

} // namespace

void step_strip3d(const GridDev& g, const StateDev& in, const StateDev& out, StepCtl* ctl, const RunParamsDev& rp,
                  int slot, int out_buf, int L, cudaStream_t s)
{
    switch (g.limiter) {
    case LIM_CONSTANT:
        launch_l<LIM_CONSTANT>(g, in, out, ctl, rp, slot, out_buf, L, s);
        break;
    case LIM_VANLEER:
        launch_l<LIM_VANLEER>(g, in, out, ctl, rp, slot, out_buf, L, s);
        break;
    case LIM_MINMOD:
        launch_l<LIM_MINMOD>(g, in, out, ctl, rp, slot, out_buf, L, s);
        break;
    default:
        launch_l<LIM_VANALBADA>(g, in, out, ctl, rp, slot, out_buf, L, s);
        break;
    }
    ++g_launches;
}

} // namespace hcl::fused
