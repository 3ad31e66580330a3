// fused_fp64_fast.cu -- the fast-FP64 fused step (precision HCL_FP64_FAST):
// the FP64 tile kernels of fused_step.cuh with the perfect gas in its fast
// forms (EOS_PERFECT_GAS_FAST in physics_exact.cuh: P = (gamma-1) e, one
// reciprocal of rho per state, limiters on raw differences, one reciprocal
// in HLLC), compiled with FMA contraction.  Everything is FP64; the results
// differ from the reference's FP64 arithmetic by rounding only, and are held
// to 1e-12 relative L1 per variable against the oracle.
#include <cuda_runtime.h>

#include "fused_step.cuh"
#include "per_device.hpp"
#include "stages.hpp"

namespace hcl::fused {

namespace {
bool big_tile_3d_fits_fast(const GridDev& g)
{
    return FusedLauncher<3, true, 8, 8, 4>::smem(g.nfx) + kFusedStaticSmemMargin <= (size_t)smem_optin();
}
} // namespace

void step_fast64(const GridDev& g, const StateDev& in, const StateDev& out, StepCtl* ctl, const RunParamsDev& rp,
                 int slot, int out_buf, cudaStream_t s)
{
    switch (g.ndim) {
    case 1:
        FusedLauncher<1, true, 128, 1, 1>::launch_kind<EOS_PERFECT_GAS_FAST>(g, in, out, ctl, rp, slot, out_buf, s);
        break;
    case 2:
        FusedLauncher<2, true, 16, 16, 1>::launch_kind<EOS_PERFECT_GAS_FAST>(g, in, out, ctl, rp, slot, out_buf, s);
        break;
    default:
        if (big_tile_3d_fits_fast(g)) {
            FusedLauncher<3, true, 8, 8, 4>::launch_kind<EOS_PERFECT_GAS_FAST>(g, in, out, ctl, rp, slot, out_buf, s);
        } else {
            FusedLauncher<3, true, 8, 4, 4>::launch_kind<EOS_PERFECT_GAS_FAST>(g, in, out, ctl, rp, slot, out_buf, s);
        }
        break;
    }
}

void configure_fast64()
{
    FusedLauncher<1, true, 128, 1, 1>::configure_fast();
    FusedLauncher<2, true, 16, 16, 1>::configure_fast();
    FusedLauncher<3, true, 8, 4, 4>::configure_fast();
    FusedLauncher<3, true, 8, 8, 4>::configure_fast();
}

} // namespace hcl::fused
