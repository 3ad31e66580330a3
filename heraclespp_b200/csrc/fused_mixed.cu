// fused_mixed.cu -- the FP32-mixed fused step (compiled with FMA contraction,
// -ftz=true -prec-div=false -prec-sqrt=false): FP32 primitives, slopes,
// face states and fluxes; FP64 stored state, internal-energy recovery,
// update accumulation and dt.
#include <cuda_runtime.h>

#include "fused_step.cuh"
#include "stages.hpp"

namespace hcl::fused {

// Schedules selectable at run time for 2-D (the autotuner picks one):
// 0-2 shared-memory tiles 16x16, 32x8, 32x16; 3-5 warp strips of 32, 64,
// 128 rows; 6 warp strips whose height fits one wave of resident warps; 9
// fitted warp strips in CTAs of 16 warps that march in step, rows staged by
// TMA; 10 the same with per-lane cp.async staging.  3-10 need a uniform
// Cartesian grid, 9 an even ghost width.  7 and 8 are unused (they were
// paired-column strips, slower than 6 and 9, and were removed).
// With passive scalars: the tiles,
// and for one or two scalars the 4-warp strips 3-6 (2-D), for one the column
// march (3-D).
// 3-D: 0 shared-memory tiles 8x8x4; 1 column march (uniform Cartesian grids).
int mixed_shape_count(int ndim)
{
    return ndim == 2 ? 11 : (ndim == 3 ? 2 : 1);
}

size_t mixed_smem_bytes(const GridDev& g, int shape)
{
    switch (g.ndim) {
    case 1:
        return FusedLauncher<1, false, 256, 1, 1>::smem(g.nfx);
    case 2:
        return shape == 1 ? FusedLauncher<2, false, 32, 8, 1>::smem(g.nfx)
                          : (shape == 2 ? FusedLauncher<2, false, 32, 16, 1>::smem(g.nfx)
                                        : FusedLauncher<2, false, 16, 16, 1>::smem(g.nfx));
    default:
        return FusedLauncher<3, false, 8, 8, 4>::smem(g.nfx);
    }
}

bool mixed_shape_valid(const GridDev& g, int shape)
{
    if (g.pressure_fix) {
        // the pressure fix rides in the shared-memory tiles only
        return (g.ndim == 2 ? shape < 3 : shape == 0) &&
               mixed_smem_bytes(g, shape) + kFusedStaticSmemMargin <= (size_t)smem_optin();
    }
    if (g.nfx > 0) {
        // passive scalars ride in the shared-memory tiles and, one or two of
        // them, in the 4-warp strips and the 3-D column march
        if (g.ndim == 2 && shape >= 3 && shape <= 6) {
            return strip2d_fx_eligible(g);
        }
        if (g.ndim == 3 && shape == 1) {
            return strip3d_fx_eligible(g);
        }
        return (g.ndim == 2 ? shape < 3 : shape == 0) && mixed_smem_bytes(g, shape) + kFusedStaticSmemMargin <= (size_t)smem_optin();
    }
    if (g.ndim == 3) {
        return shape == 0 || (shape == 1 && strip3d_eligible(g));
    }
    if (shape < 3) {
        return true;
    }
    if (shape == 9) {
        return strip2d_tma_eligible(g);
    }
    return (shape < 7 || shape == 10) && strip2d_eligible(g);
}

void configure_mixed()
{
    FusedLauncher<1, false, 256, 1, 1>::configure();
    FusedLauncher<2, false, 16, 16, 1>::configure();
    FusedLauncher<2, false, 32, 8, 1>::configure();
    FusedLauncher<2, false, 32, 16, 1>::configure();
    FusedLauncher<3, false, 8, 8, 4>::configure();
}

void step_mixed(const GridDev& g, const StateDev& in, const StateDev& out, StepCtl* ctl, const RunParamsDev& rp,
                int slot, int out_buf, int shape, cudaStream_t s)
{
    switch (g.ndim) {
    case 1:
        FusedLauncher<1, false, 256, 1, 1>::launch(g, in, out, ctl, rp, slot, out_buf, s);
        break;
    case 2:
        if ((shape == 9 && strip2d_tma_eligible(g)) || (shape == 10 && strip2d_eligible(g))) {
            step_strip2d(g, in, out, ctl, rp, slot, out_buf, 0, true, shape == 9, s);
        } else if (shape >= 3 && (strip2d_eligible(g) || (shape <= 6 && strip2d_fx_eligible(g)))) {
            step_strip2d(g, in, out, ctl, rp, slot, out_buf, shape == 3 ? 32 : (shape == 4 ? 64 : (shape == 5 ? 128 : 0)),
                         false, false, s);
        } else if (shape == 1) {
            FusedLauncher<2, false, 32, 8, 1>::launch(g, in, out, ctl, rp, slot, out_buf, s);
        } else if (shape == 2) {
            FusedLauncher<2, false, 32, 16, 1>::launch(g, in, out, ctl, rp, slot, out_buf, s);
        } else {
            FusedLauncher<2, false, 16, 16, 1>::launch(g, in, out, ctl, rp, slot, out_buf, s);
        }
        break;
    default:
        if (shape == 1 && (strip3d_eligible(g) || strip3d_fx_eligible(g))) {
            step_strip3d(g, in, out, ctl, rp, slot, out_buf, 0, s);
        } else {
            FusedLauncher<3, false, 8, 8, 4>::launch(g, in, out, ctl, rp, slot, out_buf, s);
        }
        break;
    }
}

} // namespace hcl::fused
