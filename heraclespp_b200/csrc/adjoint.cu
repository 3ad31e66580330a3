// adjoint.cu -- launchers of the discrete-adjoint kernels (FP64 and FP32-mixed
// reverse sweeps; the stored state and the adjoint state are FP64).
#include <cuda_runtime.h>

#include <algorithm>

#include "adjoint_step.cuh"
#include "stages.hpp"

namespace hcl::adjoint {

namespace {

// the device's largest dynamic shared-memory opt-in per block
int smem_optin()
{
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    return v;
}

template <int ND, class R, int TX, int TY, int TZ, int NT, bool SPH = false, bool EXACTB = true>
struct Launcher {
    using S = Shape<ND, TX, TY, TZ>;
    static size_t smem(int nfx = 0) { return AdjShape<ND, R, TX, TY, TZ>::smem(nfx); }
    static void configure()
    {
        cudaFuncSetAttribute(k_adjoint_step<ND, R, TX, TY, TZ, NT, SPH, EXACTB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem());
        // with passive scalars the size depends on their count: allow the opt-in
        cudaFuncSetAttribute(k_adjoint_step<ND, R, TX, TY, TZ, NT, SPH, EXACTB, true>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, smem_optin());
        // grids of user-defined nodes
        cudaFuncSetAttribute(k_adjoint_step<ND, R, TX, TY, TZ, NT, SPH, EXACTB, false, true>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem());
        cudaFuncSetAttribute(k_adjoint_step<ND, R, TX, TY, TZ, NT, SPH, EXACTB, true, true>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, smem_optin());
    }
    static void launch(const GridDev& g, const StateDev& U, const StateDev& lo, const StateDev& li, double dt,
                       const StateDev& lz, double* gbar, cudaStream_t s)
    {
        const int nt0 = (g.nx[0] + S::T0 - 1) / S::T0;
        const int nt1 = (g.nx[1] + S::T1 - 1) / S::T1;
        const int nt2 = (g.nx[2] + S::T2 - 1) / S::T2;
        const dim3 grid(nt0 * nt1 * nt2);
        if (!g.uniform_dx) {
            if (g.nfx > 0) {
                k_adjoint_step<ND, R, TX, TY, TZ, NT, SPH, EXACTB, true, true>
                    <<<grid, NT, smem(g.nfx), s>>>(g, U, lo, li, dt, lz, gbar);
            } else {
                k_adjoint_step<ND, R, TX, TY, TZ, NT, SPH, EXACTB, false, true>
                    <<<grid, NT, smem(), s>>>(g, U, lo, li, dt, lz, gbar);
            }
        } else if (g.nfx > 0) {
            k_adjoint_step<ND, R, TX, TY, TZ, NT, SPH, EXACTB, true><<<grid, NT, smem(g.nfx), s>>>(g, U, lo, li, dt, lz, gbar);
        } else {
            k_adjoint_step<ND, R, TX, TY, TZ, NT, SPH, EXACTB><<<grid, NT, smem(), s>>>(g, U, lo, li, dt, lz, gbar);
        }
        ++g_launches;
    }
};

// Threads per CTA: the 2-D FP32 sweep runs its 16x16 tile with 384 threads,
// so the 320 Hancock cells and the 400 stencil cells of a tile take about one
// round each (measured 8 % faster than 256 threads); the FP64 sweep keeps 256
// threads and two CTAs per SM.
template <bool SPH, bool EXACTB>
struct Launchers {
    using L1d = Launcher<1, double, 128, 1, 1, 128, SPH, EXACTB>;
    using L2d = Launcher<2, double, 16, 16, 1, 256, SPH, EXACTB>;
    using L3d = Launcher<3, double, 8, 4, 4, 128, SPH, EXACTB>;
    using L1f = Launcher<1, float, 128, 1, 1, 128, SPH, true>;
    using L2f = Launcher<2, float, 16, 16, 1, 384, SPH, true>;
    using L3f = Launcher<3, float, 8, 4, 4, 128, SPH, true>;

    static size_t smem(int ndim, bool fp64, int nfx)
    {
        if (fp64) {
            return ndim == 1 ? L1d::smem(nfx) : (ndim == 2 ? L2d::smem(nfx) : L3d::smem(nfx));
        }
        return ndim == 1 ? L1f::smem(nfx) : (ndim == 2 ? L2f::smem(nfx) : L3f::smem(nfx));
    }

    static void configure()
    {
        L1d::configure();
        L2d::configure();
        L3d::configure();
        L1f::configure();
        L2f::configure();
        L3f::configure();
    }

    static void step(const GridDev& g, const StateDev& U, const StateDev& lam_out, const StateDev& lam_in, double dt,
                     bool fp64, const StateDev& lam_zero, double* gbar, cudaStream_t s)
    {
        if (fp64) {
            if (g.ndim == 1) {
                L1d::launch(g, U, lam_out, lam_in, dt, lam_zero, gbar, s);
            } else if (g.ndim == 2) {
                L2d::launch(g, U, lam_out, lam_in, dt, lam_zero, gbar, s);
            } else {
                L3d::launch(g, U, lam_out, lam_in, dt, lam_zero, gbar, s);
            }
        } else {
            if (g.ndim == 1) {
                L1f::launch(g, U, lam_out, lam_in, dt, lam_zero, gbar, s);
            } else if (g.ndim == 2) {
                L2f::launch(g, U, lam_out, lam_in, dt, lam_zero, gbar, s);
            } else {
                L3f::launch(g, U, lam_out, lam_in, dt, lam_zero, gbar, s);
            }
        }
    }
};

} // namespace

void configure()
{
    Launchers<false, true>::configure();
    Launchers<true, true>::configure();
    Launchers<false, false>::configure();
    Launchers<true, false>::configure();
}

int scalar_sweep_fits(int ndim, bool fp64, int nfx, size_t* need, size_t* avail)
{
    // the tile shapes do not depend on the geometry
    *need = Launchers<false, true>::smem(ndim, fp64, nfx);
    *avail = (size_t)smem_optin();
    return *need <= *avail;
}

void step(const GridDev& g, const StateDev& U, const StateDev& lam_out, const StateDev& lam_in, double dt, bool fp64,
          bool exact_branches, const StateDev& lam_zero, double* gbar, cudaStream_t s)
{
    // the FP32 sweep has one form: its instantiation does not depend on EXACTB
    const bool eb = exact_branches || !fp64;
    if (g.geom == GEOM_SPHERICAL) {
        if (eb) {
            Launchers<true, true>::step(g, U, lam_out, lam_in, dt, fp64, lam_zero, gbar, s);
        } else {
            Launchers<true, false>::step(g, U, lam_out, lam_in, dt, fp64, lam_zero, gbar, s);
        }
    } else {
        if (eb) {
            Launchers<false, true>::step(g, U, lam_out, lam_in, dt, fp64, lam_zero, gbar, s);
        } else {
            Launchers<false, false>::step(g, U, lam_out, lam_in, dt, fp64, lam_zero, gbar, s);
        }
    }
}

namespace {
// Reverse of InternalMassGravity (gravity.cpp:59-128, the forward in
// stage_kernels.cu k_internal_mass_gravity): g_r[i] = -G M_i / xc_i^2 for
// i >= ng, M_i = M_c + sum over shells s of a(i, s) shell[s], with a(i, s) =
// V(xc_{s+ng}^3 - x0_{s+ng}^3) for s + ng <= i plus V(x0_{s+ng+1}^3 -
// xc_{s+ng}^3) for s + ng < i (V = 4 pi / 3), and shell[s] the dv-weighted
// mean density of radial index s + ng over the interior (j, k).  With
// c_i = gbar_i (-G / xc_i^2) and the suffix sums C_i = sum_{i' >= i} c_i':
// shell_bar[s] = C_{s+ng} V(xc^3 - x0^3)_{s+ng} + C_{s+ng+1} V(x0_{s+ng+1}^3 - xc_{s+ng}^3),
// and every cell of the shell gets shell_bar[s] dv / sum dv on its density
// adjoint (on the interior cell a ghost is filled from).  One CTA.
__global__ void k_internal_mass_reverse(GridDev g, const double* __restrict__ gbar, double* __restrict__ shell_bar,
                                        StateDev lam)
{
    const int ng = g.ng;
    const int n0 = g.n[0];
    const int nsh = g.nx[0] + ng;
    const double* x0 = g.x[0];
    const double* xc = g.xc[0];
    if (threadIdx.x == 0) {
        const double vol_s3 = 4 * kPi / 3;
        double C = 0.0;          // C_{i+1}
        for (int i = n0 - 1; i >= ng; --i) {
            const double Cn = C; // C_{i+1}
            C += gbar[i] * (-kG / (xc[i] * xc[i]));
            const int sidx_ = i - ng;
            const double xc3 = xc[i] * xc[i] * xc[i];
            const double x3 = x0[i] * x0[i] * x0[i];
            const double x3p = x0[i + 1] * x0[i + 1] * x0[i + 1];
            shell_bar[sidx_] = C * (vol_s3 * (xc3 - x3)) + Cn * (vol_s3 * (x3p - xc3));
        }
    }
    __syncthreads();
    const int g1 = g.ndim >= 2 ? ng : 0;
    const int g2 = g.ndim >= 3 ? ng : 0;
    for (int si = threadIdx.x; si < nsh; si += blockDim.x) {
        const int i = si + ng;
        double sd = 0;
        for (int j = 0; j < g.nx[1]; ++j) {
            for (int k = 0; k < g.nx[2]; ++k) {
                sd += g.dv[lidx(g, i, j + g1, k + g2)];
            }
        }
        const double f = shell_bar[si] / sd;
        if (f == 0.0) {
            continue;
        }
        int flip = 0;
        const int src = bc_source(i, n0, ng, g.bc[0], g.bc[1], &flip); // a density: no sign change
        for (int j = 0; j < g.nx[1]; ++j) {
            for (int k = 0; k < g.nx[2]; ++k) {
                const double w = f * g.dv[lidx(g, i, j + g1, k + g2)];
                atomicAdd(&lam.q[sidx(lam, g.n[1], src, j + g1, k + g2)], w);
            }
        }
    }
}
} // namespace

void internal_mass_reverse(const GridDev& g, const double* gbar, double* shell_bar, const StateDev& lam, cudaStream_t s)
{
    k_internal_mass_reverse<<<1, 256, 0, s>>>(g, gbar, shell_bar, lam);
    ++g_launches;
}

namespace {
template <int ND>
__global__ void k_zero_ghosts(GridDev g, StateDev lam)
{
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < g.N; c += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(c % g.n[0]);
        const int64_t r = c / g.n[0];
        const int j = (int)(r % g.n[1]);
        const int k = (int)(r / g.n[1]);
        const int idx[3] = {i, j, k};
        bool ghost = false;
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            ghost |= idx[d] < g.ng || idx[d] >= g.n[d] - g.ng;
        }
        if (ghost) {
            const int64_t o = sidx(lam, g.n[1], i, j, k);
            for (int v = 0; v < ND + 2 + g.nfx; ++v) {
                lam.q[o + lam.plane * v] = 0.0;
            }
        }
    }
}
} // namespace

void zero_ghosts(const GridDev& g, const StateDev& lam, cudaStream_t s)
{
    int blocks = (int)((g.N + 255) / 256);
    if (blocks > 148 * 8) {
        blocks = 148 * 8;
    }
    if (g.ndim == 1) {
        k_zero_ghosts<1><<<blocks, 256, 0, s>>>(g, lam);
    } else if (g.ndim == 2) {
        k_zero_ghosts<2><<<blocks, 256, 0, s>>>(g, lam);
    } else {
        k_zero_ghosts<3><<<blocks, 256, 0, s>>>(g, lam);
    }
    ++g_launches;
}

void fold(const GridDev& g, const StateDev& lam, cudaStream_t s)
{
    const int64_t count = (int64_t)g.nx[0] * g.nx[1] * g.nx[2];
    int blocks = (int)((count + 255) / 256);
    if (blocks > 148 * 8) {
        blocks = 148 * 8;
    }
    if (g.ndim == 1) {
        k_fold_ghosts<1><<<blocks, 256, 0, s>>>(g, lam);
    } else if (g.ndim == 2) {
        k_fold_ghosts<2><<<blocks, 256, 0, s>>>(g, lam);
    } else {
        k_fold_ghosts<3><<<blocks, 256, 0, s>>>(g, lam);
    }
    ++g_launches;
}

} // namespace hcl::adjoint
