// fused_strip2d.cuh -- the FP32-mixed 2-D fused step as a barrier-free
// warp-strip sweep (uniform Cartesian grids, uniform gravity).
//
// Same mathematics and precision split as k_fused_step<2, false, ...>; a
// different schedule:
//  * a warp owns 28 output columns x L output rows.  Lane l holds column
//    c0 - 2 + l, so x-neighbours (slopes, the left state of an x-face, the
//    right flux of a cell) come from warp shuffles; lanes 2..29 write output;
//  * the warp marches up its rows with a register window: at row r it issues
//    the copy of FP64 row r+4 into its shared-memory ring (cp.async), turns
//    row r+2 into primitives (FP64 internal-energy recovery), builds the
//    Hancock face states of row r+1, solves the y-face r+1/2 and the x-faces
//    of row r, and updates row r in FP64.  Every primitive, Hancock state and
//    face flux is computed once per lane (plus a 4-row start-up and the 4
//    halo lanes), with no barriers (a lane reads only the ring entries it
//    copied);
//  * ghost images, the internal-energy check and the CFL max of the new
//    state are done in the same pass.
// strip_work() is the per-strip body shared by the single-domain kernels
// (k_strip2d, also with one passive scalar, and k_strip2d_sync) and the
// persistent ensemble kernel.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "fused_step.cuh"
#include "hcl_device.cuh"
#include "physics_fast.cuh"
#include "stages.hpp"
#include "tma_ring.cuh"

namespace hcl::fused {

template <int LIM>
__device__ __forceinline__ float lim_fast(float dR, float dL)
{
    const float prod = dR * dL;
    if constexpr (LIM == LIM_CONSTANT) {
        return 0.f;
    }
    if (!(prod > 0.f)) {
        return 0.f;
    }
    if constexpr (LIM == LIM_VANLEER) {
        return 2.f * prod * __fdividef(1.f, dR + dL);
    } else if constexpr (LIM == LIM_MINMOD) {
        return fabsf(dR) < fabsf(dL) ? dR : dL;
    } else {
        return prod * (dR + dL) * __fdividef(1.f, fmaf(dR, dR, dL * dL));
    }
}

// Half the limited slope, lim_fast(dR, dL) / 2: the same value (scaling by a
// power of two is exact) with the factors 2 and 1/2 of van Leer cancelled.
template <int LIM>
__device__ __forceinline__ float half_lim_fast(float dR, float dL)
{
    if constexpr (LIM == LIM_VANLEER) {
        const float prod = dR * dL;
        return prod > 0.f ? prod * __fdividef(1.f, dR + dL) : 0.f;
    } else {
        return 0.5f * lim_fast<LIM>(dR, dL);
    }
}

struct StripCtx {
    fast::Eos eos;
    float cthx, cthy; // (dt/2)/dx, (dt/2)/dy
    float dgx, dgy;   // (dt/2) g
    bool gravity;     // any g component non-zero (the terms vanish exactly otherwise)
};

// FP64 state -> FP32 primitives, internal energy recovered in FP64 (the
// reciprocal starts from the hardware approximation and takes one FP64
// Newton step: ~1e-14 relative)
__device__ __forceinline__ void strip_prim(double gm1, const double q[4], float w[4])
{
    double r = (double)__fdividef(1.f, (float)q[0]);
    r = r * (2.0 - q[0] * r);
    const double u = q[1] * r;
    const double v = q[2] * r;
    const double mu = fma(q[1], u, q[2] * v);
    w[0] = (float)q[0];
    w[1] = (float)u;
    w[2] = (float)v;
    w[3] = (float)(gm1 * fma(-0.5, mu, q[3]));
}

// conservative state and physical flux of a face primitive state along l
// (hydro/euler_equations.hpp:72-86, :124-134), sharing the products
__device__ __forceinline__ void cons_and_flux(const fast::Eos& e, const float w[4], int l, float U[4], float F[4])
{
    const float m0 = w[0] * w[1];
    const float m1 = w[0] * w[2];
    const float Et = fmaf(0.5f, fmaf(m0, w[1], m1 * w[2]), w[3] * e.inv_gm1);
    U[0] = w[0];
    U[1] = m0;
    U[2] = m1;
    U[3] = Et;
    const float ml = l == 0 ? m0 : m1;
    const float ul = l == 0 ? w[1] : w[2];
    F[0] = ml;
    F[1] = ml * w[1];
    F[2] = ml * w[2];
    F[1 + l] += w[3];
    F[3] = ul * (Et + w[3]);
}

// Hancock face states of one cell: x-left, x-right, y-bottom, y-top (conservative).
// NFX > 0: also each passive scalar k's face values xo[4k..4k+3] (same order,
// fractions) from its primitives xw[3k..3k+2] = {row below, this row, row
// above}: limited slopes, times the face density before the predictor, plus
// the predictor's increment from the face states' mass fluxes, divided by the
// predicted face density (extrapolation_reconstruction.hpp:315-337, :329-339).
template <int LIM, int NFX = 0>
__device__ __forceinline__ void strip_hancock(const StripCtx& c, const float wd[4], const float wc[4], const float wu[4],
                                              float hxL[4], float hxR[4], float hyB[4], float hyT[4],
                                              const float* xw = nullptr, float* xo = nullptr)
{
    float fxL[4], fxR[4], fyB[4], fyT[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        const float wl = __shfl_up_sync(0xffffffffu, wc[v], 1);
        const float wr = __shfl_down_sync(0xffffffffu, wc[v], 1);
        const float sx = half_lim_fast<LIM>(wr - wc[v], wc[v] - wl);
        fxL[v] = wc[v] - sx;
        fxR[v] = wc[v] + sx;
        const float sy = half_lim_fast<LIM>(wu[v] - wc[v], wc[v] - wd[v]);
        fyB[v] = wc[v] - sy;
        fyT[v] = wc[v] + sy;
    }
    float FxL[4], FxR[4], FyB[4], FyT[4];
    cons_and_flux(c.eos, fxL, 0, hxL, FxL);
    cons_and_flux(c.eos, fxR, 0, hxR, FxR);
    cons_and_flux(c.eos, fyB, 1, hyB, FyB);
    cons_and_flux(c.eos, fyT, 1, hyT, FyT);
    float inc[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        inc[v] = fmaf(c.cthx, FxL[v] - FxR[v], c.cthy * (FyB[v] - FyT[v]));
    }
    float* outs[4] = {hxL, hxR, hyB, hyT};
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        float* u = outs[f];
        // gravity on the face state (extrapolation_reconstruction.hpp:306-312)
        const float r0 = u[0], m0 = u[1], m1 = u[2];
        u[0] = r0 + inc[0];
        if (c.gravity) {
            u[1] = fmaf(c.dgx, r0, m0 + inc[1]);
            u[2] = fmaf(c.dgy, r0, m1 + inc[2]);
            u[3] = fmaf(c.dgx, m0, fmaf(c.dgy, m1, u[3] + inc[3]));
        } else {
            u[1] = m0 + inc[1];
            u[2] = m1 + inc[2];
            u[3] = u[3] + inc[3];
        }
    }
    if constexpr (NFX > 0) {
        const float rho_pre[4] = {fxL[0], fxR[0], fyB[0], fyT[0]};
#pragma unroll
        for (int k = 0; k < NFX; ++k) {
            const float* xk = xw + 3 * k;
            const float xl = __shfl_up_sync(0xffffffffu, xk[1], 1);
            const float xr = __shfl_down_sync(0xffffffffu, xk[1], 1);
            const float sx = half_lim_fast<LIM>(xr - xk[1], xk[1] - xl);
            const float sy = half_lim_fast<LIM>(xk[2] - xk[1], xk[1] - xk[0]);
            const float pf[4] = {xk[1] - sx, xk[1] + sx, xk[1] - sy, xk[1] + sy};
            const float xinc =
                fmaf(c.cthx, pf[0] * FxL[0] - pf[1] * FxR[0], c.cthy * (pf[2] * FyB[0] - pf[3] * FyT[0]));
#pragma unroll
            for (int f = 0; f < 4; ++f) {
                xo[4 * k + f] = __fdividef(fmaf(pf[f], rho_pre[f], xinc), outs[f][0]);
            }
        }
    }
}

template <int RS>
__device__ __forceinline__ void strip_riemann(const fast::Eos& e, const float* L, const float* R, int l, float* F)
{
    fast::riemann<2>(e, RS, L, R, l, F);
}

// Shared-memory row ring of one warp: 8 row slots x 4 variables x 32 lanes.
// Ghost images of one scalar plane q (no sign flips): the loop of
// store_images_2d for a single value.
__device__ __forceinline__ void store_images_2d_scalar(double* __restrict__ q, int pitch, int n0, int n1, int ng, int col,
                                                       int r, unsigned xm, unsigned ym, double v)
{
    unsigned yb = ym & 0xffffu;
    int py = r;
    bool self_y = true;
    for (;;) {
        unsigned xb = xm & 0xffffu;
        int px = col;
        bool self_x = true;
        for (;;) {
            if (!(self_x && self_y)) {
                q[(int64_t)py * pitch + px] = v;
            }
            if (xb == 0u) {
                break;
            }
            const int k = __ffs(xb) - 1;
            xb &= xb - 1u;
            px = ghost_slot(k, n0, ng);
            self_x = false;
        }
        if (yb == 0u) {
            break;
        }
        const int k = __ffs(yb) - 1;
        yb &= yb - 1u;
        py = ghost_slot(k, n1, ng);
        self_y = false;
    }
}

// With a passive scalar the ring holds 5 variables.
template <int NVR>
using StripRingN = double (*)[NVR][32];
using StripRing = StripRingN<4>;
constexpr int kStripRingDoubles = 8 * 4 * 32;

// One strip (28 columns x rows [r0, r1)) of one domain: reads qin, writes qout.
// Accumulates the CFL max and the first bad cell of the lanes' output cells.
// SYNC > 0: the warp takes part in a CTA barrier after every SYNC rows and
// after row L - 1 of its strip, L barriers' worth of rows whatever the
// strip's own height (strip_idle() is the same barrier sequence without a
// strip), so that all warps of a CTA march in step.
// XIMG: border columns with up to XIMG x images (1: Periodic, Reflexive; 2:
// also NullGradient with two ghost layers) store them without a divergent
// branch.
// NFX > 0: the passive scalars (state planes 4..3+NFX) ride along: face
// values from strip_hancock, upwind fluxes from the Riemann mass fluxes
// (godunov_scheme.hpp:262-301), the update in FP64 divided by the new density
// and clamped to [0, 1], stored with the same ghost images.
// TMA: the ring rows are staged by the Tensor Memory Accelerator (tma_ring.cuh):
// lane 0 issues one box of two rows through `tmap` (the input state) into one
// of the warp's 4 ring slots, the lanes wait on the slot's mbarrier (`bars`,
// 4 per warp; `phase` counts the boxes the warp has waited for, which fixes
// each slot's next parity; `timeout` is set when a bounded wait gave up).
// Rows past r1 + 2 are not loaded.  Needs NFX == 0 and an even ghost width
// (the box's first column c0 - 2 must start on a 16-byte boundary).
template <int LIM, int RS, int SYNC = 0, int XIMG = 1, int NFX = 0, bool TMA = false>
__device__ __forceinline__ void strip_work(const GridDev& g, const double* __restrict__ qin, double* __restrict__ qout,
                                           int64_t plane, int pitch, double dt, int sx, int sy, int L, double& inv_max,
                                           int64_t& bad_cell, StripRingN<4 + NFX> ring,
                                           const CUtensorMap* tmap = nullptr, uint64_t* bars = nullptr,
                                           unsigned* phase = nullptr, bool* timeout = nullptr)
{
    static_assert(!TMA || NFX == 0, "the TMA ring carries the 4 hydro variables");
    const int lane = threadIdx.x & 31;
    const int n0 = g.n[0], n1 = g.n[1];
    const int c0 = g.ng + kStripLanesOut * sx;
    const int col = c0 - 2 + lane;
    const int colc = min(col, n0 - 1);
    const bool out_lane = lane >= 2 && lane < 2 + kStripLanesOut && col < g.ng + g.nx[0];
    const int r0 = g.ng + L * sy;
    const int r1 = min(r0 + L, g.ng + g.nx[1]);
    const unsigned xm = out_lane ? ghost_mask(col, n0, g.ng, g.bc[0], g.bc[1]) : 0u;
    // A column with at most XIMG x images stores them on every row that has
    // no y image, in step with the other lanes of the warp (which store their
    // own cell again): no divergent branch on the common border rows.  Other
    // cases take store_images_2d.
    const unsigned xbits = xm & 0xffffu;
    const int x_cnt = __popc(xbits);
    const bool x_fast = x_cnt <= XIMG;
    const bool x_any = __any_sync(0xffffffffu, x_cnt != 0);
    const bool x_two = XIMG > 1 && __any_sync(0xffffffffu, x_cnt == 2);
    const int x_img = xbits ? ghost_slot(__ffs(xbits) - 1, n0, g.ng) : col; // first image, or the cell
    const bool x_flip = xbits ? ((xm >> (15 + __ffs(xbits))) & 1u) != 0u : false;

    StripCtx c;
    c.eos = fast::Eos{(float)g.gamma, (float)g.gamma_m1, (float)(1.0 / g.gamma_m1)};
    c.cthx = (float)(0.5 * dt * g.inv_dx[0]);
    c.cthy = (float)(0.5 * dt * g.inv_dx[1]);
    c.dgx = (float)(0.5 * dt * g.g[0]);
    c.dgy = (float)(0.5 * dt * g.g[1]);
    c.gravity = g.g[0] != 0.0 || g.g[1] != 0.0;
    float inv_f = 0.f; // this strip's CFL max (NaN once a NaN was seen)
    const double cx = dt * g.inv_dx[0];
    const double cy = dt * g.inv_dx[1];
    const double dgx = dt * g.g[0];
    const double dgy = dt * g.g[1];
    const double gm1 = g.gamma_m1;

    // The FP64 rows stream through the warp's ring of 8 row slots in shared
    // memory (one 8-byte cp.async per lane and variable; a lane only reads
    // what it copied, so no barrier is needed).  Rows are issued 4 ahead.
    auto stage_row = [&](int r) {
        const int rc = min(max(r, 0), n1 - 1);
        const int64_t o = (int64_t)rc * pitch + colc;
#pragma unroll
        for (int v = 0; v < 4 + NFX; ++v) {
            const unsigned dst = (unsigned)__cvta_generic_to_shared(&ring[r & 7][v][lane]);
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(qin + o + plane * v) : "memory");
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    };
    // TMA staging: box b of this strip holds rows r0-2+2b and r0-1+2b as
    // [var][row][lane] in slot (nb0 + b) & 3; the k-th box a warp waits for
    // completes its slot's phase with parity (k >> 2) & 1.  Boxes 0..nbox-1
    // cover rows r0-2 .. r1+1 (the last may reach r1+2).
    const unsigned nb0 = TMA ? *phase : 0u;
    const int nbox = TMA ? ((r1 - r0 + 3) >> 1) + 1 : 0;
    bool tmo = false;
    const unsigned ring_s = TMA ? smem_u32(&ring[0][0][0]) : 0u;
    const unsigned bar_s = TMA ? smem_u32(bars) : 0u;
    const double* ring_d = &ring[0][0][0];
    auto tma_issue = [&](int b) {
        __syncwarp(); // the warp is done with the slot's previous box
        const unsigned sl = (nb0 + (unsigned)b) & 3u;
        tma_box_elected(ring_s + sl * kTmaBoxBytes, tmap, bar_s + 8u * sl, kTmaBoxBytes, c0 - 2, r0 - 2 + 2 * b, 0);
    };
    auto tma_wait = [&](int b) {
        const unsigned k = nb0 + (unsigned)b;
        if (!mbar_wait_bounded_s(bar_s + 8u * (k & 3u), (k >> 2) & 1u)) {
            tmo = true;
        }
    };
    auto ring_row = [&](int r, double* q) {
        if constexpr (TMA) {
            const int rel = r - (r0 - 2);
            const unsigned sl = (nb0 + (unsigned)(rel >> 1)) & 3u;
            const double* base = ring_d + sl * (kTmaBoxBytes / 8u) + (rel & 1) * 32 + lane;
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                q[v] = base[v * 64];
            }
        } else {
#pragma unroll
            for (int v = 0; v < 4 + NFX; ++v) {
                q[v] = ring[r & 7][v][lane];
            }
        }
    };

    // preamble: rows r0-2 .. r0+1 -> primitives; Hancock of rows r0-1 and r0
    float wB[4], wC[4], wD[4];
    float hxL[4], hxR[4], hyT[4];
    double Glo[4];
    // passive scalars (index k): primitives of rows r, r+1; face values of
    // row r (x-left, x-right, y-top); upwind flux of the y-face r-1/2
    constexpr int NX = NFX > 0 ? NFX : 1;
    float xC[NX], xD[NX], xoL[NX], xoR[NX], xoT[NX], gx_lo[NX];
#pragma unroll
    for (int k = 0; k < NX; ++k) {
        xC[k] = xD[k] = xoL[k] = xoR[k] = xoT[k] = gx_lo[k] = 0.f;
    }
    {
        double q[4 + NFX];
        float wA[4], hyB[4];
        float xA[NX], xB[NX];
        if constexpr (TMA) {
            for (int b = 0; b < min(4, nbox); ++b) {
                tma_issue(b);
            }
            tma_wait(0); // rows r0-2, r0-1
            tma_wait(1); // rows r0, r0+1
        } else {
            for (int rr = r0 - 2; rr <= r0 + 3; ++rr) {
                stage_row(rr);
            }
            asm volatile("cp.async.wait_group 2;\n" ::: "memory"); // rows r0-2 .. r0+1 landed
        }
        ring_row(r0 - 2, q);
        strip_prim(gm1, q, wA);
#pragma unroll
        for (int k = 0; k < NFX; ++k) {
            xA[k] = (float)q[4 + k];
        }
        ring_row(r0 - 1, q);
        strip_prim(gm1, q, wB);
#pragma unroll
        for (int k = 0; k < NFX; ++k) {
            xB[k] = (float)q[4 + k];
        }
        ring_row(r0, q);
        strip_prim(gm1, q, wC);
#pragma unroll
        for (int k = 0; k < NFX; ++k) {
            xC[k] = (float)q[4 + k];
        }
        ring_row(r0 + 1, q);
        strip_prim(gm1, q, wD);
#pragma unroll
        for (int k = 0; k < NFX; ++k) {
            xD[k] = (float)q[4 + k];
        }
        float t0[4], t1[4], t2[4], tT[4];
        float xw0[3 * NX], xw1[3 * NX];
#pragma unroll
        for (int k = 0; k < NX; ++k) {
            xw0[3 * k] = xA[k];
            xw0[3 * k + 1] = xB[k];
            xw0[3 * k + 2] = xC[k];
            xw1[3 * k] = xB[k];
            xw1[3 * k + 1] = xC[k];
            xw1[3 * k + 2] = xD[k];
        }
        float xo0[4 * NX], xo1[4 * NX];
        strip_hancock<LIM, NFX>(c, wA, wB, wC, t0, t1, t2, tT, xw0, xo0); // row r0-1: keep its top face
        strip_hancock<LIM, NFX>(c, wB, wC, wD, hxL, hxR, hyB, hyT, xw1, xo1); // row r0
        float G[4];
        strip_riemann<RS>(c.eos, tT, hyB, 1, G);
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            Glo[v] = (double)G[v];
        }
#pragma unroll
        for (int k = 0; k < NFX; ++k) {
            gx_lo[k] = (G[0] < 0.f ? xo1[4 * k + 2] : xo0[4 * k + 3]) * G[0];
            xoL[k] = xo1[4 * k];
            xoR[k] = xo1[4 * k + 1];
            xoT[k] = xo1[4 * k + 3];
        }
    }
    // window: wC = P[r], wD = P[r+1]; ring rows r+3, r+4 in flight.  Two rows
    // per iteration turn the window slide into register renaming (KH 2048^2:
    // 106.5 -> 102.7 us per step; four rows per iteration are slower).
#pragma unroll 2
    for (int i = 0; i < (SYNC > 0 ? L : r1 - r0); ++i) {
        const int r = r0 + i;
        if constexpr (SYNC > 0) {
            if (r >= r1) {
                if (i % SYNC == SYNC - 1 || i == L - 1) {
                    __syncthreads();
                }
                continue;
            }
        }
        double q[4 + NFX];
        float wN[4];
        float xN[NX];
        if constexpr (TMA) {
            if ((i & 1) == 0) {
                tma_wait((i >> 1) + 2); // rows r+2, r+3 landed
                if ((i >> 1) + 4 < nbox) {
                    tma_issue((i >> 1) + 4);
                }
            }
        } else {
            stage_row(r + 4);
            asm volatile("cp.async.wait_group 2;\n" ::: "memory"); // rows up to r+2 landed
        }
        ring_row(r, q);
        {
            double qn2[4 + NFX];
            ring_row(r + 2, qn2);
            strip_prim(gm1, qn2, wN);
#pragma unroll
            for (int k = 0; k < NFX; ++k) {
                xN[k] = (float)qn2[4 + k];
            }
        }
        // Hancock of row r+1
        float nxL[4], nxR[4], nyB[4], nyT[4];
        float xw[3 * NX];
#pragma unroll
        for (int k = 0; k < NFX; ++k) {
            xw[3 * k] = xC[k];
            xw[3 * k + 1] = xD[k];
            xw[3 * k + 2] = xN[k];
        }
        float nxo[4 * NX];
        strip_hancock<LIM, NFX>(c, wC, wD, wN, nxL, nxR, nyB, nyT, xw, nxo);
        // y-face r+1/2
        float G[4];
        strip_riemann<RS>(c.eos, hyT, nyB, 1, G);
        double Ghi[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            Ghi[v] = (double)G[v];
        }
        float gx_hi[NX];
#pragma unroll
        for (int k = 0; k < NFX; ++k) {
            // the upper cell's bottom face when the mass flows down, else the lower cell's top face
            gx_hi[k] = (G[0] < 0.f ? nxo[4 * k + 2] : xoT[k]) * G[0];
        }
        // x-faces of row r: left face at this lane, right face from lane+1
        float uL[4], Fl[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            uL[v] = __shfl_up_sync(0xffffffffu, hxR[v], 1);
        }
        strip_riemann<RS>(c.eos, uL, hxL, 0, Fl);
        double Fld[4], Frd[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            Fld[v] = (double)Fl[v];
            Frd[v] = __shfl_down_sync(0xffffffffu, Fld[v], 1);
        }
        float fx_l[NX], fx_r[NX];
#pragma unroll
        for (int k = 0; k < NFX; ++k) {
            // left face: this cell's left value when the mass flows left, else the left cell's right value
            const float up_left = __shfl_up_sync(0xffffffffu, xoR[k], 1);
            fx_l[k] = (Fl[0] < 0.f ? xoL[k] : up_left) * Fl[0];
            fx_r[k] = __shfl_down_sync(0xffffffffu, fx_l[k], 1);
        }
        if (out_lane) {
            // Godunov update of row r in FP64 (godunov_scheme.hpp:159-163, 258-260)
            double qn[4];
            const int64_t oo = (int64_t)r * pitch + col;
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                qn[v] = q[v] + fma(cx, Fld[v] - Frd[v], cy * (Glo[v] - Ghi[v]));
            }
            if (c.gravity) {
                qn[1] = fma(dgx, q[0], qn[1]);
                qn[2] = fma(dgy, q[0], qn[2]);
                qn[3] = fma(dgx, q[1], fma(dgy, q[2], qn[3]));
            }
            // health check (main.cpp:397-425): the new state fails when
            // evol = E - |m|^2 / (2 rho) is negative or NaN.  Evaluated in FP64
            // without the division, as the sign of 2 rho evol = 2 rho E - |m|^2
            // (reversed for rho < 0; rho = 0 gives -inf or NaN: fails).
            const double tre = (qn[0] + qn[0]) * qn[3];
            const double mm = fma(qn[1], qn[1], qn[2] * qn[2]);
            const bool healthy = qn[0] > 0.0 ? tre >= mm : (qn[0] < 0.0 && tre <= mm);
            if (!healthy && bad_cell < 0) {
                bad_cell = lidx(g, col, r, 0);
            }
            // CFL contribution (time_step.hpp:55-77) in FP32 from the FP64
            // internal energy: c^2 = gamma (gamma-1) evol / rho
            //                      = gamma (gamma-1) / 2 * (2 rho E - |m|^2) / rho^2
            {
                const float ir = __fdividef(1.f, (float)qn[0]);
                const float c2 = g.cfl_kc2 * (float)(tre - mm) * ir * ir;
                const float snd = sqrtf(c2);
                const float cell =
                    fmaf(fabsf((float)qn[1] * ir) + snd, g.inv_dx_f[0], (fabsf((float)qn[2] * ir) + snd) * g.inv_dx_f[1]);
                inv_f = cell > inv_f ? cell : (isnan(cell) ? cell : inv_f);
            }
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                qout[oo + plane * v] = qn[v];
            }
            double xnew[NX];
#pragma unroll
            for (int k = 0; k < NFX; ++k) {
                const double xn = fma(q[4 + k], q[0], fma(cx, (double)fx_l[k] - (double)fx_r[k],
                                                          cy * ((double)gx_lo[k] - (double)gx_hi[k])));
                double xv = xn / qn[0];
                xv = xv < 0. ? 0. : (xv > 1. ? 1. : xv);
                xnew[k] = xv;
                qout[oo + plane * (4 + k)] = xv;
            }
            const unsigned ym = (r < 2 * g.ng || r >= n1 - 2 * g.ng) ? ghost_mask(r, n1, g.ng, g.bc[2], g.bc[3]) : 0u;
            if (ym != 0u || !x_fast) {
                if ((xm | ym) != 0u) {
                    store_images_2d(qout, plane, pitch, n0, n1, g.ng, col, r, xm, ym, qn);
#pragma unroll
                    for (int k = 0; k < NFX; ++k) {
                        store_images_2d_scalar(qout + plane * (4 + k), pitch, n0, n1, g.ng, col, r, xm, ym, xnew[k]);
                    }
                }
            } else if (x_any) {
                const int64_t og = (int64_t)r * pitch + x_img;
                qout[og] = qn[0];
                qout[og + plane] = x_flip ? -qn[1] : qn[1];
                qout[og + 2 * plane] = qn[2];
                qout[og + 3 * plane] = qn[3];
#pragma unroll
                for (int k = 0; k < NFX; ++k) {
                    qout[og + (4 + k) * plane] = xnew[k];
                }
                if (XIMG > 1 && x_two) {
                    // the second image, or the first again
                    const unsigned b2 = xbits & (xbits - 1u);
                    const int px = b2 ? ghost_slot(__ffs(b2) - 1, n0, g.ng) : x_img;
                    const bool fl = b2 ? ((xm >> (15 + __ffs(b2))) & 1u) != 0u : x_flip;
                    const int64_t og2 = (int64_t)r * pitch + px;
                    qout[og2] = qn[0];
                    qout[og2 + plane] = fl ? -qn[1] : qn[1];
                    qout[og2 + 2 * plane] = qn[2];
                    qout[og2 + 3 * plane] = qn[3];
#pragma unroll
                    for (int k = 0; k < NFX; ++k) {
                        qout[og2 + (4 + k) * plane] = xnew[k];
                    }
                }
            }
        }
        // slide the window
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            wC[v] = wD[v];
            wD[v] = wN[v];
            hxL[v] = nxL[v];
            hxR[v] = nxR[v];
            hyT[v] = nyT[v];
            Glo[v] = Ghi[v];
        }
#pragma unroll
        for (int k = 0; k < NFX; ++k) {
            xC[k] = xD[k];
            xD[k] = xN[k];
            xoL[k] = nxo[4 * k];
            xoR[k] = nxo[4 * k + 1];
            xoT[k] = nxo[4 * k + 3];
            gx_lo[k] = gx_hi[k];
        }
        if constexpr (SYNC > 0) {
            if (i % SYNC == SYNC - 1 || i == L - 1) {
                __syncthreads();
            }
        }
    }
    if constexpr (TMA) {
        // every issued box has been waited for
        *phase = nb0 + (unsigned)nbox;
        if (tmo) {
            *timeout = true;
        }
    } else {
        asm volatile("cp.async.wait_all;\n" ::: "memory"); // the ring is reused by the next strip
    }
    const double inv_d = (double)inv_f;
    inv_max = inv_d > inv_max ? inv_d : (isnan(inv_d) ? inv_d : inv_max);
    (void)wB;
}

// The barrier sequence of strip_work<..., SYNC> for a warp without a strip.
template <int SYNC>
__device__ __forceinline__ void strip_idle(int L)
{
    for (int i = 0; i < L; ++i) {
        if (i % SYNC == SYNC - 1 || i == L - 1) {
            __syncthreads();
        }
    }
}

// time-loop control of one step, published by one thread (main.cpp:354-385)
__device__ __forceinline__ void publish_decision(StepCtl* ctl, const Decision& dec, const RunParamsDev& rp, int slot,
                                                 int out_buf)
{
    const int q = (slot + 1) & 1;
    if (!dec.noop) {
        ctl->t[q] = dec.t + dec.dt;
        ctl->iter[q] = dec.iter + 1;
        ctl->time_output_id[q] = dec.toid_next;
        ctl->iter_output_id[q] = dec.ioid_next;
        ctl->stop[q] = dec.stop;
        ctl->last_dt = dec.dt;
        if (dec.stop) {
            ctl->final_buf = out_buf;
        }
        if (dec.neg_dt) {
            ctl->err = 5;
            ctl->errflag[q] = 1;
            ctl->t[q] = dec.t;
            ctl->iter[q] = dec.iter;
            ctl->final_buf = out_buf ^ 1;
        }
        if (rp.dt_log && dec.iter < rp.dt_log_cap && !dec.neg_dt) {
            rp.dt_log[dec.iter] = dec.dt;
        }
    } else {
        ctl->t[q] = dec.t;
        ctl->iter[q] = dec.iter;
        ctl->time_output_id[q] = dec.toid_next;
        ctl->iter_output_id[q] = dec.ioid_next;
        ctl->stop[q] = 1;
        ctl->errflag[q] = ctl->errflag[slot & 1];
    }
    ctl->inv_dt_bits[(slot + 2) % 3] = 0ull;
}

// NFX = 1 or 2 passive scalars: (4+NFX)-variable rings; three CTAs of 4 warps
// per SM leave 170 registers for one scalar's window, two CTAs 255 for two.
// The rings of NFX = 2 (48 KB) are dynamic shared memory.
template <int LIM, int RS, int NFX = 0>
__global__ void __launch_bounds__(128, NFX > 1 ? 2 : (NFX > 0 ? 3 : 4))
k_strip2d(GridDev g, StateDev in, StateDev out, StepCtl* ctl, RunParamsDev rp, int slot, int out_buf, int L)
{
    const int lane = threadIdx.x & 31;
    const Decision dec = decide(ctl, slot, rp);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        publish_decision(ctl, dec, rp, slot, out_buf);
    }
    if (dec.noop || dec.neg_dt) {
        return;
    }
    const int ncolw = (g.nx[0] + kStripLanesOut - 1) / kStripLanesOut;
    const int nstrip = (g.nx[1] + L - 1) / L;
    const int nitems = ncolw * nstrip;
    const int wg = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (wg >= nitems) {
        return;
    }
    double inv_max = 0.0;
    int64_t bad_cell = -1;
    // grid-stride over the strips (the launcher sizes the grid to the
    // resident warps, so a warp usually takes one or two strips)
    const int wstride = gridDim.x * (blockDim.x >> 5);
    double* ring_mem;
    if constexpr (NFX > 1) {
        extern __shared__ __align__(16) double s_ring_dyn[];
        ring_mem = s_ring_dyn;
    } else {
        __shared__ __align__(16) double s_ring[4 * 8 * (4 + NFX) * 32];
        ring_mem = s_ring;
    }
    const StripRingN<4 + NFX> ring =
        reinterpret_cast<StripRingN<4 + NFX>>(ring_mem + ((threadIdx.x >> 5) & 3) * 8 * (4 + NFX) * 32);
    for (int w = wg; w < nitems; w += wstride) {
        strip_work<LIM, RS, 0, 1, NFX>(g, in.q, out.q, in.plane, in.pitch, dec.dt, w % ncolw, w / ncolw, L, inv_max,
                                       bad_cell, ring);
    }
    // warp max of 1/dt -> one atomic per warp
    const bool nan_seen = isnan(inv_max);
    double m = nan_seen ? 0.0 : inv_max;
    m = warp_max_d(m);
    const unsigned nanv = __ballot_sync(0xffffffffu, nan_seen);
    if (lane == 0) {
        atomicMax(&ctl->inv_dt_bits[(slot + 1) % 3], dbl_bits(m));
        if (nanv) {
            atomicMax(&ctl->inv_dt_bits[(slot + 1) % 3], 0x7ff8000000000000ull);
        }
    }
    if (bad_cell >= 0) {
        atomicMin(&ctl->bad_cell, (unsigned long long)bad_cell);
        ctl->err = 4;
        ctl->errflag[(slot + 1) & 1] = 1;
        ctl->final_buf = out_buf;
    }
}

// The same step with one CTA of 16 warps per SM (fitted strips, one wave).
// With four CTAs of 4 warps per SM the strips of one SM finish up to ~20 %
// apart, in the order the CTAs were launched, and the last strips run with
// few warps left to hide their latency; the warps of one CTA finish closer
// together.  A CTA barrier every kStripSyncRows rows can hold the 16 strips
// at one height; measured on KH 2048^2 (step time for 2/4/8/16/32/64 rows:
// 113.2/111.3/108.5/107.2/106.7/106.5 us) frequent barriers cost more than
// they even out, so the interval is a strip's usual height.
constexpr int kStripSyncRows = 64;
constexpr int kStripSyncWarps = 16;

// Dynamic shared memory of k_strip2d_sync: 16 row rings; with TMA also one
// mbarrier per ring slot and the slack to put the rings on a 1 KB boundary.
constexpr int kStripSyncSmem = kStripSyncWarps * kStripRingDoubles * (int)sizeof(double);
constexpr int kStripSyncSmemTma = kStripSyncSmem + kStripSyncWarps * 8 * (int)sizeof(uint64_t) + 1024;

// TMA: the rows come in through the Tensor Memory Accelerator (`tmap` is a
// 3-D tiled map of the input state: columns, rows, variables); otherwise
// per-lane cp.async and `tmap` is unused.
template <int LIM, int RS, bool TMA = false>
__global__ void __launch_bounds__(32 * kStripSyncWarps, 1)
k_strip2d_sync(GridDev g, StateDev in, StateDev out, StepCtl* ctl, RunParamsDev rp, int slot, int out_buf, int L,
               const __grid_constant__ CUtensorMap tmap)
{
    extern __shared__ __align__(16) double s_sync_rings[]; // [kStripSyncWarps][kStripRingDoubles] (+ mbarriers)
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const Decision dec = decide(ctl, slot, rp);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        publish_decision(ctl, dec, rp, slot, out_buf);
    }
    if (dec.noop || dec.neg_dt) {
        return;
    }
    const int ncolw = (g.nx[0] + kStripLanesOut - 1) / kStripLanesOut;
    const int nstrip = (g.nx[1] + L - 1) / L;
    const int nitems = ncolw * nstrip;
    double inv_max = 0.0;
    int64_t bad_cell = -1;
    double* rings = s_sync_rings;
    uint64_t* bars = nullptr;
    unsigned phase = 0u;
    bool timeout = false;
    if constexpr (TMA) {
        // rings on a 1 KB boundary, then 8 mbarriers per warp
        const unsigned base = smem_u32(s_sync_rings);
        rings = reinterpret_cast<double*>(reinterpret_cast<unsigned char*>(s_sync_rings) +
                                          (((base + 1023u) & ~1023u) - base));
        bars = reinterpret_cast<uint64_t*>(rings + kStripSyncWarps * kStripRingDoubles) + warp * 8;
        if (lane == 0) {
            for (int k = 0; k < 8; ++k) {
                mbar_init(bars + k, 1u);
            }
            mbar_init_fence();
            tma_prefetch_map(&tmap);
        }
        __syncwarp();
    }
    const StripRing ring = reinterpret_cast<StripRing>(rings + warp * kStripRingDoubles);
    // the CTA takes strips in groups of 16 (one per warp); every warp of the
    // CTA runs the same loop, so the barrier sequences match
    for (int base = blockIdx.x * kStripSyncWarps; base < nitems; base += gridDim.x * kStripSyncWarps) {
        const int w = base + warp;
        if (w < nitems) {
            strip_work<LIM, RS, kStripSyncRows, 1, 0, TMA>(g, in.q, out.q, in.plane, in.pitch, dec.dt, w % ncolw,
                                                           w / ncolw, L, inv_max, bad_cell, ring, &tmap, bars, &phase,
                                                           &timeout);
        } else {
            strip_idle<kStripSyncRows>(L);
        }
    }
    const bool nan_seen = isnan(inv_max);
    double m = nan_seen ? 0.0 : inv_max;
    m = warp_max_d(m);
    const unsigned nanv = __ballot_sync(0xffffffffu, nan_seen);
    if (lane == 0) {
        atomicMax(&ctl->inv_dt_bits[(slot + 1) % 3], dbl_bits(m));
        if (nanv) {
            atomicMax(&ctl->inv_dt_bits[(slot + 1) % 3], 0x7ff8000000000000ull);
        }
    }
    if (bad_cell >= 0) {
        atomicMin(&ctl->bad_cell, (unsigned long long)bad_cell);
        ctl->err = 4;
        ctl->errflag[(slot + 1) & 1] = 1;
        ctl->final_buf = out_buf;
    }
    if (TMA && __any_sync(0xffffffffu, timeout) && lane == 0) {
        // a staged row never arrived: stop the run with HCL_ERR_TIMEOUT
        ctl->err = 6;
        ctl->errflag[(slot + 1) & 1] = 1;
        ctl->final_buf = out_buf;
    }
}

} // namespace hcl::fused
