// fused_strip3d.cuh -- the FP32-mixed 3-D fused step as a column march
// (uniform Cartesian grids, uniform gravity).
//
// Same mathematics and precision split as k_fused_step<3, false, ...>; a
// different schedule.  A CTA of 16 warps owns a block of 28 x 12 output
// columns (x, y) and marches it along z over L planes:
//  * lane l of warp w holds the column (c0 - 2 + l, j0 - 2 + w); x-neighbours
//    come from warp shuffles, y-neighbours from the neighbouring warps through
//    shared memory, z-neighbours from a register window;
//  * at step z the CTA turns plane z+2 into primitives (FP64 internal-energy
//    recovery), builds the Hancock face states of plane z+1, solves the
//    x-faces of plane z+1, the z-face z+1/2 and the y-faces of plane z, and
//    updates plane z in FP64 with the ghost images, the health check and the
//    CFL contribution.  One CTA barrier per plane orders the shared planes.
// Lanes 2..29 and warps 2..13 write; the others are the stencil halo.  The
// halo warps solve no x- or z-face and update nothing; warp 1 solves the
// y-face above it, which row 2 reads.  (Skipping the Hancock states of warps
// 0 and 15 as well, whose neighbours read only their primitives, measured
// 2.25 against 1.93 ms per step on RT 256^2 x 512: the branch around the
// predictor cost more than the work it saved.)
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "fused_step.cuh"
#include "fused_strip2d.cuh"
#include "hcl_device.cuh"
#include "physics_fast.cuh"
#include "stages.hpp"

namespace hcl::fused {

constexpr int kS3Warps = 16;
constexpr int kS3Threads = 32 * kS3Warps;

namespace s3 {

struct Ctx {
    fast::Eos eos;
    float cth[3]; // (dt/2)/dx_d
    float dg[3];  // (dt/2) g_d
    bool gravity;
};

// FP64 state -> FP32 primitives (rho, u, v, w, P); internal energy in FP64
__device__ __forceinline__ void prim(double gm1, const double q[5], float w[5])
{
    double r = (double)__fdividef(1.f, (float)q[0]);
    r = r * (2.0 - q[0] * r);
    const double u = q[1] * r;
    const double v = q[2] * r;
    const double x = q[3] * r;
    const double mu = fma(q[1], u, fma(q[2], v, q[3] * x));
    w[0] = (float)q[0];
    w[1] = (float)u;
    w[2] = (float)v;
    w[3] = (float)x;
    w[4] = (float)(gm1 * fma(-0.5, mu, q[4]));
}

// conservative state and flux along l of a face primitive state
__device__ __forceinline__ void cons_and_flux(const fast::Eos& e, const float w[5], int l, float U[5], float F[5])
{
    const float m0 = w[0] * w[1];
    const float m1 = w[0] * w[2];
    const float m2 = w[0] * w[3];
    const float Et = fmaf(0.5f, fmaf(m0, w[1], fmaf(m1, w[2], m2 * w[3])), w[4] * e.inv_gm1);
    U[0] = w[0];
    U[1] = m0;
    U[2] = m1;
    U[3] = m2;
    U[4] = Et;
    const float ml = l == 0 ? m0 : (l == 1 ? m1 : m2);
    const float ul = w[1 + l];
    F[0] = ml;
    F[1] = ml * w[1];
    F[2] = ml * w[2];
    F[3] = ml * w[3];
    F[1 + l] += w[4];
    F[4] = ul * (Et + w[4]);
}

// Hancock face states of one cell: minus/plus faces along x, y, z
// (extrapolation_reconstruction.hpp:65-143, gravity :306-312).  wyd/wyu are
// the y-neighbours, wzd/wzu the z-neighbours; x-neighbours come by shuffle.
// NFX > 0: also each passive scalar k's face values xo[6k..6k+2] (minus faces
// x, y, z) and xo[6k+3..6k+5] (plus faces) from its primitives
// xw[5k..5k+4] = {centre, y-, y+, z-, z+}: limited slopes, times the face
// density before the predictor, plus the predictor's increment from the face
// states' mass fluxes, divided by the predicted face density
// (extrapolation_reconstruction.hpp:315-337, :329-339).
template <int LIM, int NFX = 0>
__device__ __forceinline__ void hancock(const Ctx& c, const float wc[5], const float wyd[5], const float wyu[5],
                                        const float wzd[5], const float wzu[5], float hm[3][5], float hp[3][5],
                                        const float* xw = nullptr, float* xo = nullptr)
{
    float fm[3][5], fp[3][5];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        const float wl = __shfl_up_sync(0xffffffffu, wc[v], 1);
        const float wr = __shfl_down_sync(0xffffffffu, wc[v], 1);
        const float sx = half_lim_fast<LIM>(wr - wc[v], wc[v] - wl);
        fm[0][v] = wc[v] - sx;
        fp[0][v] = wc[v] + sx;
        const float sy = half_lim_fast<LIM>(wyu[v] - wc[v], wc[v] - wyd[v]);
        fm[1][v] = wc[v] - sy;
        fp[1][v] = wc[v] + sy;
        const float sz = half_lim_fast<LIM>(wzu[v] - wc[v], wc[v] - wzd[v]);
        fm[2][v] = wc[v] - sz;
        fp[2][v] = wc[v] + sz;
    }
    float inc[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
    float mfm[3], mfp[3]; // mass fluxes of the face states before the update
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        float Fm[5], Fp[5];
        cons_and_flux(c.eos, fm[d], d, hm[d], Fm);
        cons_and_flux(c.eos, fp[d], d, hp[d], Fp);
        mfm[d] = Fm[0];
        mfp[d] = Fp[0];
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            inc[v] = fmaf(c.cth[d], Fm[v] - Fp[v], inc[v]);
        }
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            float* u = s == 0 ? hm[d] : hp[d];
            const float r0 = u[0], m0 = u[1], m1 = u[2], m2 = u[3];
#pragma unroll
            for (int v = 0; v < 5; ++v) {
                u[v] += inc[v];
            }
            if (c.gravity) {
                u[1] = fmaf(c.dg[0], r0, u[1]);
                u[2] = fmaf(c.dg[1], r0, u[2]);
                u[3] = fmaf(c.dg[2], r0, u[3]);
                u[4] = fmaf(c.dg[0], m0, fmaf(c.dg[1], m1, fmaf(c.dg[2], m2, u[4])));
            }
        }
    }
#pragma unroll
    for (int k = 0; k < NFX; ++k) {
        const float* xk = xw + 5 * k;
        float* ok = xo + 6 * k;
        const float xl = __shfl_up_sync(0xffffffffu, xk[0], 1);
        const float xr = __shfl_down_sync(0xffffffffu, xk[0], 1);
        const float s[3] = {half_lim_fast<LIM>(xr - xk[0], xk[0] - xl), half_lim_fast<LIM>(xk[2] - xk[0], xk[0] - xk[1]),
                            half_lim_fast<LIM>(xk[4] - xk[0], xk[0] - xk[3])};
        float xinc = 0.f;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            xinc = fmaf(c.cth[d], (xk[0] - s[d]) * mfm[d] - (xk[0] + s[d]) * mfp[d], xinc);
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            ok[d] = __fdividef(fmaf(xk[0] - s[d], fm[d][0], xinc), hm[d][0]);
            ok[3 + d] = __fdividef(fmaf(xk[0] + s[d], fp[d][0], xinc), hp[d][0]);
        }
    }
}

} // namespace s3

// Shared planes of one CTA: primitives of the current Hancock plane, the
// y-face states of the last two Hancock planes and the y-face fluxes.
struct S3Shared {
    float prim[2][kS3Warps][5][32];
    float yface[2][kS3Warps][2][5][32]; // [.][w][0: bottom (minus), 1: top (plus)]
    float gflux[2][kS3Warps][5][32];    // flux of the y-face above row w
};
// the same for each passive scalar
struct S3SharedFx {
    float xprim[2][kS3Warps][32];
    float xyface[2][kS3Warps][2][32];
    float xgflux[2][kS3Warps][32];
};
template <int NFX>
struct S3SharedT : S3Shared {
    S3SharedFx fx[NFX];
};
template <>
struct S3SharedT<0> : S3Shared {
};

// Ghost images of one scalar plane q (no sign flips): the loops of
// store_images_3d for a single value.
__device__ __forceinline__ void store_images_3d_scalar(double* __restrict__ q, int64_t pitch, int n0, int n1, int n2,
                                                       int ng, int col, int row, int z, unsigned xm, unsigned ym,
                                                       unsigned zm, double v)
{
    unsigned zb = zm & 0xffffu;
    int pz = z;
    bool self_z = true;
    for (;;) {
        unsigned yb = ym & 0xffffu;
        int py = row;
        bool self_y = true;
        for (;;) {
            unsigned xb = xm & 0xffffu;
            int px = col;
            bool self_x = true;
            for (;;) {
                if (!(self_x && self_y && self_z)) {
                    q[((int64_t)pz * n1 + py) * pitch + px] = v;
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
        if (zb == 0u) {
            break;
        }
        const int k = __ffs(zb) - 1;
        zb &= zb - 1u;
        pz = ghost_slot(k, n2, ng);
        self_z = false;
    }
}

// NFX > 0: the passive scalars (state planes 5 .. 4 + NFX) ride along: face
// values from hancock, upwind fluxes from the Riemann mass fluxes
// (godunov_scheme.hpp:262-301), the update in FP64 divided by the new density
// and clamped to [0, 1], stored with the same ghost images.
template <int LIM, int RS, int NFX = 0>
__global__ void __launch_bounds__(kS3Threads, 1)
k_strip3d(GridDev g, StateDev in, StateDev out, StepCtl* ctl, RunParamsDev rp, int slot, int out_buf, int L)
{
    extern __shared__ __align__(16) unsigned char s3_raw[];
    S3SharedT<NFX>& sh = *reinterpret_cast<S3SharedT<NFX>*>(s3_raw);
    S3SharedFx* fxs = nullptr; // the scalars' shared planes
    if constexpr (NFX > 0) {
        fxs = sh.fx;
    }
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    const Decision dec = decide(ctl, slot, rp);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        publish_decision(ctl, dec, rp, slot, out_buf);
    }
    if (dec.noop || dec.neg_dt) {
        return;
    }
    const double dt = dec.dt;
    const int n0 = g.n[0], n1 = g.n[1], n2 = g.n[2];
    const int ncx = (g.nx[0] + 27) / 28, ncy = (g.nx[1] + 11) / 12;
    int b = blockIdx.x;
    const int bx = b % ncx;
    b /= ncx;
    const int by = b % ncy;
    const int bz = b / ncy;
    const int col = g.ng + 28 * bx - 2 + lane;
    const int row = g.ng + 12 * by - 2 + w;
    const int colc = min(col, n0 - 1);
    const int rowc = min(row, n1 - 1);
    const bool out_cell = lane >= 2 && lane < 30 && w >= 2 && w < 14 && col < g.ng + g.nx[0] &&
                          row < g.ng + g.nx[1];
    // this column's x and y images (ghost_mask), fixed over the march
    const unsigned xm = out_cell ? ghost_mask(col, n0, g.ng, g.bc[0], g.bc[1]) : 0u;
    const unsigned ym = out_cell ? ghost_mask(row, n1, g.ng, g.bc[2], g.bc[3]) : 0u;
    const unsigned xym = xm | ym;
    const int z0 = g.ng + L * bz;
    const int z1 = min(z0 + L, g.ng + g.nx[2]);
    const int64_t pitch = in.pitch;
    const int64_t plane = in.plane;
    const double* __restrict__ qin = in.q;
    double* __restrict__ qout = out.q;

    s3::Ctx c;
    c.eos = fast::Eos{(float)g.gamma, (float)g.gamma_m1, (float)(1.0 / g.gamma_m1)};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        c.cth[d] = (float)(0.5 * dt * g.inv_dx[d]);
        c.dg[d] = (float)(0.5 * dt * g.g[d]);
    }
    c.gravity = g.g[0] != 0.0 || g.g[1] != 0.0 || g.g[2] != 0.0;
    const double gm1 = g.gamma_m1;
    float inv_f = 0.f; // CFL max of this CTA's cells (NaN once a NaN was seen)

    auto load = [&](int z, double* q) {
        const int zc = min(max(z, 0), n2 - 1);
        const int64_t o = ((int64_t)zc * n1 + rowc) * pitch + colc;
#pragma unroll
        for (int v = 0; v < 5 + NFX; ++v) {
            q[v] = __ldg(qin + o + plane * v);
        }
    };
    auto put_prim = [&](int z, const float p[5]) {
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            sh.prim[z & 1][w][v][lane] = p[v];
        }
    };
    const int wd = max(w - 1, 0), wu = min(w + 1, kS3Warps - 1);
    // warp-uniform roles of the halo warps (see the file comment)
    const bool w_update = w >= 2 && w < kS3Warps - 2;
    const bool w_yface = w >= 1 && w < kS3Warps - 2;

    // window: wC = P[z], wD = P[z+1]; qN = U[z+2] in flight
    float wC[5], wD[5];
    float hzU[5];      // z-plus face state of plane z (for the z-face z+1/2)
    double dFx[5];     // x-flux difference (left - right face) of plane z, exact in FP64
    float Gzlo[5];     // z-face flux z-1/2
    double qN[5 + NFX];
    // passive scalars (index k): primitives of planes z, z+1; z-plus face
    // value of plane z; x-flux difference of plane z; upwind flux of the
    // z-face z-1/2
    constexpr int NX = NFX > 0 ? NFX : 1;
    float xC[NX], xD[NX], xzU[NX], gzx_lo[NX];
    double dxx[NX];
#pragma unroll
    for (int k = 0; k < NX; ++k) {
        xC[k] = xD[k] = xzU[k] = gzx_lo[k] = 0.f;
        dxx[k] = 0.0;
    }
    {
        double q[5 + NFX];
        load(z0 - 2, q);
        s3::prim(gm1, q, wC);
#pragma unroll
        for (int k = 0; k < NFX; ++k) {
            xC[k] = (float)q[5 + k];
        }
        load(z0 - 1, q);
        s3::prim(gm1, q, wD);
        put_prim(z0 - 1, wD);
#pragma unroll
        for (int k = 0; k < NFX; ++k) {
            xD[k] = (float)q[5 + k];
            fxs[k].xprim[(z0 - 1) & 1][w][lane] = xD[k];
        }
        load(z0, qN);
    }
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        hzU[v] = Gzlo[v] = 0.f;
        dFx[v] = 0.0;
    }
    double inv_max = 0.0;
    int64_t bad_cell = -1;
    const double cxyz[3] = {dt * g.inv_dx[0], dt * g.inv_dx[1], dt * g.inv_dx[2]};
    const double Dg[3] = {dt * g.g[0], dt * g.g[1], dt * g.g[2]};
    __syncthreads();

    // two planes per iteration: the window slide becomes register renaming
    // (RT 256^2 x 512: 2.09 -> 2.00 ms per step)
#pragma unroll 2
    for (int z = z0 - 2; z < z1; ++z) {
        // 1. primitives of plane z+2
        float wN[5];
        s3::prim(gm1, qN, wN);
        put_prim(z + 2, wN);
        float xN[NX];
#pragma unroll
        for (int k = 0; k < NFX; ++k) {
            xN[k] = (float)qN[5 + k];
            fxs[k].xprim[(z + 2) & 1][w][lane] = xN[k];
        }
        load(z + 3, qN);
        // 2. Hancock of plane z+1 (y-neighbours' primitives of plane z+1 were shared last step)
        float wyd[5], wyu[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            wyd[v] = sh.prim[(z + 1) & 1][wd][v][lane];
            wyu[v] = sh.prim[(z + 1) & 1][wu][v][lane];
        }
        float hm[3][5], hp[3][5];
        float xw[5 * NX];
#pragma unroll
        for (int k = 0; k < NFX; ++k) {
            xw[5 * k] = xD[k];
            xw[5 * k + 1] = fxs[k].xprim[(z + 1) & 1][wd][lane];
            xw[5 * k + 2] = fxs[k].xprim[(z + 1) & 1][wu][lane];
            xw[5 * k + 3] = xC[k];
            xw[5 * k + 4] = xN[k];
        }
        float xo[6 * NX];
        s3::hancock<LIM, NFX>(c, wD, wyd, wyu, wC, wN, hm, hp, xw, xo);
        // 3. x-faces of plane z+1: left face at this lane, right face from lane+1
        double dFxN[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        double dxxN[NX];
        float gzx_hi[NX];
#pragma unroll
        for (int k = 0; k < NX; ++k) {
            dxxN[k] = 0.0;
            gzx_hi[k] = 0.f;
        }
        float Gzhi[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
        if (w_update) {
            float uL[5], Fl[5];
#pragma unroll
            for (int v = 0; v < 5; ++v) {
                uL[v] = __shfl_up_sync(0xffffffffu, hp[0][v], 1);
            }
            fast::riemann<3>(c.eos, RS, uL, hm[0], 0, Fl);
#pragma unroll
            for (int v = 0; v < 5; ++v) {
                dFxN[v] = (double)Fl[v] - (double)__shfl_down_sync(0xffffffffu, Fl[v], 1);
            }
#pragma unroll
            for (int k = 0; k < NFX; ++k) {
                // this cell's minus value when the mass flows left, else the left cell's plus value
                const float up_left = __shfl_up_sync(0xffffffffu, xo[6 * k + 3], 1);
                const float fl = (Fl[0] < 0.f ? xo[6 * k] : up_left) * Fl[0];
                dxxN[k] = (double)fl - (double)__shfl_down_sync(0xffffffffu, fl, 1);
            }
            // 4. z-face z+1/2
            fast::riemann<3>(c.eos, RS, hzU, hm[2], 2, Gzhi);
#pragma unroll
            for (int k = 0; k < NFX; ++k) {
                gzx_hi[k] = (Gzhi[0] < 0.f ? xo[6 * k + 2] : xzU[k]) * Gzhi[0];
            }
        }
        // 5. y-face states of plane z+1 for the neighbours
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            sh.yface[(z + 1) & 1][w][0][v][lane] = hm[1][v];
            sh.yface[(z + 1) & 1][w][1][v][lane] = hp[1][v];
        }
#pragma unroll
        for (int k = 0; k < NFX; ++k) {
            fxs[k].xyface[(z + 1) & 1][w][0][lane] = xo[6 * k + 1];
            fxs[k].xyface[(z + 1) & 1][w][1][lane] = xo[6 * k + 4];
        }
        // 6. y-face above this row, plane z
        const bool upd = z >= z0;
        if (upd && w_yface) {
            float yL[5], yR[5], G[5];
#pragma unroll
            for (int v = 0; v < 5; ++v) {
                yL[v] = sh.yface[z & 1][w][1][v][lane];
                yR[v] = sh.yface[z & 1][wu][0][v][lane];
            }
            fast::riemann<3>(c.eos, RS, yL, yR, 1, G);
#pragma unroll
            for (int v = 0; v < 5; ++v) {
                sh.gflux[z & 1][w][v][lane] = G[v];
            }
#pragma unroll
            for (int k = 0; k < NFX; ++k) {
                // the upper row's bottom value when the mass flows down, else this row's top value
                const float xu =
                    G[0] < 0.f ? fxs[k].xyface[z & 1][wu][0][lane] : fxs[k].xyface[z & 1][w][1][lane];
                fxs[k].xgflux[z & 1][w][lane] = xu * G[0];
            }
        }
        __syncthreads();
        // 7. update of plane z
        if (upd && out_cell) {
            double q[5 + NFX], qn[5];
            const int64_t oo = ((int64_t)z * n1 + row) * pitch + col;
#pragma unroll
            for (int v = 0; v < 5 + NFX; ++v) {
                q[v] = __ldg(qin + oo + plane * v);
            }
#pragma unroll
            for (int v = 0; v < 5; ++v) {
                const double gb = (double)sh.gflux[z & 1][wd][v][lane];
                const double gt = (double)sh.gflux[z & 1][w][v][lane];
                qn[v] = q[v] + fma(cxyz[0], dFx[v],
                                   fma(cxyz[1], gb - gt, cxyz[2] * ((double)Gzlo[v] - (double)Gzhi[v])));
            }
            if (c.gravity) {
                qn[1] = fma(Dg[0], q[0], qn[1]);
                qn[2] = fma(Dg[1], q[0], qn[2]);
                qn[3] = fma(Dg[2], q[0], qn[3]);
                qn[4] = fma(Dg[0], q[1], fma(Dg[1], q[2], fma(Dg[2], q[3], qn[4])));
            }
            // health check (main.cpp:397-425) in FP64 without the division:
            // evol = E - |m|^2 / (2 rho) has the sign of 2 rho E - |m|^2
            // (reversed for rho < 0; rho = 0 fails)
            const double tre = (qn[0] + qn[0]) * qn[4];
            const double mm = fma(qn[1], qn[1], fma(qn[2], qn[2], qn[3] * qn[3]));
            const bool healthy = qn[0] > 0.0 ? tre >= mm : (qn[0] < 0.0 && tre <= mm);
            if (!healthy && bad_cell < 0) {
                bad_cell = lidx(g, col, row, z);
            }
            // CFL contribution (time_step.hpp:55-77) in FP32 from the FP64
            // internal energy: c^2 = gamma (gamma-1) / 2 * (2 rho E - |m|^2) / rho^2
            {
                const float ir = __fdividef(1.f, (float)qn[0]);
                const float c2 = g.cfl_kc2 * (float)(tre - mm) * ir * ir;
                const float snd = sqrtf(c2);
                const float cell = fmaf(fabsf((float)qn[1] * ir) + snd, g.inv_dx_f[0],
                                        fmaf(fabsf((float)qn[2] * ir) + snd, g.inv_dx_f[1],
                                             (fabsf((float)qn[3] * ir) + snd) * g.inv_dx_f[2]));
                inv_f = cell > inv_f ? cell : (isnan(cell) ? cell : inv_f);
            }
#pragma unroll
            for (int v = 0; v < 5; ++v) {
                qout[oo + plane * v] = qn[v];
            }
            double xnew[NX];
#pragma unroll
            for (int k = 0; k < NFX; ++k) {
                const double gb = (double)fxs[k].xgflux[z & 1][wd][lane];
                const double gt = (double)fxs[k].xgflux[z & 1][w][lane];
                const double xn = fma(q[5 + k], q[0], fma(cxyz[0], dxx[k], fma(cxyz[1], gb - gt, cxyz[2] * ((double)gzx_lo[k] - (double)gzx_hi[k]))));
                double xv = xn / qn[0];
                xv = xv < 0. ? 0. : (xv > 1. ? 1. : xv);
                xnew[k] = xv;
                qout[oo + plane * (5 + k)] = xv;
            }
            // ghost images of border cells (boundary_distribute.hpp:42-76)
            const unsigned zm = (z < 2 * g.ng || z >= g.n[2] - 2 * g.ng)
                                    ? ghost_mask(z, g.n[2], g.ng, g.bc[4], g.bc[5])
                                    : 0u;
            if ((xym | zm) != 0u) {
                store_images_3d(qout, plane, pitch, n0, n1, g.n[2], g.ng, col, row, z, xm, ym, zm, qn);
#pragma unroll
                for (int k = 0; k < NFX; ++k) {
                    store_images_3d_scalar(qout + plane * (5 + k), pitch, n0, n1, g.n[2], g.ng, col, row, z, xm, ym, zm,
                                           xnew[k]);
                }
            }
        }
        // slide the window
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            wC[v] = wD[v];
            wD[v] = wN[v];
            hzU[v] = hp[2][v];
            dFx[v] = dFxN[v];
            Gzlo[v] = Gzhi[v];
        }
#pragma unroll
        for (int k = 0; k < NFX; ++k) {
            xC[k] = xD[k];
            xD[k] = xN[k];
            xzU[k] = xo[6 * k + 5];
            dxx[k] = dxxN[k];
            gzx_lo[k] = gzx_hi[k];
        }
    }

    // warp max of 1/dt -> one atomic per warp
    inv_max = (double)inv_f;
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

} // namespace hcl::fused
