// fused_strip2d_pair.cuh -- the FP32-mixed 2-D fused step with two columns
// per lane in packed FP32 pairs (uniform Cartesian grids, uniform gravity).
//
// Same mathematics, precision split and row march as fused_strip2d.cuh.  A
// lane holds columns a = c0 - 2 + 2*lane and a + 1 in the two halves of its
// float2 values, so each FP32 operation of the two cells is one packed
// FADD2 / FMUL2 / FFMA2 instruction of sm_100; the FP64 parts (primitive
// recovery, update, CFL) stay per cell.  A warp writes 60 columns (lanes
// 1..30; lanes 0 and 31 are the stencil halo).  x-neighbours: the left
// neighbour of half .x is the previous lane's .y, the right neighbour of
// half .y is the next lane's .x.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "fused_step.cuh"
#include "fused_strip2d.cuh"
#include "hcl_device.cuh"
#include "physics_fast.cuh"
#include "stages.hpp"

namespace hcl::fused {

namespace pairs {

using f2 = float2;

__device__ __forceinline__ f2 mk2(float a, float b)
{
    return make_float2(a, b);
}
__device__ __forceinline__ f2 dup2(float a)
{
    return make_float2(a, a);
}
__device__ __forceinline__ f2 add2(f2 a, f2 b)
{
    return __fadd2_rn(a, b);
}
__device__ __forceinline__ f2 sub2(f2 a, f2 b)
{
    return __fadd2_rn(a, make_float2(-b.x, -b.y));
}
__device__ __forceinline__ f2 mul2(f2 a, f2 b)
{
    return __fmul2_rn(a, b);
}
__device__ __forceinline__ f2 fma2(f2 a, f2 b, f2 c)
{
    return __ffma2_rn(a, b, c);
}
__device__ __forceinline__ f2 rcp2(f2 a)
{
    return mk2(__fdividef(1.f, a.x), __fdividef(1.f, a.y));
}
__device__ __forceinline__ f2 sel2(bool px, bool py, f2 a, f2 b)
{
    return mk2(px ? a.x : b.x, py ? a.y : b.y);
}

// limited slope on raw differences (hydro/slope_limiters.hpp:38-85 in the
// product forms of physics_fast.cuh), zero when RL <= 0
template <int LIM>
__device__ __forceinline__ f2 lim2(f2 dR, f2 dL)
{
    if constexpr (LIM == LIM_CONSTANT) {
        return dup2(0.f);
    }
    const f2 prod = mul2(dR, dL);
    f2 phi;
    if constexpr (LIM == LIM_VANLEER) {
        phi = mul2(add2(prod, prod), rcp2(add2(dR, dL)));
    } else if constexpr (LIM == LIM_MINMOD) {
        phi = mk2(fabsf(dR.x) < fabsf(dL.x) ? dR.x : dL.x, fabsf(dR.y) < fabsf(dL.y) ? dR.y : dL.y);
    } else {
        phi = mul2(mul2(prod, add2(dR, dL)), rcp2(fma2(dR, dR, mul2(dL, dL))));
    }
    return mk2(prod.x > 0.f ? phi.x : 0.f, prod.y > 0.f ? phi.y : 0.f);
}

struct Ctx {
    fast::Eos eos;
    f2 cthx, cthy;   // (dt/2)/dx, (dt/2)/dy in both halves
    f2 dgx, dgy;     // (dt/2) g
    bool gravity;
};

// FP64 state of two cells -> packed FP32 primitives (internal energy
// recovered in FP64; FP32 reciprocal plus one FP64 Newton step)
__device__ __forceinline__ void prim_pair(double gm1, const double2 q[4], f2 w[4])
{
    const double qa[4] = {q[0].x, q[1].x, q[2].x, q[3].x};
    const double qb[4] = {q[0].y, q[1].y, q[2].y, q[3].y};
    float wa[4], wb[4];
    strip_prim(gm1, qa, wa);
    strip_prim(gm1, qb, wb);
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        w[v] = mk2(wa[v], wb[v]);
    }
}

// conservative state and physical flux along direction LD of packed face
// primitives (hydro/euler_equations.hpp:72-86, :124-134)
template <int LD>
__device__ __forceinline__ void cons_flux(const fast::Eos& e, const f2 w[4], f2 U[4], f2 F[4])
{
    const f2 m0 = mul2(w[0], w[1]);
    const f2 m1 = mul2(w[0], w[2]);
    const f2 Et = fma2(dup2(0.5f), fma2(m0, w[1], mul2(m1, w[2])), mul2(w[3], dup2(e.inv_gm1)));
    U[0] = w[0];
    U[1] = m0;
    U[2] = m1;
    U[3] = Et;
    const f2 ml = LD == 0 ? m0 : m1;
    const f2 ul = LD == 0 ? w[1] : w[2];
    F[0] = ml;
    F[1] = LD == 0 ? fma2(ml, w[1], w[3]) : mul2(ml, w[1]);
    F[2] = LD == 1 ? fma2(ml, w[2], w[3]) : mul2(ml, w[2]);
    F[3] = mul2(ul, add2(Et, w[3]));
}

// Hancock face states of the two cells of a lane (conservative):
// extrapolation_reconstruction.hpp:65-143 and the gravity terms :306-312
template <int LIM>
__device__ __forceinline__ void hancock(const Ctx& c, const f2 wd[4], const f2 wc[4], const f2 wu[4], f2 hxL[4],
                                        f2 hxR[4], f2 hyB[4], f2 hyT[4])
{
    f2 fxL[4], fxR[4], fyB[4], fyT[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        const float up = __shfl_up_sync(0xffffffffu, wc[v].y, 1);
        const float dn = __shfl_down_sync(0xffffffffu, wc[v].x, 1);
        const f2 wl = mk2(up, wc[v].x);
        const f2 wr = mk2(wc[v].y, dn);
        const f2 hx = mul2(dup2(0.5f), lim2<LIM>(sub2(wr, wc[v]), sub2(wc[v], wl)));
        fxL[v] = sub2(wc[v], hx);
        fxR[v] = add2(wc[v], hx);
        const f2 hy = mul2(dup2(0.5f), lim2<LIM>(sub2(wu[v], wc[v]), sub2(wc[v], wd[v])));
        fyB[v] = sub2(wc[v], hy);
        fyT[v] = add2(wc[v], hy);
    }
    f2 FxL[4], FxR[4], FyB[4], FyT[4];
    cons_flux<0>(c.eos, fxL, hxL, FxL);
    cons_flux<0>(c.eos, fxR, hxR, FxR);
    cons_flux<1>(c.eos, fyB, hyB, FyB);
    cons_flux<1>(c.eos, fyT, hyT, FyT);
    f2 inc[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        inc[v] = fma2(c.cthx, sub2(FxL[v], FxR[v]), mul2(c.cthy, sub2(FyB[v], FyT[v])));
    }
    f2* outs[4] = {hxL, hxR, hyB, hyT};
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        f2* u = outs[f];
        const f2 r0 = u[0], m0 = u[1], m1 = u[2];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            u[v] = add2(u[v], inc[v]);
        }
        if (c.gravity) {
            u[1] = fma2(c.dgx, r0, u[1]);
            u[2] = fma2(c.dgy, r0, u[2]);
            u[3] = fma2(c.dgx, m0, fma2(c.dgy, m1, u[3]));
        }
    }
}

// primitives of packed conservative states; returns 1/rho (fast::to_prim)
__device__ __forceinline__ f2 to_prim(const fast::Eos& e, const f2 c[4], f2 p[4])
{
    const f2 ir = rcp2(c[0]);
    p[0] = c[0];
    p[1] = mul2(c[1], ir);
    p[2] = mul2(c[2], ir);
    const f2 mu = fma2(c[2], p[2], mul2(c[1], p[1]));
    p[3] = mul2(dup2(e.gm1), fma2(dup2(-0.5f), mu, c[3]));
    return ir;
}

// Riemann solvers on packed conservative face states along LD
// (hydro/riemann_solver.hpp:22-181, as fast::riemann): both halves computed,
// the HLLC branches taken by per-half selects
template <int RS, int LD>
__device__ __forceinline__ void riemann(const fast::Eos& e, const f2 cL[4], const f2 cR[4], f2 f[4])
{
    constexpr int n = 1 + LD, t = 2 - LD;
    if constexpr (RS == RS_SPLITTING) {
        float L[2][4], R[2][4], F[2][4];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            L[0][v] = cL[v].x;
            L[1][v] = cL[v].y;
            R[0][v] = cR[v].x;
            R[1][v] = cR[v].y;
        }
        fast::riemann<2>(e, RS, L[0], R[0], LD, F[0]);
        fast::riemann<2>(e, RS, L[1], R[1], LD, F[1]);
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            f[v] = mk2(F[0][v], F[1][v]);
        }
        return;
    }
    f2 pL[4], pR[4];
    const f2 irL = to_prim(e, cL, pL);
    const f2 irR = to_prim(e, cR, pR);
    const f2 sL = mul2(mul2(dup2(e.gamma), pL[3]), irL);
    const f2 sR = mul2(mul2(dup2(e.gamma), pR[3]), irR);
    const f2 aL = mk2(sqrtf(sL.x), sqrtf(sL.y));
    const f2 aR = mk2(sqrtf(sR.x), sqrtf(sR.y));
    const f2 uL = pL[n], uR = pR[n];
    const f2 l1 = sub2(uL, aL), r1 = sub2(uR, aR);
    const f2 l2 = add2(uL, aL), r2 = add2(uR, aR);
    const f2 wsL = mk2(fminf(l1.x, r1.x), fminf(l1.y, r1.y));
    const f2 wsR = mk2(fmaxf(l2.x, r2.x), fmaxf(l2.y, r2.y));
    if constexpr (RS == RS_HLL) {
        const f2 sl = mk2(fminf(wsL.x, 0.f), fminf(wsL.y, 0.f));
        const f2 sr = mk2(fmaxf(wsR.x, 0.f), fmaxf(wsR.y, 0.f));
        const f2 inv = rcp2(sub2(sr, sl));
        const f2 slsr = mul2(sl, sr);
        f2 fL[4], fR[4];
        fL[0] = cL[n];
        fR[0] = cR[n];
        fL[n] = fma2(cL[n], pL[n], pL[3]);
        fR[n] = fma2(cR[n], pR[n], pR[3]);
        fL[t] = mul2(cL[n], pL[t]);
        fR[t] = mul2(cR[n], pR[t]);
        fL[3] = mul2(uL, add2(cL[3], pL[3]));
        fR[3] = mul2(uR, add2(cR[3], pR[3]));
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            f[v] = mul2(fma2(slsr, sub2(cR[v], cL[v]), sub2(mul2(sr, fL[v]), mul2(sl, fR[v]))), inv);
        }
        return;
    }
    // HLLC
    const f2 rcL = mul2(cL[0], sub2(wsL, uL));
    const f2 rcR = mul2(cR[0], sub2(wsR, uR));
    const f2 num = sub2(fma2(rcL, uL, sub2(pR[3], pL[3])), mul2(rcR, uR));
    const f2 ustar = mul2(num, rcp2(sub2(rcL, rcR)));
    const f2 pstar =
        mul2(dup2(0.5f), fma2(rcR, sub2(ustar, uR), fma2(rcL, sub2(ustar, uL), add2(pL[3], pR[3]))));
    const bool lx = ustar.x > 0.f, ly = ustar.y > 0.f;
    const f2 S = sel2(lx, ly, wsL, wsR);
    f2 cs[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        cs[v] = sel2(lx, ly, cL[v], cR[v]);
    }
    const f2 un = sel2(lx, ly, pL[n], pR[n]);
    const f2 ut = sel2(lx, ly, pL[t], pR[t]);
    const f2 Ps = sel2(lx, ly, pL[3], pR[3]);
    const f2 mn = cs[n];
    const f2 eP = add2(cs[3], Ps);
    // supersonic: the upwind physical flux
    f2 fs[4];
    fs[0] = mn;
    fs[n] = fma2(mn, un, Ps);
    fs[t] = mul2(mn, ut);
    fs[3] = mul2(un, eP);
    // star state
    const f2 Smu = sub2(S, un);
    const f2 inv = rcp2(sub2(S, ustar));
    const f2 ratio = mul2(Smu, inv);
    const f2 rho_star = mul2(cs[0], ratio);
    const f2 rsu = mul2(rho_star, ustar);
    const f2 E_star = fma2(ratio, cs[3], mul2(mul2(sub2(ustar, un), inv), fma2(mul2(ustar, cs[0]), Smu, Ps)));
    f2 fc[4];
    fc[0] = fma2(S, sub2(rho_star, cs[0]), mn);
    fc[n] = fma2(rsu, ustar, pstar);
    fc[t] = mul2(rsu, ut);
    fc[3] = fma2(S, sub2(E_star, cs[3]), mul2(un, eP));
    const f2 wprod = mul2(wsL, wsR);
    const bool sx = wprod.x > 0.f, sy = wprod.y > 0.f;
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        f[v] = sel2(sx, sy, fs[v], fc[v]);
    }
}

} // namespace pairs

// FP64 update of one cell of a pair (godunov_scheme.hpp:159-163, 258-260),
// its health check (main.cpp:397-425), CFL contribution (time_step.hpp:55-77),
// store and ghost images (boundary_distribute.hpp:42-76)
__device__ __forceinline__ void pair_update_cell(const GridDev& g, double* __restrict__ qout, int64_t plane, int pitch,
                                                 int col, int r, const double q[4], const double Fl[4],
                                                 const double Fr[4], const double Glo[4], const double Ghi[4],
                                                 double cx, double cy, double Dgx, double Dgy, double& inv_max,
                                                 int64_t& bad_cell, bool store_pair_later, double qn[4])
{
    const int n0 = g.n[0], n1 = g.n[1];
    const double gm1 = g.gamma_m1;
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        qn[v] = q[v] + fma(cx, Fl[v] - Fr[v], cy * (Glo[v] - Ghi[v]));
    }
    qn[1] = fma(Dgx, q[0], qn[1]);
    qn[2] = fma(Dgy, q[0], qn[2]);
    qn[3] = fma(Dgx, q[1], fma(Dgy, q[2], qn[3]));
    double rr = (double)__fdividef(1.f, (float)qn[0]);
    rr = rr * (2.0 - qn[0] * rr);
    const double u = qn[1] * rr;
    const double vv = qn[2] * rr;
    const double evol = fma(-0.5, fma(qn[1], u, qn[2] * vv), qn[3]);
    const double c2 = g.gamma * gm1 * evol * rr;
    double y = (double)rsqrtf((float)c2);
    y = y * (1.5 - 0.5 * c2 * y * y);
    const double snd = c2 * y;
    const double cell = fma(fabs(u) + snd, g.inv_dx[0], (fabs(vv) + snd) * g.inv_dx[1]);
    inv_max = cell > inv_max ? cell : (isnan(cell) ? cell : inv_max);
    if (!(evol >= 0.0) && bad_cell < 0) {
        bad_cell = lidx(g, col, r, 0);
    }
    const int64_t oo = (int64_t)r * pitch + col;
    if (!store_pair_later) {
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            qout[oo + plane * v] = qn[v];
        }
    }
    if (!(col >= 2 * g.ng && col < n0 - 2 * g.ng && r >= 2 * g.ng && r < n1 - 2 * g.ng)) {
        const unsigned xm = ghost_mask(col, n0, g.ng, g.bc[0], g.bc[1]);
        const unsigned ym = ghost_mask(r, n1, g.ng, g.bc[2], g.bc[3]);
        store_images_2d(qout, plane, pitch, n0, n1, g.ng, col, r, xm, ym, qn);
    }
}

// One strip of the paired schedule: 60 columns x rows [r0, r1).
template <int LIM, int RS>
__device__ __forceinline__ void pair_strip_work(const GridDev& g, const double* __restrict__ qin,
                                                double* __restrict__ qout, int64_t plane, int pitch, double dt, int sx,
                                                int sy, int L, double& inv_max, int64_t& bad_cell)
{
    using namespace pairs;
    const int lane = threadIdx.x & 31;
    const int n0 = g.n[0], n1 = g.n[1];
    const int c0 = g.ng + kPairLanesOut * sx;
    const int a = c0 - 2 + 2 * lane; // first column of the lane (even: ng is even)
    const bool whole = a + 1 < n0;   // both columns inside the row (the vector load)
    const int col_end = g.ng + g.nx[0];
    const bool mid = lane >= 1 && lane <= 30;
    const bool out_a = mid && a < col_end;
    const bool out_b = mid && a + 1 < col_end;
    const int r0 = g.ng + L * sy;
    const int r1 = min(r0 + L, g.ng + g.nx[1]);

    Ctx c;
    c.eos = fast::Eos{(float)g.gamma, (float)g.gamma_m1, (float)(1.0 / g.gamma_m1)};
    c.cthx = dup2((float)(0.5 * dt * g.inv_dx[0]));
    c.cthy = dup2((float)(0.5 * dt * g.inv_dx[1]));
    c.dgx = dup2((float)(0.5 * dt * g.g[0]));
    c.dgy = dup2((float)(0.5 * dt * g.g[1]));
    c.gravity = g.g[0] != 0.0 || g.g[1] != 0.0;
    const double cx = dt * g.inv_dx[0];
    const double cy = dt * g.inv_dx[1];
    const double Dgx = dt * g.g[0];
    const double Dgy = dt * g.g[1];
    const double gm1 = g.gamma_m1;

    // columns beyond the row (only lanes whose cells are not written, and the
    // right neighbour of the last written cell at an odd width) read the
    // row's last column
    auto load_row = [&](int r, double2 q[4]) {
        const int64_t o = (int64_t)min(max(r, 0), n1 - 1) * pitch;
        if (whole) {
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                q[v] = __ldg(reinterpret_cast<const double2*>(qin + o + a + plane * v));
            }
        } else {
            const int ca = min(a, n0 - 1), cb = min(a + 1, n0 - 1);
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                q[v] = make_double2(__ldg(qin + o + ca + plane * v), __ldg(qin + o + cb + plane * v));
            }
        }
    };

    f2 wC[4], wD[4];
    f2 hxL[4], hxR[4], hyT[4];
    double GloA[4], GloB[4];
    double2 qPre[4];
    {
        double2 q[4];
        f2 wA[4], wB[4];
        load_row(r0 - 2, q);
        prim_pair(gm1, q, wA);
        load_row(r0 - 1, q);
        prim_pair(gm1, q, wB);
        load_row(r0, q);
        prim_pair(gm1, q, wC);
        load_row(r0 + 1, q);
        prim_pair(gm1, q, wD);
        load_row(r0 + 2, qPre);
        f2 t0[4], t1[4], t2[4], tT[4], hyB[4];
        hancock<LIM>(c, wA, wB, wC, t0, t1, t2, tT); // row r0-1: its top face
        hancock<LIM>(c, wB, wC, wD, hxL, hxR, hyB, hyT); // row r0
        f2 G[4];
        riemann<RS, 1>(c.eos, tT, hyB, G);
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            GloA[v] = (double)G[v].x;
            GloB[v] = (double)G[v].y;
        }
    }
    for (int r = r0; r < r1; ++r) {
        f2 wN[4];
        prim_pair(gm1, qPre, wN);
        load_row(r + 3, qPre);
        // Hancock of row r+1
        f2 nxL[4], nxR[4], nyB[4], nyT[4];
        hancock<LIM>(c, wC, wD, wN, nxL, nxR, nyB, nyT);
        // y-faces r+1/2 of both cells
        f2 G[4];
        riemann<RS, 1>(c.eos, hyT, nyB, G);
        // x-faces left of both cells of row r
        f2 Lx[4], F[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            Lx[v] = mk2(__shfl_up_sync(0xffffffffu, hxR[v].y, 1), hxR[v].x);
        }
        riemann<RS, 0>(c.eos, Lx, hxL, F);
        double GhiA[4], GhiB[4], FlA[4], FlB[4], FrB[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            GhiA[v] = (double)G[v].x;
            GhiB[v] = (double)G[v].y;
            FlA[v] = (double)F[v].x;
            FlB[v] = (double)F[v].y;
            FrB[v] = (double)__shfl_down_sync(0xffffffffu, F[v].x, 1);
        }
        if (out_a) {
            const int64_t oq = (int64_t)r * pitch + a;
            double qa[4], qb[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                const double2 q2 = __ldg(reinterpret_cast<const double2*>(qin + oq + plane * v));
                qa[v] = q2.x;
                qb[v] = q2.y;
            }
            double qna[4], qnb[4];
            pair_update_cell(g, qout, plane, pitch, a, r, qa, FlA, FlB, GloA, GhiA, cx, cy, Dgx, Dgy, inv_max,
                             bad_cell, out_b, qna);
            if (out_b) {
                pair_update_cell(g, qout, plane, pitch, a + 1, r, qb, FlB, FrB, GloB, GhiB, cx, cy, Dgx, Dgy, inv_max,
                                 bad_cell, true, qnb);
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    *reinterpret_cast<double2*>(qout + oq + plane * v) = make_double2(qna[v], qnb[v]);
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
            GloA[v] = GhiA[v];
            GloB[v] = GhiB[v];
        }
    }
}

template <int LIM, int RS>
__global__ void __launch_bounds__(128, 3)
k_strip2d_pair(GridDev g, StateDev in, StateDev out, StepCtl* ctl, RunParamsDev rp, int slot, int out_buf, int L)
{
    const int lane = threadIdx.x & 31;
    const Decision dec = decide(ctl, slot, rp);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        publish_decision(ctl, dec, rp, slot, out_buf);
    }
    if (dec.noop || dec.neg_dt) {
        return;
    }
    const int ncolw = (g.nx[0] + kPairLanesOut - 1) / kPairLanesOut;
    const int nstrip = (g.nx[1] + L - 1) / L;
    const int nitems = ncolw * nstrip;
    const int wg = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (wg >= nitems) {
        return;
    }
    double inv_max = 0.0;
    int64_t bad_cell = -1;
    const int wstride = gridDim.x * (blockDim.x >> 5);
    for (int w = wg; w < nitems; w += wstride) {
        pair_strip_work<LIM, RS>(g, in.q, out.q, in.plane, in.pitch, dec.dt, w % ncolw, w / ncolw, L, inv_max,
                                 bad_cell);
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
}

} // namespace hcl::fused
