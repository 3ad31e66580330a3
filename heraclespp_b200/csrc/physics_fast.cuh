// physics_fast.cuh -- FP32 per-cell physics of the mixed-precision step.
//
// Same mathematics as the reference, rewritten in algebraically equal forms
// that cost fewer divisions:
//  * PerfectGas: P = (gamma-1) e and e = P/(gamma-1); the reference's
//    temperature round trip (thermodynamics/perfect_gas.hpp:46-78) multiplies
//    and divides by the same kb*T/(mmw*mp) factors, which cancel exactly in
//    real arithmetic.
//  * limiters on raw differences (hydro/slope_limiters.hpp:38-85):
//    VanLeer 2RL/(R+L), Minmod sign*min(|R|,|L|), VanAlbada RL(R+L)/(R^2+L^2),
//    all zero when RL <= 0.
//  * fluxes use the conservative energy where the reference rebuilds it from
//    the primitives (equal in real arithmetic).
// Divisions use the hardware reciprocal approximation (this TU is compiled
// with -prec-div=false -ftz=true).  State vectors are [rho, v_0..v_{ND-1}, E|P].
#pragma once

#include "hcl_device.cuh"

namespace hcl::fast {

struct Eos {
    float gamma, gm1, inv_gm1;
};

__device__ __forceinline__ float rcp(float x)
{
    return __fdividef(1.0f, x);
}

template <int ND>
__device__ __forceinline__ void to_cons(const Eos& e, const float* p, float* c)
{
    float u2 = 0.f;
    c[0] = p[0];
#pragma unroll
    for (int d = 0; d < ND; ++d) {
        c[1 + d] = p[0] * p[1 + d];
        u2 = fmaf(p[1 + d], p[1 + d], u2);
    }
    c[1 + ND] = fmaf(0.5f * p[0], u2, p[1 + ND] * e.inv_gm1);
}

// primitive state from a conservative one, also returning 1/rho
template <int ND>
__device__ __forceinline__ float to_prim(const Eos& e, const float* c, float* p)
{
    const float ir = rcp(c[0]);
    float mu = 0.f;
    p[0] = c[0];
#pragma unroll
    for (int d = 0; d < ND; ++d) {
        p[1 + d] = c[1 + d] * ir;
        mu = fmaf(c[1 + d], p[1 + d], mu);
    }
    p[1 + ND] = e.gm1 * fmaf(-0.5f, mu, c[1 + ND]);
    return ir;
}

// physical flux from a primitive state (hydro/euler_equations.hpp:72-86)
template <int ND>
__device__ __forceinline__ void flux_prim(const Eos& e, const float* p, int l, float* f)
{
    float u2 = 0.f;
#pragma unroll
    for (int d = 0; d < ND; ++d) {
        u2 = fmaf(p[1 + d], p[1 + d], u2);
    }
    const float P = p[1 + ND];
    const float Et = fmaf(0.5f * p[0], u2, P * e.inv_gm1);
    const float ul = p[1 + l];
    f[0] = p[0] * ul;
#pragma unroll
    for (int d = 0; d < ND; ++d) {
        f[1 + d] = f[0] * p[1 + d];
    }
    f[1 + l] += P;
    f[1 + ND] = ul * (Et + P);
}

// limited slope on raw differences (see header comment)
__device__ __forceinline__ float limited(int lim, float dR, float dL)
{
    const float prod = dR * dL;
    if (lim == LIM_CONSTANT || !(prod > 0.f)) {
        return 0.f;
    }
    if (lim == LIM_VANLEER) {
        return 2.f * prod * rcp(dR + dL);
    }
    if (lim == LIM_MINMOD) {
        return fabsf(dR) < fabsf(dL) ? dR : dL;
    }
    return prod * (dR + dL) * rcp(fmaf(dR, dR, dL * dL));
}

// hydro/riemann_solver.hpp:22-181 on conservative face states
template <int ND>
__device__ __forceinline__ void riemann(const Eos& e, int solver, const float* cL, const float* cR, int l, float* f)
{
    float pL[ND + 2], pR[ND + 2];
    const float irL = to_prim<ND>(e, cL, pL);
    const float irR = to_prim<ND>(e, cR, pR);
    const float PL = pL[1 + ND], PR = pR[1 + ND];
    const float aL = sqrtf(e.gamma * PL * irL);
    const float aR = sqrtf(e.gamma * PR * irR);
    const float uL = pL[1 + l], uR = pR[1 + l];
    if (solver == RS_SPLITTING) {
        const float a = 1.1f * fmaxf(cL[0] * aL, cR[0] * aR);
        const float ustar = 0.5f * (uL + uR) - (0.5f * rcp(a)) * (PR - PL);
        const float Ma = fabsf(ustar) * rcp(fminf(aL, aR));
        const float theta = fminf(1.f, Ma);
        const float Pstar = 0.5f * (PL + PR) - 0.5f * theta * a * (uR - uL);
        const float* cs = ustar > 0.f ? cL : cR;
        f[0] = ustar * cs[0];
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            f[1 + d] = ustar * cs[1 + d];
        }
        f[1 + l] += Pstar;
        f[1 + ND] = ustar * (cs[1 + ND] + Pstar);
        return;
    }
    const float wsL = fminf(uL - aL, uR - aR);
    const float wsR = fmaxf(uL + aL, uR + aR);
    if (solver == RS_HLL) {
        const float sl = fminf(wsL, 0.f);
        const float sr = fmaxf(wsR, 0.f);
        const float inv = rcp(sr - sl);
        // physical fluxes from the conservative states
        float fL[ND + 2], fR[ND + 2];
        fL[0] = cL[1 + l];
        fR[0] = cR[1 + l];
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            fL[1 + d] = cL[1 + l] * pL[1 + d];
            fR[1 + d] = cR[1 + l] * pR[1 + d];
        }
        fL[1 + l] += PL;
        fR[1 + l] += PR;
        fL[1 + ND] = uL * (cL[1 + ND] + PL);
        fR[1 + ND] = uR * (cR[1 + ND] + PR);
        const float slsr = sl * sr;
#pragma unroll
        for (int v = 0; v < ND + 2; ++v) {
            f[v] = (sr * fL[v] - sl * fR[v] + slsr * (cR[v] - cL[v])) * inv;
        }
        return;
    }
    // HLLC
    const float rcL = cL[0] * (wsL - uL);
    const float rcR = cR[0] * (wsR - uR);
    const float ustar = (PR - PL + rcL * uL - rcR * uR) * rcp(rcL - rcR);
    const float pstar = 0.5f * (PL + PR + rcL * (ustar - uL) + rcR * (ustar - uR));
    const bool left = ustar > 0.f;
    const float S = left ? wsL : wsR;
    const float* cs = left ? cL : cR;
    const float* ps = left ? pL : pR;
    const float un = ps[1 + l];
    const float Ps = ps[1 + ND];
    const float mn = cs[1 + l];
    if (wsL * wsR > 0.f) {
        f[0] = mn;
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            f[1 + d] = mn * ps[1 + d];
        }
        f[1 + l] += Ps;
        f[1 + ND] = un * (cs[1 + ND] + Ps);
        return;
    }
    const float inv = rcp(S - ustar);
    const float ratio = (S - un) * inv;
    const float rho_star = cs[0] * ratio;
    f[0] = mn + S * (rho_star - cs[0]);
    const float rsu = rho_star * ustar;
#pragma unroll
    for (int d = 0; d < ND; ++d) {
        f[1 + d] = rsu * ps[1 + d];
    }
    f[1 + l] = fmaf(rsu, ustar, pstar);
    const float E_star = ratio * cs[1 + ND] + (ustar - un) * inv * (ustar * cs[0] * (S - un) + Ps);
    f[1 + ND] = un * (cs[1 + ND] + Ps) + S * (E_star - cs[1 + ND]);
}

} // namespace hcl::fast
