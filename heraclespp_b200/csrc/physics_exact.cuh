// physics_exact.cuh -- per-cell physics with the reference's FP64 arithmetic.
//
// Each function keeps the association order of the reference expression it
// restates, and the translation units that include this header are built
// with --fmad=false, so the device results round exactly like the reference's
// FP64 CPU build (IEEE division and square root are the CUDA defaults for
// double).  State vectors are [rho, v_0..v_{ND-1}, E or P].
//
// Eos kind EOS_PERFECT_GAS_FAST selects the fast-FP64 forms instead (used by
// the fused kernels of the fast-FP64 precision, built with FMA contraction):
// the same mathematics with fewer divisions -- P = (gamma-1) e and
// e = P/(gamma-1) (the temperature factors of perfect_gas.hpp:46-83 cancel),
// one reciprocal of rho per state, limiters on raw differences
// (slope_limiters.hpp:38-85: van Leer 2RL/(R+L), minmod the smaller of R and
// L, van Albada RL(R+L)/(R^2+L^2)) and one reciprocal of S - u* in HLLC.
// Results differ from the reference by rounding only (~1e-16 per operation).
#pragma once

#include "hcl_device.cuh"

namespace hcl::exact {

struct Eos {
    double gamma, gamma_m1, mmw;
    int kind; // EOS_PERFECT_GAS or EOS_RAD_GAS
};

__device__ __forceinline__ Eos eos_of(const GridDev& g)
{
    return Eos{g.gamma, g.gamma_m1, g.mmw, g.eos};
}

// thermodynamics/rad_gas.hpp:47-146: gas plus radiation.  The temperature
// comes from a Newton iteration (at most 100 steps, stop at |dT| <= 1e-6)
// started at the larger of the gas-only and radiation-only temperatures.
namespace rad {
__device__ __forceinline__ double evol_from_temp(const Eos& e, double rho, double T)
{
    const double T4 = T * T * T * T;
    return (rho * kKb * T / (e.mmw * kMp * e.gamma_m1)) + (kAr * T4);
}
__device__ __forceinline__ double pres_from_temp(const Eos& e, double rho, double T)
{
    const double T4 = T * T * T * T;
    return (rho * kKb * T / (e.mmw * kMp)) + (kAr * T4 / 3);
}
static __device__ __noinline__ double temp_from_pres(const Eos& e, double rho, double P)
{
    const double C1 = rho * kKb / (e.mmw * kMp);
    const double Tg = P / C1;
    const double Tr = pow(3 * P / kAr, 1. / 4);
    double T = Tr > Tg ? Tr : Tg;
    for (int i = 0; i < 100; ++i) {
        const double T3 = T * T * T;
        const double f = (kAr * T3 * T / 3) + (C1 * T) - P;
        const double df = (4 * kAr * T3 / 3) + C1;
        const double delta_T = -f / df;
        T += delta_T;
        if (fabs(delta_T) <= 1E-6) {
            break;
        }
    }
    return T;
}
static __device__ __noinline__ double temp_from_evol(const Eos& e, double rho, double evol)
{
    const double C1 = rho * kKb / (e.mmw * kMp * e.gamma_m1);
    const double Tg = evol / C1;
    const double Tr = pow(evol / kAr, 1. / 4);
    double T = Tr > Tg ? Tr : Tg;
    for (int i = 0; i < 100; ++i) {
        const double T3 = T * T * T;
        const double f = (kAr * T3 * T) + (C1 * T) - evol;
        const double df = (4 * kAr * T3) + C1;
        const double delta_T = -f / df;
        T += delta_T;
        if (fabs(delta_T) <= 1E-6 || isnan(delta_T)) {
            break;
        }
    }
    return T;
}
static __device__ __noinline__ double sound(const Eos& e, double rho, double P)
{
    const double T = temp_from_pres(e, rho, P);
    const double Pg = rho * kKb * T / (e.mmw * kMp);
    const double T4 = T * T * T * T;
    const double Pr = kAr * T4 / 3;
    const double alpha = Pr / Pg;
    const double num = (e.gamma / (e.gamma - 1)) + (20 * alpha) + (16 * alpha * alpha);
    const double den = (1. / (e.gamma - 1)) + (12 * alpha);
    const double gamma_eff = num / den;
    return sqrt(gamma_eff * Pg / rho);
}
} // namespace rad

// thermodynamics/perfect_gas.hpp:46-83: P <-> e through the temperature.
__device__ __forceinline__ double temp_from_pres(const Eos& e, double rho, double P)
{
    return P * e.mmw * kMp / (rho * kKb);
}
__device__ __forceinline__ double evol_from_temp(const Eos& e, double rho, double T)
{
    return rho * kKb * T / (e.mmw * kMp * e.gamma_m1);
}
__device__ __forceinline__ double pres_from_temp(const Eos& e, double rho, double T)
{
    return rho * kKb * T / (e.mmw * kMp);
}
__device__ __forceinline__ double temp_from_evol(const Eos& e, double rho, double evol)
{
    return evol * e.mmw * kMp * e.gamma_m1 / (rho * kKb);
}
// compute_temp_from_pres of the configured EOS (perfect_gas.hpp:64-68,
// rad_gas.hpp:71-89)
__device__ __forceinline__ double temperature(const Eos& e, double rho, double P)
{
    if (e.kind == EOS_RAD_GAS) {
        return rad::temp_from_pres(e, rho, P);
    }
    return temp_from_pres(e, rho, P);
}
__device__ __forceinline__ double evol_from_pres(const Eos& e, double rho, double P)
{
    if (e.kind == EOS_PERFECT_GAS_FAST) {
        return P * (1.0 / e.gamma_m1);
    }
    if (e.kind == EOS_RAD_GAS) {
        return rad::evol_from_temp(e, rho, rad::temp_from_pres(e, rho, P)); // rad_gas.hpp:47-51
    }
    return evol_from_temp(e, rho, temp_from_pres(e, rho, P));
}
__device__ __forceinline__ double pres_from_evol(const Eos& e, double rho, double evol)
{
    if (e.kind == EOS_PERFECT_GAS_FAST) {
        return e.gamma_m1 * evol;
    }
    if (e.kind == EOS_RAD_GAS) {
        return rad::pres_from_temp(e, rho, rad::temp_from_evol(e, rho, evol)); // rad_gas.hpp:65-69
    }
    return pres_from_temp(e, rho, temp_from_evol(e, rho, evol));
}
__device__ __forceinline__ double sound(const Eos& e, double rho, double P)
{
    if (e.kind == EOS_RAD_GAS) {
        return rad::sound(e, rho, P);
    }
    return sqrt(e.gamma * P / rho);
}

// hydro/euler_equations.hpp:41-59
template <int ND>
__device__ __forceinline__ double ek_cons(const double* c)
{
    double norm = 0;
#pragma unroll
    for (int d = 0; d < ND; ++d) {
        norm += c[1 + d] * c[1 + d];
    }
    return norm / c[0] / 2;
}
template <int ND>
__device__ __forceinline__ double ek_prim(const double* p)
{
    double norm = 0;
#pragma unroll
    for (int d = 0; d < ND; ++d) {
        norm += p[1 + d] * p[1 + d];
    }
    return p[0] * norm / 2;
}

// hydro/euler_equations.hpp:111-122
template <int ND>
__device__ __forceinline__ void to_prim(const Eos& e, const double* c, double* p)
{
    if (e.kind == EOS_PERFECT_GAS_FAST) {
        const double ir = 1.0 / c[0];
        double mu = 0;
        p[0] = c[0];
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            p[1 + d] = c[1 + d] * ir;
            mu += c[1 + d] * p[1 + d];
        }
        p[1 + ND] = e.gamma_m1 * (c[1 + ND] - 0.5 * mu);
        return;
    }
    const double evol = c[1 + ND] - ek_cons<ND>(c);
    p[0] = c[0];
#pragma unroll
    for (int d = 0; d < ND; ++d) {
        p[1 + d] = c[1 + d] / c[0];
    }
    p[1 + ND] = pres_from_evol(e, c[0], evol);
}

// hydro/euler_equations.hpp:124-134
template <int ND>
__device__ __forceinline__ void to_cons(const Eos& e, const double* p, double* c)
{
    c[0] = p[0];
#pragma unroll
    for (int d = 0; d < ND; ++d) {
        c[1 + d] = p[0] * p[1 + d];
    }
    c[1 + ND] = evol_from_pres(e, p[0], p[1 + ND]) + ek_prim<ND>(p);
}

// hydro/euler_equations.hpp:72-86
template <int ND>
__device__ __forceinline__ void flux_prim(const Eos& e, const double* p, int l, double* f)
{
    const double P = p[1 + ND];
    const double E = ek_prim<ND>(p) + evol_from_pres(e, p[0], P);
    f[0] = p[0] * p[1 + l];
#pragma unroll
    for (int d = 0; d < ND; ++d) {
        f[1 + d] = p[0] * p[1 + l] * p[1 + d];
    }
    f[1 + l] += P;
    f[1 + ND] = p[1 + l] * (E + P);
}

// hydro/slope_limiters.hpp:18-87 (division forms kept as written; the
// raw-difference forms for kind EOS_PERFECT_GAS_FAST)
__device__ __forceinline__ double slope(int lim, double diffR, double diffL, int kind = EOS_PERFECT_GAS)
{
    if (lim == LIM_CONSTANT) {
        return 0;
    }
    if (kind == EOS_PERFECT_GAS_FAST) {
        const double prod = diffR * diffL;
        if (!(prod > 0)) {
            return 0;
        }
        if (lim == LIM_VANLEER) {
            return 2 * prod / (diffR + diffL);
        }
        if (lim == LIM_MINMOD) {
            return fabs(diffR) < fabs(diffL) ? diffR : diffL;
        }
        return prod * (diffR + diffL) / (diffR * diffR + diffL * diffL);
    }
    if (diffL * diffR > 0) {
        const double ratio = diffR / diffL;
        if (lim == LIM_VANLEER) {
            return (1. / 2) * (diffR + diffL) * (4 * ratio) / ((ratio + 1) * (ratio + 1));
        }
        if (lim == LIM_MINMOD) {
            const double minmod = 2 * fmin(1., ratio) / (1 + ratio);
            return minmod * (diffL + diffR) / 2;
        }
        return (1. / 2) * (diffR + diffL) * (2 * ratio) / ((ratio * ratio) + 1);
    }
    return 0;
}

// hydro/riemann_solver.hpp:60-64, :136-140
__device__ __forceinline__ double flux_hll(double UL, double UR, double FL, double FR, double wsL, double wsR)
{
    return ((wsR * FL) - (wsL * FR) + (wsL * wsR * (UR - UL))) / (wsR - wsL);
}
__device__ __forceinline__ double flux_hllc(double F, double U, double Ustar, double ws)
{
    return F + (ws * (Ustar - U));
}

// hydro/riemann_solver.hpp:22-181.  cL/cR: conservative states; l: direction.
template <int ND>
__device__ __forceinline__ void riemann(const Eos& e, int solver, const double* cL, const double* cR, int l, double* f)
{
    double pL[ND + 2], pR[ND + 2];
    to_prim<ND>(e, cL, pL);
    to_prim<ND>(e, cR, pR);
    const double PL = pL[1 + ND];
    const double PR = pR[1 + ND];
    const double aL = sound(e, pL[0], PL);
    const double aR = sound(e, pR[0], PR);
    const double uL = pL[1 + l];
    const double uR = pR[1 + l];
    if (solver == RS_SPLITTING) {
        // :146-180
        const double a = 1.1 * fmax(pL[0] * aL, pR[0] * aR);
        const double ustar = ((uL + uR) / 2) - (1 / (2 * a) * (PR - PL));
        const double Ma = fabs(ustar) / fmin(aL, aR);
        const double theta = fmin(1., Ma);
        const double Pstar = ((PL + PR) / 2) - ((theta * a) / 2 * (uR - uL));
        const double* cs = (ustar > 0) ? cL : cR;
        f[0] = ustar * cs[0];
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            f[1 + d] = ustar * cs[1 + d];
        }
        f[1 + l] += Pstar;
        f[1 + ND] = (ustar * cs[1 + ND]) + (Pstar * ustar);
        return;
    }
    const double wsL = fmin(uL - aL, uR - aR);
    const double wsR = fmax(uL + aL, uR + aR);
    double fL[ND + 2], fR[ND + 2];
    flux_prim<ND>(e, pL, l, fL);
    flux_prim<ND>(e, pR, l, fR);
    if (solver == RS_HLL) {
        // :31-58
        const double neg_wsL = fmin(wsL, 0.);
        const double pos_wsR = fmax(wsR, 0.);
#pragma unroll
        for (int v = 0; v < ND + 2; ++v) {
            f[v] = flux_hll(cL[v], cR[v], fL[v], fR[v], neg_wsL, pos_wsR);
        }
        return;
    }
    // HLLC :70-134
    const double rcL = pL[0] * (wsL - uL);
    const double rcR = pR[0] * (wsR - uR);
    const double ustar = (PR - PL + (rcL * uL) - (rcR * uR)) / (rcL - rcR);
    const double pstar = 1. / 2 * (PL + PR + (rcL * (ustar - uL)) + (rcR * (ustar - uR)));
    const bool left = ustar > 0;
    const double S = left ? wsL : wsR;
    const double* cs = left ? cL : cR;
    const double* ps = left ? pL : pR;
    const double* fs = left ? fL : fR;
    const double un = ps[1 + l];
    if (wsL * wsR > 0) {
#pragma unroll
        for (int v = 0; v < ND + 2; ++v) {
            f[v] = fs[v];
        }
        return;
    }
    if (e.kind == EOS_PERFECT_GAS_FAST) {
        const double inv = 1.0 / (S - ustar);
        const double ratio = (S - un) * inv;
        const double rs = cs[0] * ratio;
        f[0] = flux_hllc(fs[0], cs[0], rs, S);
        const double rsu = rs * ustar;
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            f[1 + d] = rsu * ps[1 + d];
        }
        f[1 + l] = rsu * ustar + pstar;
        const double Es = ratio * cs[1 + ND] + (ustar - un) * inv * (ustar * cs[0] * (S - un) + ps[1 + ND]);
        f[1 + ND] = flux_hllc(fs[1 + ND], cs[1 + ND], Es, S);
        return;
    }
    const double rho_star = cs[0] * (S - un) / (S - ustar);
    f[0] = flux_hllc(fs[0], cs[0], rho_star, S);
#pragma unroll
    for (int d = 0; d < ND; ++d) {
        f[1 + d] = rho_star * ustar * ps[1 + d];
    }
    f[1 + l] = (rho_star * ustar * ustar) + pstar;
    const double E_star = ((S - un) / (S - ustar) * cs[1 + ND]) + ((ustar - un) / (S - ustar) * ((ustar * cs[0] * (S - un)) + ps[1 + ND]));
    f[1 + ND] = flux_hllc(fs[1 + ND], cs[1 + ND], E_star, S);
}

// hydro/source_terms.hpp:16-77 (trigonometric factors precomputed on the host
// with the same libm expressions: cot_mid = cos((x1+x1p)/2)/sin((x1+x1p)/2),
// sm = sin(x1), sp = sin(x1p)).
__device__ __forceinline__ double src_grad_pres(double dtodv, double PL, double PR, double dS, double dS_p)
{
    return dtodv * (PL + PR) / 2 * (dS_p - dS);
}
__device__ __forceinline__ double src_grad_u_r(double dtodv, double rhoL, double rhoR, double uL, double uR, double dS,
                                               double dS_p)
{
    return dtodv * ((rhoL * uL * uL) + (rhoR * uR * uR)) / 2 * (dS_p - dS) / 2;
}
__device__ __forceinline__ double src_grad_u_idir_r(double dtodv, double x0, double x0_p, double rhoL, double rhoR,
                                                    double uL_r, double uR_r, double uL_o, double uR_o, double dS,
                                                    double dS_p)
{
    return dtodv * (x0_p - x0) / (x0_p + x0) * ((rhoR * uR_o * uR_r * dS_p) + (rhoL * uL_o * uL_r * dS));
}
__device__ __forceinline__ double src_grad_u_th(double dtodv, double cot_mid, double rhoL, double rhoR, double uL,
                                                double uR, double dS, double dS_p)
{
    return dtodv * ((rhoL * uL * uL) + (rhoR * uR * uR)) / 2 * cot_mid * (dS_p - dS) / 2;
}
__device__ __forceinline__ double src_grad_u_phi(double dtodv, double sm, double sp, double rhoL, double rhoR,
                                                 double uL_th, double uR_th, double uL_phi, double uR_phi, double dS,
                                                 double dS_p)
{
    return dtodv * (sp - sm) / (sp + sm) * ((rhoR * uR_phi * uR_th * dS_p) + (rhoL * uL_phi * uL_th * dS));
}

} // namespace hcl::exact
