// adjoint_cell.cuh -- hand-written reverse-mode (discrete adjoint) of the
// per-cell and per-face pieces of the MUSCL-Hancock step.
//
// Every function pair computes a forward value and, given the adjoint of its
// outputs, accumulates the adjoint of its inputs (transpose-Jacobian product).
// Branches (limiter sign test and selection, HLL/HLLC wave-speed min/max, the
// HLLC star-side switch on ustar and the supersonic switch on wsL*wsR) are
// differentiated along the branch the forward evaluation took.  The algebra
// is the PerfectGas form P = (gamma-1) e, which is the reference's temperature
// round trip (thermodynamics/perfect_gas.hpp:46-78) with the cancelling
// factors removed: the derivatives are those of the same function.
//
// Compiles as CUDA (host+device) and as plain C++ (tests check every reverse
// against central finite differences on the CPU).
#pragma once

#include <cmath>

#if defined(__CUDACC__)
#define HCL_HD __host__ __device__ __forceinline__
#else
#define HCL_HD inline
#endif

namespace hcl::adj {

template <class R>
struct Eos {
    R gamma, gm1, inv_gm1;
};

// ---- primitive <-> conservative --------------------------------------------
// W = (rho, u_d, P) from U = (rho, m_d, E)
template <int ND, class R>
HCL_HD void prim_from_cons(const Eos<R>& e, const R* U, R* W)
{
    const R ir = R(1) / U[0];
    R mu = 0;
    W[0] = U[0];
    for (int d = 0; d < ND; ++d) {
        W[1 + d] = U[1 + d] * ir;
        mu += U[1 + d] * W[1 + d];
    }
    W[1 + ND] = e.gm1 * (U[1 + ND] - R(0.5) * mu);
}

template <int ND, class R>
HCL_HD void prim_from_cons_rev(const Eos<R>& e, const R* U, const R* Wb, R* Ub)
{
    const R ir = R(1) / U[0];
    R u2 = 0;
    R u[ND];
    for (int d = 0; d < ND; ++d) {
        u[d] = U[1 + d] * ir;
        u2 += u[d] * u[d];
    }
    const R Pb = Wb[1 + ND];
    Ub[1 + ND] += e.gm1 * Pb;
    R rb = Wb[0] + Pb * e.gm1 * R(0.5) * u2;
    for (int d = 0; d < ND; ++d) {
        Ub[1 + d] += Wb[1 + d] * ir - Pb * e.gm1 * u[d];
        rb -= Wb[1 + d] * u[d] * ir;
    }
    Ub[0] += rb;
}

// U from W (hydro/euler_equations.hpp:124-134)
template <int ND, class R>
HCL_HD void cons_from_prim(const Eos<R>& e, const R* W, R* U)
{
    R u2 = 0;
    U[0] = W[0];
    for (int d = 0; d < ND; ++d) {
        U[1 + d] = W[0] * W[1 + d];
        u2 += W[1 + d] * W[1 + d];
    }
    U[1 + ND] = W[1 + ND] * e.inv_gm1 + R(0.5) * W[0] * u2;
}

template <int ND, class R>
HCL_HD void cons_from_prim_rev(const Eos<R>& e, const R* W, const R* Ub, R* Wb)
{
    R u2 = 0;
    for (int d = 0; d < ND; ++d) {
        u2 += W[1 + d] * W[1 + d];
    }
    const R Eb = Ub[1 + ND];
    R rb = Ub[0] + Eb * R(0.5) * u2;
    for (int d = 0; d < ND; ++d) {
        rb += Ub[1 + d] * W[1 + d];
        Wb[1 + d] += Ub[1 + d] * W[0] + Eb * W[0] * W[1 + d];
    }
    Wb[0] += rb;
    Wb[1 + ND] += Eb * e.inv_gm1;
}

// ---- physical flux from primitives (hydro/euler_equations.hpp:72-86) ---------
template <int ND, class R>
HCL_HD void flux_prim(const Eos<R>& e, const R* W, int l, R* F)
{
    R u2 = 0;
    for (int d = 0; d < ND; ++d) {
        u2 += W[1 + d] * W[1 + d];
    }
    const R P = W[1 + ND];
    const R Et = P * e.inv_gm1 + R(0.5) * W[0] * u2;
    const R ul = W[1 + l];
    F[0] = W[0] * ul;
    for (int d = 0; d < ND; ++d) {
        F[1 + d] = W[0] * ul * W[1 + d];
    }
    F[1 + l] += P;
    F[1 + ND] = ul * (Et + P);
}

template <int ND, class R>
HCL_HD void flux_prim_rev(const Eos<R>& e, const R* W, int l, const R* Fb, R* Wb)
{
    R u2 = 0;
    for (int d = 0; d < ND; ++d) {
        u2 += W[1 + d] * W[1 + d];
    }
    const R rho = W[0];
    const R P = W[1 + ND];
    const R ul = W[1 + l];
    const R Et = P * e.inv_gm1 + R(0.5) * rho * u2;
    const R FEb = Fb[1 + ND];
    // F_rho = rho ul
    R rb = Fb[0] * ul;
    R ulb = Fb[0] * rho;
    // F_m_d = rho ul u_d (+P for d == l)
    for (int d = 0; d < ND; ++d) {
        rb += Fb[1 + d] * ul * W[1 + d];
        ulb += Fb[1 + d] * rho * W[1 + d];
        Wb[1 + d] += Fb[1 + d] * rho * ul; // d/du_d (for d == l adds the second u_l factor)
    }
    R Pb = Fb[1 + l];
    // F_E = ul (Et + P), Et = P/gm1 + rho u2 / 2
    ulb += FEb * (Et + P);
    rb += FEb * ul * R(0.5) * u2;
    for (int d = 0; d < ND; ++d) {
        Wb[1 + d] += FEb * ul * rho * W[1 + d];
    }
    Pb += FEb * ul * (e.inv_gm1 + R(1));
    Wb[0] += rb;
    Wb[1 + l] += ulb;
    Wb[1 + ND] += Pb;
}

// ---- spherical geometric source terms (hydro/source_terms.hpp:16-77) -----------
// The momentum sources of one direction d of a cell from its two face states
// W_L, W_R along d in primitive form, as the predictor
// (extrapolation_reconstruction.hpp:145-303, k = dt/2 / dv) and the update
// (godunov_scheme.hpp:165-256, k = dt / dv on the predicted states) add them:
//  d = 0: m_r  += k (P_L + P_R)/2 (dS_p - dS)
//         m_r  += k (rho_L u_o,L^2 + rho_R u_o,R^2)/2 (dS_p - dS)/2     (o = theta, phi)
//         m_o  -= k rf (rho_R u_o,R u_r,R dS_p + rho_L u_o,L u_r,L dS)
//  d = 1: m_th += k (P_L + P_R)/2 (dS_p - dS)
//         m_th += k (rho_L u_ph,L^2 + rho_R u_ph,R^2)/2 cot (dS_p - dS)/2  (3-D)
//         m_ph -= k sf (rho_R u_ph,R u_th,R dS_p + rho_L u_ph,L u_th,L dS)  (3-D)
// with dS, dS_p the areas of the cell's minus and plus faces along d,
// rf = (r_+ - r_-)/(r_+ + r_-) of the cell's radial faces, cot the cotangent
// of its mid polar angle and sf = (sin th_+ - sin th_-)/(sin th_+ + sin th_-).
template <class R>
struct SphGeo {
    R k;
    R dS, dSp;
    R rf, cot, sf;
};

template <int ND, class R>
HCL_HD void sph_source(const SphGeo<R>& s, int d, const R* WL, const R* WR, R* S)
{
    const R dd = s.dSp - s.dS;
    if (d == 0) {
        S[1] += s.k * (WL[1 + ND] + WR[1 + ND]) / R(2) * dd;
        for (int o = 1; o < ND; ++o) {
            S[1] += s.k * ((WL[0] * WL[1 + o] * WL[1 + o]) + (WR[0] * WR[1 + o] * WR[1 + o])) / R(2) * dd / R(2);
            S[1 + o] -= s.k * s.rf * ((WR[0] * WR[1 + o] * WR[1] * s.dSp) + (WL[0] * WL[1 + o] * WL[1] * s.dS));
        }
    } else if (d == 1 && ND >= 2) {
        S[2] += s.k * (WL[1 + ND] + WR[1 + ND]) / R(2) * dd;
        if (ND == 3) {
            S[2] += s.k * ((WL[0] * WL[3] * WL[3]) + (WR[0] * WR[3] * WR[3])) / R(2) * s.cot * dd / R(2);
            S[3] -= s.k * s.sf * ((WR[0] * WR[3] * WR[2] * s.dSp) + (WL[0] * WL[3] * WL[2] * s.dS));
        }
    }
}

// Accumulates into WLb, WRb the transpose of sph_source's Jacobian applied to Sb.
template <int ND, class R>
HCL_HD void sph_source_rev(const SphGeo<R>& s, int d, const R* WL, const R* WR, const R* Sb, R* WLb, R* WRb)
{
    const R dd = s.dSp - s.dS;
    if (d == 0) {
        const R a = s.k * dd / R(2) * Sb[1];
        WLb[1 + ND] += a;
        WRb[1 + ND] += a;
        const R b = s.k * dd / R(4) * Sb[1];
        for (int o = 1; o < ND; ++o) {
            WLb[0] += b * WL[1 + o] * WL[1 + o];
            WLb[1 + o] += b * R(2) * WL[0] * WL[1 + o];
            WRb[0] += b * WR[1 + o] * WR[1 + o];
            WRb[1 + o] += b * R(2) * WR[0] * WR[1 + o];
            const R c = -s.k * s.rf * Sb[1 + o];
            const R cR = c * s.dSp, cL = c * s.dS;
            WRb[0] += cR * WR[1 + o] * WR[1];
            WRb[1 + o] += cR * WR[0] * WR[1];
            WRb[1] += cR * WR[0] * WR[1 + o];
            WLb[0] += cL * WL[1 + o] * WL[1];
            WLb[1 + o] += cL * WL[0] * WL[1];
            WLb[1] += cL * WL[0] * WL[1 + o];
        }
    } else if (d == 1 && ND >= 2) {
        const R a = s.k * dd / R(2) * Sb[2];
        WLb[1 + ND] += a;
        WRb[1 + ND] += a;
        if (ND == 3) {
            const R b = s.k * s.cot * dd / R(4) * Sb[2];
            WLb[0] += b * WL[3] * WL[3];
            WLb[3] += b * R(2) * WL[0] * WL[3];
            WRb[0] += b * WR[3] * WR[3];
            WRb[3] += b * R(2) * WR[0] * WR[3];
            const R c = -s.k * s.sf * Sb[3];
            const R cR = c * s.dSp, cL = c * s.dS;
            WRb[0] += cR * WR[3] * WR[2];
            WRb[3] += cR * WR[0] * WR[2];
            WRb[2] += cR * WR[0] * WR[3];
            WLb[0] += cL * WL[3] * WL[2];
            WLb[3] += cL * WL[0] * WL[2];
            WLb[2] += cL * WL[0] * WL[3];
        }
    }
}

// ---- limiters on raw differences (hydro/slope_limiters.hpp) --------------------
// phi(R, L) and its partials; zero when R*L <= 0.
template <class R>
HCL_HD R limiter(int lim, R dR, R dL, R* gR, R* gL)
{
    *gR = 0;
    *gL = 0;
    const R prod = dR * dL;
    if (lim == 0 || !(prod > R(0))) {
        return R(0);
    }
    if (lim == 1) { // van Leer: 2RL/(R+L)
        // partials 2 (L/(R+L))^2 and 2 (R/(R+L))^2, formed from the ratios
        // (each in (0, 1) when RL > 0) so that tiny differences neither
        // overflow 1/(R+L)^2 nor underflow L^2 into 0 * inf
        const R s = dR + dL;
        const R is = R(1) / s;
        const R a = dL * is;
        const R b = dR * is;
        *gR = R(2) * a * a;
        *gL = R(2) * b * b;
        return R(2) * prod * is;
    }
    if (lim == 2) { // minmod
        if (std::fabs(dR) < std::fabs(dL)) {
            *gR = R(1);
            return dR;
        }
        *gL = R(1);
        return dL;
    }
    // van Albada: RL(R+L)/(R^2+L^2).  Its partials
    // L^2 (L^2 + 2RL - R^2) / (R^2+L^2)^2 and R^2 (R^2 + 2RL - L^2) / (R^2+L^2)^2
    // are homogeneous of degree 0: formed from R and L scaled by
    // 1/max(|R|, |L|), so that tiny differences do not overflow them
    const R N = prod * (dR + dL);
    const R D = dR * dR + dL * dL;
    const R iD = R(1) / D;
    const R im = R(1) / std::fmax(std::fabs(dR), std::fabs(dL));
    const R r = dR * im;
    const R l = dL * im;
    const R d = r * r + l * l;
    const R id2 = R(1) / (d * d);
    *gR = l * l * (l * l + R(2) * r * l - r * r) * id2;
    *gL = r * r * (r * r + R(2) * r * l - l * l) * id2;
    return N * iD;
}

// The limiter on raw differences along a branch decided by the caller
// (`active`: the forward step's R*L > 0, which it forms from differences
// divided by the cell spacing; the raw product can underflow to 0 where the
// scaled one does not).  Partials as in limiter().
template <class R>
HCL_HD R limiter_on(int lim, bool active, R dR, R dL, R* gR, R* gL)
{
    *gR = 0;
    *gL = 0;
    if (lim == 0 || !active) {
        return R(0);
    }
    if (lim == 1) {
        const R s = dR + dL;
        const R is = R(1) / s;
        const R a = dL * is;
        const R b = dR * is;
        *gR = R(2) * a * a;
        *gL = R(2) * b * b;
        return R(2) * (dR * dL) * is;
    }
    if (lim == 2) {
        if (std::fabs(dR) < std::fabs(dL)) {
            *gR = R(1);
            return dR;
        }
        *gL = R(1);
        return dL;
    }
    const R N = (dR * dL) * (dR + dL);
    const R D = dR * dR + dL * dL;
    const R im = R(1) / std::fmax(std::fabs(dR), std::fabs(dL));
    const R r = dR * im;
    const R l = dL * im;
    const R d = r * r + l * l;
    const R id2 = R(1) / (d * d);
    *gR = l * l * (l * l + R(2) * r * l - r * r) * id2;
    *gL = r * r * (r * r + R(2) * r * l - l * l) * id2;
    return D > R(0) ? N / D : R(0);
}

// ---- Riemann solvers (hydro/riemann_solver.hpp) on conservative states -------
// Forward flux and reverse: given Fb, accumulate ULb, URb.  Solver 0 = HLL,
// 1 = HLLC, 2 = the low-Mach splitting solver (riemann_solver.hpp:143-181).
template <int ND, class R>
HCL_HD void riemann(const Eos<R>& e, int solver, const R* UL, const R* UR, int l, R* F)
{
    R WL[ND + 2], WR[ND + 2];
    prim_from_cons<ND>(e, UL, WL);
    prim_from_cons<ND>(e, UR, WR);
    const R PL = WL[1 + ND], PR = WR[1 + ND];
    const R aL = std::sqrt(e.gamma * PL / UL[0]);
    const R aR = std::sqrt(e.gamma * PR / UR[0]);
    const R uL = WL[1 + l], uR = WR[1 + l];
    if (solver == 2) {
        const R a = R(1.1) * (UL[0] * aL > UR[0] * aR ? UL[0] * aL : UR[0] * aR);
        const R ustar = R(0.5) * (uL + uR) - (PR - PL) / (R(2) * a);
        const R amin = aL < aR ? aL : aR;
        const R Ma = std::fabs(ustar) / amin;
        const R theta = Ma < R(1) ? Ma : R(1);
        const R Pstar = R(0.5) * (PL + PR) - R(0.5) * theta * a * (uR - uL);
        const R* U = ustar > R(0) ? UL : UR;
        for (int v = 0; v < ND + 2; ++v) {
            F[v] = ustar * U[v];
        }
        F[1 + l] += Pstar;
        F[1 + ND] += Pstar * ustar;
        return;
    }
    const R wsL = (uL - aL) < (uR - aR) ? (uL - aL) : (uR - aR);
    const R wsR = (uL + aL) > (uR + aR) ? (uL + aL) : (uR + aR);
    R FL[ND + 2], FR[ND + 2];
    flux_prim<ND>(e, WL, l, FL);
    flux_prim<ND>(e, WR, l, FR);
    if (solver == 0) {
        const R sl = wsL < R(0) ? wsL : R(0);
        const R sr = wsR > R(0) ? wsR : R(0);
        const R inv = R(1) / (sr - sl);
        for (int v = 0; v < ND + 2; ++v) {
            F[v] = (sr * FL[v] - sl * FR[v] + sl * sr * (UR[v] - UL[v])) * inv;
        }
        return;
    }
    const R rcL = UL[0] * (wsL - uL);
    const R rcR = UR[0] * (wsR - uR);
    const R ustar = (PR - PL + rcL * uL - rcR * uR) / (rcL - rcR);
    const R pstar = R(0.5) * (PL + PR + rcL * (ustar - uL) + rcR * (ustar - uR));
    const bool left = ustar > R(0);
    const R S = left ? wsL : wsR;
    const R* U = left ? UL : UR;
    const R* W = left ? WL : WR;
    const R* Fk = left ? FL : FR;
    const R un = W[1 + l];
    if (wsL * wsR > R(0)) {
        for (int v = 0; v < ND + 2; ++v) {
            F[v] = Fk[v];
        }
        return;
    }
    const R q = R(1) / (S - ustar);
    const R ratio = (S - un) * q;
    const R rs = U[0] * ratio;
    F[0] = Fk[0] + S * (rs - U[0]);
    for (int d = 0; d < ND; ++d) {
        F[1 + d] = rs * ustar * W[1 + d];
    }
    F[1 + l] = rs * ustar * ustar + pstar;
    const R Es = ratio * U[1 + ND] + (ustar - un) * q * (ustar * U[0] * (S - un) + W[1 + ND]);
    F[1 + ND] = Fk[1 + ND] + S * (Es - U[1 + ND]);
}

template <int ND, class R>
HCL_HD void riemann_rev(const Eos<R>& e, int solver, const R* UL, const R* UR, int l, const R* Fb, R* ULb, R* URb)
{
    constexpr int NV = ND + 2;
    R WL[NV], WR[NV];
    prim_from_cons<ND>(e, UL, WL);
    prim_from_cons<ND>(e, UR, WR);
    const R PL = WL[1 + ND], PR = WR[1 + ND];
    const R cL2 = e.gamma * PL / UL[0];
    const R cR2 = e.gamma * PR / UR[0];
    const R aL = std::sqrt(cL2);
    const R aR = std::sqrt(cR2);
    const R uL = WL[1 + l], uR = WR[1 + l];
    if (solver == 2) {
        // forward values along the branches the forward evaluation took
        const bool selLa = UL[0] * aL > UR[0] * aR;
        const R a = R(1.1) * (selLa ? UL[0] * aL : UR[0] * aR);
        const R ustar = R(0.5) * (uL + uR) - (PR - PL) / (R(2) * a);
        const bool selLm = aL < aR;
        const R amin = selLm ? aL : aR;
        const R Ma = std::fabs(ustar) / amin;
        const bool sub = Ma < R(1);
        const R theta = sub ? Ma : R(1);
        const R Pstar = R(0.5) * (PL + PR) - R(0.5) * theta * a * (uR - uL);
        const bool left = ustar > R(0);
        const R* U = left ? UL : UR;
        R* Ub = left ? ULb : URb;
        // F_v = ustar U_v (+ Pstar on the normal momentum, + Pstar ustar on E)
        R ustarb = Fb[1 + ND] * Pstar;
        const R Pstarb = Fb[1 + l] + Fb[1 + ND] * ustar;
        for (int v = 0; v < NV; ++v) {
            ustarb += Fb[v] * U[v];
            Ub[v] += Fb[v] * ustar;
        }
        // Pstar = (PL + PR)/2 - theta a (uR - uL)/2
        R WLb[NV], WRb[NV];
        for (int v = 0; v < NV; ++v) {
            WLb[v] = WRb[v] = R(0);
        }
        WLb[1 + ND] += R(0.5) * Pstarb;
        WRb[1 + ND] += R(0.5) * Pstarb;
        const R thetab = -R(0.5) * Pstarb * a * (uR - uL);
        R ab = -R(0.5) * Pstarb * theta * (uR - uL);
        WRb[1 + l] -= R(0.5) * Pstarb * theta * a;
        WLb[1 + l] += R(0.5) * Pstarb * theta * a;
        // theta = min(1, Ma); Ma = |ustar| / min(aL, aR)
        R aLb = 0, aRb = 0;
        if (sub) {
            const R sgn = ustar > R(0) ? R(1) : (ustar < R(0) ? R(-1) : R(0));
            ustarb += thetab * sgn / amin;
            const R aminb = -thetab * Ma / amin;
            if (selLm) {
                aLb += aminb;
            } else {
                aRb += aminb;
            }
        }
        // ustar = (uL + uR)/2 - (PR - PL)/(2a)
        WLb[1 + l] += R(0.5) * ustarb;
        WRb[1 + l] += R(0.5) * ustarb;
        WRb[1 + ND] -= ustarb / (R(2) * a);
        WLb[1 + ND] += ustarb / (R(2) * a);
        ab += ustarb * (PR - PL) / (R(2) * a * a);
        // a = 1.1 max(rhoL aL, rhoR aR)
        if (selLa) {
            WLb[0] += R(1.1) * ab * aL;
            aLb += R(1.1) * ab * UL[0];
        } else {
            WRb[0] += R(1.1) * ab * aR;
            aRb += R(1.1) * ab * UR[0];
        }
        if (aL > R(0)) {
            const R c2b = aLb * R(0.5) / aL;
            WLb[1 + ND] += c2b * e.gamma / UL[0];
            ULb[0] -= c2b * cL2 / UL[0];
        }
        if (aR > R(0)) {
            const R c2b = aRb * R(0.5) / aR;
            WRb[1 + ND] += c2b * e.gamma / UR[0];
            URb[0] -= c2b * cR2 / UR[0];
        }
        prim_from_cons_rev<ND>(e, UL, WLb, ULb);
        prim_from_cons_rev<ND>(e, UR, WRb, URb);
        return;
    }
    const bool selL_min = (uL - aL) < (uR - aR);
    const bool selL_max = (uL + aL) > (uR + aR);
    const R wsL = selL_min ? (uL - aL) : (uR - aR);
    const R wsR = selL_max ? (uL + aL) : (uR + aR);
    R FL[NV], FR[NV];
    flux_prim<ND>(e, WL, l, FL);
    flux_prim<ND>(e, WR, l, FR);
    // adjoints of intermediates
    R WLb[NV], WRb[NV], FLb[NV], FRb[NV];
    for (int v = 0; v < NV; ++v) {
        WLb[v] = WRb[v] = FLb[v] = FRb[v] = R(0);
    }
    R wsLb = 0, wsRb = 0;
    if (solver == 0) {
        const bool cl = wsL < R(0);
        const bool cr = wsR > R(0);
        const R sl = cl ? wsL : R(0);
        const R sr = cr ? wsR : R(0);
        const R inv = R(1) / (sr - sl);
        R slb = 0, srb = 0;
        for (int v = 0; v < NV; ++v) {
            const R num = sr * FL[v] - sl * FR[v] + sl * sr * (UR[v] - UL[v]);
            const R f = num * inv;
            const R nb = Fb[v] * inv;
            const R invb = Fb[v] * num;
            // inv = 1/(sr - sl): d inv = -inv^2 (d sr - d sl)
            srb += -invb * inv * inv;
            slb += invb * inv * inv;
            FLb[v] += nb * sr;
            FRb[v] -= nb * sl;
            srb += nb * (FL[v] + sl * (UR[v] - UL[v]));
            slb += nb * (-FR[v] + sr * (UR[v] - UL[v]));
            URb[v] += nb * sl * sr;
            ULb[v] -= nb * sl * sr;
            (void)f;
        }
        if (cl) {
            wsLb += slb;
        }
        if (cr) {
            wsRb += srb;
        }
    } else {
        const R rcL = UL[0] * (wsL - uL);
        const R rcR = UR[0] * (wsR - uR);
        const R num = PR - PL + rcL * uL - rcR * uR;
        const R den = rcL - rcR;
        const R ustar = num / den;
        const bool left = ustar > R(0);
        const R S = left ? wsL : wsR;
        const R* U = left ? UL : UR;
        const R* W = left ? WL : WR;
        R* Ub = left ? ULb : URb;
        R* Wb = left ? WLb : WRb;
        R* Fkb = left ? FLb : FRb;
        const R un = W[1 + l];
        R ustarb = 0, pstarb = 0, Sb = 0;
        if (wsL * wsR > R(0)) {
            for (int v = 0; v < NV; ++v) {
                Fkb[v] += Fb[v];
            }
        } else {
            const R q = R(1) / (S - ustar);
            const R ratio = (S - un) * q;
            const R rs = U[0] * ratio;
            const R A = ustar * U[0] * (S - un) + W[1 + ND];
            const R Es = ratio * U[1 + ND] + (ustar - un) * q * A;
            // F_E = Fk_E + S (Es - E)
            const R FEb = Fb[1 + ND];
            Fkb[1 + ND] += FEb;
            Sb += FEb * (Es - U[1 + ND]);
            R Esb = FEb * S;
            Ub[1 + ND] -= FEb * S;
            // Es = ratio E + (ustar - un) q A
            R ratiob = Esb * U[1 + ND];
            Ub[1 + ND] += Esb * ratio;
            ustarb += Esb * q * A;
            R unb = -Esb * q * A;
            R qb = Esb * (ustar - un) * A;
            R Ab = Esb * (ustar - un) * q;
            // A = ustar rho (S - un) + P
            ustarb += Ab * U[0] * (S - un);
            Ub[0] += Ab * ustar * (S - un);
            Sb += Ab * ustar * U[0];
            unb -= Ab * ustar * U[0];
            Wb[1 + ND] += Ab;
            // F_m_l = rs ustar^2 + pstar ; F_m_d = rs ustar u_d (d != l)
            R rsb = 0;
            for (int d = 0; d < ND; ++d) {
                if (d == l) {
                    rsb += Fb[1 + d] * ustar * ustar;
                    ustarb += Fb[1 + d] * R(2) * rs * ustar;
                    pstarb += Fb[1 + d];
                } else {
                    rsb += Fb[1 + d] * ustar * W[1 + d];
                    ustarb += Fb[1 + d] * rs * W[1 + d];
                    Wb[1 + d] += Fb[1 + d] * rs * ustar;
                }
            }
            // F_rho = Fk_rho + S (rs - rho)
            Fkb[0] += Fb[0];
            Sb += Fb[0] * (rs - U[0]);
            rsb += Fb[0] * S;
            Ub[0] -= Fb[0] * S;
            // rs = rho ratio
            Ub[0] += rsb * ratio;
            ratiob += rsb * U[0];
            // ratio = (S - un) q
            Sb += ratiob * q;
            unb -= ratiob * q;
            qb += ratiob * (S - un);
            // q = 1/(S - ustar)
            const R dq = -qb * q * q;
            Sb += dq;
            ustarb -= dq;
            Wb[1 + l] += unb;
        }
        if (left) {
            wsLb += Sb;
        } else {
            wsRb += Sb;
        }
        // pstar = (PL + PR + rcL (ustar - uL) + rcR (ustar - uR)) / 2
        R PLb = R(0.5) * pstarb;
        R PRb = R(0.5) * pstarb;
        R rcLb = R(0.5) * pstarb * (ustar - uL);
        R rcRb = R(0.5) * pstarb * (ustar - uR);
        ustarb += R(0.5) * pstarb * (rcL + rcR);
        R uLb = -R(0.5) * pstarb * rcL;
        R uRb = -R(0.5) * pstarb * rcR;
        // ustar = num / den
        const R numb = ustarb / den;
        const R denb = -ustarb * ustar / den;
        PRb += numb;
        PLb -= numb;
        rcLb += numb * uL + denb;
        uLb += numb * rcL;
        rcRb += -numb * uR - denb;
        uRb -= numb * rcR;
        // rcL = rhoL (wsL - uL), rcR = rhoR (wsR - uR)
        ULb[0] += rcLb * (wsL - uL);
        wsLb += rcLb * UL[0];
        uLb -= rcLb * UL[0];
        URb[0] += rcRb * (wsR - uR);
        wsRb += rcRb * UR[0];
        uRb -= rcRb * UR[0];
        WLb[1 + l] += uLb;
        WRb[1 + l] += uRb;
        WLb[1 + ND] += PLb;
        WRb[1 + ND] += PRb;
    }
    // wave speeds: wsL = min(uL - aL, uR - aR), wsR = max(uL + aL, uR + aR)
    R aLb = 0, aRb = 0;
    if (selL_min) {
        WLb[1 + l] += wsLb;
        aLb -= wsLb;
    } else {
        WRb[1 + l] += wsLb;
        aRb -= wsLb;
    }
    if (selL_max) {
        WLb[1 + l] += wsRb;
        aLb += wsRb;
    } else {
        WRb[1 + l] += wsRb;
        aRb += wsRb;
    }
    // a = sqrt(gamma P / rho)
    if (aL > R(0)) {
        const R c2b = aLb * R(0.5) / aL;
        WLb[1 + ND] += c2b * e.gamma / UL[0];
        ULb[0] -= c2b * cL2 / UL[0];
    }
    if (aR > R(0)) {
        const R c2b = aRb * R(0.5) / aR;
        WRb[1 + ND] += c2b * e.gamma / UR[0];
        URb[0] -= c2b * cR2 / UR[0];
    }
    flux_prim_rev<ND>(e, WL, l, FLb, WLb);
    flux_prim_rev<ND>(e, WR, l, FRb, WRb);
    prim_from_cons_rev<ND>(e, UL, WLb, ULb);
    prim_from_cons_rev<ND>(e, UR, WRb, URb);
}

} // namespace hcl::adj
