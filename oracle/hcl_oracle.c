/*
 * hcl_oracle.c -- CPU restatement of the HERACLES++ MUSCL-Hancock step.
 *
 * TEST INFRASTRUCTURE ONLY (see hcl_oracle.h).  Nothing in the product
 * library links or loads this file.
 *
 * Build flags matter: it must be compiled without FMA contraction and
 * without fast-math (-O2 -ffp-contract=off -fno-fast-math, no -march=native)
 * so that each expression rounds exactly as the reference's FP64 CPU build.
 * Every expression keeps the reference's association order; comments give
 * the reference path:line it restates.
 */
#include "hcl_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* units.hpp:176-177 (Joule/Kelvin and kg are exactly 1.0) */
static const double KB = 1.380649E-23;
static const double MP = 1.672649E-27;
/* units.hpp:179 */
static const double GRAV_G = 6.6743015E-11;
static const double OR_PI = 3.141592653589793238462643383279502884; /* Kokkos::numbers::pi */
/* Kokkos::numbers::pi */
static const double PI = 3.141592653589793238462643383279502884;

#define MAXV 5 /* rho + 3 momenta + E */

/* ------------------------------------------------------------------ */
/* threads                                                             */
/* ------------------------------------------------------------------ */
void or_set_threads(int nthreads)
{
#ifdef _OPENMP
    if (nthreads > 0) {
        omp_set_num_threads(nthreads);
    }
#else
    (void)nthreads;
#endif
}

int or_get_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------ */
/* EOS: thermodynamics/perfect_gas.hpp:46-89                            */
/* ------------------------------------------------------------------ */
static inline double temp_from_pres(const or_ctx* c, double rho, double P)
{
    return P * c->mmw * MP / (rho * KB); /* :69-72 */
}
static inline double evol_from_temp(const or_ctx* c, double rho, double T)
{
    return rho * KB * T / (c->mmw * MP * c->gamma_m1); /* :52-56 */
}
static inline double pres_from_temp(const or_ctx* c, double rho, double T)
{
    return rho * KB * T / (c->mmw * MP); /* :64-67 */
}
static inline double temp_from_evol(const or_ctx* c, double rho, double evol)
{
    return evol * c->mmw * MP * c->gamma_m1 / (rho * KB); /* :74-78 */
}

/* ------------------------------------------------------------------ */
/* EOS: thermodynamics/rad_gas.hpp:47-141 (gas plus radiation)          */
/* ------------------------------------------------------------------ */
/* units.hpp:69-74 (Joule, m, K are 1 there) */
#define OR_PI5 (3.141592653589793238462643383279502884 * 3.141592653589793238462643383279502884 * \
                3.141592653589793238462643383279502884 * 3.141592653589793238462643383279502884 * \
                3.141592653589793238462643383279502884)
#define OR_KB4 (1.380649E-23 * 1.380649E-23 * 1.380649E-23 * 1.380649E-23)
#define OR_HPLANCK3 (6.62607015E-34 * 6.62607015E-34 * 6.62607015E-34)
#define OR_C3 ((2.99792458E8 * 2.99792458E8) * 2.99792458E8)
static const double AR = (8 * OR_PI5 * OR_KB4) / (15 * OR_HPLANCK3 * OR_C3); /* radiation constant */

static double rad_evol_from_temp(const or_ctx* c, double rho, double T)
{
    const double T4 = T * T * T * T; /* :58-63 */
    return (rho * KB * T / (c->mmw * MP * c->gamma_m1)) + (AR * T4);
}
static double rad_pres_from_temp(const or_ctx* c, double rho, double T)
{
    const double T4 = T * T * T * T; /* :71-75 */
    return (rho * KB * T / (c->mmw * MP)) + (AR * T4 / 3);
}
static double rad_temp_from_pres(const or_ctx* c, double rho, double P)
{
    /* :77-104: Newton from the larger of the gas-only and radiation-only
       temperatures, at most 100 steps, stop when |dT| <= 1e-6 */
    const double C1 = rho * KB / (c->mmw * MP);
    const double Tg = P / C1;
    const double Tr = pow(3 * P / AR, 1. / 4);
    double T = Tr > Tg ? Tr : Tg;
    for (int i = 0; i < 100; ++i) {
        const double T3 = T * T * T;
        const double f = (AR * T3 * T / 3) + (C1 * T) - P;
        const double df = (4 * AR * T3 / 3) + C1;
        const double delta_T = -f / df;
        T += delta_T;
        if (fabs(delta_T) <= 1E-6) {
            break;
        }
    }
    return T;
}
static double rad_temp_from_evol(const or_ctx* c, double rho, double evol)
{
    /* :106-133: as above on evol = rho eint; also stops on a NaN step */
    const double C1 = rho * KB / (c->mmw * MP * c->gamma_m1);
    const double Tg = evol / C1;
    const double Tr = pow(evol / AR, 1. / 4);
    double T = Tr > Tg ? Tr : Tg;
    for (int i = 0; i < 100; ++i) {
        const double T3 = T * T * T;
        const double f = (AR * T3 * T) + (C1 * T) - evol;
        const double df = (4 * AR * T3) + C1;
        const double delta_T = -f / df;
        T += delta_T;
        if (fabs(delta_T) <= 1E-6 || isnan(delta_T)) {
            break;
        }
    }
    return T;
}
static double rad_speed_of_sound(const or_ctx* c, double rho, double P)
{
    /* :135-146: effective adiabatic index of the gas-radiation mixture */
    const double T = rad_temp_from_pres(c, rho, P);
    const double Pg = rho * KB * T / (c->mmw * MP);
    const double T4 = T * T * T * T;
    const double Pr = AR * T4 / 3;
    const double alpha = Pr / Pg;
    const double num = (c->gamma / (c->gamma - 1)) + (20 * alpha) + (16 * alpha * alpha);
    const double den = (1. / (c->gamma - 1)) + (12 * alpha);
    const double gamma_eff = num / den;
    return sqrt(gamma_eff * Pg / rho);
}

void or_set_eos(or_ctx* c, int eos)
{
    c->eos = eos;
}
double or_temperature(const or_ctx* c, double rho, double P)
{
    return c->eos == OR_EOS_RAD_GAS ? rad_temp_from_pres(c, rho, P) : temp_from_pres(c, rho, P);
}
double or_evol_from_pres(const or_ctx* c, double rho, double P)
{
    if (c->eos == OR_EOS_RAD_GAS) {
        return rad_evol_from_temp(c, rho, rad_temp_from_pres(c, rho, P)); /* rad_gas.hpp:47-51 */
    }
    return evol_from_temp(c, rho, temp_from_pres(c, rho, P)); /* :46-50 */
}
double or_pres_from_evol(const or_ctx* c, double rho, double evol)
{
    if (c->eos == OR_EOS_RAD_GAS) {
        return rad_pres_from_temp(c, rho, rad_temp_from_evol(c, rho, evol)); /* rad_gas.hpp:65-69 */
    }
    return pres_from_temp(c, rho, temp_from_evol(c, rho, evol)); /* :58-62 */
}
double or_speed_of_sound(const or_ctx* c, double rho, double P)
{
    if (c->eos == OR_EOS_RAD_GAS) {
        return rad_speed_of_sound(c, rho, P);
    }
    return sqrt(c->gamma * P / rho); /* :80-83 */
}
int or_eos_valid(double rho, double P)
{
    return isfinite(rho) && rho > 0 && isfinite(P) && P > 0; /* :85-89 */
}

/* ------------------------------------------------------------------ */
/* Euler algebra: hydro/euler_equations.hpp                             */
/* state vectors: [rho, v_0 .. v_{ndim-1}, E or P]                      */
/* ------------------------------------------------------------------ */
double or_ek_cons(const or_ctx* c, const double* cons)
{
    double norm_rhou = 0; /* :41-49 */
    for (int d = 0; d < c->ndim; ++d) {
        norm_rhou += cons[1 + d] * cons[1 + d];
    }
    return norm_rhou / cons[0] / 2;
}

double or_ek_prim(const or_ctx* c, const double* prim)
{
    double norm_u = 0; /* :51-59 */
    for (int d = 0; d < c->ndim; ++d) {
        norm_u += prim[1 + d] * prim[1 + d];
    }
    return prim[0] * norm_u / 2;
}

static inline double evol_cons(const or_ctx* c, const double* cons)
{
    return cons[1 + c->ndim] - or_ek_cons(c, cons); /* :61-65 */
}

void or_flux_from_prim(const or_ctx* c, const double* prim, int l, double* flux)
{
    /* :72-86 */
    const int nd = c->ndim;
    const double rho = prim[0];
    const double P = prim[1 + nd];
    const double E = or_ek_prim(c, prim) + or_evol_from_pres(c, rho, P);
    flux[0] = rho * prim[1 + l];
    for (int d = 0; d < nd; ++d) {
        flux[1 + d] = rho * prim[1 + l] * prim[1 + d];
    }
    flux[1 + l] += P;
    flux[1 + nd] = prim[1 + l] * (E + P);
}

void or_flux_from_cons(const or_ctx* c, const double* cons, int l, double* flux)
{
    /* :93-109 */
    const int nd = c->ndim;
    const double evol = evol_cons(c, cons);
    const double P = or_pres_from_evol(c, cons[0], evol);
    const double u = cons[1 + l] / cons[0];
    flux[0] = u * cons[0];
    for (int d = 0; d < nd; ++d) {
        flux[1 + d] = u * cons[1 + d];
    }
    flux[1 + l] += P;
    flux[1 + nd] = u * (cons[1 + nd] + P);
}

void or_to_prim(const or_ctx* c, const double* cons, double* prim)
{
    /* :111-122 */
    const int nd = c->ndim;
    const double evol = evol_cons(c, cons);
    prim[0] = cons[0];
    for (int d = 0; d < nd; ++d) {
        prim[1 + d] = cons[1 + d] / cons[0];
    }
    prim[1 + nd] = or_pres_from_evol(c, cons[0], evol);
}

void or_to_cons(const or_ctx* c, const double* prim, double* cons)
{
    /* :124-134 */
    const int nd = c->ndim;
    cons[0] = prim[0];
    for (int d = 0; d < nd; ++d) {
        cons[1 + d] = prim[0] * prim[1 + d];
    }
    cons[1 + nd] = or_evol_from_pres(c, prim[0], prim[1 + nd]) + or_ek_prim(c, prim);
}

/* ------------------------------------------------------------------ */
/* Slope limiters: hydro/slope_limiters.hpp:18-87                      */
/* ------------------------------------------------------------------ */
double or_slope(int limiter, double diffR, double diffL)
{
    switch (limiter) {
    case OR_LIM_CONSTANT:
        return 0; /* :18-27 */
    case OR_LIM_VANLEER:
        if (diffL * diffR > 0) { /* :38-46 */
            const double ratio = diffR / diffL;
            return (1. / 2) * (diffR + diffL) * (4 * ratio) / ((ratio + 1) * (ratio + 1));
        }
        return 0;
    case OR_LIM_MINMOD:
        if (diffL * diffR > 0) { /* :57-66 */
            const double ratio = diffR / diffL;
            const double minmod = 2 * fmin(1., ratio) / (1 + ratio);
            return minmod * (diffL + diffR) / 2;
        }
        return 0;
    case OR_LIM_VANALBADA:
        if (diffL * diffR > 0) { /* :77-85 */
            const double ratio = diffR / diffL;
            return (1. / 2) * (diffR + diffL) * (2 * ratio) / ((ratio * ratio) + 1);
        }
        return 0;
    default:
        return 0;
    }
}

/* ------------------------------------------------------------------ */
/* Riemann solvers: hydro/riemann_solver.hpp                            */
/* ------------------------------------------------------------------ */
static inline double flux_hll(double UL, double UR, double FL, double FR, double wsL, double wsR)
{
    return ((wsR * FL) - (wsL * FR) + (wsL * wsR * (UR - UL))) / (wsR - wsL); /* :60-64 */
}

static inline double flux_hllc(double F, double U, double Ustar, double ws)
{
    return F + (ws * (Ustar - U)); /* :136-140 */
}

static void riemann_hll(const or_ctx* c, const double* consL, const double* consR, int l, double* flux)
{
    /* :31-58 */
    const int nd = c->ndim;
    double primL[MAXV], primR[MAXV], fluxL[MAXV], fluxR[MAXV];
    or_to_prim(c, consL, primL);
    or_to_prim(c, consR, primR);
    const double cL = or_speed_of_sound(c, primL[0], primL[1 + nd]);
    const double cR = or_speed_of_sound(c, primR[0], primR[1 + nd]);
    const double wsL = fmin(primL[1 + l] - cL, primR[1 + l] - cR);
    const double wsR = fmax(primL[1 + l] + cL, primR[1 + l] + cR);
    const double neg_wsL = fmin(wsL, 0.);
    const double pos_wsR = fmax(wsR, 0.);
    or_flux_from_prim(c, primL, l, fluxL);
    or_flux_from_prim(c, primR, l, fluxR);
    for (int v = 0; v < nd + 2; ++v) {
        flux[v] = flux_hll(consL[v], consR[v], fluxL[v], fluxR[v], neg_wsL, pos_wsR);
    }
}

static void riemann_hllc(const or_ctx* c, const double* consL, const double* consR, int l, double* flux)
{
    /* :70-134 */
    const int nd = c->ndim;
    double primL[MAXV], primR[MAXV], fluxL[MAXV], fluxR[MAXV];
    or_to_prim(c, consL, primL);
    or_to_prim(c, consR, primR);
    const double PL = primL[1 + nd];
    const double PR = primR[1 + nd];
    const double cL = or_speed_of_sound(c, primL[0], PL);
    const double cR = or_speed_of_sound(c, primR[0], PR);
    const double wsL = fmin(primL[1 + l] - cL, primR[1 + l] - cR);
    const double wsR = fmax(primL[1 + l] + cL, primR[1 + l] + cR);
    or_flux_from_prim(c, primL, l, fluxL);
    or_flux_from_prim(c, primR, l, fluxR);

    const double rcL = primL[0] * (wsL - primL[1 + l]);
    const double rcR = primR[0] * (wsR - primR[1 + l]);
    const double ustar = (PR - PL + (rcL * primL[1 + l]) - (rcR * primR[1 + l])) / (rcL - rcR);
    const double pstar = 1. / 2 * (PL + PR + (rcL * (ustar - primL[1 + l])) + (rcR * (ustar - primR[1 + l])));

    double S;
    const double *cons_state, *prim_state, *flux_state;
    if (ustar > 0) {
        S = wsL;
        cons_state = consL;
        prim_state = primL;
        flux_state = fluxL;
    } else {
        S = wsR;
        cons_state = consR;
        prim_state = primR;
        flux_state = fluxR;
    }
    const double un = prim_state[1 + l];
    if (wsL * wsR > 0) {
        for (int v = 0; v < nd + 2; ++v) {
            flux[v] = flux_state[v];
        }
    } else {
        const double rho_star = cons_state[0] * (S - un) / (S - ustar);
        flux[0] = flux_hllc(flux_state[0], cons_state[0], rho_star, S);
        for (int d = 0; d < nd; ++d) {
            flux[1 + d] = rho_star * ustar * prim_state[1 + d];
        }
        flux[1 + l] = (rho_star * ustar * ustar) + pstar;
        const double E_star = ((S - un) / (S - ustar) * cons_state[1 + nd])
                              + ((ustar - un) / (S - ustar) * ((ustar * cons_state[0] * (S - un)) + prim_state[1 + nd]));
        flux[1 + nd] = flux_hllc(flux_state[1 + nd], cons_state[1 + nd], E_star, S);
    }
}

static void riemann_splitting(const or_ctx* c, const double* consL, const double* consR, int l, double* flux)
{
    /* :146-180 */
    const int nd = c->ndim;
    double primL[MAXV], primR[MAXV];
    or_to_prim(c, consL, primL);
    or_to_prim(c, consR, primR);
    const double PL = primL[1 + nd];
    const double PR = primR[1 + nd];
    const double cL = or_speed_of_sound(c, primL[0], PL);
    const double cR = or_speed_of_sound(c, primR[0], PR);
    const double a = 1.1 * fmax(primL[0] * cL, primR[0] * cR);
    const double ustar = ((primL[1 + l] + primR[1 + l]) / 2) - (1 / (2 * a) * (PR - PL));
    const double Ma = fabs(ustar) / fmin(cL, cR);
    const double theta = fmin(1, Ma);
    const double Pstar = ((PL + PR) / 2) - ((theta * a) / 2 * (primR[1 + l] - primL[1 + l]));
    const double* cons_state = (ustar > 0) ? consL : consR;
    flux[0] = ustar * cons_state[0];
    for (int d = 0; d < nd; ++d) {
        flux[1 + d] = ustar * cons_state[1 + d];
    }
    flux[1 + l] += Pstar;
    flux[1 + nd] = (ustar * cons_state[1 + nd]) + (Pstar * ustar);
}

void or_riemann(const or_ctx* c, int solver, const double* consL, const double* consR, int l, double* flux)
{
    switch (solver) {
    case OR_RS_HLL:
        riemann_hll(c, consL, consR, l, flux);
        break;
    case OR_RS_HLLC:
        riemann_hllc(c, consL, consR, l, flux);
        break;
    default:
        riemann_splitting(c, consL, consR, l, flux);
        break;
    }
}

/* ------------------------------------------------------------------ */
/* Spherical source terms: hydro/source_terms.hpp:16-77                 */
/* ------------------------------------------------------------------ */
static inline double source_grad_pres(double dtodv, double PL, double PR, double dS, double dS_p)
{
    return dtodv * (PL + PR) / 2 * (dS_p - dS);
}
static inline double source_grad_u_r(double dtodv, double rhoL, double rhoR, double uL, double uR, double dS, double dS_p)
{
    return dtodv * ((rhoL * uL * uL) + (rhoR * uR * uR)) / 2 * (dS_p - dS) / 2;
}
static inline double source_grad_u_idir_r(double dtodv, double x0, double x0_p, double rhoL, double rhoR, double uL_r,
                                          double uR_r, double uL_other, double uR_other, double dS, double dS_p)
{
    return dtodv * (x0_p - x0) / (x0_p + x0) * ((rhoR * uR_other * uR_r * dS_p) + (rhoL * uL_other * uL_r * dS));
}
static inline double source_grad_u_th(double dtodv, double x1, double x1_p, double rhoL, double rhoR, double uL_phi,
                                      double uR_phi, double dS, double dS_p)
{
    return dtodv * ((rhoL * uL_phi * uL_phi) + (rhoR * uR_phi * uR_phi)) / 2 * (cos((x1 + x1_p) / 2) / sin((x1 + x1_p) / 2))
           * (dS_p - dS) / 2;
}
static inline double source_grad_u_phi(double dtodv, double x1, double x1_p, double rhoL, double rhoR, double uL_th,
                                       double uR_th, double uL_phi, double uR_phi, double dS, double dS_p)
{
    const double sm = sin(x1);
    const double sp = sin(x1_p);
    return dtodv * (sp - sm) / (sp + sm) * ((rhoR * uR_phi * uR_th * dS_p) + (rhoL * uL_phi * uL_th * dS));
}

/* ------------------------------------------------------------------ */
/* Grid                                                                 */
/* ------------------------------------------------------------------ */
long or_ncells(const or_ctx* c)
{
    return (long)c->n[0] * c->n[1] * c->n[2];
}

static inline long IDX(const or_ctx* c, int i, int j, int k)
{
    return i + (long)c->n[0] * (j + (long)c->n[1] * k);
}

static inline double gravity_at(const or_ctx* c, int i, int dir)
{
    /* gravity.hpp:36-40 (uniform), :63-70 (point mass) and the same radial
       table for the internal mass */
    if (c->gravity != OR_GRAV_UNIFORM) {
        return dir == 0 ? c->g_r[i] : 0;
    }
    return c->g[dir];
}

static void fill_geometry(or_ctx* c)
{
    const long N = or_ncells(c);
    for (int d = 0; d < 3; ++d) {
        /* grid.cpp:31-44 */
        for (int i = 0; i < c->n[d]; ++i) {
            c->dx[d][i] = c->x[d][i + 1] - c->x[d][i];
            c->xc[d][i] = (c->x[d][i] + c->x[d][i + 1]) / 2;
        }
    }
    double* ds = c->ds;
    double* dv = c->dv;
    const double* x0 = c->x[0];
    const double* x1 = c->x[1];
    const double *dx0 = c->dx[0], *dx1 = c->dx[1], *dx2 = c->dx[2];
    /* geometry.cpp: the reference fills all_ghosts, i.e. every cell */
    for (int k = 0; k < c->n[2]; ++k) {
        for (int j = 0; j < c->n[1]; ++j) {
            for (int i = 0; i < c->n[0]; ++i) {
                const long id = IDX(c, i, j, k);
                if (c->geom == OR_GEOM_CARTESIAN) {
                    /* geometry.cpp:43-57 */
                    for (int idim = 0; idim < 3; ++idim) {
                        double dxi[3] = {dx0[i], dx1[j], dx2[k]};
                        dxi[idim] = 1;
                        ds[id + N * idim] = dxi[0] * dxi[1] * dxi[2];
                    }
                    dv[id] = dx0[i] * dx1[j] * dx2[k];
                } else if (c->ndim == 1) {
                    /* geometry.cpp:71-85 */
                    ds[id] = 4 * PI * x0[i] * x0[i];
                    dv[id] = (4 * PI * ((x0[i + 1] * x0[i + 1] * x0[i + 1]) - (x0[i] * x0[i] * x0[i]))) / 3;
                } else if (c->ndim == 2) {
                    /* geometry.cpp:87-105 */
                    const double dcos = cos(x1[j]) - cos(x1[j + 1]);
                    ds[id] = 2 * PI * x0[i] * x0[i] * dcos;
                    ds[id + N] = (2 * PI / 2) * ((x0[i + 1] * x0[i + 1]) - (x0[i] * x0[i])) * sin(x1[j]);
                    dv[id] = (2 * PI / 3) * ((x0[i + 1] * x0[i + 1] * x0[i + 1]) - (x0[i] * x0[i] * x0[i])) * dcos;
                } else {
                    /* geometry.cpp:107-125 */
                    const double dcos = cos(x1[j]) - cos(x1[j + 1]);
                    ds[id] = x0[i] * x0[i] * dcos * dx2[k];
                    ds[id + N] = (1. / 2) * ((x0[i + 1] * x0[i + 1]) - (x0[i] * x0[i])) * sin(x1[j]) * dx2[k];
                    ds[id + 2 * N] = x0[i] * dx0[i] * dx1[j];
                    dv[id] = (1. / 3) * ((x0[i + 1] * x0[i + 1] * x0[i + 1]) - (x0[i] * x0[i] * x0[i])) * dcos * dx2[k];
                }
            }
        }
    }
    if (c->gravity == OR_GRAV_POINT_MASS) {
        /* gravity.cpp:49-55 */
        for (int i = 0; i < c->n[0]; ++i) {
            c->g_r[i] = -GRAV_G * c->central_mass / (c->xc[0][i] * c->xc[0][i]);
        }
    }
}

static int ctx_alloc(or_ctx* c, int ndim, const int nx[3], int ng, int nfx, int geom, double gamma, double mmw,
                     int limiter, int riemann, const int bc[6], int gravity, const double g[3], double central_mass)
{
    memset(c, 0, sizeof(*c));
    /* perfect_gas.cpp:13-22 */
    if (!isfinite(gamma) || gamma <= 1) {
        return -1;
    }
    if (!isfinite(mmw) || mmw <= 0) {
        return -2;
    }
    c->ndim = ndim;
    c->ng = ng;
    c->nfx = nfx;
    c->geom = geom;
    c->gamma = gamma;
    c->gamma_m1 = gamma - 1;
    c->mmw = mmw;
    c->limiter = limiter;
    c->riemann = riemann;
    c->gravity = gravity;
    c->central_mass = central_mass;
    for (int d = 0; d < 3; ++d) {
        c->g[d] = g ? g[d] : 0.0;
        c->nx[d] = d < ndim ? nx[d] : 1;
        /* grid.cpp:56-58,119: ghosts only on active dims */
        c->n[d] = c->nx[d] + (d < ndim ? 2 * ng : 0);
    }
    for (int f = 0; f < 6; ++f) {
        c->bc[f] = bc ? bc[f] : OR_BC_PERIODIC;
        c->bc_order[f] = f; /* boundary_distribute.cpp:35-38 (empty priority) */
    }
    const long N = or_ncells(c);
    for (int d = 0; d < 3; ++d) {
        c->x[d] = (double*)calloc((size_t)c->n[d] + 1, sizeof(double));
        c->dx[d] = (double*)calloc((size_t)c->n[d], sizeof(double));
        c->xc[d] = (double*)calloc((size_t)c->n[d], sizeof(double));
    }
    c->ds = (double*)calloc((size_t)N * 3, sizeof(double));
    c->dv = (double*)calloc((size_t)N, sizeof(double));
    if (gravity != OR_GRAV_UNIFORM) {
        c->g_r = (double*)calloc((size_t)c->n[0], sizeof(double));
    }
    return 0;
}

int or_ctx_init(or_ctx* c, int ndim, const int nx[3], int ng, int nfx, int geom, double gamma, double mmw, int limiter,
                int riemann, const int bc[6], int gravity, const double g[3], double central_mass,
                const double xmin[3], const double xmax[3])
{
    const int rc = ctx_alloc(c, ndim, nx, ng, nfx, geom, gamma, mmw, limiter, riemann, bc, gravity, g, central_mass);
    if (rc) {
        return rc;
    }
    /* grid_type.cpp:151-158 and :176-186: x(i) = xmin + (i - ng) * dx */
    for (int d = 0; d < 3; ++d) {
        const int ngd = d < ndim ? ng : 0;
        const double dxd = (xmax[d] - xmin[d]) / c->nx[d];
        for (int i = 0; i < c->n[d] + 1; ++i) {
            c->x[d][i] = xmin[d] + ((i - ngd) * dxd);
        }
    }
    fill_geometry(c);
    return 0;
}

int or_ctx_init_nodes(or_ctx* c, int ndim, const int nx[3], int ng, int nfx, int geom, double gamma, double mmw,
                      int limiter, int riemann, const int bc[6], int gravity, const double g[3], double central_mass,
                      const double* x0, const double* x1, const double* x2)
{
    const int rc = ctx_alloc(c, ndim, nx, ng, nfx, geom, gamma, mmw, limiter, riemann, bc, gravity, g, central_mass);
    if (rc) {
        return rc;
    }
    const double* xs[3] = {x0, x1, x2};
    for (int d = 0; d < 3; ++d) {
        memcpy(c->x[d], xs[d], sizeof(double) * ((size_t)c->n[d] + 1));
    }
    fill_geometry(c);
    return 0;
}

void or_ctx_free(or_ctx* c)
{
    for (int d = 0; d < 3; ++d) {
        free(c->x[d]);
        free(c->dx[d]);
        free(c->xc[d]);
    }
    free(c->ds);
    free(c->dv);
    free(c->g_r);
    memset(c, 0, sizeof(*c));
}

/* Range::with_ghosts(ng_eff) -> [begin, end) per dim, range.cpp:388-403 */
static void cell_range(const or_ctx* c, int ng_eff, int b[3], int e[3])
{
    for (int d = 0; d < 3; ++d) {
        if (d < c->ndim) {
            b[d] = c->ng - ng_eff;
            e[d] = c->ng + c->nx[d] + ng_eff;
        } else {
            b[d] = 0;
            e[d] = 1;
        }
    }
}

/* ------------------------------------------------------------------ */
/* Array conversions: hydro/array_conversion.hpp                        */
/* ------------------------------------------------------------------ */
void or_conv_prim_to_cons(const or_ctx* c, int ng_eff, const double* rho, const double* u, const double* P,
                          double* rhou, double* E)
{
    int b[3], e[3];
    cell_range(c, ng_eff, b, e);
    const long N = or_ncells(c);
    const int nd = c->ndim;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = b[2]; k < e[2]; ++k) {
        for (int j = b[1]; j < e[1]; ++j) {
            for (int i = b[0]; i < e[0]; ++i) {
                const long id = IDX(c, i, j, k);
                double prim[MAXV], cons[MAXV];
                prim[0] = rho[id];
                for (int d = 0; d < nd; ++d) {
                    prim[1 + d] = u[id + N * d];
                }
                prim[1 + nd] = P[id];
                or_to_cons(c, prim, cons);
                for (int d = 0; d < nd; ++d) {
                    rhou[id + N * d] = cons[1 + d];
                }
                E[id] = cons[1 + nd];
            }
        }
    }
}

void or_conv_cons_to_prim(const or_ctx* c, int ng_eff, const double* rho, const double* rhou, const double* E,
                          double* u, double* P)
{
    int b[3], e[3];
    cell_range(c, ng_eff, b, e);
    const long N = or_ncells(c);
    const int nd = c->ndim;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = b[2]; k < e[2]; ++k) {
        for (int j = b[1]; j < e[1]; ++j) {
            for (int i = b[0]; i < e[0]; ++i) {
                const long id = IDX(c, i, j, k);
                double cons[MAXV], prim[MAXV];
                cons[0] = rho[id];
                for (int d = 0; d < nd; ++d) {
                    cons[1 + d] = rhou[id + N * d];
                }
                cons[1 + nd] = E[id];
                or_to_prim(c, cons, prim);
                for (int d = 0; d < nd; ++d) {
                    u[id + N * d] = prim[1 + d];
                }
                P[id] = prim[1 + nd];
            }
        }
    }
}

/* ------------------------------------------------------------------ */
/* Face reconstruction: hydro/limited_linear_reconstruction.hpp:46-64  */
/* var_rec(i,j,k,s,idim) = var_rec[id + N*s + rec_stride_d*idim]         */
/* ------------------------------------------------------------------ */
void or_face_reconstruction(const or_ctx* c, int ng_eff, const double* var, double* var_rec, long rec_stride_d)
{
    int b[3], e[3];
    cell_range(c, ng_eff, b, e);
    const long N = or_ncells(c);
    const int nd = c->ndim;
    const double *dx0 = c->dx[0], *dx1 = c->dx[1], *dx2 = c->dx[2];
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = b[2]; k < e[2]; ++k) {
        for (int j = b[1]; j < e[1]; ++j) {
            for (int i = b[0]; i < e[0]; ++i) {
                const long id = IDX(c, i, j, k);
                for (int idim = 0; idim < nd; ++idim) {
                    const int ki = idim == 0, kj = idim == 1, kk = idim == 2; /* kronecker.hpp:15-35 */
                    const int im = i - ki, jm = j - kj, km = k - kk;
                    const int ip = i + ki, jp = j + kj, kp = k + kk;
                    const double dl = (ki * dx0[i]) + (kj * dx1[j]) + (kk * dx2[k]);
                    const double dl_m = (ki * dx0[im]) + (kj * dx1[jm]) + (kk * dx2[km]);
                    const double dl_p = (ki * dx0[ip]) + (kj * dx1[jp]) + (kk * dx2[kp]);
                    const double v = var[id];
                    const double slope = or_slope(c->limiter, (var[IDX(c, ip, jp, kp)] - v) / ((dl + dl_p) / 2),
                                                  (v - var[IDX(c, im, jm, km)]) / ((dl_m + dl) / 2));
                    var_rec[id + rec_stride_d * idim] = v - ((dl / 2) * slope);
                    var_rec[id + N + rec_stride_d * idim] = v + ((dl / 2) * slope);
                }
            }
        }
    }
}

/* ------------------------------------------------------------------ */
/* MUSCL-Hancock reconstruction                                         */
/* hydro_reconstruction.hpp:85-129, extrapolation_reconstruction.hpp    */
/* ------------------------------------------------------------------ */
void or_hydro_reconstruction(const or_ctx* c, int ng_eff, double dt, const double* rho, const double* u,
                             const double* P, const double* fx, double* rho_rec, double* rhou_rec, double* E_rec,
                             double* fx_rec, double* u_rec, double* P_rec)
{
    const long N = or_ncells(c);
    const int nd = c->ndim;
    const int nfx = c->nfx;
    /* strides of the (.., s, idim) and (.., s, idim, r) arrays */
    const long S5 = 2 * N;          /* per idim in a 5-D rec array */
    const long S6r = 2 * N * nd;    /* per component r in a 6-D rec array */

    /* hydro_reconstruction.hpp:99-109 */
    or_face_reconstruction(c, ng_eff, rho, rho_rec, S5);
    for (int d = 0; d < nd; ++d) {
        or_face_reconstruction(c, ng_eff, u + N * d, u_rec + S6r * d, S5);
    }
    or_face_reconstruction(c, ng_eff, P, P_rec, S5);
    for (int f = 0; f < nfx; ++f) {
        or_face_reconstruction(c, ng_eff, fx + N * f, fx_rec + 2 * N * nd * f, S5);
    }

    int b[3], e[3];
    cell_range(c, ng_eff, b, e);

    /* hydro_reconstruction.hpp:111-126: prim -> cons for every side and dim */
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = b[2]; k < e[2]; ++k) {
        for (int j = b[1]; j < e[1]; ++j) {
            for (int i = b[0]; i < e[0]; ++i) {
                const long id = IDX(c, i, j, k);
                for (int idim = 0; idim < nd; ++idim) {
                    for (int s = 0; s < 2; ++s) {
                        const long o = id + N * s + S5 * idim;
                        double prim[MAXV], cons[MAXV];
                        prim[0] = rho_rec[o];
                        for (int r = 0; r < nd; ++r) {
                            prim[1 + r] = u_rec[o + S6r * r];
                        }
                        prim[1 + nd] = P_rec[o];
                        or_to_cons(c, prim, cons);
                        for (int r = 0; r < nd; ++r) {
                            rhou_rec[o + S6r * r] = cons[1 + r];
                        }
                        E_rec[o] = cons[1 + nd];
                    }
                }
            }
        }
    }

    /* extrapolation_reconstruction.hpp:87-88: fx_rec_old copy */
    double* fx_rec_old = NULL;
    if (nfx > 0) {
        fx_rec_old = (double*)malloc(sizeof(double) * (size_t)(2 * N * nd * nfx));
        memcpy(fx_rec_old, fx_rec, sizeof(double) * (size_t)(2 * N * nd * nfx));
    }

    const double* x0 = c->x[0];
    const double* x1 = c->x[1];
    const double* ds = c->ds;
    const double* dv = c->dv;
    const int sph = c->geom == OR_GEOM_SPHERICAL;

    /* extrapolation_reconstruction.hpp:90-325 "Hancock_extrapolation" */
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = b[2]; k < e[2]; ++k) {
        for (int j = b[1]; j < e[1]; ++j) {
            for (int i = b[0]; i < e[0]; ++i) {
                const long id = IDX(c, i, j, k);
                double rho_old[2][3];
                double rhou_old[2][3][3];
                for (int idim = 0; idim < nd; ++idim) {
                    rho_old[0][idim] = rho_rec[id + S5 * idim];
                    rho_old[1][idim] = rho_rec[id + N + S5 * idim];
                    for (int r = 0; r < nd; ++r) {
                        rhou_old[0][idim][r] = rhou_rec[id + S5 * idim + S6r * r];
                        rhou_old[1][idim][r] = rhou_rec[id + N + S5 * idim + S6r * r];
                    }
                    for (int f = 0; f < nfx; ++f) {
                        const long of = id + S5 * idim + 2 * N * nd * f;
                        fx_rec[of] *= rho_rec[id + S5 * idim];
                        fx_rec[of + N] *= rho_rec[id + N + S5 * idim];
                    }
                }

                for (int idim = 0; idim < nd; ++idim) {
                    const int ip = i + (idim == 0), jp = j + (idim == 1), kp = k + (idim == 2);
                    const long idp = IDX(c, ip, jp, kp);
                    double primL[MAXV], primR[MAXV], fluxL[MAXV], fluxR[MAXV];
                    primL[0] = rho_old[0][idim];
                    for (int r = 0; r < nd; ++r) {
                        primL[1 + r] = u_rec[id + S5 * idim + S6r * r];
                    }
                    primL[1 + nd] = P_rec[id + S5 * idim];
                    or_flux_from_prim(c, primL, idim, fluxL);

                    primR[0] = rho_old[1][idim];
                    for (int r = 0; r < nd; ++r) {
                        primR[1 + r] = u_rec[id + N + S5 * idim + S6r * r];
                    }
                    primR[1 + nd] = P_rec[id + N + S5 * idim];
                    or_flux_from_prim(c, primR, idim, fluxR);

                    const double dtodv = dt / dv[id];
                    const double dsc = ds[id + N * idim];
                    const double dsp = ds[idp + N * idim];

                    for (int ipos = 0; ipos < nd; ++ipos) {
                        const long o0 = id + S5 * ipos;
                        const long o1 = o0 + N;
                        rho_rec[o0] += dtodv * ((fluxL[0] * dsc) - (fluxR[0] * dsp));
                        rho_rec[o1] += dtodv * ((fluxL[0] * dsc) - (fluxR[0] * dsp));
                        for (int r = 0; r < nd; ++r) {
                            rhou_rec[o0 + S6r * r] += dtodv * ((fluxL[1 + r] * dsc) - (fluxR[1 + r] * dsp));
                            rhou_rec[o1 + S6r * r] += dtodv * ((fluxL[1 + r] * dsc) - (fluxR[1 + r] * dsp));
                        }
                        E_rec[o0] += dtodv * ((fluxL[1 + nd] * dsc) - (fluxR[1 + nd] * dsp));
                        E_rec[o1] += dtodv * ((fluxL[1 + nd] * dsc) - (fluxR[1 + nd] * dsp));
                    }

                    if (sph) {
                        /* :145-303 */
                        const double PL = primL[1 + nd], PR = primR[1 + nd];
                        for (int ipos = 0; ipos < nd; ++ipos) {
                            const long o0 = id + S5 * ipos;
                            const long o1 = o0 + N;
                            if (idim == 0) {
                                const double sp = source_grad_pres(dtodv, PL, PR, dsc, dsp);
                                rhou_rec[o0 + S6r * idim] += sp;
                                rhou_rec[o1 + S6r * idim] += sp;
                                if (nd == 2 || nd == 3) {
                                    const double sr = source_grad_u_r(dtodv, primL[0], primR[0], primL[2], primR[2], dsc, dsp);
                                    rhou_rec[o0 + S6r * idim] += sr;
                                    rhou_rec[o1 + S6r * idim] += sr;
                                    const double st = source_grad_u_idir_r(dtodv, x0[i], x0[i + 1], primL[0], primR[0], primL[1],
                                                                           primR[1], primL[2], primR[2], dsc, dsp);
                                    rhou_rec[o0 + S6r * 1] -= st;
                                    rhou_rec[o1 + S6r * 1] -= st;
                                }
                                if (nd == 3) {
                                    const double sr = source_grad_u_r(dtodv, primL[0], primR[0], primL[3], primR[3], dsc, dsp);
                                    rhou_rec[o0 + S6r * idim] += sr;
                                    rhou_rec[o1 + S6r * idim] += sr;
                                    const double sph2 = source_grad_u_idir_r(dtodv, x0[i], x0[i + 1], primL[0], primR[0], primL[1],
                                                                             primR[1], primL[3], primR[3], dsc, dsp);
                                    rhou_rec[o0 + S6r * 2] -= sph2;
                                    rhou_rec[o1 + S6r * 2] -= sph2;
                                }
                            }
                            if (idim == 1) {
                                const double sp = source_grad_pres(dtodv, PL, PR, dsc, dsp);
                                rhou_rec[o0 + S6r * idim] += sp;
                                rhou_rec[o1 + S6r * idim] += sp;
                                if (nd == 3) {
                                    const double sth = source_grad_u_th(dtodv, x1[j], x1[j + 1], primL[0], primR[0], primL[3],
                                                                        primR[3], dsc, dsp);
                                    rhou_rec[o0 + S6r * idim] += sth;
                                    rhou_rec[o1 + S6r * idim] += sth;
                                    const double sphi = source_grad_u_phi(dtodv, x1[j], x1[j + 1], primL[0], primR[0], primL[2],
                                                                          primR[2], primL[3], primR[3], dsc, dsp);
                                    rhou_rec[o0 + S6r * 2] -= sphi;
                                    rhou_rec[o1 + S6r * 2] -= sphi;
                                }
                            }
                        }
                    }

                    /* gravity :306-312 */
                    const double gd = gravity_at(c, i, idim);
                    for (int ipos = 0; ipos < nd; ++ipos) {
                        const long o0 = id + S5 * ipos;
                        const long o1 = o0 + N;
                        rhou_rec[o0 + S6r * idim] += dt * gd * rho_old[0][ipos];
                        rhou_rec[o1 + S6r * idim] += dt * gd * rho_old[1][ipos];
                        E_rec[o0] += dt * gd * rhou_old[0][ipos][idim];
                        E_rec[o1] += dt * gd * rhou_old[1][ipos][idim];
                    }

                    /* passive scalars :315-337 */
                    for (int f = 0; f < nfx; ++f) {
                        const long off = 2 * N * nd * f;
                        const double flux_fx_L = fx_rec_old[id + S5 * idim + off] * fluxL[0];
                        const double flux_fx_R = fx_rec_old[id + N + S5 * idim + off] * fluxR[0];
                        for (int ipos = 0; ipos < nd; ++ipos) {
                            const long o0 = id + S5 * ipos + off;
                            fx_rec[o0] += dtodv * ((flux_fx_L * dsc) - (flux_fx_R * dsp));
                            fx_rec[o0 + N] += dtodv * ((flux_fx_L * dsc) - (flux_fx_R * dsp));
                        }
                    }
                }
            }
        }
    }

    if (nfx > 0) {
        /* "passive_scalar_extrapolation" :329-339 */
#pragma omp parallel for collapse(2) schedule(static)
        for (int k = b[2]; k < e[2]; ++k) {
            for (int j = b[1]; j < e[1]; ++j) {
                for (int i = b[0]; i < e[0]; ++i) {
                    const long id = IDX(c, i, j, k);
                    for (int idim = 0; idim < nd; ++idim) {
                        for (int f = 0; f < nfx; ++f) {
                            const long off = id + S5 * idim + 2 * N * nd * f;
                            fx_rec[off] /= rho_rec[id + S5 * idim];
                            fx_rec[off + N] /= rho_rec[id + N + S5 * idim];
                        }
                    }
                }
            }
        }
        free(fx_rec_old);
    }
}

/* ------------------------------------------------------------------ */
/* Godunov update: hydro/godunov_scheme.hpp:77-302                      */
/* ------------------------------------------------------------------ */
void or_godunov(const or_ctx* c, int ng_eff, double dt, const double* rho, const double* rhou, const double* E,
                const double* fx, const double* rho_rec, const double* rhou_rec, const double* E_rec,
                const double* fx_rec, double* rho_new, double* rhou_new, double* E_new, double* fx_new)
{
    int b[3], e[3];
    cell_range(c, ng_eff, b, e);
    const long N = or_ncells(c);
    const int nd = c->ndim;
    const int nfx = c->nfx;
    const long S5 = 2 * N;
    const long S6r = 2 * N * nd;
    const double* x0 = c->x[0];
    const double* x1 = c->x[1];
    const double* ds = c->ds;
    const double* dv = c->dv;
    const int sph = c->geom == OR_GEOM_SPHERICAL;

#pragma omp parallel for collapse(2) schedule(static)
    for (int k = b[2]; k < e[2]; ++k) {
        for (int j = b[1]; j < e[1]; ++j) {
            for (int i = b[0]; i < e[0]; ++i) {
                const long id = IDX(c, i, j, k);
                double rn = rho[id];
                double En = E[id];
                double mn[3] = {0, 0, 0};
                for (int d = 0; d < nd; ++d) {
                    mn[d] = rhou[id + N * d];
                }
                for (int f = 0; f < nfx; ++f) {
                    fx_new[id + N * f] = fx[id + N * f] * rho[id];
                }

                for (int idim = 0; idim < nd; ++idim) {
                    const int im = i - (idim == 0), jm = j - (idim == 1), km = k - (idim == 2);
                    const int ip = i + (idim == 0), jp = j + (idim == 1), kp = k + (idim == 2);
                    const long idm = IDX(c, im, jm, km);
                    const long idp = IDX(c, ip, jp, kp);
                    double mR[MAXV], vL[MAXV], vR[MAXV], pL[MAXV], FL[MAXV], FR[MAXV];
                    /* minus_oneR = rec(i-1, side 1), var_L = rec(i, side 0) */
                    mR[0] = rho_rec[idm + N + S5 * idim];
                    vL[0] = rho_rec[id + S5 * idim];
                    vR[0] = rho_rec[id + N + S5 * idim];
                    pL[0] = rho_rec[idp + S5 * idim];
                    for (int r = 0; r < nd; ++r) {
                        mR[1 + r] = rhou_rec[idm + N + S5 * idim + S6r * r];
                        vL[1 + r] = rhou_rec[id + S5 * idim + S6r * r];
                        vR[1 + r] = rhou_rec[id + N + S5 * idim + S6r * r];
                        pL[1 + r] = rhou_rec[idp + S5 * idim + S6r * r];
                    }
                    mR[1 + nd] = E_rec[idm + N + S5 * idim];
                    vL[1 + nd] = E_rec[id + S5 * idim];
                    vR[1 + nd] = E_rec[id + N + S5 * idim];
                    pL[1 + nd] = E_rec[idp + S5 * idim];
                    or_riemann(c, c->riemann, mR, vL, idim, FL);
                    or_riemann(c, c->riemann, vR, pL, idim, FR);

                    const double dtodv = dt / dv[id];
                    const double dsc = ds[id + N * idim];
                    const double dsp = ds[idp + N * idim];
                    rn += dtodv * ((FL[0] * dsc) - (FR[0] * dsp));
                    for (int r = 0; r < nd; ++r) {
                        mn[r] += dtodv * ((FL[1 + r] * dsc) - (FR[1 + r] * dsp));
                    }
                    En += dtodv * ((FL[1 + nd] * dsc) - (FR[1 + nd] * dsp));

                    if (sph) {
                        /* :165-256 */
                        double primL[MAXV], primR[MAXV];
                        or_to_prim(c, vL, primL);
                        or_to_prim(c, vR, primR);
                        if (idim == 0) {
                            mn[idim] += source_grad_pres(dtodv, primL[1 + nd], primR[1 + nd], dsc, dsp);
                            if (nd == 2 || nd == 3) {
                                mn[idim] += source_grad_u_r(dtodv, primL[0], primR[0], primL[2], primR[2], dsc, dsp);
                                mn[1] -= source_grad_u_idir_r(dtodv, x0[i], x0[i + 1], primL[0], primR[0], primL[1], primR[1],
                                                              primL[2], primR[2], dsc, dsp);
                            }
                            if (nd == 3) {
                                mn[idim] += source_grad_u_r(dtodv, primL[0], primR[0], primL[3], primR[3], dsc, dsp);
                                mn[2] -= source_grad_u_idir_r(dtodv, x0[i], x0[i + 1], primL[0], primR[0], primL[1], primR[1],
                                                              primL[3], primR[3], dsc, dsp);
                            }
                        }
                        if (idim == 1) {
                            mn[idim] += source_grad_pres(dtodv, primL[1 + nd], primR[1 + nd], dsc, dsp);
                            if (nd == 3) {
                                mn[idim] += source_grad_u_th(dtodv, x1[j], x1[j + 1], primL[0], primR[0], primL[3], primR[3], dsc, dsp);
                                mn[2] -= source_grad_u_phi(dtodv, x1[j], x1[j + 1], primL[0], primR[0], primL[2], primR[2], primL[3],
                                                           primR[3], dsc, dsp);
                            }
                        }
                    }

                    /* gravity :258-260 */
                    const double gd = gravity_at(c, i, idim);
                    mn[idim] += dt * gd * rho[id];
                    En += dt * gd * rhou[id + N * idim];

                    /* passive scalars :262-290 */
                    for (int f = 0; f < nfx; ++f) {
                        const long off = 2 * N * nd * f;
                        long iL = idm, iR = id;
                        long sL = 1, sR = 1;
                        if (FL[0] < 0) {
                            iL = id;
                            sL = 0;
                        }
                        if (FR[0] < 0) {
                            iR = idp;
                            sR = 0;
                        }
                        const double flux_fx_L = fx_rec[iL + N * sL + S5 * idim + off] * FL[0];
                        const double flux_fx_R = fx_rec[iR + N * sR + S5 * idim + off] * FR[0];
                        fx_new[id + N * f] += dtodv * ((flux_fx_L * dsc) - (flux_fx_R * dsp));
                    }
                }
                rho_new[id] = rn;
                for (int d = 0; d < nd; ++d) {
                    rhou_new[id + N * d] = mn[d];
                }
                E_new[id] = En;
            }
        }
    }

    if (nfx > 0) {
        /* "passive_scalar_Godunov" :294-301 */
#pragma omp parallel for collapse(2) schedule(static)
        for (int k = b[2]; k < e[2]; ++k) {
            for (int j = b[1]; j < e[1]; ++j) {
                for (int i = b[0]; i < e[0]; ++i) {
                    const long id = IDX(c, i, j, k);
                    for (int f = 0; f < nfx; ++f) {
                        double v = fx_new[id + N * f] / rho_new[id];
                        fx_new[id + N * f] = v < 0. ? 0. : (v > 1. ? 1. : v);
                    }
                }
            }
        }
    }
}

/* ------------------------------------------------------------------ */
/* Boundaries: boundary_distribute.hpp:42-76 with one MPI rank,         */
/* boundary_distribute.cpp:75-120 (ghost_sync), boundary.cpp:54-107     */
/* ------------------------------------------------------------------ */
static void copy_cell(const or_ctx* c, double* rho, double* rhou, double* E, double* fx, long dst, long src)
{
    const long N = or_ncells(c);
    rho[dst] = rho[src];
    for (int d = 0; d < c->ndim; ++d) {
        rhou[dst + N * d] = rhou[src + N * d];
    }
    E[dst] = E[src];
    for (int f = 0; f < c->nfx; ++f) {
        fx[dst + N * f] = fx[src + N * f];
    }
}

/* pressure_fix.hpp:19-172 on the no_ghosts range (main.cpp:459-474): where the
 * old internal energy is below eps times the kinetic energy, E_new is rebuilt
 * from a blend of the Godunov increment and a pressure-work estimate from the
 * face velocities.  The loops and the overwrite of E_new inside the inner loop
 * follow the reference. */
void or_internal_mass_gravity(const or_ctx* c, const double* rho)
{
    /* gravity.cpp:59-128 on one rank.  Shells: the nx0 interior cells of
       dimension 0 and the ng ghost cells after them (offset i + ng).  Sums
       over the interior (j, k), j outer and k inner (Kokkos' default
       right-most-fastest MDRange order; the reference's threaded reduction
       may associate differently). */
    const int ng = c->ng;
    const int nsh = c->nx[0] + ng;
    const int g1 = c->ndim >= 2 ? ng : 0;
    const int g2 = c->ndim >= 3 ? ng : 0;
    double* rho_mean = (double*)calloc((size_t)nsh, sizeof(double));
    for (int i = 0; i < nsh; ++i) {
        double sm = 0;
        double sd = 0;
        for (int j = 0; j < c->nx[1]; ++j) {
            for (int k = 0; k < c->nx[2]; ++k) {
                const long id = IDX(c, i + ng, j + g1, k + g2);
                sm += rho[id] * c->dv[id];
                sd += c->dv[id];
            }
        }
        rho_mean[i] = sm / sd; /* :96-100 */
    }
    const double* x0 = c->x[0];
    const double* xc = c->xc[0];
    const double vol_s3 = 4 * OR_PI / 3;
    double* M = c->g_r; /* the enclosed mass first, then g in place */
    for (int i = 0; i < ng; ++i) {
        M[i] = c->central_mass; /* :102 */
    }
    double partial = 0; /* :104-120, a sequential running sum */
    for (int i = ng; i < c->nx[0] + 2 * ng; ++i) {
        const int off = i - ng;
        const double x3 = x0[i] * x0[i] * x0[i];
        if (i == ng) {
            partial += c->central_mass + (vol_s3 * ((xc[i] * xc[i] * xc[i]) - x3) * rho_mean[off]);
        } else {
            partial += (vol_s3 * (x3 - (xc[i - 1] * xc[i - 1] * xc[i - 1])) * rho_mean[off - 1])
                       + (vol_s3 * ((xc[i] * xc[i] * xc[i]) - x3) * rho_mean[off]);
        }
        M[i] = partial;
    }
    for (int i = 0; i < c->n[0]; ++i) {
        M[i] = -GRAV_G * M[i] / (xc[i] * xc[i]); /* :122-125 */
    }
    free(rho_mean);
}

void or_pressure_fix(const or_ctx* c, double dt, double eps, const double* rho, const double* rhou, const double* E,
                     const double* rho_rec, const double* rhou_rec, const double* E_rec, const double* rho_new,
                     const double* rhou_new, double* E_new)
{
    int b[3], e[3];
    cell_range(c, 0, b, e);
    const long N = or_ncells(c);
    const int nd = c->ndim;
    const long S5 = 2 * N;
    const long S6r = 2 * N * nd;
    const double* ds = c->ds;
    const double* dv = c->dv;
    const double eps2 = eps / 10;

#pragma omp parallel for collapse(2) schedule(static)
    for (int k = b[2]; k < e[2]; ++k) {
        for (int j = b[1]; j < e[1]; ++j) {
            for (int i = b[0]; i < e[0]; ++i) {
                const long id = IDX(c, i, j, k);
                double cons[MAXV], cons_new[MAXV], prim[MAXV];
                cons[0] = rho[id];
                cons_new[0] = rho_new[id];
                for (int r = 0; r < nd; ++r) {
                    cons[1 + r] = rhou[id + N * r];
                    cons_new[1 + r] = rhou_new[id + N * r];
                }
                cons[1 + nd] = E[id];
                cons_new[1 + nd] = E_new[id];
                or_to_prim(c, cons, prim);
                const double ekin = or_ek_cons(c, cons);
                const double evol = E[id] - ekin;
                const double evol_new = E_new[id] - or_ek_cons(c, cons_new);
                const double de_god = evol_new - evol;
                if (evol < eps * ekin) {
                    E_new[id] = E[id];
                    double divU = 0;
                    double divUE = 0;
                    double einL = 0;
                    double einR = 0;
                    double alpha = (evol * evol) / (ekin * ekin * eps * eps);
                    if (evol < eps2 * ekin) {
                        alpha = 0;
                    }
                    for (int idim = 0; idim < nd; ++idim) {
                        const long idm = IDX(c, i - (idim == 0), j - (idim == 1), k - (idim == 2));
                        const long idp = IDX(c, i + (idim == 0), j + (idim == 1), k + (idim == 2));
                        for (int ipos = 0; ipos < nd; ++ipos) {
                            double vL[MAXV], vR[MAXV], mR[MAXV], pL[MAXV];
                            double primL[MAXV], primR[MAXV], prim_mR[MAXV], prim_pL[MAXV];
                            double cons_p[MAXV], cons_m[MAXV];
                            vL[0] = rho_rec[id + S5 * idim];
                            vR[0] = rho_rec[id + N + S5 * idim];
                            mR[0] = rho_rec[idm + N + S5 * idim];
                            pL[0] = rho_rec[idp + S5 * idim];
                            cons_p[0] = rho[idp];
                            cons_m[0] = rho[idm];
                            for (int r = 0; r < nd; ++r) {
                                vL[1 + r] = rhou_rec[id + S5 * idim + S6r * r];
                                vR[1 + r] = rhou_rec[id + N + S5 * idim + S6r * r];
                                mR[1 + r] = rhou_rec[idm + N + S5 * idim + S6r * r];
                                pL[1 + r] = rhou_rec[idp + S5 * idim + S6r * r];
                                cons_p[1 + r] = rhou[idp + N * r];
                                cons_m[1 + r] = rhou[idm + N * r];
                            }
                            vL[1 + nd] = E_rec[id + S5 * idim];
                            vR[1 + nd] = E_rec[id + N + S5 * idim];
                            mR[1 + nd] = E_rec[idm + N + S5 * idim];
                            pL[1 + nd] = E_rec[idp + S5 * idim];
                            cons_p[1 + nd] = E[idp];
                            cons_m[1 + nd] = E[idm];
                            or_to_prim(c, vL, primL);
                            or_to_prim(c, vR, primR);
                            or_to_prim(c, mR, prim_mR);
                            or_to_prim(c, pL, prim_pL);
                            const double us = (prim_mR[1 + ipos] + primL[1 + ipos]) / 2;
                            const double us_p = (primR[1 + ipos] + prim_pL[1 + ipos]) / 2;
                            divU += ((us_p * ds[idp + N * ipos]) - (us * ds[id + N * ipos])) / dv[id];
                            if (us_p > 0) {
                                einR = E[id] - or_ek_cons(c, cons);
                            } else {
                                einR = E[idp] - or_ek_cons(c, cons_p);
                            }
                            if (us < 0) {
                                einL = E[id] - or_ek_cons(c, cons);
                            } else {
                                einL = E[idm] - or_ek_cons(c, cons_m);
                            }
                            divUE += ((us_p * einR * ds[idp + N * ipos]) - (us * einL * ds[id + N * ipos])) / dv[id];
                            const double de_pf = dt * ((-prim[1 + nd] * divU) - divUE);
                            double sum = 0;
                            for (int idr = 0; idr < nd; ++idr) {
                                sum += cons[1 + idr] * cons[1 + idr] / cons[0];
                            }
                            const double de_tot = (alpha * de_god) + ((1 - alpha) * de_pf);
                            E_new[id] = evol + de_tot + (1. / 2 * sum);
                        }
                    }
                }
            }
        }
    }
}

void or_boundaries(const or_ctx* c, double* rho, double* rhou, double* E, double* fx)
{
    const long N = or_ncells(c);
    const int nd = c->ndim;
    /* ghost_sync for every dim and face: with a single rank in a periodic
     * Cartesian topology, MPI_Sendrecv_replace returns the rank's own slab,
     * so the ng first interior layers go to the right ghosts (iface 0) and
     * the ng last interior layers go to the left ghosts (iface 1). */
    for (int idim = 0; idim < nd; ++idim) {
        const int ng = c->ng;
        const int nn = c->n[idim];
        for (int iface = 0; iface < 2; ++iface) {
            const int src0 = iface == 0 ? ng : nn - 2 * ng;
            const int dst0 = iface == 0 ? nn - ng : 0;
            for (int k = 0; k < c->n[2]; ++k) {
                for (int j = 0; j < c->n[1]; ++j) {
                    for (int i = 0; i < c->n[0]; ++i) {
                        int idx[3] = {i, j, k};
                        const int l = idx[idim];
                        if (l < dst0 || l >= dst0 + ng) {
                            continue;
                        }
                        int sidx[3] = {i, j, k};
                        sidx[idim] = src0 + (l - dst0);
                        copy_cell(c, rho, rhou, E, fx, IDX(c, i, j, k), IDX(c, sidx[0], sidx[1], sidx[2]));
                    }
                }
            }
        }
    }
    /* physical conditions on border faces in m_bc_order (all faces are
     * border faces on one rank) */
    for (int o = 0; o < 2 * nd; ++o) {
        const int bc_id = c->bc_order[o];
        const int idim = bc_id / 2;
        const int iface = bc_id % 2;
        const int kind = c->bc[bc_id];
        if (kind == OR_BC_PERIODIC) {
            continue; /* boundary.hpp:118-137: no-op */
        }
        const int ng = c->ng;
        const int nn = c->n[idim];
        const int begin = iface == 1 ? nn - ng : 0;
        const int end = begin + ng;
        for (int k = 0; k < c->n[2]; ++k) {
            for (int j = 0; j < c->n[1]; ++j) {
                for (int i = 0; i < c->n[0]; ++i) {
                    int idx[3] = {i, j, k};
                    const int l = idx[idim];
                    if (l < begin || l >= end) {
                        continue;
                    }
                    int sidx[3] = {i, j, k};
                    if (kind == OR_BC_NULLGRADIENT) {
                        sidx[idim] = iface == 0 ? end : begin - 1; /* boundary.cpp:241 */
                    } else {
                        const int mirror = iface == 0 ? ((2 * ng) - 1) : ((2 * (nn - ng)) - 1); /* boundary.cpp:279 */
                        sidx[idim] = mirror - l;
                    }
                    const long dst = IDX(c, i, j, k);
                    copy_cell(c, rho, rhou, E, fx, dst, IDX(c, sidx[0], sidx[1], sidx[2]));
                    if (kind == OR_BC_REFLEXIVE) {
                        rhou[dst + N * idim] = -rhou[dst + N * idim]; /* boundary.cpp:290 */
                    }
                }
            }
        }
    }
}

/* ------------------------------------------------------------------ */
/* Reductions                                                           */
/* ------------------------------------------------------------------ */
double or_time_step(const or_ctx* c, int ng_eff, const double* rho, const double* u, const double* P)
{
    /* time_step.hpp:55-82 */
    int b[3], e[3];
    cell_range(c, ng_eff, b, e);
    const long N = or_ncells(c);
    const int nd = c->ndim;
    const int sph = c->geom == OR_GEOM_SPHERICAL;
    double inverse_dt = 0;
#pragma omp parallel for collapse(2) reduction(max : inverse_dt) schedule(static)
    for (int k = b[2]; k < e[2]; ++k) {
        for (int j = b[1]; j < e[1]; ++j) {
            for (int i = b[0]; i < e[0]; ++i) {
                const long id = IDX(c, i, j, k);
                const double sound = or_speed_of_sound(c, rho[id], P[id]);
                double dxg[3] = {c->dx[0][i], c->dx[1][j], c->dx[2][k]};
                if (sph) {
                    if (nd == 2) {
                        dxg[1] *= c->xc[0][i];
                    }
                    if (nd == 3) {
                        dxg[1] *= c->xc[0][i];
                        dxg[2] *= c->xc[0][i] * sin(c->xc[1][j]);
                    }
                }
                double cell_inverse_dt = 0;
                for (int d = 0; d < nd; ++d) {
                    cell_inverse_dt += (fabs(u[id + N * d]) + sound) / dxg[d];
                }
                inverse_dt = inverse_dt > cell_inverse_dt ? inverse_dt : cell_inverse_dt;
            }
        }
    }
    return 1 / inverse_dt;
}

double or_min_internal_energy(const or_ctx* c, const double* rho, const double* rhou, const double* E)
{
    /* internal_energy.cpp:20-45 over no_ghosts */
    int b[3], e[3];
    cell_range(c, 0, b, e);
    const long N = or_ncells(c);
    const int nd = c->ndim;
    double evol = INFINITY;
    int has_nan = 0;
#pragma omp parallel for collapse(2) reduction(min : evol) reduction(| : has_nan) schedule(static)
    for (int k = b[2]; k < e[2]; ++k) {
        for (int j = b[1]; j < e[1]; ++j) {
            for (int i = b[0]; i < e[0]; ++i) {
                const long id = IDX(c, i, j, k);
                double cons[MAXV];
                cons[0] = rho[id];
                for (int d = 0; d < nd; ++d) {
                    cons[1 + d] = rhou[id + N * d];
                }
                cons[1 + nd] = E[id];
                const double ce = evol_cons(c, cons);
                if (isnan(ce)) {
                    has_nan = 1;
                }
                evol = ce < evol ? ce : evol;
            }
        }
    }
    return has_nan ? NAN : evol;
}

double or_integrate(const or_ctx* c, const double* var)
{
    /* integration.cpp:22-37 over no_ghosts; Kahan-compensated here so the
     * result does not depend on the thread count */
    int b[3], e[3];
    cell_range(c, 0, b, e);
    double s = 0, comp = 0;
    for (int k = b[2]; k < e[2]; ++k) {
        for (int j = b[1]; j < e[1]; ++j) {
            for (int i = b[0]; i < e[0]; ++i) {
                const long id = IDX(c, i, j, k);
                const double y = var[id] * c->dv[id] - comp;
                const double t = s + y;
                comp = (t - s) - y;
                s = t;
            }
        }
    }
    return s;
}

/* ------------------------------------------------------------------ */
/* Initial state and time loop                                          */
/* ------------------------------------------------------------------ */
void or_init_from_prim(const or_ctx* c, const double* rho_prim, const double* u, const double* P, double* rho,
                       double* rhou, double* E, double* fx)
{
    /* main.cpp:305-307: conv_prim_to_cons(no_ghosts) then bcs */
    const long N = or_ncells(c);
    memcpy(rho, rho_prim, sizeof(double) * (size_t)N);
    or_conv_prim_to_cons(c, 0, rho_prim, u, P, rhou, E);
    or_boundaries(c, rho, rhou, E, fx);
}

int or_run(const or_ctx* c, double* rho, double* rhou, double* E, double* fx, const or_run_params* p,
           or_run_result* res, double* dts_out)
{
    const long N = or_ncells(c);
    const int nd = c->ndim;
    const int nfx = c->nfx;
    double* u = (double*)calloc((size_t)N * nd, sizeof(double));
    double* P = (double*)calloc((size_t)N, sizeof(double));
    double* rho_rec = (double*)calloc((size_t)N * 2 * nd, sizeof(double));
    double* rhou_rec = (double*)calloc((size_t)N * 2 * nd * nd, sizeof(double));
    double* E_rec = (double*)calloc((size_t)N * 2 * nd, sizeof(double));
    double* fx_rec = (double*)calloc((size_t)N * 2 * nd * (nfx > 0 ? nfx : 1), sizeof(double));
    double* u_rec = (double*)calloc((size_t)N * 2 * nd * nd, sizeof(double));
    double* P_rec = (double*)calloc((size_t)N * 2 * nd, sizeof(double));
    double* rho_new = (double*)calloc((size_t)N, sizeof(double));
    double* rhou_new = (double*)calloc((size_t)N * nd, sizeof(double));
    double* E_new = (double*)calloc((size_t)N, sizeof(double));
    double* fx_new = (double*)calloc((size_t)N * (nfx > 0 ? nfx : 1), sizeof(double));

    int status = 0;
    double t = p->t_ini;
    int iter = 0;
    int iter_output_id = -1;  /* main.cpp:207-209 */
    int time_output_id = -1;
    int should_exit = 0;
    /* main.cpp:315-316: an initial output bumps iter_output_id */
    if (p->iter_frequency > 0 || p->time_frequency > 0) {
        ++iter_output_id;
    }

    /* main.cpp:309-311 */
    if (c->gravity == OR_GRAV_INTERNAL_MASS) {
        or_internal_mass_gravity(c, rho);
    }
    or_conv_cons_to_prim(c, c->ng, rho, rhou, E, u, P);
    res->initial_mass = or_integrate(c, rho);

    while (!should_exit) {
        double dt;
        if (p->fixed_dt) {
            dt = p->dts[iter];
        } else {
            dt = p->cfl * or_time_step(c, c->ng, rho, u, P); /* main.cpp:355 */
        }
        if (p->iter_frequency > 0) { /* :358-364 */
            const int next_output = (iter_output_id + 1) * p->iter_frequency;
            if ((iter + 1) >= next_output) {
                ++iter_output_id;
            }
        }
        if (p->time_frequency > 0) { /* :365-375 */
            const double next_output = p->time_first_output + ((time_output_id + 1) * p->time_frequency);
            if ((t + dt) >= next_output) {
                dt = next_output - t;
                if (dt <= 0) {
                    status = 2;
                    break;
                }
                ++time_output_id;
            }
        }
        if ((t + dt) >= p->t_end) { /* :377-381 */
            dt = p->t_end - t;
            should_exit = 1;
        }
        if ((iter + 1) >= p->max_iter) { /* :382-385 */
            should_exit = 1;
        }
        const double min_evol = or_min_internal_energy(c, rho, rhou, E); /* :397-425 */
        if (isnan(min_evol) || min_evol < 0) {
            status = 1;
            break;
        }
        if (dts_out) {
            dts_out[iter] = dt;
        }
        or_hydro_reconstruction(c, 1, dt / 2, rho, u, P, fx, rho_rec, rhou_rec, E_rec, fx_rec, u_rec, P_rec);
        or_godunov(c, 0, dt, rho, rhou, E, fx, rho_rec, rhou_rec, E_rec, fx_rec, rho_new, rhou_new, E_new, fx_new);
        if (p->pressure_fix) { /* :459-474 */
            or_pressure_fix(c, dt, p->eps_pf, rho, rhou, E, rho_rec, rhou_rec, E_rec, rho_new, rhou_new, E_new);
        }
        or_boundaries(c, rho_new, rhou_new, E_new, fx_new); /* :479 */
        memcpy(rho, rho_new, sizeof(double) * (size_t)N);   /* :481-484 */
        memcpy(rhou, rhou_new, sizeof(double) * (size_t)N * nd);
        memcpy(E, E_new, sizeof(double) * (size_t)N);
        if (nfx > 0) {
            memcpy(fx, fx_new, sizeof(double) * (size_t)N * nfx);
        }
        or_conv_cons_to_prim(c, c->ng, rho, rhou, E, u, P); /* :526 */
        if (c->gravity == OR_GRAV_INTERNAL_MASS) {
            or_internal_mass_gravity(c, rho); /* :528 */
        }
        t += dt;                                             /* :530-531 */
        ++iter;
    }
    res->t = t;
    res->iter = iter;
    res->status = status;
    res->final_mass = or_integrate(c, rho);

    free(u);
    free(P);
    free(rho_rec);
    free(rhou_rec);
    free(E_rec);
    free(fx_rec);
    free(u_rec);
    free(P_rec);
    free(rho_new);
    free(rhou_new);
    free(E_new);
    free(fx_new);
    return status;
}
